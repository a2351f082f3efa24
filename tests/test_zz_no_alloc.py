"""The allocation-free CG entry point (tpf_ppe_solve_cg_static) against the
handle-based solve (tpf_ppe_solve, CG, FP64), both called through the C ABI.

The entry point is for callers that cannot allocate device memory while they
run (a caching allocator that already holds the device, a memory budget fixed
at start-up).  It runs the same kernels on the same grid shape, so its
iterates match the handle path: the test asks for the same iteration count and
solutions within 1e-12 of the solution's magnitude, on two calls in a row (the
second call reuses the workspace left by the first), and checks that a call
after the first leaves the device's free memory unchanged.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from twophaseflow_b200 import _lib
from twophaseflow_b200.workloads import divergence_rhs, droplet_density, node_coords

pytestmark = pytest.mark.gpu


def _coords_arg(coords):
    arrs = [np.ascontiguousarray(c, dtype=np.float64) for c in coords]
    ptrs = (C.POINTER(C.c_double) * len(arrs))(*[a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs])
    return arrs, ptrs


def _handle_solve(lib, N, coords, pin, rhs_d, rho_d, p_d, precond, tol, maxiter, stream):
    o = _lib.tpf_ppe_options()
    lib.tpf_ppe_default_options(C.byref(o))
    o.method, o.precond, o.precision = _lib.TPF_PPE_CG, precond, _lib.TPF_PREC_F64
    o.tol, o.maxiter = tol, maxiter
    keep, cptr = _coords_arg(coords)
    Na = (C.c_int64 * len(N))(*N)
    h = C.c_void_p()
    _lib.check(lib.tpf_ppe_create(C.byref(h), len(N), Na, cptr, pin, C.byref(o)))
    try:
        res = _lib.tpf_ppe_result()
        _lib.check(lib.tpf_ppe_solve(h, _lib.dptr(rhs_d), _lib.dptr(rho_d), _lib.dptr(p_d), None, stream,
                                     C.byref(res)))
    finally:
        lib.tpf_ppe_destroy(h)
    return res


def _static_solve(lib, N, coords, pin, rhs_d, rho_d, p_d, precond, tol, maxiter, stream):
    keep, cptr = _coords_arg(coords)
    Na = (C.c_int64 * len(N))(*N)
    res = _lib.tpf_ppe_result()
    st = lib.tpf_ppe_solve_cg_static(len(N), Na, cptr, pin, _lib.dptr(rhs_d), _lib.dptr(rho_d), _lib.dptr(p_d),
                                     None, precond, tol, maxiter, stream, C.byref(res))
    _lib.check(st)
    return res


CASES = [
    ((64, 64), "jacobi"),
    ((96, 40), "none"),
    ((24, 20, 28), "jacobi"),
    ((256, 256), "jacobi"),
    ((39, 39, 39), "jacobi"),   # 40^3 = 64 000 nodes: the 3-D size at the limit
]


@pytest.mark.parametrize("N,precond", CASES)
def test_static_cg_matches_handle_solve(cuda_device, N, precond):
    import torch
    lib = _lib.load()
    pc = _lib.TPF_PRECOND_JACOBI if precond == "jacobi" else _lib.TPF_PRECOND_NONE
    coords = node_coords(N)
    if len(N) == 2:
        # a non-uniform first axis: the grid metrics come from the coordinates
        x = coords[0]
        coords = [x + 0.15 * np.sin(np.pi * x) / np.pi * (x[1] - x[0]) * 4, coords[1]]
    rho = droplet_density(N, n_drops=6, rho_g=1e-2)
    rhs = divergence_rhs(N)
    pin = 0
    rho_d = torch.from_numpy(rho).to(cuda_device)
    rhs_d = torch.from_numpy(rhs).to(cuda_device)
    stream = _lib.current_stream_handle()
    tol, maxiter = 1e-10, 20000
    p_ref = torch.zeros_like(rho_d)
    r_ref = _handle_solve(lib, N, coords, pin, rhs_d, rho_d, p_ref, pc, tol, maxiter, stream)
    scale = float(p_ref.abs().max())
    assert scale > 0.0
    for call in range(2):
        p = torch.full_like(rho_d, float("nan"))
        r = _static_solve(lib, N, coords, pin, rhs_d, rho_d, p, pc, tol, maxiter, stream)
        torch.cuda.synchronize()
        assert r.info == 0
        assert r.iterations == r_ref.iterations, (call, r.iterations, r_ref.iterations)
        assert r.rel_residual < tol
        err = float((p - p_ref).abs().max())
        assert err <= 1e-12 * scale, (call, err, scale)
        assert float(p.flatten()[pin]) == 0.0


def test_static_cg_allocates_no_device_memory(cuda_device):
    """After the first call on the device (which looks the workspace up and,
    under lazy module loading, loads it), further calls change the device's
    free memory by nothing: no cudaMalloc, no allocating library call."""
    import torch
    lib = _lib.load()
    N = (128, 128)
    coords = node_coords(N)
    rho_d = torch.from_numpy(droplet_density(N, n_drops=6, rho_g=1e-2)).to(cuda_device)
    rhs_d = torch.from_numpy(divergence_rhs(N)).to(cuda_device)
    p = torch.zeros_like(rho_d)
    stream = _lib.current_stream_handle()
    _static_solve(lib, N, coords, 0, rhs_d, rho_d, p, _lib.TPF_PRECOND_JACOBI, 1e-10, 20000, stream)
    torch.cuda.synchronize()
    reserved = torch.cuda.memory_reserved()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        r = _static_solve(lib, N, coords, 0, rhs_d, rho_d, p, _lib.TPF_PRECOND_JACOBI, 1e-10, 20000, stream)
        assert r.info == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert torch.cuda.memory_reserved() == reserved


def test_static_cg_rejects_oversize_and_bad_arguments(cuda_device):
    import torch
    lib = _lib.load()
    stream = _lib.current_stream_handle()
    dummy = torch.zeros(4, dtype=torch.float64, device=cuda_device)
    res = _lib.tpf_ppe_result()

    def call(N, precond=_lib.TPF_PRECOND_JACOBI, tol=1e-8):
        keep, cptr = _coords_arg(node_coords(N))
        Na = (C.c_int64 * len(N))(*N)
        return lib.tpf_ppe_solve_cg_static(len(N), Na, cptr, 0, _lib.dptr(dummy), _lib.dptr(dummy),
                                           _lib.dptr(dummy), None, precond, tol, 100, stream, C.byref(res))

    # 257 x 257 cells = 258^2 nodes > TPF_PPE_STATIC_MAX_DOF
    assert call((257, 257)) == _lib.TPF_EINVAL
    assert "exceed the maximum" in _lib.last_error()
    # per-axis limit
    assert call((_lib.TPF_PPE_STATIC_MAX_AXIS, 8)) == _lib.TPF_EINVAL
    assert call((8, 8), precond=_lib.TPF_PRECOND_LINE) == _lib.TPF_EINVAL
    assert call((8, 8), tol=0.0) == _lib.TPF_EINVAL
