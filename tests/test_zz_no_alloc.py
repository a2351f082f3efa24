"""The allocation-free CG entry point (tpf_ppe_solve_cg_static) against the
handle-based solve (tpf_ppe_solve, CG, FP64), both called through the C ABI.

The static entry point runs the same kernels on the same grid shape, so its
iterates match the handle path: the test asks for the same iteration count and
solutions within 1e-12 of the solution's magnitude, on two calls in a row (the
second call reuses the workspace left by the first).
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
