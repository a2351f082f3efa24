"""GPU tests of the CLS transport: the FCCD flux-form right-hand side and the
TVD-RK3 level-set step, against the reference's outputs
(tests/golden/advect_golden.npz) and the oracle."""

from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from oracle import advect as oa

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "advect_golden.npz")
CASES = ["wall2d", "per2d", "wall3d", "per3d"]
# the CCD second derivatives agree with the reference to ~1e-13 relative
TOL = 1e-10


@pytest.fixture(scope="module")
def golden():
    with np.load(GOLDEN) as d:
        return {k: d[k] for k in d.files}


def _setup(g, name):
    from twophaseflow_b200 import CCDSolver, FCCDSolver, UniformGrid
    N = tuple(int(n) for n in g[f"{name}/N"])
    L = tuple(float(x) for x in g[f"{name}/L"])
    bc = str(g[f"{name}/bc"])
    grid = UniformGrid(N, L)
    ccd = CCDSolver(grid, None, bc_type=bc)
    return N, grid, FCCDSolver(grid, None, bc_type=bc, ccd_solver=ccd)


@pytest.mark.parametrize("name", CASES)
def test_rhs_matches_reference(cuda_device, golden, name):
    N, grid, fccd = _setup(golden, name)
    vel = [golden[f"{name}/u{a}"] for a in range(len(N))]
    r = fccd.advection_rhs(vel, scalar=golden[f"{name}/psi"], mode="flux")[0]
    ref = golden[f"{name}/rhs_scalar"]
    assert isinstance(r, np.ndarray)
    assert np.abs(r - ref).max() <= TOL * np.abs(ref).max()
    mom = fccd.advection_rhs(vel, mode="flux")
    for a in range(len(N)):
        ref = golden[f"{name}/rhs_mom{a}"]
        assert np.abs(mom[a] - ref).max() <= TOL * np.abs(ref).max()


@pytest.mark.parametrize("name", CASES)
def test_rk3_step_matches_reference(cuda_device, golden, name):
    from twophaseflow_b200 import FCCDLevelSetAdvection
    N, grid, fccd = _setup(golden, name)
    vel = [golden[f"{name}/u{a}"] for a in range(len(N))]
    dt = float(golden[f"{name}/dt"])
    adv = FCCDLevelSetAdvection(None, grid, fccd, mode="flux")
    out = adv.advance(golden[f"{name}/psi"].copy(), vel, dt)
    assert np.abs(out - golden[f"{name}/psi_new"]).max() <= 1e-12
    assert out.min() >= 0.0 and out.max() <= 1.0
    out = adv.advance(golden[f"{name}/psi"].copy(), vel, dt, clip_bounds=None)
    assert np.abs(out - golden[f"{name}/psi_new_noclip"]).max() <= 1e-12


@pytest.mark.parametrize("shape,periodic", [((1025, 1025), False), ((1025, 1025), True), ((129, 130, 131), False),
                                            ((129, 130, 131), True)])
def test_flux_kernel_bit_exact(cuda_device, shape, periodic):
    """The face-value + divergence kernel alone on every axis, given the same
    product and second derivative as the oracle: bit-identical."""
    import torch
    from twophaseflow_b200 import _lib
    rng = np.random.default_rng(23)
    prod = rng.standard_normal(shape)
    q = rng.standard_normal(shape)
    P, Q = torch.from_numpy(prod).cuda(), torch.from_numpy(q).cuda()
    acc = torch.empty_like(P)
    sh = (C.c_int64 * len(shape))(*shape)
    ref = np.zeros(shape)
    lib = _lib.load()
    for ax in range(len(shape)):
        H = 1.0 / (shape[ax] - 1) * (1.0 + 0.25 * ax)
        _lib.check(lib.tpf_fccd_flux_divergence_axis(len(shape), sh, ax, int(periodic), H, _lib.dptr(P), _lib.dptr(Q),
                                                     1 if ax else 0, _lib.dptr(acc), _lib.TPF_F64,
                                                     _lib.current_stream_handle()))
        ref += oa.flux_divergence(prod, q, ax, H, periodic)
    np.testing.assert_array_equal(acc.cpu().numpy(), ref)


def test_stage_and_image_kernels_bit_exact(cuda_device):
    """TVD-RK3 stage arithmetic, clip (NaN kept) and periodic image nodes on a
    periodic-wall box against NumPy."""
    import torch
    from twophaseflow_b200 import _lib
    rng = np.random.default_rng(29)
    shape = (65, 66)
    q0, q, L = (rng.uniform(-0.2, 1.2, shape) for _ in range(3))
    q[3, 4] = np.nan
    T = [torch.from_numpy(a).cuda() for a in (q0, q, L)]
    out = torch.empty_like(T[0])
    sh = (C.c_int64 * 2)(*shape)
    per = (C.c_int * 2)(1, 0)
    lib = _lib.load()
    for stage, ca, cb in ((1, 0.0, 0.0), (2, 0.75, 0.25), (3, 1.0 / 3.0, 2.0 / 3.0)):
        _lib.check(lib.tpf_tvd_rk3_stage(2, sh, per, stage, ca, cb, 0.013, _lib.dptr(T[0]), _lib.dptr(T[1]),
                                         _lib.dptr(T[2]), 1, 0.0, 1.0, _lib.dptr(out), _lib.TPF_F64,
                                         _lib.current_stream_handle()))
        up = q + 0.013 * L
        ref = up if stage == 1 else ca * q0 + cb * up
        ref = np.clip(ref, 0.0, 1.0)
        ref[-1, :] = ref[0, :]
        np.testing.assert_array_equal(out.cpu().numpy(), ref)
    a = torch.from_numpy(q0.copy()).cuda()
    per3 = (C.c_int * 2)(1, 1)
    _lib.check(lib.tpf_sync_periodic_images(2, sh, per3, _lib.dptr(a), _lib.TPF_F64, _lib.current_stream_handle()))
    np.testing.assert_array_equal(a.cpu().numpy(), oa.sync_images(q0.copy(), "periodic"))


def test_transport_full_size_properties(cuda_device):
    """257^3 periodic box, device tensors: the flux form conserves the sum over
    the unique nodes (to rounding), the step keeps psi in [0, 1] and equals
    the oracle's RK3 step on a 65^3 crop of the same construction."""
    import torch
    from twophaseflow_b200 import CCDSolver, FCCDLevelSetAdvection, FCCDSolver, UniformGrid
    for n, check_oracle in ((256, False), (64, True)):
        N = (n, n, n)
        x = torch.linspace(0.0, 1.0, n + 1, dtype=torch.float64, device="cuda")
        X = torch.meshgrid(x, x, x, indexing="ij")
        r = torch.sqrt((X[0] - 0.5) ** 2 + (X[1] - 0.5) ** 2 + (X[2] - 0.5) ** 2)
        psi = torch.sigmoid((0.25 - r) / (1.5 / n)).contiguous()
        vel = [torch.sin(2 * np.pi * X[(a + 1) % 3]).contiguous() for a in range(3)]
        del X, r
        grid = UniformGrid(N)
        fccd = FCCDSolver(grid, None, bc_type="periodic", ccd_solver=CCDSolver(grid, None, bc_type="periodic"))
        rhs = fccd.advection_rhs(vel, scalar=psi)[0]
        s = rhs[:-1, :-1, :-1]
        assert abs(float(s.sum())) <= 1e-9 * float(s.abs().sum())
        out = FCCDLevelSetAdvection(None, grid, fccd).advance(psi, vel, 0.2 / n)
        assert float(out.min()) >= 0.0 and float(out.max()) <= 1.0
        if check_oracle:
            ref = oa.advance(psi.cpu().numpy(), [v.cpu().numpy() for v in vel], 0.2 / n, (1.0,) * 3, N, "periodic")
            assert np.abs(out.cpu().numpy() - ref).max() <= 1e-12
