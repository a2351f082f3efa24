"""GPU tests of the steps either side of the PPE: the velocity corrector fused
into the CCD line solve and the CFL time step, against the reference's outputs
(tests/golden/step_golden.npz) and the oracle."""

from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

from oracle import step as ostep

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "step_golden.npz")
CASES = ["wall2d", "per2d", "wall3d"]
# the CCD derivatives agree with the reference to ~1e-13 relative (test_ccd_gpu)
TOL = 1e-10


@pytest.fixture(scope="module")
def golden():
    with np.load(GOLDEN) as d:
        return {k: d[k] for k in d.files}


def _grid(g, name):
    from twophaseflow_b200 import CCDSolver, UniformGrid
    N = tuple(int(n) for n in g[f"{name}/N"])
    L = tuple(float(x) for x in g[f"{name}/L"])
    grid = UniformGrid(N, L)
    bc = str(g[f"{name}/bc"])
    return N, grid, CCDSolver(grid, None, bc_type=bc)


@pytest.mark.parametrize("name", CASES)
def test_corrector_matches_reference(cuda_device, golden, name):
    """NumPy in, NumPy out, like the reference's CPU backend; the wall planes
    keep u* exactly."""
    from twophaseflow_b200 import VelocityCorrector, ccd_pressure_gradient
    N, grid, ccd = _grid(golden, name)
    vel = [golden[f"{name}/u{a}"] for a in range(len(N))]
    p, rho, dt = golden[f"{name}/p"], golden[f"{name}/rho"], float(golden[f"{name}/dt"])
    out = VelocityCorrector(None, grid, ccd).correct(vel, p, rho, dt)
    grad = ccd_pressure_gradient(ccd, p, len(N))
    for ax in range(len(N)):
        assert isinstance(out[ax], np.ndarray)
        ref = golden[f"{name}/unew{ax}"]
        assert np.abs(out[ax] - ref).max() <= TOL * np.abs(ref).max()
        ref_g = golden[f"{name}/grad{ax}"]
        assert np.abs(grad[ax] - ref_g).max() <= TOL * np.abs(ref_g).max()
        if str(golden[f"{name}/bc"]) == "wall":
            assert np.array_equal(np.take(out[ax], [0, -1], axis=ax), np.take(vel[ax], [0, -1], axis=ax))


@pytest.mark.parametrize("bc", ["wall", "periodic"])
def test_corrector_lane_kernel_epilogue_against_oracle(cuda_device, bc):
    """160^3 (161^3 nodes): every axis runs the lane-per-line kernel (strided
    and contiguous store paths) with the corrector epilogue."""
    import torch
    from twophaseflow_b200 import CCDSolver, UniformGrid, VelocityCorrector
    N = (160, 160, 160)
    grid = UniformGrid(N)
    ccd = CCDSolver(grid, None, bc_type=bc)
    rng = np.random.default_rng(31)
    shape = tuple(n + 1 for n in N)
    x = [np.linspace(0.0, 1.0, n + 1) for n in N]
    X = np.meshgrid(*x, indexing="ij")
    p = np.sin(2 * np.pi * X[0]) * np.cos(4 * np.pi * X[1]) * np.sin(2 * np.pi * X[2]) + 0.1 * rng.standard_normal(shape)
    rho = 1e-3 + rng.uniform(0.0, 1.0, shape)
    vel = [rng.standard_normal(shape) for _ in range(3)]
    dt = 0.01
    dev = [torch.from_numpy(v).to(cuda_device) for v in vel]
    out = VelocityCorrector(None, grid, ccd).correct(dev, torch.from_numpy(p).to(cuda_device),
                                                     torch.from_numpy(rho).to(cuda_device), dt)
    ref = ostep.correct(vel, p, rho, dt, [1.0 / n for n in N], bc)
    for ax in range(3):
        o = out[ax].cpu().numpy()
        assert np.abs(o - ref[ax]).max() <= TOL * np.abs(ref[ax]).max()


def test_corrector_in_place_through_the_c_abi(cuda_device, golden):
    """u_out == u_star is allowed (the correction is applied exactly once)."""
    import torch
    from twophaseflow_b200 import _lib
    from twophaseflow_b200.arrays import line_split
    name = "wall3d"
    N, grid, ccd = _grid(golden, name)
    p = torch.from_numpy(golden[f"{name}/p"]).to(cuda_device)
    rho = torch.from_numpy(golden[f"{name}/rho"]).to(cuda_device)
    dt = float(golden[f"{name}/dt"])
    lib = _lib.load()
    for ax in range(len(N)):
        u = torch.from_numpy(golden[f"{name}/u{ax}"]).to(cuda_device).contiguous()
        outer, n, inner = line_split(u.shape, ax)
        plan = ccd._plan(ax, False)
        _lib.check(lib.tpf_ccd_apply_corrector(plan, outer, inner, _lib.dptr(p), _lib.dptr(u), _lib.dptr(rho),
                                               C.c_double(dt), _lib.dptr(u), 0, _lib.current_stream_handle()))
        ref = golden[f"{name}/unew{ax}"]
        assert np.abs(u.cpu().numpy() - ref).max() <= TOL * np.abs(ref).max()


def test_corrector_rejects_aliasing_pressure(cuda_device, golden):
    import torch
    from twophaseflow_b200 import _lib
    from twophaseflow_b200.arrays import line_split
    name = "wall2d"
    N, grid, ccd = _grid(golden, name)
    p = torch.from_numpy(golden[f"{name}/p"]).to(cuda_device)
    rho = torch.from_numpy(golden[f"{name}/rho"]).to(cuda_device)
    lib = _lib.load()
    outer, n, inner = line_split(p.shape, 0)
    st = lib.tpf_ccd_apply_corrector(ccd._plan(0, False), outer, inner, _lib.dptr(p), _lib.dptr(p), _lib.dptr(rho),
                                     C.c_double(0.1), _lib.dptr(p), 0, None)
    assert st == _lib.TPF_EINVAL


@pytest.mark.parametrize("name", CASES)
def test_cfl_matches_reference_exactly(cuda_device, golden, name):
    """The maxima are exact, the formula is the reference's: identical dt."""
    import torch
    from twophaseflow_b200 import CFLCalculator
    N, grid, ccd = _grid(golden, name)
    vel = [torch.from_numpy(golden[f"{name}/u{a}"]).to(cuda_device) for a in range(len(N))]
    mu = torch.from_numpy(golden[f"{name}/mu"]).to(cuda_device)
    rho = torch.from_numpy(golden[f"{name}/rho"]).to(cuda_device)
    for tag, kw in (("cn", dict(cn_viscous=True)), ("expl", dict(cn_viscous=False)),
                    ("cap", dict(We=0.01, rho_ratio=0.1, cn_viscous=True))):
        assert CFLCalculator(None, grid, 0.3, **kw).compute(vel, mu, rho) == float(golden[f"{name}/dt_{tag}"])


def test_cfl_maxima_large_and_nan(cuda_device):
    """Maxima over 2^24 + 3 values (grid-stride loop, warp shuffles, one atomic
    per warp) equal NumPy's; a NaN propagates as in the reference."""
    import torch
    from twophaseflow_b200 import CFLCalculator, UniformGrid
    rng = np.random.default_rng(5)
    n = (1 << 24) + 3
    u = rng.standard_normal(n)
    v = rng.standard_normal(n) * 3.0
    mu = rng.uniform(0.1, 1.0, n)
    rho = rng.uniform(0.1, 1.0, n)
    calc = CFLCalculator(None, UniformGrid((16, 16)), 0.3)
    dev = lambda a: torch.from_numpy(a).to(cuda_device)
    sp, nu = calc.maxima([dev(u), dev(v)], dev(mu), dev(rho))
    assert sp == [float(np.max(np.abs(u))), float(np.max(np.abs(v)))]
    assert nu == float(np.max(mu / rho))
    u[12345] = np.nan
    sp, _ = calc.maxima([dev(u), dev(v)])
    assert np.isnan(sp[0]) and sp[1] == float(np.max(np.abs(v)))


RCG = os.path.join(os.path.dirname(__file__), "golden", "rhiechow_golden.npz")
RC_CASES = ["wall2d", "per2d", "wall3d", "per3d"]


@pytest.fixture(scope="module")
def rc_golden():
    with np.load(RCG) as d:
        return {k: d[k] for k in d.files}


@pytest.mark.parametrize("name", RC_CASES)
def test_rc_divergence_matches_reference(cuda_device, rc_golden, name):
    """NumPy in and out; within the CCD's rounding of the reference."""
    from twophaseflow_b200 import RhieChowInterpolator
    g = rc_golden
    N, grid, ccd = _grid(g, name)
    rc = RhieChowInterpolator(None, grid, ccd, bc_type=str(g[f"{name}/bc"]))
    vel = [g[f"{name}/u{a}"] for a in range(len(N))]
    p, rho, dt = g[f"{name}/p"], g[f"{name}/rho"], float(g[f"{name}/dt"])
    d = rc.face_velocity_divergence(vel, p, rho, dt)
    ref = g[f"{name}/div"]
    assert isinstance(d, np.ndarray)
    assert np.abs(d - ref).max() <= TOL * np.abs(ref).max()
    d = rc.face_velocity_divergence(vel, p, rho, dt, kappa=g[f"{name}/kappa"], psi=g[f"{name}/psi"],
                                    we=float(g[f"{name}/we"]))
    ref = g[f"{name}/div_bf"]
    assert np.abs(d - ref).max() <= TOL * np.abs(ref).max()


@pytest.mark.parametrize("shape,periodic", [((1025, 1025), False), ((1025, 1025), True), ((129, 130, 131), False),
                                            ((129, 130, 131), True)])
def test_rc_axis_kernel_bit_exact(cuda_device, shape, periodic):
    """The divergence kernel alone, every axis, plain and balanced-force, with
    the same derivative arrays given to the oracle: bit-identical."""
    import torch
    from twophaseflow_b200 import _lib
    rng = np.random.default_rng(17)
    f = {k: rng.standard_normal(shape) for k in ("u", "p", "dp", "kappa", "psi", "dpsi")}
    f["rho"] = 1e-3 + rng.uniform(0.0, 1.0, shape)
    T = {k: torch.from_numpy(v).cuda() for k, v in f.items()}
    sh = (C.c_int64 * len(shape))(*shape)
    lib = _lib.load()
    for bf in (False, True):
        div = torch.empty(shape, dtype=torch.float64, device="cuda")
        ref = np.zeros(shape)
        for ax in range(len(shape)):
            h = 1.0 / (shape[ax] - 1) * (1.0 + 0.1 * ax)
            extra = [_lib.dptr(T["kappa"]), _lib.dptr(T["psi"]), _lib.dptr(T["dpsi"]), 0.7] if bf else \
                [None, None, None, 0.0]
            _lib.check(lib.tpf_rc_divergence_axis(len(shape), sh, ax, int(periodic), h, 0.013, _lib.dptr(T["u"]),
                                                  _lib.dptr(T["p"]), _lib.dptr(T["rho"]), _lib.dptr(T["dp"]),
                                                  *extra, 1 if ax else 0, _lib.dptr(div), _lib.TPF_F64,
                                                  _lib.current_stream_handle()))
            ref += ostep._rc_axis(f["u"], f["p"], f["rho"], f["dp"], ax, h, 0.013, periodic,
                                  f["kappa"] if bf else None, f["psi"] if bf else None,
                                  f["dpsi"] if bf else None, 0.7 if bf else None)
        np.testing.assert_array_equal(div.cpu().numpy(), ref)


def test_rc_refuses_partial_balanced_force(cuda_device):
    import torch
    from twophaseflow_b200 import _lib
    x = torch.zeros((8, 8), dtype=torch.float64, device="cuda")
    sh = (C.c_int64 * 2)(8, 8)
    st = _lib.load().tpf_rc_divergence_axis(2, sh, 0, 0, 0.1, 0.01, _lib.dptr(x), _lib.dptr(x), _lib.dptr(x),
                                            _lib.dptr(x), _lib.dptr(x), None, None, 0.7, 0, _lib.dptr(x),
                                            _lib.TPF_F64, None)
    assert st != 0 and "balanced-force" in _lib.last_error()
