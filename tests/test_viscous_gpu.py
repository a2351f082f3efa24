"""GPU tests of the viscous stress divergence (ViscousTerm.compute_explicit)
against the reference's outputs (tests/golden/viscous_golden.npz) and the oracle."""

from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import viscous as ov

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "viscous_golden.npz")
SCHEMES = ["ccd_bulk", "conservative_stress", "ccd_stress_legacy"]
TOL = 1e-10   # CCD rounding against the reference's dense LU


@pytest.fixture(scope="module")
def golden():
    with np.load(GOLDEN) as d:
        return {k: d[k] for k in d.files}


@pytest.mark.parametrize("name", ["wall2d", "per2d", "wall3d"])
@pytest.mark.parametrize("scheme", SCHEMES)
def test_viscous_matches_reference(cuda_device, golden, name, scheme):
    """The low-order scheme involves no CCD solve: bit-identical; the CCD
    schemes within the CCD's rounding."""
    from twophaseflow_b200 import CCDSolver, UniformGrid, ViscousTerm
    N = tuple(int(n) for n in golden[f"{name}/N"])
    L = tuple(float(x) for x in golden[f"{name}/L"])
    grid = UniformGrid(N, L)
    ccd = CCDSolver(grid, None, bc_type=str(golden[f"{name}/bc"]))
    vel = [golden[f"{name}/u{a}"] for a in range(len(N))]
    v = ViscousTerm(None, 100.0, spatial_scheme=scheme).compute_explicit(vel, golden[f"{name}/mu"],
                                                                         golden[f"{name}/rho"], ccd)
    for a in range(len(N)):
        ref = golden[f"{name}/{scheme}/v{a}"]
        assert isinstance(v[a], np.ndarray)
        if scheme == "conservative_stress":
            np.testing.assert_array_equal(v[a], ref)
        else:
            assert np.abs(v[a] - ref).max() <= TOL * np.abs(ref).max()


@pytest.mark.parametrize("shape", [(513, 385), (65, 66, 67)])
def test_low_order_scheme_bit_exact_large(cuda_device, shape):
    """The low-order kernel (stress formed inside, accumulation, division by
    Re rho) on a larger grid with device tensors: bit-identical to the oracle."""
    import torch
    from twophaseflow_b200 import CCDSolver, UniformGrid, ViscousTerm
    rng = np.random.default_rng(61)
    N = tuple(n - 1 for n in shape)
    L = tuple(1.0 + 0.3 * a for a in range(len(shape)))
    vel = [rng.standard_normal(shape) for _ in shape]
    mu = 0.01 + rng.uniform(0.0, 1.0, shape)
    rho = 0.001 + rng.uniform(0.0, 1.0, shape)
    grid = UniformGrid(N, L)
    ccd = CCDSolver(grid, None, bc_type="wall")
    T = lambda a: torch.from_numpy(a).cuda()
    v = ViscousTerm(None, 37.0, spatial_scheme="conservative_stress").compute_explicit(
        [T(x) for x in vel], T(mu), T(rho), ccd)
    ref = ov.viscous(vel, mu, rho, 37.0, L, N, "wall", "conservative_stress")
    for a in range(len(shape)):
        assert v[a].is_cuda
        np.testing.assert_array_equal(v[a].cpu().numpy(), ref[a])


def test_viscous_of_rigid_rotation_vanishes(cuda_device):
    """u = -y, v = x with constant mu: grad u + grad u^T = 0, so V = 0."""
    import torch
    from twophaseflow_b200 import CCDSolver, UniformGrid, ViscousTerm
    n = 128
    x = np.linspace(0.0, 1.0, n + 1)
    X, Y = np.meshgrid(x, x, indexing="ij")
    grid = UniformGrid((n, n))
    ccd = CCDSolver(grid, None, bc_type="wall")
    for scheme in SCHEMES:
        v = ViscousTerm(None, 10.0, spatial_scheme=scheme).compute_explicit([-Y, X], np.full(X.shape, 0.3),
                                                                            np.ones(X.shape), ccd)
        assert max(np.abs(c).max() for c in v) < 1e-9


@pytest.mark.parametrize("name", ["wall2d", "per2d", "wall3d"])
@pytest.mark.parametrize("tag,cn", [("cn", True), ("fe", False)])
def test_cn_predictor_matches_reference(cuda_device, golden, name, tag, cn):
    from twophaseflow_b200 import CCDSolver, UniformGrid, ViscousTerm
    N = tuple(int(n) for n in golden[f"{name}/N"])
    L = tuple(float(x) for x in golden[f"{name}/L"])
    ccd = CCDSolver(UniformGrid(N, L), None, bc_type=str(golden[f"{name}/bc"]))
    vel = [golden[f"{name}/u{a}"] for a in range(len(N))]
    e = [golden[f"{name}/e{a}"] for a in range(len(N))]
    u = ViscousTerm(None, 100.0, cn_viscous=cn).apply_cn_predictor(vel, e, golden[f"{name}/mu"],
                                                                   golden[f"{name}/rho"], ccd, 0.003)
    for a in range(len(N)):
        ref = golden[f"{name}/pred_{tag}{a}"]
        assert isinstance(u[a], np.ndarray)
        assert np.abs(u[a] - ref).max() <= TOL * np.abs(ref).max()


def test_cn_combine_kernel_bit_exact(cuda_device):
    """Both combinations against NumPy on the same operands."""
    import torch
    from twophaseflow_b200 import _lib
    rng = np.random.default_rng(67)
    shape = (129, 130, 131)
    u, e, vn, vs = (rng.standard_normal(shape) for _ in range(4))
    rho = 0.001 + rng.uniform(0.0, 1.0, shape)
    T = [torch.from_numpy(a).cuda() for a in (u, e, rho, vn, vs)]
    out = torch.empty_like(T[0])
    lib = _lib.load()
    for mode in (0, 1):
        _lib.check(lib.tpf_cn_predictor_combine(u.size, mode, 0.0037, *[_lib.dptr(t) for t in T], _lib.dptr(out),
                                                _lib.TPF_F64, _lib.current_stream_handle()))
        ref = u + 0.0037 * (e / rho + vn) if mode == 0 else u + 0.0037 * (e / rho + 0.5 * vn + 0.5 * vs)
        np.testing.assert_array_equal(out.cpu().numpy(), ref)
