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


@pytest.mark.parametrize("name", ["wall2d", "per2d", "wall3d"])
def test_interface_band_viscous_matches_reference(cuda_device, golden, name):
    """ccd_bulk with psi (compute_explicit and the Picard CN predictor) against
    the reference's own outputs at the viscous bar."""
    from twophaseflow_b200 import CCDSolver, UniformGrid, ViscousTerm
    N = tuple(int(n) for n in golden[f"{name}/N"])
    L = tuple(float(x) for x in golden[f"{name}/L"])
    ccd = CCDSolver(UniformGrid(N, L), None, bc_type=str(golden[f"{name}/bc"]))
    vel = [golden[f"{name}/u{a}"] for a in range(len(N))]
    e = [golden[f"{name}/e{a}"] for a in range(len(N))]
    mu, rho, psi = golden[f"{name}/mu"], golden[f"{name}/rho"], golden[f"{name}/psi"]
    v = ViscousTerm(None, 100.0, spatial_scheme="ccd_bulk").compute_explicit(vel, mu, rho, ccd, psi=psi)
    u = ViscousTerm(None, 100.0, cn_viscous=True).apply_cn_predictor(vel, e, mu, rho, ccd, 0.003, psi=psi)
    for a in range(len(N)):
        ref = golden[f"{name}/ccd_bulk_band/v{a}"]
        assert np.abs(v[a] - ref).max() <= TOL * np.abs(ref).max(), (a, np.abs(v[a] - ref).max())
        ref = golden[f"{name}/pred_band{a}"]
        assert np.abs(u[a] - ref).max() <= TOL * np.abs(ref).max()


@pytest.mark.parametrize("shape", [(129, 130), (41, 38, 45)])
def test_band_mask_kernel_bit_exact(cuda_device, shape):
    """The band and normal-axis masks against the oracle on seeded psi with
    exact 0 / 1 plateaus, ties between axes and a flat region."""
    import ctypes as C
    import torch
    from oracle import viscous as ov
    from twophaseflow_b200 import _lib
    rng = np.random.default_rng(71)
    nd = len(shape)
    psi = rng.uniform(0.0, 1.0, shape)
    psi[psi < 0.3] = 0.0
    psi[psi > 0.7] = 1.0
    psi[tuple(slice(0, 5) for _ in shape)] = 0.5        # flat: every axis normal
    coords = [np.linspace(0.0, 1.0 + 0.2 * a, n) for a, n in enumerate(shape)]
    band, normal = ov.band_masks(psi, coords)
    grads = [torch.from_numpy(ov.low_order_derivative(psi, a, coords[a])).cuda() for a in range(nd)]
    tp = torch.from_numpy(psi).cuda()
    b = torch.empty(shape, dtype=torch.uint8, device="cuda")
    m = [torch.empty_like(b) for _ in range(nd)]
    lib = _lib.load()
    _lib.check(lib.tpf_visc_band_masks(nd, (C.c_int64 * nd)(*shape), _lib.dptr(tp),
                                       (C.c_void_p * nd)(*[_lib.dptr(g) for g in grads]), _lib.dptr(b),
                                       (C.c_void_p * nd)(*[_lib.dptr(x) for x in m]), _lib.TPF_F64,
                                       _lib.current_stream_handle()))
    np.testing.assert_array_equal(b.cpu().numpy().astype(bool), band)
    for a in range(nd):
        np.testing.assert_array_equal(m[a].cpu().numpy().astype(bool), normal[a])


@pytest.mark.parametrize("name", ["wall2d", "per2d", "wall3d"])
def test_richardson_cn_predictor_matches_reference(cuda_device, golden, name):
    """cn_mode='richardson_picard' (RichardsonCNAdvance around Picard, three
    Picard steps and one combination kernel) against the reference's own
    output, at the CN predictor's bar; the factory rejects unknown modes."""
    from types import SimpleNamespace
    from twophaseflow_b200 import CCDSolver, RichardsonCNAdvance, UniformGrid, ViscousTerm, make_cn_advance
    from twophaseflow_b200.predictor import Predictor
    N = tuple(int(n) for n in golden[f"{name}/N"])
    L = tuple(float(x) for x in golden[f"{name}/L"])
    ccd = CCDSolver(UniformGrid(N, L), None, bc_type=str(golden[f"{name}/bc"]))
    vel = [golden[f"{name}/u{a}"] for a in range(len(N))]
    e = [golden[f"{name}/e{a}"] for a in range(len(N))]
    adv = make_cn_advance(None, "richardson_picard")
    assert isinstance(adv, RichardsonCNAdvance)
    u = ViscousTerm(None, 100.0, cn_viscous=True, cn_advance=adv).apply_cn_predictor(
        vel, e, golden[f"{name}/mu"], golden[f"{name}/rho"], ccd, 0.003)
    for a in range(len(N)):
        ref = golden[f"{name}/pred_rich{a}"]
        assert np.abs(u[a] - ref).max() <= TOL * np.abs(ref).max()
    with pytest.raises(ValueError, match="cn_mode"):
        make_cn_advance(None, "pade22")
    cfg = SimpleNamespace(grid=SimpleNamespace(ndim=len(N)), fluid=SimpleNamespace(Re=100.0, Fr=1.0, We=10.0),
                          numerics=SimpleNamespace(cn_viscous=True, cn_mode="richardson_picard"))
    assert isinstance(Predictor(None, cfg, ccd).viscous.cn_advance, RichardsonCNAdvance)


def test_cn_combine_kernel_bit_exact(cuda_device):
    """The combinations against NumPy on the same operands."""
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
    # mode 3: the Richardson extrapolation (4 u - vn) / 3, e and rho unused
    _lib.check(lib.tpf_cn_predictor_combine(u.size, 3, 0.0, _lib.dptr(T[0]), None, None, _lib.dptr(T[3]), None,
                                            _lib.dptr(out), _lib.TPF_F64, _lib.current_stream_handle()))
    np.testing.assert_array_equal(out.cpu().numpy(), (4.0 * u - vn) / 3.0)


PGOLD = os.path.join(os.path.dirname(__file__), "golden", "predictor_golden.npz")


@pytest.fixture(scope="module")
def pgolden():
    with np.load(PGOLD) as d:
        return {k: d[k] for k in d.files}


@pytest.mark.parametrize("name", ["wall2d", "per2d", "wall3d"])
def test_predictor_matches_reference(cuda_device, pgolden, name):
    """Two consecutive steps (the second uses the stored convection: AB2)."""
    from types import SimpleNamespace
    from twophaseflow_b200 import CCDSolver, FlowState, Predictor, UniformGrid
    g = pgolden
    N = tuple(int(x) for x in g[f"{name}/N"])
    L = tuple(float(x) for x in g[f"{name}/L"])
    bc = str(g[f"{name}/bc"])
    cfg = SimpleNamespace(grid=SimpleNamespace(ndim=len(N)), fluid=SimpleNamespace(Re=50.0, Fr=0.8, We=4.0),
                          numerics=SimpleNamespace(cn_viscous=bool(g[f"{name}/cn"]), cn_mode="picard"))
    ccd = CCDSolver(UniformGrid(N, L), None, bc_type=bc)
    pred = Predictor(None, cfg, ccd, use_gfm=bool(g[f"{name}/gfm"]))
    for s in range(2):
        vel = [g[f"{name}/s{s}/u{a}"] for a in range(len(N))]
        psi = g[f"{name}/s{s}/psi"]
        st = FlowState(velocity=vel, psi=psi, rho=0.1 + 0.9 * psi, mu=0.01 + 0.99 * psi, kappa=g[f"{name}/s{s}/kappa"],
                       pressure=g[f"{name}/s{s}/p"])
        u = pred.compute(st, float(g[f"{name}/s{s}/dt"]))
        for a in range(len(N)):
            ref = g[f"{name}/s{s}/ustar{a}"]
            assert isinstance(u[a], np.ndarray)
            assert np.abs(u[a] - ref).max() <= TOL * np.abs(ref).max()


def test_predictor_kernels_bit_exact(cuda_device):
    """Convection accumulation, gravity / CSF scaling, the explicit right-hand
    side (first step and AB2) and the explicit viscous update against NumPy."""
    import torch
    from twophaseflow_b200 import _lib
    rng = np.random.default_rng(73)
    shape = (129, 130, 131)
    a, b, c, d, e = (rng.standard_normal(shape) for _ in range(5))
    rho = 0.1 + rng.uniform(0.0, 1.0, shape)
    T = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    lib = _lib.load()
    st = _lib.current_stream_handle()
    n = a.size
    acc = T(c.copy())
    ta, tb, trho = T(a), T(b), T(rho)   # held: a temporary's memory could be reused before the kernel runs
    _lib.check(lib.tpf_ns_conv_accumulate(n, 0, _lib.dptr(ta), _lib.dptr(tb), _lib.dptr(acc), _lib.TPF_F64, st))
    np.testing.assert_array_equal(acc.cpu().numpy(), c - a * b)
    out = torch.empty_like(acc)
    _lib.check(lib.tpf_ns_scaled(n, 0, _lib.dptr(trho), None, 0.64, _lib.dptr(out), _lib.TPF_F64, st))
    np.testing.assert_array_equal(out.cpu().numpy(), -rho / 0.64)
    _lib.check(lib.tpf_ns_scaled(n, 1, _lib.dptr(ta), _lib.dptr(tb), 4.0, _lib.dptr(out), _lib.TPF_F64, st))
    np.testing.assert_array_equal(out.cpu().numpy(), a * b / 4.0)
    tc, td, te = T(c), T(d), T(e)
    for ab2 in (0, 1):
        _lib.check(lib.tpf_ns_explicit_rhs(n, ab2, _lib.dptr(ta), _lib.dptr(tb), _lib.dptr(trho), _lib.dptr(tc),
                                           _lib.dptr(td), _lib.dptr(te), _lib.dptr(out), _lib.TPF_F64, st))
        cv = (1.5 * a - 0.5 * b) if ab2 else a
        np.testing.assert_array_equal(out.cpu().numpy(), rho * cv + c + d + (-e))
    _lib.check(lib.tpf_cn_predictor_combine(n, 2, 0.003, _lib.dptr(ta), _lib.dptr(tb), _lib.dptr(trho),
                                            _lib.dptr(tc), None, _lib.dptr(out), _lib.TPF_F64, st))
    np.testing.assert_array_equal(out.cpu().numpy(), a + 0.003 * (b + rho * c) / rho)


@pytest.mark.parametrize("scheme", SCHEMES)
def test_viscous_nonuniform_grid_matches_reference(cuda_device, scheme):
    """The three schemes on the reference's interface-fitted 32^2 wall grid
    (cell widths 0.019..0.033; tests/golden/viscous_nonuniform_golden.npz):
    the low-order stencil from the node coordinates, the CCD derivatives with
    the grid metric; the conservative scheme has no CCD solve, so it is bit
    for bit."""
    from types import SimpleNamespace
    from twophaseflow_b200 import CCDSolver, ViscousTerm
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "viscous_nonuniform_golden.npz"))
    N = tuple(int(n) for n in g["N"])
    coords = [g["coords0"], g["coords1"]]
    grid = SimpleNamespace(N=N, ndim=2, L=(1.0, 1.0), shape=tuple(n + 1 for n in N), uniform=False,
                           J=[g["J0"], g["J1"]], dJ_dxi=[g["dJ0"], g["dJ1"]], coords=coords)
    ccd = CCDSolver(grid, None, bc_type="wall")
    v = ViscousTerm(None, 100.0, spatial_scheme=scheme).compute_explicit([g["u0"], g["u1"]], g["mu"], g["rho"], ccd)
    for a in range(2):
        ref = g[f"{scheme}/v{a}"]
        if scheme == "conservative_stress":
            np.testing.assert_array_equal(v[a], ref)
        else:
            assert np.abs(v[a] - ref).max() <= TOL * np.abs(ref).max(), (a, np.abs(v[a] - ref).max())
