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
def test_node_mode_matches_reference(cuda_device, golden, name):
    """Option C (mode="node"): node gradients, nodal right-hand sides and one
    RK3 step against the reference's own outputs."""
    from twophaseflow_b200 import FCCDLevelSetAdvection
    N, grid, fccd = _setup(golden, name)
    vel = [golden[f"{name}/u{a}"] for a in range(len(N))]
    psi = golden[f"{name}/psi"]
    for a in range(len(N)):
        g = fccd.node_gradient(psi, a)
        ref = golden[f"{name}/node_grad_psi{a}"]
        assert np.abs(g - ref).max() <= TOL * np.abs(ref).max(), (a, np.abs(g - ref).max())
    r = fccd.advection_rhs(vel, scalar=psi, mode="node")[0]
    ref = golden[f"{name}/rhs_scalar_node"]
    assert np.abs(r - ref).max() <= TOL * np.abs(ref).max()
    mom = fccd.advection_rhs(vel, mode="node")
    for a in range(len(N)):
        ref = golden[f"{name}/rhs_mom_node{a}"]
        assert np.abs(mom[a] - ref).max() <= TOL * np.abs(ref).max()
    out = FCCDLevelSetAdvection(None, grid, fccd, mode="node").advance(psi.copy(), vel, float(golden[f"{name}/dt"]))
    assert np.abs(out - golden[f"{name}/psi_new_node"]).max() <= 1e-12


@pytest.mark.parametrize("shape,periodic", [((1025, 1025), False), ((129, 130, 131), True)])
def test_node_gradient_kernel_bit_exact(cuda_device, shape, periodic):
    """The Option C kernel alone on every axis, given the oracle's operands:
    bit-identical gradient and accumulation."""
    import torch
    from twophaseflow_b200 import _lib
    rng = np.random.default_rng(29)
    u, q, uk = (rng.standard_normal(shape) for _ in range(3))
    U, Q, K = (torch.from_numpy(a).cuda() for a in (u, q, uk))
    out = torch.empty_like(U)
    acc = torch.empty_like(U)
    sh = (C.c_int64 * len(shape))(*shape)
    lib = _lib.load()
    ref_acc = np.zeros(shape)
    for ax in range(len(shape)):
        H = 1.0 / (shape[ax] - 1) * (1.0 + 0.25 * ax)
        for mode, dst in ((0, out), (1 if ax == 0 else 2, acc)):
            _lib.check(lib.tpf_fccd_node_gradient_axis(len(shape), sh, ax, int(periodic), H, _lib.dptr(U),
                                                       _lib.dptr(Q), _lib.dptr(K), mode, _lib.dptr(dst),
                                                       _lib.TPF_F64, _lib.current_stream_handle()))
        g = oa.node_gradient(u, q, ax, H, periodic)
        np.testing.assert_array_equal(out.cpu().numpy(), g)
        ref_acc = ref_acc - uk * g
    np.testing.assert_array_equal(acc.cpu().numpy(), ref_acc)


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


RGOLD = os.path.join(os.path.dirname(__file__), "golden", "reinit_golden.npz")
REINIT = ["zero2d", "per2d", "neu2d", "zero3d"]


@pytest.fixture(scope="module")
def rgolden():
    with np.load(RGOLD) as d:
        return {k: d[k] for k in d.files}


@pytest.mark.parametrize("name", REINIT)
def test_reinit_matches_reference(cuda_device, rgolden, name):
    """Within 1e-11 of the reference (the CCD's rounding differs; the oracle's
    output moves by ~5e-14 for 1e-14 input noise on these fields)."""
    from twophaseflow_b200 import CCDSolver, SplitReinitializer, UniformGrid
    g = rgolden
    N = tuple(int(x) for x in g[f"{name}/N"])
    L = tuple(float(x) for x in g[f"{name}/L"])
    grid = UniformGrid(N, L)
    ccd = CCDSolver(grid, None, bc_type=str(g[f"{name}/ccd_bc"]))
    r = SplitReinitializer(None, grid, ccd, float(g[f"{name}/eps"]), n_steps=int(g[f"{name}/n_steps"]),
                           bc=str(g[f"{name}/bc"]), mass_correction=bool(g[f"{name}/mass"]))
    out = r.reinitialize(g[f"{name}/psi"])
    assert isinstance(out, np.ndarray)
    assert np.abs(out - g[f"{name}/psi_reinit"]).max() <= 1e-11


@pytest.mark.parametrize("name", CASES)
def test_mass_corrected_transport_matches_reference(cuda_device, golden, name):
    from twophaseflow_b200 import FCCDLevelSetAdvection
    N, grid, fccd = _setup(golden, name)
    vel = [golden[f"{name}/u{a}"] for a in range(len(N))]
    adv = FCCDLevelSetAdvection(None, grid, fccd, mode="flux", mass_correction=True)
    out = adv.advance(golden[f"{name}/psi"].copy(), vel, float(golden[f"{name}/dt"]))
    assert np.abs(out - golden[f"{name}/psi_new_mass"]).max() <= 1e-12


@pytest.mark.parametrize("shape", [(1025, 1025), (129, 130, 131)])
def test_reinit_kernels_bit_exact(cuda_device, shape):
    """Compression flux, filtered divergence (all three paddings) and the CN
    line solve alone, every axis, against the oracle's arithmetic."""
    import torch
    from twophaseflow_b200 import _lib
    rng = np.random.default_rng(41)
    nd = len(shape)
    lib = _lib.load()
    st = _lib.current_stream_handle()
    sh = (C.c_int64 * nd)(*shape)
    psi = rng.uniform(0.0, 1.0, shape)
    d1 = [rng.standard_normal(shape) for _ in range(nd)]
    d1[0][0, 0] = 1e-9   # below the |grad| floor
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    tp, td = T(psi), [T(a) for a in d1]
    flux = [torch.empty_like(tp) for _ in range(nd)]
    P = C.c_void_p * nd
    _lib.check(lib.tpf_reinit_compression_flux(nd, tp.numel(), _lib.dptr(tp), P(*[_lib.dptr(t) for t in td]),
                                               P(*[_lib.dptr(t) for t in flux]), _lib.TPF_F64, st))
    gs = sum(x * x for x in d1)
    sg = np.maximum(np.sqrt(np.maximum(gs, 1e-12)), 1e-6)
    for a in range(nd):
        np.testing.assert_array_equal(flux[a].cpu().numpy(), (psi * (1.0 - psi)) * (d1[a] / sg))
    for pad, label in ((0, "zero"), (1, "periodic"), (2, "neumann")):
        div = torch.empty_like(tp)
        ref = np.zeros(shape)
        for a in range(nd):
            _lib.check(lib.tpf_reinit_filtered_divergence_axis(nd, sh, a, pad, 0.05, _lib.dptr(td[a]), 1 if a else 0,
                                                               _lib.dptr(div), _lib.TPF_F64, st))
            gp = oa._pad(d1[a], a, label)
            n = gp.shape[a]
            c = np.take(gp, range(1, n - 1), axis=a)
            ref = ref + (c + 0.05 * (np.take(gp, range(2, n), axis=a) - 2.0 * c + np.take(gp, range(0, n - 2), axis=a)))
        np.testing.assert_array_equal(div.cpu().numpy(), ref)
    # CN line solve with factors built as the reference builds them
    for a in range(nd):
        n = shape[a]
        mu = 0.7
        c_L, d_L = oa.BETA2 - 3.0 * mu, 1.0 + 6.0 * mu
        sup, sub, m = np.full(n - 1, c_L), np.full(n - 1, c_L), np.full(n, d_L)
        sup[0] = 2.0 * c_L
        sub[-1] = 2.0 * c_L
        f = np.empty(n - 1)
        for i in range(1, n):
            f[i - 1] = sub[i - 1] / m[i - 1]
            m[i] -= f[i - 1] * sup[i - 1]
        cR, dR = oa.BETA2 + 3.0 * mu, 1.0 - 6.0 * mu
        out = torch.empty_like(tp)
        tf, tm, ts = T(f), T(m), T(sup)   # held until the kernel has run
        _lib.check(lib.tpf_reinit_cn_axis(nd, sh, a, cR, dR, _lib.dptr(tf), _lib.dptr(tm), _lib.dptr(ts),
                                          _lib.dptr(tp), _lib.dptr(out), _lib.TPF_F64, st))
        torch.cuda.synchronize()
        p = np.moveaxis(psi, a, 0)
        d = np.empty_like(p)
        d[1:-1] = cR * p[:-2] + dR * p[1:-1] + cR * p[2:]
        d[0] = dR * p[0] + 2.0 * cR * p[1]
        d[-1] = 2.0 * cR * p[-2] + dR * p[-1]
        for i in range(1, n):
            d[i] = d[i] - f[i - 1] * d[i - 1]
        x = np.empty_like(d)
        x[-1] = d[-1] / m[-1]
        for i in range(n - 2, -1, -1):
            x[i] = (d[i] - sup[i] * x[i + 1]) / m[i]
        np.testing.assert_array_equal(out.cpu().numpy(), np.moveaxis(x, 0, a))


def test_mass_correction_kernels(cuda_device):
    """Device sums within rounding of NumPy's; the corrected field restores the
    target mass and stays in [0, 1]; W <= 1e-12 leaves q unchanged."""
    import torch
    from twophaseflow_b200 import _lib
    rng = np.random.default_rng(43)
    q = rng.uniform(0.0, 1.0, (257, 257, 65))
    dV = np.full(q.shape, 1.0 / 256 ** 2 / 64)
    lib = _lib.load()
    st = _lib.current_stream_handle()
    tq, tv = torch.from_numpy(q).cuda(), torch.from_numpy(dV).cuda()
    part = torch.empty(2048, dtype=torch.float64, device="cuda")
    sums = torch.empty(2, dtype=torch.float64, device="cuda")
    _lib.check(lib.tpf_mass_sums(q.size, _lib.dptr(tq), _lib.dptr(tv), _lib.dptr(part), _lib.dptr(sums),
                                 _lib.TPF_F64, st))
    s = sums.cpu().numpy()
    assert abs(s[0] - np.sum(q * dV)) <= 1e-13 * abs(s[0])
    assert abs(s[1] - np.sum(4.0 * q * (1.0 - q) * dV)) <= 1e-13 * abs(s[1])
    target = torch.tensor([s[0] * 1.001], dtype=torch.float64, device="cuda")
    out = torch.empty_like(tq)
    _lib.check(lib.tpf_mass_correction_apply(q.size, _lib.dptr(tq), _lib.dptr(target), _lib.dptr(sums),
                                             _lib.dptr(out), _lib.TPF_F64, st))
    ref = oa.mass_correction(q, dV, s[0] * 1.001)
    assert np.abs(out.cpu().numpy() - ref).max() <= 1e-15
    z = torch.zeros_like(tq)
    _lib.check(lib.tpf_mass_sums(q.size, _lib.dptr(z), _lib.dptr(tv), _lib.dptr(part), _lib.dptr(sums),
                                 _lib.TPF_F64, st))
    _lib.check(lib.tpf_mass_correction_apply(q.size, _lib.dptr(z), _lib.dptr(target), _lib.dptr(sums),
                                             _lib.dptr(out), _lib.TPF_F64, st))
    assert float(out.abs().max()) == 0.0


@pytest.mark.parametrize("name", CASES)
def test_uccd6_matches_reference(cuda_device, golden, name):
    """Within the CCD chain's rounding (the oracle moves by ~2e-15 relative for
    1e-15 input noise)."""
    from twophaseflow_b200 import CCDSolver, UCCD6ConvectionTerm, UniformGrid
    N = tuple(int(n) for n in golden[f"{name}/N"])
    L = tuple(float(x) for x in golden[f"{name}/L"])
    grid = UniformGrid(N, L)
    ccd = CCDSolver(grid, None, bc_type=str(golden[f"{name}/bc"]))
    vel = [golden[f"{name}/u{a}"] for a in range(len(N))]
    u = UCCD6ConvectionTerm(None, grid, ccd, sigma=1.0e-3).compute(vel)
    for a in range(len(N)):
        ref = golden[f"{name}/uccd6_{a}"]
        assert isinstance(u[a], np.ndarray)
        assert np.abs(u[a] - ref).max() <= TOL * np.abs(ref).max()


def test_uccd6_accumulate_kernel_bit_exact(cuda_device):
    import torch
    from twophaseflow_b200 import _lib
    rng = np.random.default_rng(71)
    shape = (257, 129, 65)
    uk, d1, cons, d8, acc0 = (rng.standard_normal(shape) for _ in range(5))
    T = [torch.from_numpy(a).cuda() for a in (uk, d1, cons, d8)]
    ur = torch.tensor([float(np.abs(uk).max())], dtype=torch.float64, device="cuda")
    lib = _lib.load()
    for first in (1, 0):
        acc = torch.from_numpy(acc0.copy()).cuda()
        _lib.check(lib.tpf_uccd6_accumulate(uk.size, first, *[_lib.dptr(t) for t in T], 3.7e-9, _lib.dptr(ur),
                                            _lib.dptr(acc), _lib.TPF_F64, _lib.current_stream_handle()))
        a = (np.zeros(shape) if first else acc0) - 0.5 * (uk * d1 + cons)
        a = a - 3.7e-9 * (np.abs(uk).max() * d8)
        np.testing.assert_array_equal(acc.cpu().numpy(), a)


def test_fccd_nonuniform_grid_matches_reference(cuda_device):
    """Flux and node forms, node gradients and one RK3 step of each on the
    reference's interface-fitted 32^2 wall grid (cell widths 0.024..0.049;
    tests/golden/fccd_nonuniform_golden.npz): the reference's per-face and
    per-node weights, the CCD second derivatives with the grid metric."""
    from types import SimpleNamespace
    from twophaseflow_b200 import CCDSolver, FCCDLevelSetAdvection, FCCDSolver
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "fccd_nonuniform_golden.npz"))
    N = tuple(int(n) for n in g["N"])
    grid = SimpleNamespace(N=N, ndim=2, L=(1.0, 1.0), shape=tuple(n + 1 for n in N), uniform=False,
                           J=[g["J0"], g["J1"]], dJ_dxi=[g["dJ0"], g["dJ1"]], coords=[g["coords0"], g["coords1"]])
    fccd = FCCDSolver(grid, None, bc_type="wall", ccd_solver=CCDSolver(grid, None, bc_type="wall"))
    vel, psi = [g["u0"], g["u1"]], g["psi"]

    def close(a, ref, tol=TOL):
        assert np.abs(a - ref).max() <= tol * np.abs(ref).max(), np.abs(a - ref).max() / np.abs(ref).max()

    for a in range(2):
        close(fccd.node_gradient(psi, a), g[f"node_grad_psi{a}"])
    for mode in ("flux", "node"):
        close(fccd.advection_rhs(vel, scalar=psi, mode=mode)[0], g[f"rhs_scalar_{mode}"])
        mom = fccd.advection_rhs(vel, mode=mode)
        for a in range(2):
            close(mom[a], g[f"rhs_mom_{mode}{a}"])
        out = FCCDLevelSetAdvection(None, grid, fccd, mode=mode).advance(psi.copy(), vel, 0.004)
        assert np.abs(out - g[f"psi_new_{mode}"]).max() <= 1e-11
    with pytest.raises(NotImplementedError, match="wall axes"):
        FCCDSolver(grid, None, bc_type="periodic")


@pytest.mark.parametrize("tag,bc,mass", [("zero_mass", "zero", True), ("neumann", "neumann", False)])
def test_reinit_nonuniform_grid_matches_reference(cuda_device, tag, bc, mass):
    """Split reinitialization on the reference's interface-fitted 32^2 wall
    grid (tests/golden/reinit_nonuniform_golden.npz): dtau from the smallest
    node spacing equal bit for bit, the result within the uniform reinit bar."""
    from types import SimpleNamespace
    from twophaseflow_b200 import CCDSolver, SplitReinitializer
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "reinit_nonuniform_golden.npz"))
    N = tuple(int(n) for n in g["N"])
    grid = SimpleNamespace(N=N, ndim=2, L=(1.0, 1.0), shape=tuple(n + 1 for n in N), uniform=False,
                           J=[g["J0"], g["J1"]], dJ_dxi=[g["dJ0"], g["dJ1"]], coords=[g["coords0"], g["coords1"]],
                           h=[g["h0"], g["h1"]])
    ccd = CCDSolver(grid, None, bc_type="wall")
    r = SplitReinitializer(None, grid, ccd, float(g["eps"]), n_steps=3, bc=bc, mass_correction=mass)
    assert r.dtau == float(g[f"{tag}/dtau"])
    out = r.reinitialize(g["psi"].copy())
    assert np.abs(out - g[f"{tag}/psi_reinit"]).max() <= 1e-11, np.abs(out - g[f"{tag}/psi_reinit"]).max()
