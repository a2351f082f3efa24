"""CCD parity on the GPU: the CUDA line kernels against the reference's own
outputs (golden fixtures) and the CPU oracle.

Tolerances: FP64 results within 1e-12 of the oracle relative to the field's
max magnitude (the reference's pivoted dense LU and the block-Thomas chunked
solve differ only by round-off); FP32 within 2e-5 relative.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import ccd as occd
from twophaseflow_b200.workloads import fourier_field

pytestmark = pytest.mark.gpu

FP64_RTOL = 1e-12
FP32_RTOL = 2e-5


class _Grid:
    def __init__(self, N, L, uniform=True, J=None, dJ=None, coords=None):
        self.N = tuple(int(n) for n in N)
        self.ndim = len(self.N)
        self.L = tuple(float(v) for v in L)
        self.shape = tuple(n + 1 for n in self.N)
        self.uniform = uniform
        self.J = J
        self.dJ_dxi = dJ
        self.coords = coords if coords is not None else [np.linspace(0, l, n + 1) for n, l in zip(self.N, self.L)]


def _close(a, b, rtol, closure=0.0):
    """max|a-b| <= rtol * max|b| + closure.  ``closure`` is the round-off that
    the wall closure's own sum carries in any implementation (see _closure_atol)."""
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    err = np.abs(a - b).max()
    assert err <= rtol * scale + closure, f"max err {err:.3e} > {rtol:.1e} * {scale:.3e} + {closure:.3e}"


def _closure_atol(f, h, order):
    """Round-off bound of the one-sided wall closure c . f (ccd_solver.py:429-432):
    8 eps * max|f| * sum|c|, with sum|c_I| = 10.58/h and sum|c_II| = 640/(12 h^2).
    The reference's own dense-LU and dense-inverse paths differ by up to this much."""
    eps = np.finfo(np.float64).eps
    s = 10.58 / h if order == 1 else 640.0 / (12.0 * h * h)
    return 8.0 * eps * float(np.abs(np.asarray(f)).max()) * s


CASES = [("wall2d", "wall"), ("wall3d", "wall"), ("wall2d_big", "wall"), ("per2d", "periodic"),
         ("per3d", "periodic")]


@pytest.mark.parametrize("name,bc", CASES)
def test_ccd_matches_reference_golden(cuda_device, ccd_golden, name, bc):
    import torch
    from twophaseflow_b200 import CCDSolver
    g = ccd_golden
    grid = _Grid(g[f"{name}/N"], g[f"{name}/L"])
    ccd = CCDSolver(grid, None, bc_type=bc)
    f = torch.from_numpy(g[f"{name}/f"]).to(cuda_device)
    for ax in range(grid.ndim):
        d1, d2 = ccd.differentiate(f, ax)
        _close(d1.cpu().numpy(), g[f"{name}/d1_ax{ax}"], FP64_RTOL)
        _close(d2.cpu().numpy(), g[f"{name}/d2_ax{ax}"], FP64_RTOL)
        _close(ccd.first_derivative(f, ax).cpu().numpy(), g[f"{name}/first_ax{ax}"], FP64_RTOL)
        _close(ccd.second_derivative(f, ax).cpu().numpy(), g[f"{name}/second_ax{ax}"], FP64_RTOL)


@pytest.mark.parametrize("name", ["wall2d", "wall3d", "wall2d_big"])
def test_ccd_bc_override(cuda_device, ccd_golden, name):
    from twophaseflow_b200 import CCDSolver
    g = ccd_golden
    grid = _Grid(g[f"{name}/N"], g[f"{name}/L"])
    ccd = CCDSolver(grid, None, bc_type="wall")
    d1, d2 = ccd.differentiate(g[f"{name}/f"], 0, bc_left=(0.3, -1.2), bc_right=(0.0, 2.5))
    assert isinstance(d1, np.ndarray)   # NumPy in -> NumPy out
    _close(d1, g[f"{name}/bcov_d1"], FP64_RTOL)
    _close(d2, g[f"{name}/bcov_d2"], FP64_RTOL)
    # one-sided override: the other side keeps the compact closure
    h = float(g[f"{name}/L"][0]) / float(g[f"{name}/N"][0])
    o1, o2 = occd.differentiate(g[f"{name}/f"], 0, h, bc_left=(0.3, -1.2))
    d1, d2 = ccd.differentiate(g[f"{name}/f"], 0, bc_left=(0.3, -1.2))
    _close(d1, o1, FP64_RTOL)
    _close(d2, o2, FP64_RTOL)


@pytest.mark.parametrize("bc", ["wall", "periodic"])
def test_ccd_sin_reference_case(cuda_device, ccd_golden, bc):
    from twophaseflow_b200 import CCDSolver
    g = ccd_golden
    grid = _Grid((32, 4), (1.0, 1.0))
    ccd = CCDSolver(grid, None, bc_type=bc)
    d1, d2 = ccd.differentiate(g[f"sin_{bc}/f"], 0)
    _close(d1, g[f"sin_{bc}/d1"], FP64_RTOL)
    _close(d2, g[f"sin_{bc}/d2"], FP64_RTOL)
    if bc == "periodic":
        # image node equals node 0 (test_ccd.py:65-81)
        np.testing.assert_allclose(d1[-1], d1[0], atol=1e-12)


def test_ccd_nonuniform_metric(cuda_device, ccd_golden):
    from twophaseflow_b200 import CCDSolver
    g = ccd_golden
    J = [g["nonuni/J0"], g["nonuni/J1"]]
    dJ = [g["nonuni/dJ0"], g["nonuni/dJ1"]]
    grid = _Grid((32, 32), (1.0, 1.0), uniform=False, J=J, dJ=dJ,
                 coords=[g["nonuni/coords0"], g["nonuni/coords1"]])
    ccd = CCDSolver(grid, None, bc_type="wall")
    f = g["nonuni/f"]
    for ax in range(2):
        d1, d2 = ccd.differentiate(f, ax)
        _close(d1, g[f"nonuni/d1_ax{ax}"], 1e-11)
        _close(d2, g[f"nonuni/d2_ax{ax}"], 1e-11)
        _close(ccd.first_derivative(f, ax), g[f"nonuni/first_ax{ax}"], 1e-11)
        _close(ccd.second_derivative(f, ax), g[f"nonuni/second_ax{ax}"], 1e-11)
        r1, r2 = ccd.differentiate(f, ax, apply_metric=False)
        _close(r1, g[f"nonuni/raw_d1_ax{ax}"], FP64_RTOL)
        _close(r2, g[f"nonuni/raw_d2_ax{ax}"], FP64_RTOL)


@pytest.mark.parametrize("n", [6, 7, 9, 17, 33, 34, 65, 100, 129, 257, 300, 1025, 1500])
@pytest.mark.parametrize("bc", ["wall", "periodic"])
def test_ccd_line_lengths(cuda_device, n, bc):
    """Ragged lengths around the chunk size, single-chunk and many-chunk lines,
    batches that are not a multiple of the CTA's line count."""
    import torch
    from twophaseflow_b200 import CCDSolver
    rng = np.random.default_rng(n)
    for shape, ax in [((n, 4), 0), ((5, n), 1), ((4, n, 7), 1), ((4, 5, n), 2)]:
        N = tuple(s - 1 for s in shape)
        grid = _Grid(N, tuple(1.0 + 0.1 * i for i in range(len(N))))
        ccd = CCDSolver(grid, None, bc_type=bc)
        f = rng.standard_normal(shape)
        h = grid.L[ax] / N[ax]
        o1, o2 = occd.differentiate(f, ax, h, bc=bc)
        d1, d2 = ccd.differentiate(torch.from_numpy(f).to(cuda_device), ax)
        cl = bc == "wall"
        _close(d1.cpu().numpy(), o1, FP64_RTOL, _closure_atol(f, h, 1) if cl else 0.0)
        _close(d2.cpu().numpy(), o2, FP64_RTOL, _closure_atol(f, h, 2) if cl else 0.0)


@pytest.mark.parametrize("bc", ["wall", "periodic"])
def test_ccd_fp32(cuda_device, bc):
    import torch
    from twophaseflow_b200 import CCDSolver
    N = (256, 200)
    grid = _Grid(N, (1.0, 1.0))
    f = fourier_field(N, n_modes=8, kmax=8, seed=3)
    ccd32 = CCDSolver(grid, None, bc_type=bc, dtype=torch.float32)
    f = f.astype(np.float32).astype(np.float64)   # the FP32 input the kernel sees
    for ax in range(2):
        h = 1.0 / N[ax]
        o1, o2 = occd.differentiate(f, ax, h, bc=bc)
        d1, d2 = ccd32.differentiate(torch.from_numpy(f).to(cuda_device), ax)
        assert d1.dtype == torch.float32
        _close(d1.double().cpu().numpy(), o1, FP32_RTOL)
        _close(d2.double().cpu().numpy(), o2, 5 * FP32_RTOL)


def test_ccd_full_size_2d_against_oracle(cuda_device):
    """Workload size: 2-D 1025^2 Fourier field, wall and periodic, both axes."""
    import torch
    from twophaseflow_b200 import CCDSolver
    N = (1024, 1024)
    grid = _Grid(N, (1.0, 1.0))
    f = fourier_field(N, seed=0)
    ft = torch.from_numpy(f).to(cuda_device)
    for bc in ("wall", "periodic"):
        ccd = CCDSolver(grid, None, bc_type=bc)
        for ax in range(2):
            h = 1.0 / 1024
            o1, o2 = occd.differentiate(f, ax, h, bc=bc)
            d1, d2 = ccd.differentiate(ft, ax)
            cl = bc == "wall"
            _close(d1.cpu().numpy(), o1, FP64_RTOL, _closure_atol(f, h, 1) if cl else 0.0)
            _close(d2.cpu().numpy(), o2, FP64_RTOL, _closure_atol(f, h, 2) if cl else 0.0)


def test_ccd_full_size_3d_properties(cuda_device):
    """3-D 257^3: exact derivatives of a low-degree polynomial (the scheme is
    exact for cubics, test_ccd.py:201-252) and axis consistency."""
    import torch
    from twophaseflow_b200 import CCDSolver
    N = (256, 256, 256)
    grid = _Grid(N, (1.0, 1.0, 1.0))
    x = torch.linspace(0, 1, 257, dtype=torch.float64, device=cuda_device)
    X = x.view(-1, 1, 1)
    Y = x.view(1, -1, 1)
    Z = x.view(1, 1, -1)
    f = (X ** 3 * Y ** 2 + Z ** 3).expand(257, 257, 257).contiguous()
    ccd = CCDSolver(grid, None, bc_type="wall")
    d1, d2 = ccd.differentiate(f, 0)
    assert torch.max(torch.abs(d1 - 3 * X ** 2 * Y ** 2)).item() < 1e-9
    assert torch.max(torch.abs(d2 - 6 * X * Y ** 2)).item() < 1e-7
    d1, d2 = ccd.differentiate(f, 2)
    assert torch.max(torch.abs(d1 - 3 * Z ** 2)).item() < 1e-9
    d1, _ = ccd.differentiate(f, 1)
    assert torch.max(torch.abs(d1 - 2 * X ** 3 * Y)).item() < 1e-9


def test_ccd_oracle_3d_slab(cuda_device):
    """3-D wall/periodic against the oracle on a 257 x 40 x 257 slab (all axes)."""
    import torch
    from twophaseflow_b200 import CCDSolver
    N = (256, 39, 256)
    grid = _Grid(N, (1.0, 0.5, 2.0))
    f = fourier_field(N, L=grid.L, n_modes=8, kmax=16, seed=5)
    ft = torch.from_numpy(f).to(cuda_device)
    for bc in ("wall", "periodic"):
        ccd = CCDSolver(grid, None, bc_type=bc)
        for ax in range(3):
            h = grid.L[ax] / N[ax]
            o1, o2 = occd.differentiate(f, ax, h, bc=bc)
            d1, d2 = ccd.differentiate(ft, ax)
            cl = bc == "wall"
            _close(d1.cpu().numpy(), o1, FP64_RTOL, _closure_atol(f, h, 1) if cl else 0.0)
            _close(d2.cpu().numpy(), o2, FP64_RTOL, _closure_atol(f, h, 2) if cl else 0.0)


def test_differentiate_raw_and_neumann(cuda_device):
    import torch
    from twophaseflow_b200 import CCDSolver
    N = (40, 24)
    grid = _Grid(N, (1.0, 1.0))
    ccd = CCDSolver(grid, None, bc_type="wall")
    x = np.linspace(0.0, 1.0, 41) ** 1.3
    d1, d2 = ccd.differentiate_raw(x, 0)
    o1, o2 = occd.differentiate_wall(x[:, None], 0, 1.0 / 40)
    _close(d1, o1[:, 0], FP64_RTOL)
    _close(d2, o2[:, 0], FP64_RTOL)
    gt = torch.ones((41, 25), dtype=torch.float64, device=cuda_device)
    ccd.enforce_wall_neumann(gt, 1)
    assert gt[:, 0].abs().max().item() == 0 and gt[:, -1].abs().max().item() == 0
    assert gt[:, 1:-1].min().item() == 1.0


def test_ccd_rejects_short_wall_axis(cuda_device):
    from twophaseflow_b200 import CCDSolver
    grid = _Grid((4, 4), (1.0, 1.0))
    ccd = CCDSolver(grid, None, bc_type="wall")
    with pytest.raises(ValueError, match="n_pts >= 6"):
        ccd.differentiate(np.zeros(grid.shape), axis=0)


# shapes whose differentiated axis has 131 nodes and >= 19 200 lines, so every
# axis runs on the lane-per-line kernel (strided axes and the contiguous one)
_LANE_SHAPES = {0: (131, 150, 128), 1: (150, 131, 128), 2: (150, 128, 131)}


@pytest.mark.parametrize("bc", ["wall", "periodic"])
@pytest.mark.parametrize("ax", [0, 1, 2])
def test_ccd_lane_kernel_against_oracle(cuda_device, bc, ax):
    """Many-line 3-D fields: d1/d2 and the single-output calls against the oracle."""
    import torch
    from twophaseflow_b200 import CCDSolver
    shape = _LANE_SHAPES[ax]
    N = tuple(s - 1 for s in shape)
    grid = _Grid(N, (1.0, 1.3, 0.7))
    f = fourier_field(N, L=grid.L, n_modes=6, kmax=6, seed=11 + ax)
    ft = torch.from_numpy(f).to(cuda_device)
    ccd = CCDSolver(grid, None, bc_type=bc)
    h = grid.L[ax] / N[ax]
    o1, o2 = occd.differentiate(f, ax, h, bc=bc)
    cl = bc == "wall"
    a1 = _closure_atol(f, h, 1) if cl else 0.0
    a2 = _closure_atol(f, h, 2) if cl else 0.0
    d1, d2 = ccd.differentiate(ft, ax)
    _close(d1.cpu().numpy(), o1, FP64_RTOL, a1)
    _close(d2.cpu().numpy(), o2, FP64_RTOL, a2)
    _close(ccd.first_derivative(ft, ax).cpu().numpy(), o1, FP64_RTOL, a1)
    _close(ccd.second_derivative(ft, ax).cpu().numpy(), o2, FP64_RTOL, a2)


@pytest.mark.parametrize("bc", ["wall", "periodic"])
@pytest.mark.parametrize("ax", [0, 2])
def test_ccd_lane_kernel_fp32(cuda_device, bc, ax):
    import torch
    from twophaseflow_b200 import CCDSolver
    shape = _LANE_SHAPES[ax]
    N = tuple(s - 1 for s in shape)
    grid = _Grid(N, (1.0, 1.0, 1.0))
    f = fourier_field(N, n_modes=6, kmax=6, seed=21 + ax).astype(np.float32).astype(np.float64)
    ccd32 = CCDSolver(grid, None, bc_type=bc, dtype=torch.float32)
    h = 1.0 / N[ax]
    o1, o2 = occd.differentiate(f, ax, h, bc=bc)
    d1, d2 = ccd32.differentiate(torch.from_numpy(f).to(cuda_device), ax)
    _close(d1.double().cpu().numpy(), o1, FP32_RTOL)
    _close(d2.double().cpu().numpy(), o2, 5 * FP32_RTOL)


@pytest.mark.parametrize("ax", [0, 2])
def test_ccd_lane_kernel_metric_and_vd(cuda_device, ax):
    """Non-uniform metric epilogue and the variable-density (L_H) epilogue on
    the lane kernel: against J d1_xi, J^2 d2_xi + J J' d1_xi and against
    d2/rho - (drho/rho^2) d1 built from the raw derivatives."""
    import torch
    from twophaseflow_b200 import CCDSolver
    from twophaseflow_b200.arrays import line_split
    from twophaseflow_b200 import _lib
    shape = _LANE_SHAPES[ax]
    N = tuple(s - 1 for s in shape)
    xi = [np.linspace(0, 1, n + 1) for n in N]
    J = [1.0 + 0.3 * np.cos(2 * np.pi * x) for x in xi]
    dJ = [-0.6 * np.pi * np.sin(2 * np.pi * x) for x in xi]
    grid = _Grid(N, (1.0, 1.0, 1.0), uniform=False, J=J, dJ=dJ)
    f = fourier_field(N, n_modes=5, kmax=5, seed=31 + ax)
    ft = torch.from_numpy(f).to(cuda_device)
    ccd = CCDSolver(grid, None, bc_type="wall")
    r1, r2 = ccd.differentiate(ft, ax, apply_metric=False)
    m1, m2 = ccd.differentiate(ft, ax)
    bshape = [1, 1, 1]
    bshape[ax] = -1
    Jt = torch.from_numpy(J[ax]).to(cuda_device).view(bshape)
    dJt = torch.from_numpy(dJ[ax]).to(cuda_device).view(bshape)
    _close(m1.cpu().numpy(), (Jt * r1).cpu().numpy(), 1e-13)
    _close(m2.cpu().numpy(), (Jt * Jt * r2 + Jt * dJt * r1).cpu().numpy(), 1e-13)
    # variable-density epilogue on the uniform plan
    ccdu = CCDSolver(_Grid(N, (1.0, 1.0, 1.0)), None, bc_type="wall")
    rho = torch.from_numpy(1.5 + np.cos(np.linspace(0, 3, f.size)).reshape(f.shape)).to(cuda_device)
    drho = torch.from_numpy(0.2 * np.sin(np.linspace(0, 5, f.size)).reshape(f.shape)).to(cuda_device)
    u1, u2 = ccdu.differentiate(ft, ax)
    out = torch.empty_like(ft)
    outer, n, inner = line_split(ft.shape, ax)
    plan = ccdu._plan(ax, False)
    _lib.check(ccdu.lib.tpf_ccd_apply_vd(plan, outer, inner, _lib.dptr(ft), _lib.dptr(rho), _lib.dptr(drho),
                                         _lib.dptr(out), 0, 0, _lib.current_stream_handle()))
    ref = u2 / rho - (drho / (rho * rho)) * u1
    _close(out.cpu().numpy(), ref.cpu().numpy(), 1e-13)


@pytest.mark.parametrize("bc", ["wall", "periodic"])
def test_ccd_autotune_is_bitwise_neutral(cuda_device, bc):
    """The launch-shape autotuner (first call per shape) changes only the
    speed: tuned, cached and untuned results are bitwise identical."""
    import torch
    from twophaseflow_b200 import CCDSolver, _lib
    shape = _LANE_SHAPES[0]
    N = tuple(s - 1 for s in shape)
    grid = _Grid(N, (1.0, 1.0, 1.0))
    f = torch.from_numpy(fourier_field(N, n_modes=4, kmax=4, seed=5)).to(cuda_device)
    tuned = CCDSolver(grid, None, bc_type=bc)
    plain = CCDSolver(grid, None, bc_type=bc)
    plan = plain._plan(0, bc == "periodic")
    _lib.check(plain.lib.tpf_ccd_plan_set_autotune(plan, 0))
    a1, a2 = tuned.differentiate(f, 0)      # tunes
    b1, b2 = tuned.differentiate(f, 0)      # cached shape
    c1, c2 = plain.differentiate(f, 0)      # default shape
    assert torch.equal(a1, c1) and torch.equal(a2, c2)
    assert torch.equal(b1, c1) and torch.equal(b2, c2)


@pytest.mark.parametrize("N,bc,axis", [((1024, 600), "wall", 0), ((1024, 600), "periodic", 1),
                                       ((300, 200), "wall", 1), ((200, 64), "periodic", 0)])
def test_ccd_warp_kernel_autotune_is_bitwise_neutral(cuda_device, N, bc, axis):
    """2-D grids (the warp kernel, 1-4 warps per line): the tuned launch shape
    (lines per block, tile buffers), the cached one and the heuristic one give
    bitwise identical derivatives, which match the oracle."""
    import torch
    from twophaseflow_b200 import CCDSolver, UniformGrid, _lib
    f = fourier_field(N, n_modes=6, kmax=6, seed=8)
    ft = torch.from_numpy(f).to(cuda_device)
    tuned = CCDSolver(UniformGrid(N), None, bc_type=bc)
    plain = CCDSolver(UniformGrid(N), None, bc_type=bc)
    plan = plain._plan(axis, bc == "periodic")
    _lib.check(plain.lib.tpf_ccd_plan_set_autotune(plan, 0))
    a1, a2 = tuned.differentiate(ft, axis)
    b1, b2 = tuned.differentiate(ft, axis)
    c1, c2 = plain.differentiate(ft, axis)
    assert torch.equal(a1, c1) and torch.equal(a2, c2)
    assert torch.equal(b1, c1) and torch.equal(b2, c2)
    o1, o2 = occd.differentiate(f, axis, 1.0 / N[axis], bc=bc)
    assert np.abs(c1.cpu().numpy() - o1).max() <= 1e-11 * np.abs(o1).max()
    assert np.abs(c2.cpu().numpy() - o2).max() <= 1e-11 * np.abs(o2).max()


@pytest.mark.parametrize("N,axis", [((128, 96), 0), ((128, 96), 1), ((40, 36, 48), 2), ((40, 36, 48), 0)])
def test_ccd_refined_fp32_reaches_fp64(cuda_device, N, axis):
    """FP32 line solves under FP64 iterative refinement: without refinement the
    error is FP32-level; two refinements bring d1 and d2 to the FP64 solve
    within 1e-12 of max|d| (and the FP64 oracle within the wall bar)."""
    import torch
    from oracle import ccd as occd
    from twophaseflow_b200 import CCDSolver, UniformGrid
    from twophaseflow_b200.workloads import fourier_field
    f = fourier_field(N, n_modes=16, kmax=12, seed=3)
    ft = torch.from_numpy(f).to(cuda_device)
    ccd = CCDSolver(UniformGrid(N), None, bc_type="wall")
    d1, d2 = ccd.differentiate(ft, axis)
    errs = []
    for r in (0, 1, 2):
        a1, a2 = ccd.differentiate_refined(ft, axis, r)
        errs.append((float((a1 - d1).abs().max() / d1.abs().max()), float((a2 - d2).abs().max() / d2.abs().max())))
    assert max(errs[0]) > 1e-9          # FP32 alone
    assert errs[1][0] < errs[0][0] and errs[1][1] < errs[0][1]
    assert max(errs[2]) <= 1e-12, errs
    o1, o2 = occd.differentiate(f, axis, 1.0 / N[axis])
    a1, a2 = ccd.differentiate_refined(f, axis, 2)
    assert np.abs(a1 - o1).max() <= 1e-11 * np.abs(o1).max()
    assert np.abs(a2 - o2).max() <= 1e-11 * np.abs(o2).max()


def test_ccd_refined_rejects_periodic(cuda_device):
    from twophaseflow_b200 import CCDSolver, UniformGrid
    ccd = CCDSolver(UniformGrid((32, 32)), None, bc_type="periodic")
    with pytest.raises(NotImplementedError):
        ccd.differentiate_refined(np.zeros((33, 33)), 0)
