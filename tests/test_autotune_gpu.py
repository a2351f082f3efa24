"""Launch-shape autotuning of the stencil kernels (tpf_set_launch_autotune):
every candidate shape the tuner may pick -- nodes per thread of the CLS flux
and Rhie-Chow march kernels, threads per block of the reinitialization's CN
line solves -- gives bit-for-bit the output of the heuristic shape, on the
march axes (strided) of 3-D grids and on 2-D grids; tuning caches one choice
per signature and stays out of stream capture."""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MODES = [0, 2, 3, 4, 5, 6, 1]   # heuristic, each forced candidate, tuned


@pytest.fixture
def tune_mode():
    from twophaseflow_b200 import _lib
    lib = _lib.load()
    yield lambda m: _lib.check(lib.tpf_set_launch_autotune(m))
    _lib.check(lib.tpf_set_launch_autotune(1))


def _flux_and_cn(shape, periodic):
    import torch
    from twophaseflow_b200 import _lib
    lib = _lib.load()
    st = _lib.current_stream_handle()
    rng = np.random.default_rng(5)
    nd = len(shape)
    sh = (C.c_int64 * nd)(*shape)
    P = torch.from_numpy(rng.standard_normal(shape)).cuda()
    Q = torch.from_numpy(rng.standard_normal(shape)).cuda()
    acc = torch.empty_like(P)
    for ax in range(nd):
        _lib.check(lib.tpf_fccd_flux_divergence_axis(nd, sh, ax, int(periodic), 1.0 / shape[ax], _lib.dptr(P),
                                                     _lib.dptr(Q), 1 if ax else 0, _lib.dptr(acc), _lib.TPF_F64, st))
    outs = [acc.clone()]
    for ax in range(nd):
        n = shape[ax]
        f = torch.from_numpy(rng.uniform(0.1, 0.2, n - 1)).cuda()
        m = torch.from_numpy(rng.uniform(1.5, 2.0, n)).cuda()
        sup = torch.from_numpy(rng.uniform(-0.3, -0.2, n - 1)).cuda()
        out = torch.empty_like(P)
        _lib.check(lib.tpf_reinit_cn_axis(nd, sh, ax, 0.3, 0.4, _lib.dptr(f), _lib.dptr(m), _lib.dptr(sup),
                                          _lib.dptr(P), _lib.dptr(out), _lib.TPF_F64, st))
        torch.cuda.synchronize()
        outs.append(out)
    return [o.cpu().numpy() for o in outs]


def _rhie_chow(N):
    import torch
    from twophaseflow_b200 import CCDSolver, RhieChowInterpolator, UniformGrid
    grid = UniformGrid(N)
    ccd = CCDSolver(grid, None, bc_type="wall")
    rng = np.random.default_rng(9)
    shape = grid.shape
    vel = [torch.from_numpy(rng.standard_normal(shape)).cuda() for _ in N]
    p = torch.from_numpy(rng.standard_normal(shape)).cuda()
    rho = torch.from_numpy(rng.uniform(0.1, 1.0, shape)).cuda()
    kappa = torch.from_numpy(rng.standard_normal(shape)).cuda()
    psi = torch.from_numpy(rng.uniform(0.0, 1.0, shape)).cuda()
    rc = RhieChowInterpolator(None, grid, ccd, bc_type="wall")
    a = rc.face_velocity_divergence(vel, p, rho, 1e-3)
    b = rc.face_velocity_divergence(vel, p, rho, 1e-3, kappa=kappa, psi=psi, we=10.0)
    return [a.cpu().numpy(), b.cpu().numpy()]


@pytest.mark.parametrize("shape,periodic", [((40, 36, 48), False), ((33, 70, 41), True), ((513, 257), False)])
def test_every_candidate_shape_gives_the_same_bits(cuda_device, tune_mode, shape, periodic):
    res = {}
    for m in MODES:
        tune_mode(m)
        res[m] = _flux_and_cn(shape, periodic)
    for m in MODES[1:]:
        for a, b in zip(res[0], res[m]):
            np.testing.assert_array_equal(a, b, err_msg=f"mode {m}")


def test_rhie_chow_every_candidate_gives_the_same_bits(cuda_device, tune_mode):
    res = {}
    for m in MODES:
        tune_mode(m)
        res[m] = _rhie_chow((40, 36, 48))
    for m in MODES[1:]:
        for a, b in zip(res[0], res[m]):
            np.testing.assert_array_equal(a, b, err_msg=f"mode {m}")


def test_tuning_caches_per_signature_and_skips_capture(cuda_device, tune_mode):
    import torch
    from twophaseflow_b200 import _lib
    lib = _lib.load()
    tune_mode(0)
    tune_mode(1)
    assert lib.tpf_launch_autotune_entries() == 0
    _flux_and_cn((40, 36, 48), False)
    n1 = lib.tpf_launch_autotune_entries()
    assert n1 == 4          # flux march and CN lines on the two strided axes
    _flux_and_cn((40, 36, 48), False)
    assert lib.tpf_launch_autotune_entries() == n1   # cached
    # a new signature under stream capture is not tuned (the heuristic runs)
    shape = (24, 28, 36)
    sh = (C.c_int64 * 3)(*shape)
    P = torch.randn(shape, dtype=torch.float64, device="cuda")
    acc = torch.empty_like(P)
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            _lib.check(lib.tpf_fccd_flux_divergence_axis(3, sh, 0, 0, 0.1, _lib.dptr(P), _lib.dptr(P), 0,
                                                         _lib.dptr(acc), _lib.TPF_F64, _lib.current_stream_handle()))
    torch.cuda.current_stream().wait_stream(s)
    g.replay()
    torch.cuda.synchronize()
    assert lib.tpf_launch_autotune_entries() == n1
    with pytest.raises(ValueError):
        _lib.check(lib.tpf_set_launch_autotune(-1))
