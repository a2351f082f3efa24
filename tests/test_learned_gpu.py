"""GPU tests of the learned preconditioner: the tcgen05 U-Net forward/backward
against the NumPy oracle, training, and the network-preconditioned flexible CG
against the direct solution of the same PPE."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import ppe as oppe
from oracle import unet as ou

pytestmark = pytest.mark.gpu

# BF16 activations are rounded at every layer; GPU (FP32 sums) and oracle
# (float64 sums) round a few values to neighbouring BF16 numbers, so outputs
# and gradients agree to about 1e-2 of their magnitude.
FWD_TOL = 3e-2


def _net(H, W, B, params):
    from twophaseflow_b200.learned import UNet
    return UNet(H, W, B, params=params)


@pytest.mark.parametrize("H,W,B", [(16, 16, 2), (24, 40, 1)])
def test_unet_forward_matches_oracle(cuda_device, H, W, B):
    import torch
    rng = np.random.default_rng(7)
    p = ou.init_params(seed=2)
    p[ou.param_layout()[0][3][1]:ou.param_layout()[0][3][1] + 32] = 0.05  # nonzero biases somewhere
    x = rng.standard_normal((B, H, W, 4)).astype(np.float32)
    net = _net(H, W, B, p)
    y = net.forward(torch.from_numpy(x).to(cuda_device)).cpu().numpy()
    yo, _ = ou.forward(p, x, precision="bf16")
    scale = np.abs(yo).max()
    assert scale > 0
    err = np.abs(y - yo).max() / scale
    assert err < FWD_TOL, err
    assert np.abs(y - yo).mean() / np.abs(yo).mean() < 1e-2


@pytest.mark.parametrize("H,W,B", [(136, 136, 1), (64, 48, 3), (16, 16, 2), (8, 8, 1)])
def test_persistent_forward_matches_layered(cuda_device, H, W, B):
    """The one-launch forward (grid barriers, output channels split over
    CTAs, fused 1x1 output) gives the layered forward's outputs bit for bit:
    every output element sees the same MMA sequence, only the MMA width
    differs."""
    import torch
    rng = np.random.default_rng(5)
    p = ou.init_params(seed=4)
    offs = ou.param_layout()[0]
    for l in (0, 6, 8, 13):
        p[offs[l][1]:offs[l][1] + ou.LAYERS[l][1]] = rng.uniform(-0.1, 0.1, ou.LAYERS[l][1])
    x = torch.from_numpy(rng.standard_normal((B, H, W, 4)).astype(np.float32)).to(cuda_device)
    net = _net(H, W, B, p)
    net.set_forward_mode(0)
    y0 = net.forward(x)
    net.set_forward_mode(1)
    y1 = net.forward(x)
    y1b = net.forward(x)
    assert torch.equal(y1, y1b)
    assert float(y0.abs().max()) > 0
    assert torch.equal(y0, y1), float((y0 - y1).abs().max())
    # backward after a persistent forward uses the activations it stored
    dy = torch.from_numpy(rng.standard_normal((B, H, W)).astype(np.float32)).to(cuda_device)
    g1 = net.backward(dy).clone()
    net.set_forward_mode(0)
    net.forward(x)
    g0 = net.backward(dy)
    # weight gradients accumulate with atomics: equal up to summation order
    assert float((g0 - g1).norm() / g0.norm()) < 1e-5


def _layer_rel(g, ref):
    offs, wo, bo, _ = ou.param_layout()
    segs = [(w, b + ou.LAYERS[l][1]) for l, (w, b) in enumerate(offs)] + [(wo, bo + 1)]
    out = []
    for a, b in segs:
        nrm = np.linalg.norm(ref[a:b])
        out.append(np.linalg.norm(g[a:b] - ref[a:b]) / nrm if nrm > 0 else np.linalg.norm(g[a:b]))
    return np.array(out)


def test_unet_backward_matches_oracle(cuda_device):
    """GPU gradients vs the BF16 oracle, measured against the oracle's own
    sensitivity: BF16 storage makes the gradients chaotic (a 1e-6 relative
    change of the parameters already moves them by several percent), so the
    bar per layer is a multiple of that measured sensitivity, plus a cosine
    check that catches any systematic error."""
    import torch
    rng = np.random.default_rng(11)
    H, W, B = 16, 24, 2
    p = ou.init_params(seed=5)
    x = rng.standard_normal((B, H, W, 4)).astype(np.float32)
    dy = rng.standard_normal((B, H, W)).astype(np.float32)
    net = _net(H, W, B, p)
    net.forward(torch.from_numpy(x).to(cuda_device))
    g = net.backward(torch.from_numpy(dy).to(cuda_device)).cpu().numpy().astype(np.float64)
    _, A = ou.forward(p, x, precision="bf16")
    go = ou.backward(p, A, dy, precision="bf16")
    p2 = (p * (1.0 + 1e-6 * rng.standard_normal(p.shape))).astype(np.float32)
    _, A2 = ou.forward(p2, x, precision="bf16")
    sens = _layer_rel(ou.backward(p2, A2, dy, precision="bf16"), go)
    rels = _layer_rel(g, go)
    assert np.all(rels <= 3.0 * np.maximum(sens, 2e-2)), (rels, sens)
    offs, wo, bo, _ = ou.param_layout()
    cos = g @ go / (np.linalg.norm(g) * np.linalg.norm(go))
    assert cos > 0.995, cos


def test_train_step_reduces_loss(cuda_device):
    import torch
    from twophaseflow_b200.learned import UNet
    rng = np.random.default_rng(0)
    H = W = 32
    B = 4
    x = rng.standard_normal((B, H, W, 4)).astype(np.float32)
    # target: a smooth function of the first input channel
    t = np.cumsum(np.cumsum(x[..., 0], axis=1), axis=2) / 32.0
    net = UNet(H, W, B, seed=3)
    xt = torch.from_numpy(x).to(cuda_device)
    tt = torch.from_numpy(t.astype(np.float32)).to(cuda_device)
    losses = [net.train_step(xt, tt, 1e-3) for _ in range(60)]
    assert np.isfinite(losses).all()
    assert losses[-1] < 0.5 * losses[0], (losses[0], losses[-1])
    # the loss matches the oracle's on the updated parameters
    p = net.get_params()
    y = net.forward(xt).cpu().numpy()
    L_gpu, _ = ou.loss(y, t)
    yo, _ = ou.forward(p, x, precision="bf16")
    L_or, _ = ou.loss(yo, t)
    assert abs(L_gpu - L_or) < 0.05 * L_or + 1e-3


class _Cfg:
    def __init__(self, **kw):
        self.__dict__.update(kw)


def _case(N, seed, ratio=1000.0):
    from twophaseflow_b200.workloads import divergence_rhs, droplet_density
    rho = droplet_density(N, n_drops=6, rho_l=1.0, rho_g=1.0 / ratio, seed=seed)
    rhs = divergence_rhs(N, seed=seed + 1)
    return rho, rhs


@pytest.mark.parametrize("smooth,coarsen", [(1, 1), (2, 1), (1, 4)])
def test_flexible_cg_matches_direct_solution(cuda_device, smooth, coarsen):
    """With all-zero network parameters the preconditioner reduces to damped
    Jacobi sweeps (a fixed SPD map), so the flexible CG must converge like
    PCG: this checks the FCG recurrences, the pinning and the true-residual
    exit independently of training."""
    import torch
    from twophaseflow_b200 import UniformGrid
    from twophaseflow_b200.learned import PPESolverLearned, num_params
    N = (64, 64)
    rho, rhs = _case(N, seed=3)
    cfg = _Cfg(pseudo_tol=1e-10, pseudo_maxiter=4000, ppe_learned_smooth=smooth, ppe_learned_fallback=False,
               ppe_learned_coarsen=coarsen, ppe_learned_outer="fcg")
    s = PPESolverLearned(None, cfg, UniformGrid(N), params=np.zeros(num_params(), np.float32))
    p = s.solve(torch.from_numpy(rhs).to(cuda_device), torch.from_numpy(rho).to(cuda_device)).cpu().numpy()
    d = s.last_diagnostics
    assert d["ppe_learned_info"] == 0 and not d["ppe_learned_fell_back"]
    assert d["ppe_learned_relative_residual"] <= 1e-10
    pd = oppe.spsolve_fvm(rhs, rho, oppe.uniform_coords(N, (1.0, 1.0)))
    assert np.abs(p - pd).max() <= 1e-7 * np.abs(pd).max()
    pin = s._pin_dof
    assert p.ravel()[pin] == 0.0


@pytest.mark.parametrize("outer", ["fcg", "fgmres"])
def test_learned_solve_falls_back_to_pcg_on_stall(cuda_device, outer):
    import torch
    from twophaseflow_b200 import UniformGrid
    from twophaseflow_b200.learned import PPESolverLearned
    N = (48, 48)
    rho, rhs = _case(N, seed=5)
    # an all-zero network without smoothing gives z = 0: no progress -> fallback
    from twophaseflow_b200.learned import num_params
    cfg = _Cfg(pseudo_tol=1e-9, pseudo_maxiter=400, ppe_learned_smooth=0, ppe_learned_maxiter=400,
               ppe_learned_coarsen=1, ppe_learned_outer=outer)
    s = PPESolverLearned(None, cfg, UniformGrid(N), params=np.zeros(num_params(), np.float32))
    p = s.solve(torch.from_numpy(rhs).to(cuda_device), torch.from_numpy(rho).to(cuda_device)).cpu().numpy()
    d = s.last_diagnostics
    assert d["ppe_learned_fell_back"] and d["ppe_learned_info"] == 0
    pd = oppe.spsolve_fvm(rhs, rho, oppe.uniform_coords(N, (1.0, 1.0)))
    assert np.abs(p - pd).max() <= 1e-6 * np.abs(pd).max()


def test_pairs_are_consistent(cuda_device):
    """in2 channel 0 is D^-1/2 S e / s and target is D^1/2 e / s for the same s."""
    import torch
    from twophaseflow_b200.learned import generate_pairs
    in2, tgt = generate_pairs(N=(32, 32), n_cases=2, snapshots=(0, 5), seed=1, coarsen=1)
    assert in2.shape == (4, 40, 40, 4) and tgt.shape == (4, 40, 40)
    a = in2.cpu().numpy()
    t = tgt.cpu().numpy()
    assert np.isfinite(a).all() and np.isfinite(t).all()
    # scaled residual has unit RMS over the grid nodes; padding is zero
    rms = np.sqrt((a[:, :33, :33, 0] ** 2).mean(axis=(1, 2)))
    assert np.allclose(rms, 1.0, rtol=1e-4)
    assert np.all(a[:, 33:, :, :] == 0) and np.all(t[:, :, 33:] == 0)
    assert np.all((a[..., 1] >= 0) & (a[..., 1] <= 1))


def test_two_level_pairs(cuda_device):
    """Two-level pairs: coarse image of ceil(33/4) = 9 aggregates (padded to 16),
    unit-RMS scaled restricted residual, zero padding."""
    from twophaseflow_b200.learned import generate_pairs
    in2, tgt = generate_pairs(N=(32, 32), n_cases=2, snapshots=(0, 5), seed=1, coarsen=4)
    assert in2.shape == (4, 16, 16, 4) and tgt.shape == (4, 16, 16)
    a = in2.cpu().numpy()
    t = tgt.cpu().numpy()
    assert np.isfinite(a).all() and np.isfinite(t).all()
    rms = np.sqrt((a[:, :9, :9, 0] ** 2).mean(axis=(1, 2)))
    assert np.allclose(rms, 1.0, rtol=1e-4)
    assert np.all(a[:, 9:, :, :] == 0) and np.all(t[:, :, 9:] == 0)


def test_energy_pairs_and_loss(cuda_device):
    """Energy-loss data: a zero network leaves the whole error (loss exactly 1);
    a few training steps reduce the A-norm error left by the coarse correction."""
    import torch
    from twophaseflow_b200.learned import UNet, generate_pairs, net_image, num_params
    N = (64, 64)
    in2, coupl, esc = generate_pairs(N=N, n_cases=3, snapshots=(0, 20, 80), seed=2, coarsen=4, energy=True)
    H, W = net_image((65, 65), 4)
    assert in2.shape == (9, H, W, 4) and coupl.shape == (9, H, W, 2) and esc.shape == (9,)
    # the coupling input channels are the energy loss's couplings
    assert torch.equal(in2[..., 2:], coupl)
    assert torch.all(esc > 0)
    c = coupl.cpu().numpy()
    assert np.all(c >= 0) and np.all(c[:, 17:, :, :] == 0)
    net = UNet(H, W, 9, params=np.zeros(num_params(), np.float32))
    l0 = net.train_step_energy(in2, coupl, esc, 17, 17, 0.0)
    assert abs(l0 - 1.0) < 1e-6, l0
    net = UNet(H, W, 9, seed=4)
    losses = [net.train_step_energy(in2, coupl, esc, 17, 17, 1e-3) for _ in range(40)]
    assert np.isfinite(losses).all() and losses[-1] < min(1.0, losses[0]), (losses[0], losses[-1])


@pytest.mark.parametrize("outer,smooth,bar", [("fcg", 3, 2.5), ("fgmres", 16, 1.5)])
def test_trained_network_gain(cuda_device, outer, smooth, bar):
    """The shipped network (trained on 512^2 solver pairs, energy loss) against
    the same two-level method without it (all-zero network: the Jacobi
    two-grid cycle with no coarse correction) on a held-out 256^2 density at
    ratio 1000: flexible CG with 3 sweeps needs at least 2.5x fewer iterations
    with the network (about 3x measured), the default flexible GMRES(60) with
    16 sweeps at least 1.5x; same solution."""
    import torch
    from twophaseflow_b200 import UniformGrid
    from twophaseflow_b200.learned import PPESolverLearned, load_params, num_params
    from twophaseflow_b200.workloads import divergence_rhs, droplet_density
    N = (256, 256)
    rho = torch.from_numpy(droplet_density(N, seed=101)).to(cuda_device)
    rhs = torch.from_numpy(divergence_rhs(N, seed=102)).to(cuda_device)
    cfg = _Cfg(pseudo_tol=1e-8, pseudo_maxiter=5000, ppe_learned_maxiter=5000, ppe_learned_fallback=False,
               ppe_learned_outer=outer, ppe_learned_smooth=smooth)
    its = {}
    sol = {}
    for name, params in (("trained", load_params()), ("none", np.zeros(num_params(), np.float32))):
        s = PPESolverLearned(None, cfg, UniformGrid(N), params=params)
        sol[name] = s.solve(rhs, rho).cpu().numpy()
        d = s.last_diagnostics
        assert d["ppe_learned_info"] == 0 and not d["ppe_learned_fell_back"]
        its[name] = d["ppe_learned_iterations"]
    print(outer, smooth, its)
    assert its["trained"] * bar <= its["none"], its
    scale = np.abs(sol["none"]).max()
    assert np.abs(sol["trained"] - sol["none"]).max() <= 1e-6 * scale


def test_learned_solve_is_deterministic(cuda_device):
    """Repeated solves (eager first chunk, then graph replays) are bitwise
    identical: every reduction and the coarse-operator assembly run in a fixed
    order, so the BF16 network sees the same inputs each time."""
    import torch
    from twophaseflow_b200 import UniformGrid
    from twophaseflow_b200.learned import PPESolverLearned
    N = (128, 128)
    rho = torch.from_numpy(_case(N, seed=9)[0]).to(cuda_device)
    rhs = torch.from_numpy(_case(N, seed=9)[1]).to(cuda_device)
    s = PPESolverLearned(None, _Cfg(pseudo_tol=1e-8, pseudo_maxiter=5000, ppe_learned_fallback=False), UniformGrid(N))
    p1 = s.solve(rhs, rho)
    it1 = s.last_diagnostics["ppe_learned_iterations"]
    p2 = s.solve(rhs, rho)
    it2 = s.last_diagnostics["ppe_learned_iterations"]
    assert it1 == it2
    assert torch.equal(p1, p2)


@pytest.mark.parametrize("N,ratio,smooth,restart", [((11, 11), 1000.0, 1, 128), ((32, 32), 10.0, 2, 30),
                                                     ((24, 20), 10.0, 1, 7)])
def test_flexible_gmres_matches_direct_solution(cuda_device, N, ratio, smooth, restart):
    """ppe_learned_outer='fgmres': with all-zero network parameters the
    preconditioner is damped Jacobi (a fixed map), so flexible GMRES is
    Jacobi-GMRES: without restarts (144 unknowns, restart 128 plus one
    restart) it reaches the tolerance within the system size even at density
    ratio 1000; restarted (30, 7) on milder systems it converges too (at
    ratio 1000 restarted Jacobi-GMRES stalls, as the reference's does).
    Checked on the true residual and against the direct solution."""
    import torch
    from twophaseflow_b200 import UniformGrid
    from twophaseflow_b200.learned import PPESolverLearned, num_params
    coarsen = 1
    rho, rhs = _case(N, seed=3, ratio=ratio)
    cfg = _Cfg(pseudo_tol=1e-10, pseudo_maxiter=4000, ppe_learned_smooth=smooth, ppe_learned_fallback=False,
               ppe_learned_coarsen=coarsen, ppe_learned_outer="fgmres", ppe_learned_restart=restart,
               ppe_learned_maxiter=4000)
    s = PPESolverLearned(None, cfg, UniformGrid(N), params=np.zeros(num_params(), np.float32))
    p = s.solve(torch.from_numpy(rhs).to(cuda_device), torch.from_numpy(rho).to(cuda_device)).cpu().numpy()
    d = s.last_diagnostics
    assert d["ppe_learned_info"] == 0 and not d["ppe_learned_fell_back"], d
    assert d["ppe_learned_relative_residual"] <= 1e-10
    pd = oppe.spsolve_fvm(rhs, rho, oppe.uniform_coords(N, (1.0, 1.0)))
    assert np.abs(p - pd).max() <= 1e-7 * np.abs(pd).max()
    assert p.ravel()[s._pin_dof] == 0.0


def test_flexible_gmres_with_trained_network(cuda_device):
    """The shipped network under flexible GMRES(30) on the held-out 256^2
    density: converges without the fallback to the flexible CG's solution,
    deterministically."""
    import torch
    from twophaseflow_b200 import UniformGrid
    from twophaseflow_b200.learned import PPESolverLearned
    from twophaseflow_b200.workloads import divergence_rhs, droplet_density
    N = (256, 256)
    rho = torch.from_numpy(droplet_density(N, seed=101)).to(cuda_device)
    rhs = torch.from_numpy(divergence_rhs(N, seed=102)).to(cuda_device)
    base = dict(pseudo_tol=1e-8, pseudo_maxiter=5000, ppe_learned_maxiter=5000, ppe_learned_fallback=False)
    sg = PPESolverLearned(None, _Cfg(ppe_learned_outer="fgmres", **base), UniformGrid(N))
    pg = sg.solve(rhs, rho)
    dg = dict(sg.last_diagnostics)
    assert dg["ppe_learned_info"] == 0 and not dg["ppe_learned_fell_back"], dg
    pg2 = sg.solve(rhs, rho)
    assert torch.equal(pg, pg2) and sg.last_diagnostics["ppe_learned_iterations"] == dg["ppe_learned_iterations"]
    sc = PPESolverLearned(None, _Cfg(ppe_learned_outer="fcg", **base), UniformGrid(N))
    pc = sc.solve(rhs, rho)
    print("fgmres", dg["ppe_learned_iterations"], "fcg", sc.last_diagnostics["ppe_learned_iterations"])
    scale = float(torch.max(torch.abs(pc)))
    assert float(torch.max(torch.abs(pg - pc))) <= 1e-6 * scale
    with pytest.raises(ValueError, match="ppe_learned_outer"):
        PPESolverLearned(None, _Cfg(ppe_learned_outer="bicgstab", **base), UniformGrid(N))


def test_flexible_gmres_stall_rule_hands_over_to_pcg(cuda_device):
    """Restarted Jacobi-GMRES(7) (all-zero network, one sweep) at density ratio
    1000 stalls: the stall rule (best true residual not halved within 128
    Arnoldi columns, checked after each cycle) stops it long before the
    iteration budget and plain PCG finishes the solve."""
    import torch
    from twophaseflow_b200 import UniformGrid
    from twophaseflow_b200.learned import PPESolverLearned, num_params
    N = (48, 48)
    rho, rhs = _case(N, seed=5)
    cfg = _Cfg(pseudo_tol=1e-9, pseudo_maxiter=4000, ppe_learned_smooth=1, ppe_learned_maxiter=4000,
               ppe_learned_coarsen=1, ppe_learned_outer="fgmres", ppe_learned_restart=7)
    s = PPESolverLearned(None, cfg, UniformGrid(N), params=np.zeros(num_params(), np.float32))
    p = s.solve(torch.from_numpy(rhs).to(cuda_device), torch.from_numpy(rho).to(cuda_device)).cpu().numpy()
    d = s.last_diagnostics
    print(d)
    assert d["ppe_learned_fell_back"] and d["ppe_learned_info"] == 0
    assert d["ppe_learned_iterations"] < 2000
    pd = oppe.spsolve_fvm(rhs, rho, oppe.uniform_coords(N, (1.0, 1.0)))
    assert np.abs(p - pd).max() <= 1e-6 * np.abs(pd).max()


@pytest.mark.parametrize("N,coarsen", [((64, 64), 1), ((100, 77), 4), ((256, 256), 4)])
def test_blocked_smoother_equals_single_sweeps(cuda_device, N, coarsen):
    """The preconditioner with 1, 3 or 4 damped-Jacobi sweeps per launch
    (temporally blocked smoother) gives the same bits for 1, 5 and 16 sweeps,
    on the fine-grid and the two-level form, with the pinned node inside."""
    import torch
    from twophaseflow_b200 import UniformGrid, _lib
    from twophaseflow_b200.learned import PPESolverLearned
    rho, rhs = _case(N, seed=7)
    s = PPESolverLearned(None, _Cfg(pseudo_tol=1e-8, pseudo_maxiter=100, ppe_learned_coarsen=coarsen),
                         UniformGrid(N))
    s.prepare_operator(torch.from_numpy(rho).to(cuda_device))
    r = torch.from_numpy(rhs).to(cuda_device)
    for smooth in (1, 5, 16):
        s.smooth = smooth
        outs = []
        for blk in (1, 3, 4):
            _lib.check(s.lib.tpf_lppe_set_smooth_block(s._lp, blk))
            outs.append(s.precondition(r).clone())
        for o in outs[1:]:
            assert torch.equal(outs[0], o), smooth
    with pytest.raises(ValueError):
        _lib.check(s.lib.tpf_lppe_set_smooth_block(s._lp, 5))
