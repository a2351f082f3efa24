"""GPU tests of the composed two-phase time step (TwoPhaseStep): replaying
the captured CUDA graphs gives the same fields as eager execution, and a
rising-bubble run stays bounded, finite and nearly mass-conserving."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bubble(N):
    x = [np.linspace(0.0, 1.0, n + 1) for n in N]
    X = np.meshgrid(*x, indexing="ij")
    c = [0.5] * (len(N) - 1) + [0.3]
    r = np.sqrt(sum((X[a] - c[a]) ** 2 for a in range(len(N))))
    return 1.0 / (1.0 + np.exp(-(r - 0.2) / (1.5 / max(N))))


@pytest.mark.parametrize("N", [(64, 64), (32, 32, 32)])
def test_graph_replay_equals_eager(cuda_device, N):
    import torch
    from twophaseflow_b200 import TwoPhaseStep, UniformGrid
    psi = _bubble(N)
    dt = 0.25 / max(N)
    runs = []
    for graphs in (False, True):
        s = TwoPhaseStep(UniformGrid(N), psi, use_graphs=graphs)
        for _ in range(4):
            s.step(dt)
        torch.cuda.synchronize()
        runs.append([s.psi.cpu().numpy(), s.p.cpu().numpy()] + [v.cpu().numpy() for v in s.vel])
    for a, b in zip(*runs):
        np.testing.assert_array_equal(a, b)


def test_step_physics_2d(cuda_device):
    """64^2, 6 steps: psi in [0, 1], liquid mass within 1e-3 relative (the
    reinitialization restores mass; transport clipping may move a little),
    finite fields, a positive PPE iteration count and CFL time step."""
    import torch
    from twophaseflow_b200 import TwoPhaseStep, UniformGrid
    N = (64, 64)
    psi0 = _bubble(N)
    s = TwoPhaseStep(UniformGrid(N), psi0)
    dt = 0.25 / 64
    for _ in range(6):
        s.step(dt)
    torch.cuda.synchronize()
    psi = s.psi.cpu().numpy()
    assert np.isfinite(psi).all() and psi.min() >= 0.0 and psi.max() <= 1.0
    assert abs(psi.sum() - psi0.sum()) <= 1e-3 * psi0.sum()
    for v in s.vel:
        assert np.isfinite(v.cpu().numpy()).all()
    assert s.last_ppe_iterations > 0
    assert s.cfl_dt() > 0.0


@pytest.mark.parametrize("N", [(64, 64), (24, 20, 28)])
def test_whole_step_one_graph_equals_two_graphs(cuda_device, N):
    """The step with the pressure solve recorded inside the same CUDA graph
    (one replay per step; the 3-D streaming PCG as a conditional WHILE node)
    gives the same fields, bit for bit, and the same iteration counts as the
    step with the solve between two graphs."""
    import torch
    from twophaseflow_b200 import TwoPhaseStep, UniformGrid
    psi = _bubble(N)
    dt = 0.25 / max(N) / 4
    runs = []
    for in_graph in (False, True):
        s = TwoPhaseStep(UniformGrid(N), psi, ppe_in_graph=in_graph)
        its = []
        for _ in range(4):
            s.step(dt)
            its.append(s.last_ppe_iterations)
        torch.cuda.synchronize()
        runs.append(([s.psi.cpu().numpy(), s.p.cpu().numpy()] + [v.cpu().numpy() for v in s.vel], its))
        if in_graph:
            assert s._g2 is None   # one graph per step
    (f0, i0), (f1, i1) = runs
    assert i0 == i1 and min(i1) > 0
    for a, b in zip(f0, f1):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("N", [(96, 80), (20, 24, 16)])
def test_captured_cg_solve_replays(cuda_device, N):
    """A CG solve recorded under stream capture: each replay solves for the
    current right-hand side (written into the same buffer), equals the eager
    solve, and reports its iterations through read_result; the GMRES route
    refuses capture."""
    import torch
    from twophaseflow_b200 import PPESolverFVMMatrixFree, UniformGrid
    from twophaseflow_b200.workloads import divergence_rhs, droplet_density

    class Cfg:
        pseudo_tol = 1e-10
        pseudo_maxiter = 100000
        ppe_iteration_method = "cg"
        ppe_preconditioner = "jacobi"

    rho = torch.from_numpy(droplet_density(N, seed=2)).cuda()
    rhs_a = torch.from_numpy(divergence_rhs(N, seed=3)).cuda()
    rhs_b = torch.from_numpy(divergence_rhs(N, seed=4)).cuda()
    s = PPESolverFVMMatrixFree(None, Cfg(), UniformGrid(N))
    ref = []
    for r in (rhs_a, rhs_b):
        ref.append((s.solve(r, rho).clone(), s.last_diagnostics["ppe_low_order_cg_iterations"]))
    rhs = rhs_a.clone()
    out = torch.empty_like(rhs)
    st = torch.cuda.Stream()
    st.wait_stream(torch.cuda.current_stream())
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(st):
        with torch.cuda.graph(g, stream=st):
            out.copy_(s.solve(rhs, rho))
    torch.cuda.current_stream().wait_stream(st)
    for k, r in enumerate((rhs_a, rhs_b, rhs_a)):
        rhs.copy_(r)
        g.replay()
        d = s.read_result()
        p_ref, it_ref = ref[k % 2]
        assert d["ppe_low_order_cg_iterations"] == it_ref
        np.testing.assert_array_equal(out.cpu().numpy(), p_ref.cpu().numpy())

    class Gm(Cfg):
        ppe_iteration_method = "gmres"
        ppe_preconditioner = "line_pcr"

    sg = PPESolverFVMMatrixFree(None, Gm(), UniformGrid(N))
    sg.solve(rhs_a, rho)
    g2 = torch.cuda.CUDAGraph()
    with torch.cuda.stream(st):
        with pytest.raises(ValueError, match="cannot be captured"):
            with torch.cuda.graph(g2, stream=st):
                sg.solve(rhs, rho)
    torch.cuda.synchronize()
