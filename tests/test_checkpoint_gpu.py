"""Restart of the GPU two-phase step from checkpoints.

* A checkpoint the reference's own writer produced after three quick-start
  steps (tests/golden/c1_checkpoint_ref.npz, tests/golden/make_golden.py
  ``checkpoint``) restores into ``TwoPhaseStep`` with the quick-start
  selection; the restored step's CFL time step equals the reference's fourth
  dt bit for bit, and the fourth step lands on the reference's fourth-step
  fields at the one-step bars of the quick-start parity test, with the
  reference's GMRES iteration count.  Without the AB2 history the same step
  misses those bars by orders of magnitude, so the restored history is what
  the reference's next step reads.
* A checkpoint this package writes mid-run restores into a fresh step that
  then continues bit for bit like the uninterrupted run.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(__file__)
G = np.load(os.path.join(HERE, "golden", "c1_golden.npz"))
REF_CKPT = os.path.join(HERE, "golden", "c1_checkpoint_ref.npz")
REF_YAML = os.path.join(HERE, "golden", "c1_checkpoint.yaml")
REF_GMRES_ITERATIONS = (240, 293, 297, 277, 227, 262)
ONE_STEP_TOL = {"psi": 2e-11, "u": 5e-11, "v": 5e-11, "p": 1e-12}
FREE_RUN_TOL = {"psi": 2e-6, "u": 1e-4, "v": 1e-4, "p": 5e-7}


def _c1(use_graphs=True, psi=None):
    from twophaseflow_b200 import TwoPhaseStep, UniformGrid
    return TwoPhaseStep(UniformGrid((64, 64)), G["psi0"] if psi is None else psi, rho_ratio=0.1, mu_ratio=0.1,
                        convection="uccd6", transport_mass_correction=True, reinit_bc="neumann",
                        ppe_method="gmres", ppe_maxiter=500, no_slip=True, zero_velocity_shortcut=True,
                        use_graphs=use_graphs)


def _errs(s, k):
    import torch
    torch.cuda.synchronize()
    out = {"psi": s.psi, "u": s.vel[0], "v": s.vel[1], "p": s.p}
    return {f: float(np.abs(out[f].cpu().numpy() - G[f"s{k}/{f}"]).max() / np.abs(G[f"s{k}/{f}"]).max())
            for f in out}


@pytest.mark.parametrize("use_graphs", [False, True])
def test_restart_from_reference_checkpoint(cuda_device, use_graphs):
    from twophaseflow_b200.checkpoint import load_checkpoint
    s = _c1(use_graphs, psi=np.zeros((65, 65)))
    st = load_checkpoint(REF_CKPT, solver=s, config_path=REF_YAML, verify_code=False)
    assert st["step"] == 3
    assert st["psi"] is s.psi and st["u"] is s.vel[0]
    assert s.cfl_dt() == float(G["s3/dt"])
    for k in range(3, 6):
        s.step(float(G[f"s{k}/dt"]))
        e = _errs(s, k)
        print(f"restart k={k} gmres={s.last_ppe_iterations} " + " ".join(f"{f}={v:.2e}" for f, v in e.items()))
        tol = ONE_STEP_TOL if k == 3 else FREE_RUN_TOL
        for f in e:
            assert e[f] <= tol[f], (k, f, e)
        if k == 3:
            assert abs(s.last_ppe_iterations - REF_GMRES_ITERATIONS[3]) <= 1, s.last_ppe_iterations


def test_restart_without_history_misses(cuda_device):
    """The control: the same restart with the AB2 history dropped."""
    import torch
    from twophaseflow_b200.checkpoint import load_checkpoint
    s = _c1(False, psi=np.zeros((65, 65)))
    load_checkpoint(REF_CKPT, solver=s, config_path=REF_YAML, verify_code=False)
    s.predictor._ab2_ready = False
    s.step(float(G["s3/dt"]))
    torch.cuda.synchronize()
    e = _errs(s, 3)
    assert e["u"] > 1e3 * ONE_STEP_TOL["u"], e


def test_own_checkpoint_continues_bitwise(cuda_device, tmp_path):
    import torch
    from twophaseflow_b200.checkpoint import load_checkpoint, load_manifest
    a = _c1(True)
    t = 0.0
    for k in range(3):
        dt = float(G[f"s{k}/dt"])
        a.step(dt)
        t += dt
    path = tmp_path / "checkpoint_final.npz"
    a.save_checkpoint(path, t=t, step=3)
    m = load_manifest(path)
    assert m["backend_device"] == "gpu" and m["step"] == 3 and m["grid_shape"] == [65, 65]
    b = _c1(True, psi=np.zeros((65, 65)))
    st = load_checkpoint(path, solver=b)
    assert st["t"] == t
    assert b.cfl_dt() == a.cfl_dt()
    for _ in range(3):
        dt = a.cfl_dt()
        a.step(dt)
        b.step(dt)
        assert a.last_ppe_iterations == b.last_ppe_iterations
    torch.cuda.synchronize()
    for x, y in ((a.psi, b.psi), (a.vel[0], b.vel[0]), (a.vel[1], b.vel[1]), (a.p, b.p)):
        np.testing.assert_array_equal(x.cpu().numpy(), y.cpu().numpy())


def test_checkpoint_3d_roundtrip(cuda_device, tmp_path):
    """A 3-D step (CG route, one graph per step) writes state/w and resumes
    bit for bit."""
    import torch
    from twophaseflow_b200 import TwoPhaseStep, UniformGrid
    from twophaseflow_b200.checkpoint import CheckpointError, load_checkpoint
    from twophaseflow_b200.workloads import quickstart_psi
    N = (24, 24, 24)
    psi = quickstart_psi(N, centre=(0.5, 0.5, 0.4), radius=0.2)
    a = TwoPhaseStep(UniformGrid(N), psi, rho_ratio=0.1, mu_ratio=0.1)
    dt = 1e-3
    for _ in range(2):
        a.step(dt)
    path = tmp_path / "c3.npz"
    a.save_checkpoint(path, t=2 * dt, step=2)
    with np.load(path) as d:
        assert "state/w" in d.files and int(d["solver/conv_prev/count"]) == 3
    b = TwoPhaseStep(UniformGrid(N), psi, rho_ratio=0.1, mu_ratio=0.1)
    load_checkpoint(path, solver=b)
    for _ in range(2):
        a.step(dt)
        b.step(dt)
    torch.cuda.synchronize()
    for x, y in zip([a.psi, a.p, *a.vel], [b.psi, b.p, *b.vel]):
        np.testing.assert_array_equal(x.cpu().numpy(), y.cpu().numpy())
    other = TwoPhaseStep(UniformGrid(N), psi, rho_ratio=0.5, mu_ratio=0.1)
    with pytest.raises(CheckpointError, match="config fingerprint"):
        load_checkpoint(path, solver=other)
