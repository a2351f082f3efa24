"""The oracle of the steps either side of the PPE (velocity corrector, CFL
time step) against the reference's own outputs (tests/golden/step_golden.npz,
made by tests/golden/make_golden.py from the reference)."""

from __future__ import annotations

import os

import numpy as np
import pytest

from oracle import step as ostep

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "step_golden.npz")
CASES = ["wall2d", "per2d", "wall3d"]


@pytest.fixture(scope="module")
def golden():
    with np.load(GOLDEN) as d:
        return {k: d[k] for k in d.files}


def _case(g, name):
    N = tuple(int(n) for n in g[f"{name}/N"])
    L = tuple(float(x) for x in g[f"{name}/L"])
    h = [L[a] / N[a] for a in range(len(N))]
    vel = [g[f"{name}/u{a}"] for a in range(len(N))]
    return N, L, h, vel, str(g[f"{name}/bc"])


@pytest.mark.parametrize("name", CASES)
def test_corrector_oracle_matches_reference(golden, name):
    N, L, h, vel, bc = _case(golden, name)
    p, rho, dt = golden[f"{name}/p"], golden[f"{name}/rho"], float(golden[f"{name}/dt"])
    grad = ostep.pressure_gradient(p, h, bc)
    out = ostep.correct(vel, p, rho, dt, h, bc)
    for ax in range(len(N)):
        ref_g = golden[f"{name}/grad{ax}"]
        assert np.abs(grad[ax] - ref_g).max() <= 1e-12 * np.abs(ref_g).max()
        ref = golden[f"{name}/unew{ax}"]
        assert np.abs(out[ax] - ref).max() <= 1e-12 * np.abs(ref).max()
        if bc == "wall":   # wall planes: the velocity is left as it was
            assert np.array_equal(np.take(out[ax], [0, -1], axis=ax), np.take(vel[ax], [0, -1], axis=ax))


@pytest.mark.parametrize("name", CASES)
def test_cfl_oracle_matches_reference(golden, name):
    N, L, h, vel, bc = _case(golden, name)
    mu, rho = golden[f"{name}/mu"], golden[f"{name}/rho"]
    for tag, kw in (("cn", dict(cn_viscous=True)), ("expl", dict(cn_viscous=False)),
                    ("cap", dict(We=0.01, rho_ratio=0.1, cn_viscous=True))):
        assert ostep.cfl_dt(vel, mu, rho, L, N, 0.3, **kw) == float(golden[f"{name}/dt_{tag}"])


RC = np.load(os.path.join(os.path.dirname(__file__), "golden", "rhiechow_golden.npz"))


@pytest.mark.parametrize("name", ["wall2d", "per2d", "wall3d", "per3d"])
def test_rc_divergence_matches_reference(name):
    """The oracle's Rhie-Chow divergence, plain and balanced-force, equals the
    reference's bit for bit (same CCD, same operation order)."""
    N, L, bc = RC[f"{name}/N"], RC[f"{name}/L"], str(RC[f"{name}/bc"])
    vel = [RC[f"{name}/u{a}"] for a in range(len(N))]
    args = (vel, RC[f"{name}/p"], RC[f"{name}/rho"], float(RC[f"{name}/dt"]), L, N, bc, bc)
    np.testing.assert_array_equal(ostep.rc_divergence(*args), RC[f"{name}/div"])
    bf = dict(kappa=RC[f"{name}/kappa"], psi=RC[f"{name}/psi"], we=float(RC[f"{name}/we"]))
    np.testing.assert_array_equal(ostep.rc_divergence(*args, **bf), RC[f"{name}/div_bf"])


def test_rc_divergence_of_uniform_flow_vanishes():
    """u* = const, p = 0 on a periodic box: zero divergence."""
    N = (12, 10)
    vel = [np.full((13, 11), 0.3), np.full((13, 11), -1.1)]
    d = ostep.rc_divergence(vel, np.zeros((13, 11)), np.ones((13, 11)), 0.01, (1.0, 1.0), N, "periodic", "periodic")
    assert np.abs(d).max() < 1e-12
