"""The FCCD matrix-free PPE oracle (default path) against the reference's own
outputs (tests/golden/fccd_ppe_golden.npz, written by tests/golden/make_golden.py)."""

import os

import numpy as np
import pytest

from oracle.fccd_ppe import FCCDPPE

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "fccd_ppe_golden.npz"))
CASES = ["wall2d", "per2d", "wall3d"]


def _solver(name):
    return FCCDPPE(G[f"{name}/L"], G[f"{name}/N"], str(G[f"{name}/bc"]), tol=1e-9, maxiter=500,
                   preconditioner=str(G[f"{name}/pre"]))


@pytest.mark.parametrize("name", CASES)
def test_apply_and_jacobi_match_reference(name):
    s = _solver(name)
    s.prepare(G[f"{name}/rho"])
    np.testing.assert_array_equal(s.apply(G[f"{name}/p"]), G[f"{name}/apply"])
    if s.diag_inv is not None:
        np.testing.assert_array_equal(s.diag_inv, G[f"{name}/diag_inv"])


@pytest.mark.parametrize("name", CASES)
def test_gmres_solution_matches_reference(name):
    """Same operator, same SciPy GMRES restatement: the same solution bit for
    bit (wall Jacobi-GMRES in 2-D and 3-D; periodic unpreconditioned, whose
    corner image node takes its value through two image syncs)."""
    sol, info, its = _solver(name).solve(G[f"{name}/rhs"], G[f"{name}/rho"])
    assert info == 0 and its > 0
    np.testing.assert_array_equal(sol, G[f"{name}/sol"])


def test_constant_pressure_is_in_the_kernel():
    """A constant field has zero face gradient: the operator returns the pin
    row's value and zeros elsewhere (wall box)."""
    s = FCCDPPE((1.0, 1.0), (10, 8), "wall")
    rng = np.random.default_rng(1)
    s.prepare(0.5 + rng.uniform(0.0, 1.0, (11, 9)))
    out = s.apply(np.full((11, 9), 2.5))
    expect = np.zeros((11, 9))
    expect.ravel()[s.pin] = 2.5
    assert np.abs(out - expect).max() < 1e-12
