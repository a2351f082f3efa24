"""Pin the CPU oracle against outputs of the reference itself (golden fixtures).

The fixtures were produced by ``tests/golden/make_golden.py``, which runs the
reference's own ``CCDSolver`` / ``PPESolverFVMMatrixFree`` /
``PPESolverFVMSpsolve`` / tridiagonal helpers / ``compute_ccd_laplacian``.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import ccd as occd
from oracle import ppe as oppe

CCD_WALL = ["wall2d", "wall3d", "wall2d_big"]
CCD_PER = ["per2d", "per3d"]
PPE_CASES = ["apply2d", "gmres_line2d", "gmres_jac2d", "cg_jac2d", "cg_jac3d",
             "gmres_line3d", "cg_drop32", "gmres_drop16", "cg_rect"]


def _h(g, name):
    N = g[f"{name}/N"]
    L = g[f"{name}/L"]
    return [float(L[a]) / float(N[a]) for a in range(len(N))]


@pytest.mark.parametrize("name", CCD_WALL + CCD_PER)
def test_ccd_oracle_matches_reference(ccd_golden, name):
    g = ccd_golden
    f = g[f"{name}/f"]
    bc = "periodic" if name.startswith("per") else "wall"
    for ax, h in enumerate(_h(g, name)):
        d1, d2 = occd.differentiate(f, ax, h, bc=bc)
        np.testing.assert_allclose(d1, g[f"{name}/d1_ax{ax}"], rtol=0, atol=1e-12 * np.abs(g[f"{name}/d1_ax{ax}"]).max())
        np.testing.assert_allclose(d2, g[f"{name}/d2_ax{ax}"], rtol=0, atol=1e-12 * np.abs(g[f"{name}/d2_ax{ax}"]).max())
        # first/second-only paths agree with the full solve in the reference
        np.testing.assert_allclose(g[f"{name}/first_ax{ax}"], g[f"{name}/d1_ax{ax}"], rtol=1e-12, atol=1e-9)
        np.testing.assert_allclose(g[f"{name}/second_ax{ax}"], g[f"{name}/d2_ax{ax}"], rtol=1e-12, atol=1e-9)


@pytest.mark.parametrize("name", CCD_WALL)
def test_ccd_oracle_bc_override(ccd_golden, name):
    g = ccd_golden
    h = _h(g, name)[0]
    d1, d2 = occd.differentiate(g[f"{name}/f"], 0, h, bc_left=(0.3, -1.2), bc_right=(0.0, 2.5))
    np.testing.assert_allclose(d1, g[f"{name}/bcov_d1"], rtol=1e-12, atol=1e-12 * np.abs(d1).max())
    np.testing.assert_allclose(d2, g[f"{name}/bcov_d2"], rtol=1e-12, atol=1e-12 * np.abs(d2).max())


@pytest.mark.parametrize("bc", ["wall", "periodic"])
def test_ccd_oracle_sin(ccd_golden, bc):
    g = ccd_golden
    d1, d2 = occd.differentiate(g[f"sin_{bc}/f"], 0, 1.0 / 32, bc=bc)
    np.testing.assert_allclose(d1, g[f"sin_{bc}/d1"], atol=1e-12)
    np.testing.assert_allclose(d2, g[f"sin_{bc}/d2"], atol=1e-10)


def test_ccd_oracle_nonuniform_metric(ccd_golden):
    g = ccd_golden
    f = g["nonuni/f"]
    for ax in range(2):
        d1, d2 = occd.differentiate(f, ax, 1.0 / 32, J=g[f"nonuni/J{ax}"], dJ=g[f"nonuni/dJ{ax}"])
        np.testing.assert_allclose(d1, g[f"nonuni/d1_ax{ax}"], rtol=1e-12, atol=1e-11 * np.abs(d1).max())
        np.testing.assert_allclose(d2, g[f"nonuni/d2_ax{ax}"], rtol=1e-12, atol=1e-11 * np.abs(d2).max())
        r1, r2 = occd.differentiate(f, ax, 1.0 / 32)
        np.testing.assert_allclose(r1, g[f"nonuni/raw_d1_ax{ax}"], atol=1e-12 * np.abs(r1).max())
        np.testing.assert_allclose(r2, g[f"nonuni/raw_d2_ax{ax}"], atol=1e-12 * np.abs(r2).max())


def test_block_lu_equals_dense_lu():
    """The unpivoted 2x2 block LU the CUDA kernels implement agrees with the
    reference's pivoted dense LU to round-off."""
    for n_pts, h in [(6, 0.2), (33, 1 / 32), (257, 1 / 256)]:
        diag, lower, upper = occd.wall_blocks(n_pts, h)
        fac = occd.block_lu_factor(diag, lower, upper)
        rng = np.random.default_rng(n_pts)
        rhs = rng.standard_normal((n_pts - 2, 2, 3))
        x = occd.block_lu_solve(fac, rhs)
        A = occd.wall_dense_matrix(n_pts, h)
        xd = np.linalg.solve(A, rhs.reshape(2 * (n_pts - 2), -1)).reshape(n_pts - 2, 2, -1)
        np.testing.assert_allclose(x, xd, rtol=0, atol=1e-12 * np.abs(xd).max())


def test_block_lu_rejects_singular_pivot():
    """Reference test_ccd.py:51-62: singular pivot fails closed."""
    diag = [np.array([[1.0, 2.0], [2.0, 4.0]]), np.eye(2)]
    lower = [np.zeros((2, 2)), np.eye(2)]
    upper = [np.eye(2), np.zeros((2, 2))]
    with pytest.raises(np.linalg.LinAlgError):
        occd.block_lu_factor(diag, lower, upper)


def test_wall_rejects_small_n():
    """Reference test_ccd.py:42-48: n_pts < 6 is rejected."""
    with pytest.raises(ValueError, match="n_pts >= 6"):
        occd.differentiate(np.zeros((5, 5)), 0, 0.25)


def _solver_for(g, name):
    N = tuple(int(n) for n in g[f"{name}/N"])
    coords = oppe.uniform_coords(N, (1.0,) * len(N))
    return oppe.FVMMatrixFree(
        coords, method=str(g[f"{name}/method"]), preconditioner=str(g[f"{name}/precond"]),
        tol=float(g[f"{name}/tol"]), maxiter=int(g[f"{name}/maxiter"]),
        restart=int(g[f"{name}/restart"]))


@pytest.mark.parametrize("name", PPE_CASES)
def test_ppe_apply_and_precond_match_reference(ppe_golden, name):
    g = ppe_golden
    s = _solver_for(g, name)
    assert s.pin == int(g[f"{name}/pin"])
    s.prepare_operator(g[f"{name}/rho"])
    np.testing.assert_allclose(s.apply(g[f"{name}/p_rand"]), g[f"{name}/apply"], rtol=1e-13, atol=1e-12)
    r = g[f"{name}/r_rand"]
    if s.preconditioner == "line_pcr":
        pco = oppe.line_precond_coeffs(s.coeffs, g[f"{name}/rho"], s.c_tau, s.h_min)
        np.testing.assert_allclose(oppe.line_precond(r, pco, s.pin), g[f"{name}/line_thomas"], rtol=1e-13, atol=1e-14)
        np.testing.assert_allclose(oppe.line_precond(r, pco, s.pin, 4), g[f"{name}/line_pcr4"], rtol=1e-13, atol=1e-14)
    else:
        dinv = oppe.jacobi_diag_inv(s.coeffs, s.pin)
        z = r * dinv
        z.ravel()[s.pin] = 0.0
        np.testing.assert_allclose(z, g[f"{name}/jacobi"], rtol=1e-14, atol=0)


@pytest.mark.parametrize("name", PPE_CASES)
def test_ppe_solve_matches_reference(ppe_golden, name):
    g = ppe_golden
    s = _solver_for(g, name)
    p = s.solve(g[f"{name}/rhs"], g[f"{name}/rho"])
    pref = g[f"{name}/p"]
    scale = np.abs(pref).max()
    np.testing.assert_allclose(p, pref, rtol=0, atol=1e-10 * scale)
    # same Krylov iteration count (operator applies) as the reference run
    applies = int(g[f"{name}/applies"])
    if s.method == "cg":
        assert s.last_iterations + 0 == applies
    # and the direct solution agrees with the reference's spsolve
    pd = oppe.spsolve_fvm(g[f"{name}/rhs"], g[f"{name}/rho"], s.coords)
    np.testing.assert_allclose(pd, g[f"{name}/p_direct"], rtol=0, atol=1e-11 * np.abs(pd).max())


@pytest.mark.parametrize("name", ["lh2d", "lh3d"])
def test_ccd_laplacian_matches_reference(ppe_golden, name):
    g = ppe_golden
    N = g[f"{name}/N"]
    h = [1.0 / float(n) for n in N]
    rho = g[f"{name}/rho"]
    drho = [occd.differentiate_wall(rho, ax, h[ax])[0] for ax in range(len(N))]
    Lp = oppe.ccd_laplacian(g[f"{name}/p"], rho, drho, h)
    np.testing.assert_allclose(Lp, g[f"{name}/Lp"], rtol=0, atol=1e-11 * np.abs(Lp).max())


def test_defect_correction_matches_reference(ppe_golden):
    """Oracle DC loop + CCD operator vs the reference's PPESolverDefectCorrection
    (exact FVM base solve, CCD L_H target)."""
    g = ppe_golden
    rho, rhs = g["dc32/rho"], g["dc32/rhs"]
    N = (32, 32)
    coords = oppe.uniform_coords(N, (1.0, 1.0))
    h = [1.0 / n for n in N]
    drho = [occd.differentiate_wall(rho, ax, h[ax])[0] for ax in range(2)]
    pin = oppe.pin_dof(N)
    p, hist = oppe.defect_correction(rhs, rho, lambda r: oppe.spsolve_fvm(r, rho, coords, pin),
                                     lambda q: oppe.ccd_laplacian(q, rho, drho, h), pin,
                                     max_corrections=3, tolerance=1e-10)
    np.testing.assert_allclose(p, g["dc32/p"], rtol=0, atol=1e-10 * np.abs(g["dc32/p"]).max())
    np.testing.assert_allclose(hist, g["dc32/history"], rtol=1e-9)
