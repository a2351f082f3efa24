"""CCD variable-density operator L_H and defect correction on the GPU against
the reference's compute_ccd_laplacian (golden fixtures) and the oracle's
restatement of PPESolverDefectCorrection.

Tolerances: L_H within 1e-10 of the reference relative to max|L_H p| (two CCD
solves per axis, each at the 1e-12 bar, scaled by 1/rho and d(rho)/rho^2);
defect-correction pressure within 1e-8 relative of the oracle run with an
exact base solve (the GPU base solve stops at 1e-12).
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import ccd as occd
from oracle import ppe as oppe
from twophaseflow_b200.workloads import divergence_rhs, droplet_density

pytestmark = pytest.mark.gpu


class _Cfg:
    def __init__(self, **kw):
        self.__dict__.update(kw)


@pytest.mark.parametrize("name", ["lh2d", "lh3d"])
def test_ccd_laplacian_matches_reference(cuda_device, ppe_golden, name):
    import torch
    from twophaseflow_b200 import CCDVariableDensityOperator, UniformGrid
    g = ppe_golden
    N = tuple(int(n) for n in g[f"{name}/N"])
    op = CCDVariableDensityOperator(UniformGrid(N))
    op.prepare_operator(torch.from_numpy(g[f"{name}/rho"]).to(cuda_device))
    Lp = op.apply(torch.from_numpy(g[f"{name}/p"]).to(cuda_device)).cpu().numpy()
    ref = g[f"{name}/Lp"]
    assert np.abs(Lp - ref).max() <= 1e-10 * np.abs(ref).max()


def test_defect_correction_matches_oracle(cuda_device, ppe_golden):
    import torch
    from twophaseflow_b200 import (CCDVariableDensityOperator, PPESolverDefectCorrection,
                                   PPESolverFVMMatrixFree, UniformGrid)
    N = (32, 32)
    grid = UniformGrid(N)
    rho = droplet_density(N, n_drops=3, rho_g=0.1, seed=2)
    rhs = divergence_rhs(N, seed=3)
    base = PPESolverFVMMatrixFree(None, _Cfg(pseudo_tol=1e-13, pseudo_maxiter=100000, ppe_iteration_method="cg",
                                             ppe_preconditioner="jacobi"), grid)
    op = CCDVariableDensityOperator(grid)
    dc = PPESolverDefectCorrection(None, grid, base, op, max_corrections=3, tolerance=1e-10)
    p = dc.solve(torch.from_numpy(rhs).to(cuda_device), torch.from_numpy(rho).to(cuda_device)).cpu().numpy()
    # oracle: exact FVM base solve, CCD operator restated
    coords = oppe.uniform_coords(N, (1.0, 1.0))
    h = [1.0 / n for n in N]
    drho = [occd.differentiate_wall(rho, ax, h[ax])[0] for ax in range(2)]
    pin = oppe.pin_dof(N)
    po, hist = oppe.defect_correction(rhs, rho, lambda r: oppe.spsolve_fvm(r, rho, coords, pin),
                                      lambda q: oppe.ccd_laplacian(q, rho, drho, h), pin,
                                      max_corrections=3, tolerance=1e-10)
    assert np.abs(p - po).max() <= 1e-8 * np.abs(po).max()
    np.testing.assert_allclose(dc.last_residual_history, hist, rtol=1e-5)
    # and the reference's own DC run (same inputs as the golden fixture)
    g = ppe_golden
    np.testing.assert_allclose(rho, g["dc32/rho"])
    assert np.abs(p - g["dc32/p"]).max() <= 1e-8 * np.abs(g["dc32/p"]).max()
    # the correction loop reduces the L_H residual
    assert hist[-1] < hist[0]
