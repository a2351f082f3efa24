"""CPU restatement of the steps either side of the PPE (TEST INFRASTRUCTURE: the oracle).

* ``correct`` -- the velocity corrector u^{n+1} = u* - (dt/rho) D1 p with the
  wall-normal gradient zeroed on wall planes (reference
  ``src/twophase/coupling/velocity_corrector.py:41-89``), on the oracle's CCD
  (``oracle.ccd.differentiate``).
* ``cfl_dt`` -- the CFL-limited time step (reference
  ``src/twophase/time_integration/cfl.py:41-137``).

Pinned against the reference's own outputs in ``tests/golden/step_golden.npz``.
Only tests, smoke() and bench.py's CPU-baseline leg may use this module.
"""

from __future__ import annotations

import math

import numpy as np

from . import ccd as occd


def pressure_gradient(p, h, bc: str):
    """ccd_pressure_gradient (velocity_corrector.py:41-55)."""
    grad = []
    for ax in range(p.ndim):
        d1, _ = occd.differentiate(p, ax, h[ax], bc=bc)
        d1 = np.array(d1, copy=True)
        if bc == "wall":   # enforce_wall_neumann (ccd_solver.py:264-281)
            lo = [slice(None)] * p.ndim
            hi = [slice(None)] * p.ndim
            lo[ax] = 0
            hi[ax] = -1
            d1[tuple(lo)] = 0.0
            d1[tuple(hi)] = 0.0
        grad.append(d1)
    return grad


def correct(vel_star, p, rho, dt: float, h, bc: str):
    """VelocityCorrector.correct (velocity_corrector.py:68-89)."""
    grad = pressure_gradient(p, h, bc)
    return [vel_star[ax] - (dt / rho) * grad[ax] for ax in range(len(vel_star))]


def cfl_dt(vel, mu, rho, L, N, cfl: float, We=None, rho_ratio: float = 0.0, cn_viscous: bool = True) -> float:
    """CFLCalculator.compute (cfl.py:85-137) with its constructor's bounds (:58-83)."""
    h = min(float(L[ax] / N[ax]) for ax in range(len(N)))
    dt_sigma = None
    if We is not None and We > 0.0:
        dt_sigma = math.sqrt((1.0 + rho_ratio) * We * h ** 3 / (2.0 * math.pi))
    u_sum = np.sum(np.stack([np.max(np.abs(np.asarray(v))) for v in vel]))
    dt_conv = cfl * h / np.maximum(u_sum, 1.0e-14)
    cands = [dt_conv]
    if not cn_viscous:
        nu_max = np.max(np.asarray(mu) / np.asarray(rho))
        cands.append(cfl * h * h / (4.0 * np.maximum(nu_max, 1.0e-14)))
    if dt_sigma is not None:
        cands.append(np.asarray(cfl * dt_sigma, dtype=np.float64))
    return float(np.maximum(np.min(np.stack(cands)), 1.0e-8))
