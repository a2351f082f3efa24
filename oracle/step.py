"""CPU restatement of the steps either side of the PPE (TEST INFRASTRUCTURE: the oracle).

* ``correct`` -- the velocity corrector u^{n+1} = u* - (dt/rho) D1 p with the
  wall-normal gradient zeroed on wall planes (reference
  ``src/twophase/coupling/velocity_corrector.py:41-89``), on the oracle's CCD
  (``oracle.ccd.differentiate``).
* ``cfl_dt`` -- the CFL-limited time step (reference
  ``src/twophase/time_integration/cfl.py:41-137``).
* ``rc_divergence`` -- the Rhie-Chow face-velocity divergence (reference
  ``src/twophase/spatial/rhie_chow.py:55-284``).

Pinned against the reference's own outputs in ``tests/golden/step_golden.npz`` and
``tests/golden/rhiechow_golden.npz``.
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


def _rc_axis(u, p, rho, dp, ax: int, h: float, dt: float, periodic: bool, kappa=None, psi=None, dpsi=None, we=None):
    """Face velocities of one axis and their divergence (rhie_chow.py:117-284),
    restated on lines moved to axis 0."""
    mv = lambda a: np.moveaxis(np.asarray(a), ax, 0) if a is not None else None
    u, p, rho, dp = mv(u), mv(p), mv(rho), np.array(mv(dp), copy=True)
    kappa, psi, dpsi = mv(kappa), mv(psi), mv(dpsi)
    bf = kappa is not None
    N = p.shape[0] - 1
    fs = None
    if bf:
        fs = (kappa * dpsi) / we
    if not periodic:
        dp[0] = (p[1] - p[0]) / h
        dp[N] = (p[N] - p[N - 1]) / h
        if bf:
            fs = np.array(fs, copy=True)
            fs[0] = (kappa[0] * (psi[1] - psi[0])) / (h * we)
            fs[N] = (kappa[N] * (psi[N] - psi[N - 1])) / (h * we)

    def face(l, r):
        ubar = 0.5 * (u[l] + u[r])
        br = (p[r] - p[l]) / h - 0.5 * (dp[l] + dp[r])
        if bf:
            kf = 0.5 * (kappa[l] + kappa[r])
            br = br - ((kf * (psi[r] - psi[l])) / (h * we) - 0.5 * (fs[l] + fs[r]))
        return ubar - (dt * (2.0 / (rho[l] + rho[r]))) * br

    flux = np.zeros_like(p)
    flux[1:] = face(slice(0, N), slice(1, N + 1))
    if periodic:
        flux[0] = face(N, 0)
    div = np.empty_like(p)
    div[:N] = (flux[1:] - flux[:N]) / h
    div[N] = (flux[0] - flux[N]) / h if periodic else (-flux[N]) / h
    return np.moveaxis(div, 0, ax)


def rc_divergence(vel_star, p, rho, dt: float, L, N, ccd_bc: str, rc_bc: str, kappa=None, psi=None, we=None):
    """RhieChowInterpolator.face_velocity_divergence (rhie_chow.py:55-115) on the
    oracle CCD; rc_bc: 'wall' or 'periodic' for every axis."""
    p = np.asarray(p, dtype=np.float64)
    bf = kappa is not None and psi is not None and we is not None
    div = np.zeros_like(p)
    for ax in range(p.ndim):
        h = float(L[ax] / N[ax])
        dp, _ = occd.differentiate(p, ax, h, bc=ccd_bc)
        dpsi = occd.differentiate(np.asarray(psi), ax, h, bc=ccd_bc)[0] if bf else None
        div += _rc_axis(vel_star[ax], p, rho, dp, ax, h, dt, rc_bc == "periodic",
                        kappa if bf else None, psi if bf else None, dpsi, we if bf else None)
    return div
