"""CPU restatement of the CLS transport (TEST INFRASTRUCTURE: the oracle).

* ``flux_rhs`` -- the FCCD flux-form advection right-hand side
  -sum_k div(P_f(u_k phi)) (reference ``src/twophase/ccd/fccd_advection_helpers.py:8-72``,
  face value ``ccd/fccd.py:279-299``, face slices ``:213-233``, face divergence
  ``:464-520``) on the oracle's CCD second derivative.
* ``advance`` -- one TVD-RK3 level-set step with clip and periodic image sync
  (``levelset/fccd_advection.py:86-129``, ``time_integration/tvd_rk3.py:26-48``,
  ``core/boundary.py:116-133``).

Pinned against the reference's own outputs in ``tests/golden/advect_golden.npz``.
Only tests, smoke() and bench.py's CPU-baseline leg may use this module.
"""

from __future__ import annotations

import numpy as np

from . import ccd as occd
from .levelset import axis_kinds


def flux_divergence(prod, q, ax: int, H: float, periodic: bool):
    """-face_divergence(face_value(prod, q)) along ``ax`` (fccd.py:213-233,279-299,464-520)."""
    p = np.moveaxis(np.asarray(prod), ax, 0)
    qa = np.moveaxis(np.asarray(q), ax, 0)
    N = p.shape[0] - 1
    inv_H = 1.0 / H
    c = H * H / 16.0
    if periodic:
        lo, hi = p[:N], np.roll(p[:N], -1, axis=0)
        qlo, qhi = qa[:N], np.roll(qa[:N], -1, axis=0)
    else:
        lo, hi, qlo, qhi = p[:-1], p[1:], qa[:-1], qa[1:]
    F = 0.5 * (lo + hi) - c * (qlo + qhi)
    out = np.zeros_like(p)
    if periodic:
        du = (F - np.roll(F, 1, axis=0)) * inv_H
        out[:N] = du
        out[N] = du[0]
    else:
        out[1:N] = (F[1:] - F[:-1]) * inv_H
    return -np.moveaxis(out, 0, ax)


def _flux_contribution(u_k, phi, ax: int, H: float, h: float, periodic: bool):
    prod = u_k * phi
    q = occd.differentiate(prod, ax, h, bc="periodic" if periodic else "wall")[1]
    return flux_divergence(prod, q, ax, H, periodic)


def flux_rhs(vel, scalar, L, N, bc: str):
    """advection_rhs(..., mode='flux'): [acc] for a scalar, one acc per velocity
    component when scalar is None."""
    nd = len(vel)
    kinds = axis_kinds(bc, nd)
    H = [float(np.linspace(0.0, L[a], N[a] + 1)[1]) for a in range(nd)]
    h = [float(L[a] / N[a]) for a in range(nd)]
    targets = [scalar] if scalar is not None else list(vel)
    out = []
    for phi in targets:
        acc = np.zeros_like(np.asarray(phi, dtype=np.float64))
        for k in range(nd):
            acc += _flux_contribution(np.asarray(vel[k]), np.asarray(phi), k, H[k], h[k], kinds[k] == "periodic")
        out.append(acc)
    return out


def sync_images(a, bc: str):
    for ax, kind in enumerate(axis_kinds(bc, a.ndim)):
        if kind == "periodic":
            src = [slice(None)] * a.ndim
            img = [slice(None)] * a.ndim
            src[ax] = 0
            img[ax] = -1
            a[tuple(img)] = a[tuple(src)]
    return a


def advance(psi, vel, dt: float, L, N, bc: str, clip=(0.0, 1.0)):
    q0 = sync_images(np.array(psi, dtype=np.float64, copy=True), bc)

    def P(q):
        if clip is not None:
            q = np.clip(q, clip[0], clip[1])
        return sync_images(q, bc)

    R = lambda q: flux_rhs(vel, q, L, N, bc)[0]
    q1 = P(q0 + dt * R(q0))
    q2 = P(0.75 * q0 + 0.25 * (q1 + dt * R(q1)))
    return P((1.0 / 3.0) * q0 + (2.0 / 3.0) * (q2 + dt * R(q2)))
