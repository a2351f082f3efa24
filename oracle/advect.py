"""CPU restatement of the CLS transport (TEST INFRASTRUCTURE: the oracle).

* ``flux_rhs`` -- the FCCD flux-form advection right-hand side
  -sum_k div(P_f(u_k phi)) (reference ``src/twophase/ccd/fccd_advection_helpers.py:8-72``,
  face value ``ccd/fccd.py:279-299``, face slices ``:213-233``, face divergence
  ``:464-520``) on the oracle's CCD second derivative.
* ``node_gradient`` / ``node_rhs`` -- Option C: the R_4 Hermite node gradient
  and the nodal right-hand side -sum_k u_k grad_k phi (``ccd/fccd.py:392-462``,
  ``fccd_advection_helpers.py:46-72``).
* ``advance`` -- one TVD-RK3 level-set step with clip and periodic image sync
  (``levelset/fccd_advection.py:86-129``, ``time_integration/tvd_rk3.py:26-48``,
  ``core/boundary.py:116-133``).
* ``reinitialize`` -- the split reinitialization: compression + CN-ADI
  diffusion + mass correction (``levelset/reinit_split.py:73-102``,
  ``levelset/reinit_ops.py:34-204``, ``levelset/heaviside.py:118-149``).

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


def node_gradient(u, q, ax: int, H: float, periodic: bool):
    """Option C R_4 node gradient (fccd.py:90-94,131-134,243-277,392-462):
    face gradients (u_hi - u_lo)/H - (H/24)(q_hi - q_lo), then
    0.5 (d_L + d_R) - (H/16)(q_{i+1} - q_{i-1}); wall nodes take their one
    face gradient, periodic node N repeats node 0."""
    a = np.moveaxis(np.asarray(u), ax, 0)
    qa = np.moveaxis(np.asarray(q), ax, 0)
    N = a.shape[0] - 1
    inv_H, h24, h16 = 1.0 / H, H / 24.0, H / 16.0
    if periodic:
        lo, hi = a[:N], np.roll(a[:N], -1, axis=0)
        qlo, qhi = qa[:N], np.roll(qa[:N], -1, axis=0)
    else:
        lo, hi, qlo, qhi = a[:-1], a[1:], qa[:-1], qa[1:]
    d = (hi - lo) * inv_H - h24 * (qhi - qlo)
    out = np.empty_like(a)
    if periodic:
        qu = qa[:N]
        g = 0.5 * (np.roll(d, 1, axis=0) + d) - h16 * (np.roll(qu, -1, axis=0) - np.roll(qu, 1, axis=0))
        out[:N] = g
        out[N] = g[0]
    else:
        out[1:N] = 0.5 * (d[:-1] + d[1:]) - h16 * (qa[2:] - qa[:-2])
        out[0] = d[0]
        out[N] = d[N - 1]
    return np.moveaxis(out, 0, ax)


def node_rhs(vel, scalar, L, N, bc: str):
    """advection_rhs(..., mode='node'): -sum_k u_k (R_4 grad_k phi)
    (fccd_advection_helpers.py:46-72)."""
    nd = len(vel)
    kinds = axis_kinds(bc, nd)
    H = [float(np.linspace(0.0, L[a], N[a] + 1)[1]) for a in range(nd)]
    h = [float(L[a] / N[a]) for a in range(nd)]
    targets = [scalar] if scalar is not None else list(vel)
    out = []
    for phi in targets:
        phi = np.asarray(phi, dtype=np.float64)
        acc = np.zeros_like(phi)
        for k in range(nd):
            per = kinds[k] == "periodic"
            q = occd.differentiate(phi, k, h[k], bc="periodic" if per else "wall")[1]
            acc -= np.asarray(vel[k]) * node_gradient(phi, q, k, H[k], per)
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


def advance(psi, vel, dt: float, L, N, bc: str, clip=(0.0, 1.0), mode: str = "flux"):
    q0 = sync_images(np.array(psi, dtype=np.float64, copy=True), bc)
    if all(not np.any(np.asarray(v)) for v in vel):
        # the reference's CPU backend skips the stages for an exactly zero
        # velocity (fccd_advection.py:99-110): clip and image sync only
        q = np.clip(q0, clip[0], clip[1]) if clip is not None else q0
        return sync_images(q, bc)

    def P(q):
        if clip is not None:
            q = np.clip(q, clip[0], clip[1])
        return sync_images(q, bc)

    rhs = node_rhs if mode == "node" else flux_rhs
    R = lambda q: rhs(vel, q, L, N, bc)[0]
    q1 = P(q0 + dt * R(q0))
    q2 = P(0.75 * q0 + 0.25 * (q1 + dt * R(q1)))
    return P((1.0 / 3.0) * q0 + (2.0 / 3.0) * (q2 + dt * R(q2)))


# ── split reinitialization (levelset/reinit_split.py:73-102) ─────────────────

BETA2 = -1.0 / 8.0


def periodic_flags(bc, ndim):
    """periodic_axis_flags (core/boundary.py:94-113)."""
    if bc in ("zero", "neumann", "outflow"):
        return [False] * ndim
    return [k == "periodic" for k in axis_kinds(bc, ndim)]


def cell_volumes(L, N, flags):
    """Grid.cell_volumes for a uniform grid (core/grid.py:1123-1170)."""
    ws = []
    for a in range(len(N)):
        coords = np.linspace(0.0, L[a], N[a] + 1)
        if flags[a]:
            cw = np.diff(coords)
            w = np.empty_like(coords)
            w[:-1] = 0.5 * (np.roll(cw, 1) + cw)
            w[-1] = 0.0
        else:
            w = np.full(N[a] + 1, L[a] / N[a])
        ws.append(w)
    vol = ws[0]
    for a in range(1, len(N)):
        vol = np.expand_dims(vol, axis=a) * ws[a]
    return vol


def mass_correction(q, dV, M_target):
    """apply_mass_correction (levelset/heaviside.py:118-149)."""
    M_new = np.sum(q * dV)
    w = 4.0 * q * (1.0 - q)
    W = np.sum(w * dV)
    W_safe = W if W > 1e-12 else 1.0
    gate = 1.0 if W > 1e-12 else 0.0
    return np.clip(q + (gate * ((M_target - M_new) / W_safe)) * w, 0.0, 1.0)


def _pad(g, ax, bc):
    label = bc.strip().lower()
    n = g.shape[ax]
    take = lambda i: np.take(g, [i], axis=ax)
    if label == "periodic":
        lo, hi = take(n - 2), take(1)
    elif label in ("neumann", "outflow"):
        lo, hi = take(0), take(n - 1)
    else:
        lo, hi = np.zeros_like(take(0)), np.zeros_like(take(0))
    return np.concatenate([lo, g, hi], axis=ax)


def reinitialize(psi, L, N, ccd_bc: str, eps: float, n_steps: int = 4, bc: str = "zero", eps_d: float = 0.05,
                 mass: bool = True):
    """SplitReinitializer.reinitialize (reinit_split.py:73-102, reinit_ops.py:34-204)."""
    nd = len(N)
    h = [float(L[a] / N[a]) for a in range(nd)]
    dx = min(h)
    dtau = min(0.5 * dx ** 2 / (2.0 * nd * float(np.min(eps))), 0.5 * dx)
    kinds = axis_kinds(ccd_bc, nd)
    flags = periodic_flags(bc, nd)
    dV = cell_volumes(L, N, flags)

    def sync(a):
        for ax in range(nd):
            if flags[ax]:
                src = [slice(None)] * nd
                img = [slice(None)] * nd
                src[ax] = 0
                img[ax] = -1
                a[tuple(img)] = a[tuple(src)]
        return a

    def D1(f, ax):
        return np.asarray(occd.differentiate(f, ax, h[ax], bc=kinds[ax])[0])

    q = sync(np.array(psi, dtype=np.float64, copy=True))
    M_old = np.sum(q * dV)
    for _ in range(n_steps):
        g = [D1(q, ax) for ax in range(nd)]
        gs = sum(x * x for x in g)
        sg = np.maximum(np.sqrt(np.maximum(gs, 1e-12)), 1e-6)
        pp = q * (1.0 - q)
        div = np.zeros_like(q)
        for ax in range(nd):
            gp = _pad(D1(pp * (g[ax] / sg), ax), ax, bc)
            n = gp.shape[ax]
            c = np.take(gp, range(1, n - 1), axis=ax)
            pl = np.take(gp, range(2, n), axis=ax)
            mi = np.take(gp, range(0, n - 2), axis=ax)
            div = div + (c + eps_d * (pl - 2.0 * c + mi))
        q_new = sync(np.clip(q - dtau * div, 0.0, 1.0))
        for ax in range(nd):
            mu = eps * dtau / (2.0 * h[ax] ** 2)
            n = N[ax] + 1
            d_L, c_L = 1.0 + 6.0 * mu, BETA2 - 3.0 * mu
            main, sup, sub = np.full(n, d_L), np.full(n - 1, c_L), np.full(n - 1, c_L)
            sup[0] = 2.0 * c_L
            sub[-1] = 2.0 * c_L
            m = main.copy()
            f = np.empty(n - 1)
            for i in range(1, n):
                f[i - 1] = sub[i - 1] / m[i - 1]
                m[i] -= f[i - 1] * sup[i - 1]
            dR, cR = 1.0 - 6.0 * mu, BETA2 + 3.0 * mu
            p = np.moveaxis(q_new, ax, 0)
            d = np.empty_like(p)
            d[1:-1] = cR * p[:-2] + dR * p[1:-1] + cR * p[2:]
            d[0] = dR * p[0] + 2.0 * cR * p[1]
            d[-1] = 2.0 * cR * p[-2] + dR * p[-1]
            for i in range(1, n):
                d[i] = d[i] - f[i - 1] * d[i - 1]
            x = np.empty_like(d)
            x[-1] = d[-1] / m[-1]
            for i in range(n - 2, -1, -1):
                x[i] = (d[i] - sup[i] * x[i + 1]) / m[i]
            q_new = sync(np.moveaxis(x, 0, ax).copy())
        q = sync(np.clip(q_new, 0.0, 1.0))
    if mass:
        q = sync(mass_correction(q, dV, M_old))
    return q


def uccd6(vel, L, N, bc: str, sigma: float = 1.0e-3):
    """UCCD6ConvectionTerm.compute (ns_terms/uccd6_convection.py:83-128)."""
    nd = len(vel)
    kinds = axis_kinds(bc, nd)
    h = [float(L[a] / N[a]) for a in range(nd)]
    h7 = [(float(L[a]) / int(N[a])) ** 7 for a in range(nd)]
    D = lambda f, ax: occd.differentiate(f, ax, h[ax], bc=kinds[ax])
    out = []
    for j in range(nd):
        acc = np.zeros_like(vel[j])
        for k in range(nd):
            d1, d2 = D(vel[j], k)
            cons = D(vel[k] * vel[j], k)[0]
            acc = acc - 0.5 * (vel[k] * d1 + cons)
            d8 = D(D(D(d2, k)[1], k)[1], k)[1]
            acc = acc - (sigma * h7[k]) * (np.abs(vel[k]).max() * d8)
        out.append(acc)
    return out
