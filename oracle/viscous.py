"""CPU restatement of the viscous stress divergence (TEST INFRASTRUCTURE: the
oracle): ViscousSpatialEvaluator.evaluate (reference
``src/twophase/ns_terms/viscous_spatial.py:28-221``, the three schemes and
the interface-band form of ccd_bulk when psi is given) on the oracle's CCD.

Pinned against the reference's own outputs in ``tests/golden/viscous_golden.npz``.
Only tests, smoke() and bench.py's CPU-baseline leg may use this module.
"""

from __future__ import annotations

import numpy as np

from . import ccd as occd
from .levelset import axis_kinds


def low_order_derivative(arr, axis: int, coords):
    """_low_order_derivative (viscous_spatial.py:70-104)."""
    arr = np.asarray(arr)
    dx = coords[1:] - coords[:-1]
    d = np.empty_like(arr)
    n = arr.shape[axis]
    a = np.moveaxis(arr, axis, 0)
    o = np.moveaxis(d, axis, 0)
    o[0] = (a[1] - a[0]) / dx[0]
    o[n - 1] = (a[n - 1] - a[n - 2]) / dx[-1]
    shape = [1] * arr.ndim
    shape[0] = n - 2
    h_l = dx[:-1].reshape(shape)
    h_r = dx[1:].reshape(shape)
    o[1:n - 1] = (-(h_r / (h_l * (h_l + h_r))) * a[:n - 2] + ((h_r - h_l) / (h_l * h_r)) * a[1:n - 1]
                  + (h_l / (h_r * (h_l + h_r))) * a[2:])
    return d


def band_masks(psi, coords):
    """_interface_band_mask and _normal_axis_masks (viscous_spatial.py:175-200):
    the band 1e-6 < psi < 1 - 1e-6 dilated by one node along each axis in
    turn; per axis, whether |d psi / dx_a| (low-order) is the largest."""
    p = np.asarray(psi)
    band = (p > 1.0e-6) & (p < 1.0 - 1.0e-6)
    for ax in range(p.ndim):
        base = band.copy()
        lo = [slice(None)] * p.ndim
        hi = [slice(None)] * p.ndim
        lo[ax] = slice(1, None)
        hi[ax] = slice(None, -1)
        band[tuple(lo)] = band[tuple(lo)] | base[tuple(hi)]
        band[tuple(hi)] = band[tuple(hi)] | base[tuple(lo)]
    ag = [np.abs(low_order_derivative(p, ax, coords[ax])) for ax in range(p.ndim)]
    mx = ag[0]
    for g in ag[1:]:
        mx = np.maximum(mx, g)
    flat = mx <= 1.0e-14
    return band, [((g >= mx) & (mx > 1.0e-14)) | flat for g in ag]


def viscous(vel, mu, rho, Re: float, L, N, bc: str, scheme: str = "ccd_bulk", psi=None):
    nd = len(vel)
    kinds = axis_kinds(bc, nd)
    coords = [np.linspace(0.0, L[a], N[a] + 1) for a in range(nd)]
    h = [float(L[a] / N[a]) for a in range(nd)]
    D = lambda f, ax: np.asarray(occd.differentiate(f, ax, h[ax], bc=kinds[ax])[0])
    lo = lambda f, ax: low_order_derivative(f, ax, coords[ax])
    if psi is not None and scheme == "ccd_bulk":
        band, normal = band_masks(psi, coords)
        sw = lambda f, ax: np.where(normal[ax], lo(f, ax), D(f, ax))
        out = []
        for al in range(nd):
            total = np.zeros_like(vel[al])
            for be in range(nd):
                total += sw(mu * (sw(vel[al], be) + sw(vel[be], al)), be)
            lap = np.zeros_like(vel[al])
            for ax in range(nd):
                lap += np.asarray(occd.differentiate(vel[al], ax, h[ax], bc=kinds[ax])[1])
            out.append(np.where(band, total, mu * lap) / (Re * rho))
        return out
    out = []
    for al in range(nd):
        total = np.zeros_like(vel[al])
        for be in range(nd):
            if scheme == "conservative_stress":
                a, b = lo(vel[al], be), lo(vel[be], al)
                total += lo(mu * (a + b), be)
            elif scheme == "ccd_stress_legacy":
                a, b = D(vel[al], be), D(vel[be], al)
                total += D(mu * (a + b), be)
            else:
                a, b = D(vel[al], be), D(vel[be], al)
                total += lo(mu * (a + b), be)
        out.append(total / (Re * rho))
    return out


def cn_predictor(u_old, e, mu, rho, Re, L, N, bc, dt, cn_viscous=True, scheme="ccd_bulk"):
    """ViscousTerm.apply_cn_predictor (ns_terms/viscous.py:135-181) with the
    default PicardCNAdvance (time_integration/cn_advance/picard_cn.py:43-96)."""
    nd = len(u_old)
    vn = viscous(u_old, mu, rho, Re, L, N, bc, scheme)
    pred = [u_old[c] + dt * (e[c] / rho + vn[c]) for c in range(nd)]
    if not cn_viscous:
        return pred
    vs = viscous(pred, mu, rho, Re, L, N, bc, scheme)
    return [u_old[c] + dt * (e[c] / rho + 0.5 * vn[c] + 0.5 * vs[c]) for c in range(nd)]


def cn_predictor_richardson(u_old, e, mu, rho, Re, L, N, bc, dt, scheme="ccd_bulk"):
    """ViscousTerm.apply_cn_predictor with RichardsonCNAdvance(PicardCNAdvance)
    (time_integration/cn_advance/richardson_cn.py:76-109): one Picard step of
    dt, two of dt/2 with the explicit right-hand side frozen, then
    (4 u_{dt/2,2} - u_dt) / 3."""
    u1 = cn_predictor(u_old, e, mu, rho, Re, L, N, bc, dt, True, scheme)
    uh = cn_predictor(u_old, e, mu, rho, Re, L, N, bc, 0.5 * dt, True, scheme)
    u2 = cn_predictor(uh, e, mu, rho, Re, L, N, bc, 0.5 * dt, True, scheme)
    return [(4.0 * u2[c] - u1[c]) / 3.0 for c in range(len(u_old))]


def predictor_steps(states, dts, Re, Fr, We, L, N, bc, cn_viscous=True, use_gfm=False):
    """Predictor.compute called once per state in turn (ab2_predictor.py:110-209):
    AB2 convection (forward Euler first), gravity, CSF, IPC, viscous predictor."""
    nd = len(N)
    kinds = axis_kinds(bc, nd)
    h = [float(L[a] / N[a]) for a in range(nd)]
    D = lambda f, ax: np.asarray(occd.differentiate(f, ax, h[ax], bc=kinds[ax])[0])
    prev = None
    outs = []
    for st, dt in zip(states, dts):
        vel, rho, mu, kappa, psi, p = st
        conv = []
        for c in range(nd):
            acc = np.zeros_like(vel[c])
            for ax in range(nd):
                acc -= vel[ax] * D(vel[c], ax)
            conv.append(acc)
        ab2 = [1.5 * conv[c] - 0.5 * prev[c] for c in range(nd)] if prev is not None else conv
        grav = [np.zeros(rho.shape) for _ in range(nd)]
        grav[nd - 1] = -rho / (Fr ** 2)
        stf = [np.zeros_like(vel[c]) for c in range(nd)] if use_gfm else [kappa * D(psi, ax) / We for ax in range(nd)]
        gp = []
        for ax in range(nd):
            g = D(p, ax).copy()
            if kinds[ax] == "wall":
                lo = [slice(None)] * nd
                hi = [slice(None)] * nd
                lo[ax] = 0
                hi[ax] = -1
                g[tuple(lo)] = 0.0
                g[tuple(hi)] = 0.0
            gp.append(g)
        e = [rho * ab2[c] + grav[c] + stf[c] + (-gp[c]) for c in range(nd)]
        if cn_viscous:
            u = cn_predictor(vel, e, mu, rho, Re, L, N, bc, dt, True)
        else:
            v = viscous(vel, mu, rho, Re, L, N, bc)
            u = [vel[c] + dt * (e[c] + rho * v[c]) / rho for c in range(nd)]
        outs.append(u)
        prev = [c.copy() for c in conv]
    return outs
