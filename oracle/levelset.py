"""CPU restatement of the interface geometry and material properties from the
CLS field psi (TEST INFRASTRUCTURE: the oracle).

* ``dccd_filter_nd`` -- the 3-point DCCD dissipative filter applied along every
  axis in turn, wall planes restored afterwards (reference
  ``src/twophase/levelset/curvature.py:60-127``).
* ``curvature_psi`` -- kappa straight from psi (reference
  ``src/twophase/levelset/curvature_psi.py:72-173``) on the oracle's CCD.
* ``gaussian3x3`` -- the optional 2-D smoothing (curvature_psi.py:176-197).
* ``update_properties`` -- rho and mu from psi (heaviside.py:167-187).

Pinned against the reference's own outputs in ``tests/golden/levelset_golden.npz``.
Only tests, smoke() and bench.py's CPU-baseline leg may use this module.
"""

from __future__ import annotations

import numpy as np

from . import ccd as occd

EPS_GRAD = 1e-30


def axis_kinds(bc: str, ndim: int):
    if bc == "wall":
        return ["wall"] * ndim
    if bc == "periodic":
        return ["periodic"] * ndim
    if bc == "periodic_wall" and ndim == 2:
        return ["periodic", "wall"]
    if bc == "wall_periodic" and ndim == 2:
        return ["wall", "periodic"]
    raise ValueError(f"unknown boundary type {bc!r}")


def _filter_axis(f, ax: int, coeff, periodic: bool):
    """One axis of the filter (curvature.py:60-102): nodes 1..N-1 on a wall
    axis; the N unique nodes with wrap-around on a periodic one, the image node
    N taking node 0's result."""
    fa = np.moveaxis(f, ax, 0)
    ca = np.moveaxis(np.broadcast_to(coeff, f.shape), ax, 0)
    res = fa.copy()
    N = fa.shape[0] - 1
    if periodic:
        u = fa[:N]
        res[:N] = u + ca[:N] * ((np.roll(u, -1, axis=0) - 2.0 * u) + np.roll(u, 1, axis=0))
        res[N] = res[0]
    else:
        c = fa[1:N]
        res[1:N] = c + ca[1:N] * ((fa[2:N + 1] - 2.0 * c) + fa[0:N - 1])
    return np.moveaxis(res, 0, ax)


def dccd_filter_nd(f, eps: float, bc: str = "wall", switch=None):
    """curvature.py:105-127."""
    f = np.asarray(f, dtype=np.float64)
    kinds = axis_kinds(bc, f.ndim)
    coeff = eps if switch is None else eps * np.asarray(switch)
    out = f
    for ax in range(f.ndim):
        out = _filter_axis(out, ax, coeff, kinds[ax] == "periodic")
    out = np.array(out, copy=True)
    for ax in range(f.ndim):
        if kinds[ax] == "periodic":
            continue
        lo = [slice(None)] * f.ndim
        hi = [slice(None)] * f.ndim
        lo[ax] = 0
        hi[ax] = -1
        out[tuple(lo)] = f[tuple(lo)]
        out[tuple(hi)] = f[tuple(hi)]
    return out


def gaussian3x3(k):
    """[1 2 1; 2 4 2; 1 2 1] / 16 with edge replication (curvature_psi.py:176-197)."""
    p = np.pad(np.asarray(k), 1, mode="edge")
    w = ((1.0, 2.0, 1.0), (2.0, 4.0, 2.0), (1.0, 2.0, 1.0))
    n0, n1 = k.shape
    r = None
    for dy in range(3):
        for dx in range(3):
            term = w[dy][dx] * p[dy:dy + n0, dx:dx + n1]
            r = term if r is None else r + term
    return r / 16.0


def curvature_psi(psi, h, bc: str = "wall", psi_min: float = 0.01, gaussian_filter: bool = False,
                  dccd_eps: float = 0.05):
    """CurvatureCalculatorPsi.compute (curvature_psi.py:72-173) with the oracle CCD;
    h: cell size per axis."""
    psi = np.asarray(psi, dtype=np.float64)
    nd = psi.ndim
    kinds = axis_kinds(bc, nd)

    def D(f, ax):
        return occd.differentiate(f, ax, h[ax], bc=kinds[ax])

    sw = (2.0 * psi - 1.0) ** 2 if dccd_eps > 0 else None

    def F(g):
        return dccd_filter_nd(g, dccd_eps, bc, sw) if dccd_eps > 0 else np.asarray(g)

    d1, d2 = [], []
    for ax in range(nd):
        g1, g2 = D(psi, ax)
        d1.append(F(g1))
        d2.append(F(g2))
    gsq = d1[0] * d1[0]
    for a in range(1, nd):
        gsq = gsq + d1[a] * d1[a]
    if nd == 2:
        pxy = F(D(d1[0], 1)[0])
        px, py = d1
        num = ((py * py) * d2[0] - ((2.0 * px) * py) * pxy) + (px * px) * d2[1]
        kappa = -num / (gsq + EPS_GRAD) ** 1.5
    else:
        lap = (d2[0] + d2[1]) + d2[2]
        con = (d1[0] * d1[0]) * d2[0]
        con = con + (d1[1] * d1[1]) * d2[1]
        con = con + (d1[2] * d1[2]) * d2[2]
        for i in range(3):
            for j in range(i + 1, 3):
                con = con + ((2.0 * d1[i]) * d1[j]) * D(d1[i], j)[0]
        gs = gsq + EPS_GRAD
        kappa = -(lap - con / gs) / np.sqrt(gs)
    kappa = np.array(kappa, copy=True)
    kappa[(psi <= psi_min) | (psi >= 1.0 - psi_min)] = 0.0
    if gaussian_filter and nd == 2:
        kappa = gaussian3x3(kappa)
    return kappa


def update_properties(psi, rho_l: float, rho_g: float, mu_l: float, mu_g: float):
    """heaviside.py:167-187."""
    psi = np.asarray(psi)
    return rho_g + (rho_l - rho_g) * psi, mu_g + (mu_l - mu_g) * psi
