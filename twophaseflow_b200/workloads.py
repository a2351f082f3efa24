"""Seeded synthetic inputs for the CCD and PPE workloads.

These restate, with NumPy generators, the input recipes of the benchmark cases:

* CCD field: f = sum_{m<32} a_m prod_d cos(2 pi k_{m,d} x_d + phi_{m,d}),
  k uniform in 1..64, a_m ~ N(0,1)/|k|^2, phi ~ U(0, 2 pi), on the node-centred
  grid x = linspace(0, L, N+1) (the reference's grid, tp/core/grid.py:62-66).
* PPE density: 12 non-overlapping liquid droplets (radii U[0.02, 0.08], gap
  0.02, rejection-sampled) in gas, psi = 1/(1+exp(phi/eps)) with eps = 1.5 h,
  rho = rho_g + (rho_l - rho_g) psi (the CLS mixing rule of
  tp/levelset/heaviside.py:167-187).
* PPE right-hand side: divergence of a smooth 8-mode seeded velocity field.

No public dataset is involved; everything is generated from a seed.
"""

from __future__ import annotations

import numpy as np


def node_coords(N, L=None):
    L = L if L is not None else (1.0,) * len(N)
    return [np.linspace(0.0, float(l), int(n) + 1) for n, l in zip(N, L)]


def fourier_modes(ndim: int, n_modes: int = 32, kmax: int = 64, seed: int = 0):
    rng = np.random.default_rng(seed)
    k = rng.integers(1, kmax + 1, size=(n_modes, ndim))
    knorm2 = np.sum(k.astype(np.float64) ** 2, axis=1)
    amp = rng.standard_normal(n_modes) / knorm2
    phase = rng.uniform(0.0, 2.0 * np.pi, size=(n_modes, ndim))
    return k, amp, phase


def fourier_field(N, L=None, n_modes: int = 32, kmax: int = 64, seed: int = 0,
                  deriv_axis: int | None = None, dtype=np.float64):
    """Field (and optionally its exact first and second derivative along
    ``deriv_axis``) on the (N+1)^d node grid."""
    ndim = len(N)
    L = L if L is not None else (1.0,) * ndim
    coords = node_coords(N, L)
    k, amp, phase = fourier_modes(ndim, n_modes, kmax, seed)
    shape = tuple(int(n) + 1 for n in N)
    f = np.zeros(shape)
    d1 = np.zeros(shape) if deriv_axis is not None else None
    d2 = np.zeros(shape) if deriv_axis is not None else None
    for m in range(n_modes):
        facs, dfacs, d2facs = [], [], []
        for d in range(ndim):
            w = 2.0 * np.pi * k[m, d] / L[d]
            arg = w * coords[d] + phase[m, d]
            bshape = [1] * ndim
            bshape[d] = -1
            facs.append(np.cos(arg).reshape(bshape))
            if deriv_axis == d:
                dfacs.append((-w * np.sin(arg)).reshape(bshape))
                d2facs.append((-w * w * np.cos(arg)).reshape(bshape))
        term = amp[m]
        for d in range(ndim):
            term = term * facs[d]
        f += term
        if deriv_axis is not None:
            t1 = amp[m]
            t2 = amp[m]
            for d in range(ndim):
                if d == deriv_axis:
                    t1 = t1 * dfacs[0]
                    t2 = t2 * d2facs[0]
                else:
                    t1 = t1 * facs[d]
                    t2 = t2 * facs[d]
            d1 += t1
            d2 += t2
    f = f.astype(dtype)
    if deriv_axis is None:
        return f
    return f, d1, d2


def droplet_centres(ndim: int = 2, n_drops: int = 12, rmin: float = 0.02,
                    rmax: float = 0.08, gap: float = 0.02, seed: int = 0,
                    max_tries: int = 100000):
    rng = np.random.default_rng(seed)
    centres, radii = [], []
    tries = 0
    while len(centres) < n_drops:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("droplet rejection sampling did not finish")
        r = rng.uniform(rmin, rmax)
        c = rng.uniform(r + gap, 1.0 - r - gap, size=ndim)
        ok = all(np.linalg.norm(c - c2) >= r + r2 + gap for c2, r2 in zip(centres, radii))
        if ok:
            centres.append(c)
            radii.append(r)
    return np.array(centres), np.array(radii)


def droplet_density(N, n_drops: int = 12, rho_l: float = 1.0, rho_g: float = 1e-3,
                    eps_factor: float = 1.5, seed: int = 0):
    """Density of ``n_drops`` liquid droplets in gas on the unit box."""
    ndim = len(N)
    coords = node_coords(N)
    h = 1.0 / float(max(N))
    eps = eps_factor * h
    centres, radii = droplet_centres(ndim, n_drops, seed=seed)
    grids = np.meshgrid(*coords, indexing="ij")
    phi = np.full(grids[0].shape, np.inf)
    for c, r in zip(centres, radii):
        dist = np.sqrt(sum((g - cc) ** 2 for g, cc in zip(grids, c))) - r
        phi = np.minimum(phi, dist)
    psi = 1.0 / (1.0 + np.exp(np.clip(phi / eps, -700.0, 700.0)))
    return rho_g + (rho_l - rho_g) * psi


def bubble_density(N, centre=(0.5, 0.5), radius: float = 0.25, rho_l: float = 1.0,
                   rho_g: float = 0.1, eps_factor: float = 1.5):
    """Single gas bubble (psi ~ 0 inside) in liquid: the rising-bubble layout."""
    coords = node_coords(N)
    grids = np.meshgrid(*coords, indexing="ij")
    h = 1.0 / float(max(N))
    eps = eps_factor * h
    r = np.sqrt(sum((g - c) ** 2 for g, c in zip(grids, centre)))
    psi = 1.0 / (1.0 + np.exp(-np.clip((r - radius) / eps, -700.0, 700.0)))
    return rho_g + (rho_l - rho_g) * psi


def quickstart_psi(N=(64, 64), centre=(0.5, 0.5), radius: float = 0.25, eps_factor: float = 1.5):
    """CLS field of the quick-start rising bubble: a gas bubble (psi ~ 0
    inside) of radius 0.25 at the box centre, psi = 1/(1+exp(-(r-R)/eps)) with
    eps = 1.5 h on the unit box (the reference's quick-start initial state)."""
    coords = node_coords(N)
    grids = np.meshgrid(*coords, indexing="ij")
    eps = eps_factor / float(max(N))
    r = np.sqrt(sum((g - c) ** 2 for g, c in zip(grids, centre)))
    return 1.0 / (1.0 + np.exp(-(r - radius) / eps))


def divergence_rhs(N, n_modes: int = 8, seed: int = 1):
    """rhs = div u for u_d = sum_m a_{m,d} prod_e sin/cos(pi k_{m,e} x_e + phi)."""
    ndim = len(N)
    rng = np.random.default_rng(seed)
    coords = node_coords(N)
    grids = np.meshgrid(*coords, indexing="ij")
    rhs = np.zeros(grids[0].shape)
    for _m in range(n_modes):
        k = rng.integers(1, 9, size=ndim).astype(np.float64)
        phase = rng.uniform(0.0, 2.0 * np.pi, size=ndim)
        amp = rng.standard_normal(ndim)
        for d in range(ndim):
            # u_d = amp_d * sin(pi k_d x_d + phase_d) * prod_{e != d} cos(pi k_e x_e + phase_e)
            term = amp[d] * np.pi * k[d] * np.cos(np.pi * k[d] * grids[d] + phase[d])
            for e in range(ndim):
                if e != d:
                    term = term * np.cos(np.pi * k[e] * grids[e] + phase[e])
            rhs += term
    return rhs
