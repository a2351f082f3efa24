"""CPU restatement of the reference CCD operator (TEST INFRASTRUCTURE: the oracle).

Follows ``src/twophase/ccd/ccd_solver.py`` and ``ccd_solver_helpers.py`` of the
reference: the wall-bounded axis is solved as one dense (2(N-1))^2 system with
pivoted LU (LAPACK getrf/getrs), the periodic axis as one dense 2N x 2N
block-circulant system, exactly as the reference's CPU path does.  Also holds the
unpivoted 2x2 block-LU restatement (``block_tridiag.py``) that the CUDA line
kernels implement, so that the two factorizations can be compared on the CPU.

Only tests, smoke() and bench.py's CPU-baseline leg may use this module.
"""

from __future__ import annotations

import numpy as np
import scipy.linalg as sla

# Interior coefficients, Table 1 of the CCD scheme
# (reference src/twophase/ccd/ccd_solver.py:70-76).
ALPHA1 = 7.0 / 16.0
A1 = 15.0 / 16.0
B1 = 1.0 / 16.0
BETA2 = -1.0 / 8.0
A2 = 3.0
B2 = -9.0 / 8.0


def lower_block(h: float) -> np.ndarray:
    """Coupling of node i to node i-1 (ccd_solver_helpers.py:235,239)."""
    return np.array([[ALPHA1, B1 * h], [B2 / h, BETA2]])


def upper_block(h: float) -> np.ndarray:
    """Coupling of node i to node i+1 (ccd_solver_helpers.py:236,240)."""
    return np.array([[ALPHA1, -B1 * h], [-B2 / h, BETA2]])


def boundary_coeffs(h: float, n_pts: int, side: str) -> dict:
    """Wall closure [f'_b; f''_b] = M [f'_nb; f''_nb] + [c_I.f ; c_II.f].

    Reference: ccd_solver.py:408-465 (_boundary_coeffs_left/right and the
    n_pts >= 6 requirement of the six-point Eq-II closure).
    """
    if n_pts < 6:
        raise ValueError(
            "CCD wall Eq-II boundary closure requires n_pts >= 6 for the "
            "six-point O(h^4) formula"
        )
    c_II = np.array([45.0, -154.0, 214.0, -156.0, 61.0, -10.0]) / (12.0 * h * h)
    if side == "left":
        M = np.array([[-1.5, 1.5 * h], [0.0, 0.0]])
        c_I = np.array([-23.0 / 6.0, 21.0 / 4.0, -1.5, 1.0 / 12.0]) / h
    else:
        M = np.array([[-1.5, -1.5 * h], [0.0, 0.0]])
        c_I = np.array([23.0 / 6.0, -21.0 / 4.0, 1.5, -1.0 / 12.0]) / h
    return {"M": M, "c_I": c_I, "c_II": c_II}


def wall_blocks(n_pts: int, h: float):
    """Block rows of the folded interior system (ccd_solver_helpers.py:227-245).

    Returns (diag, lower, upper) lists of n_int = N-1 (2,2) blocks with the
    boundary closure folded into the first/last diagonal blocks.
    """
    N = n_pts - 1
    n_int = N - 1
    bl = boundary_coeffs(h, n_pts, "left")
    br = boundary_coeffs(h, n_pts, "right")
    Lb, Ub = lower_block(h), upper_block(h)
    diag = [np.eye(2) for _ in range(n_int)]
    lower = [Lb.copy() for _ in range(n_int)]
    upper = [Ub.copy() for _ in range(n_int)]
    diag[0] = diag[0] + lower[0] @ bl["M"]
    lower[0] = np.zeros((2, 2))
    diag[-1] = diag[-1] + upper[-1] @ br["M"]
    upper[-1] = np.zeros((2, 2))
    return diag, lower, upper


def wall_dense_matrix(n_pts: int, h: float) -> np.ndarray:
    """Dense A of the interior system (ccd_solver_helpers.py:247-253)."""
    diag, lower, upper = wall_blocks(n_pts, h)
    n_int = len(diag)
    A = np.zeros((2 * n_int, 2 * n_int))
    for i in range(n_int):
        A[2 * i:2 * i + 2, 2 * i:2 * i + 2] = diag[i]
        if i >= 1:
            A[2 * i:2 * i + 2, 2 * (i - 1):2 * i] = lower[i]
        if i <= n_int - 2:
            A[2 * i:2 * i + 2, 2 * (i + 1):2 * (i + 2)] = upper[i]
    return A


class WallAxis:
    """Per-axis wall solver state (ccd_solver_helpers.py:227-314, CPU branch)."""

    def __init__(self, n_pts: int, h: float):
        self.n_pts = int(n_pts)
        self.N = self.n_pts - 1
        self.n_int = self.N - 1
        self.h = float(h)
        self.bl = boundary_coeffs(h, n_pts, "left")
        self.br = boundary_coeffs(h, n_pts, "right")
        self.L0 = lower_block(h)
        self.UN = upper_block(h)
        self.lu, self.piv = sla.lu_factor(wall_dense_matrix(n_pts, h))


def _to_lines(data, axis):
    f = np.moveaxis(np.asarray(data, dtype=np.float64), axis, 0)
    shape = f.shape
    return f.reshape(shape[0], -1), shape


def _from_lines(flat, shape, axis):
    return np.moveaxis(flat.reshape(shape), 0, axis)


def differentiate_wall(data, axis: int, h: float, bc_left=None, bc_right=None,
                       solver: WallAxis | None = None):
    """Wall-bounded CCD along ``axis`` (ccd_solver_helpers.py:38-77 and
    ccd_boundary_helpers.py:64-116).  Returns (d1, d2) in the input layout."""
    f, shape = _to_lines(data, axis)
    n_pts = f.shape[0]
    s = solver if solver is not None else WallAxis(n_pts, h)
    N, n_int, h = s.N, s.n_int, s.h
    batch = f.shape[1]
    fm, f0, fp = f[0:n_int], f[1:n_int + 1], f[2:n_int + 2]
    rhs = np.empty((n_int, 2, batch))
    rhs[:, 0, :] = (A1 / h) * (fp - fm)
    rhs[:, 1, :] = (A2 / (h * h)) * (fm - 2.0 * f0 + fp)
    if bc_left is not None:
        bc_lo = np.empty((2, batch))
        bc_lo[0] = float(bc_left[0])
        bc_lo[1] = float(bc_left[1])
    else:
        bc_lo = np.stack([s.bl["c_I"] @ f[:4], s.bl["c_II"] @ f[:6]])
    if bc_right is not None:
        bc_hi = np.empty((2, batch))
        bc_hi[0] = float(bc_right[0])
        bc_hi[1] = float(bc_right[1])
    else:
        f_rev = f[N::-1]
        bc_hi = np.stack([s.br["c_I"] @ f_rev[:4], s.br["c_II"] @ f_rev[:6]])
    rhs[0] -= s.L0 @ bc_lo
    rhs[-1] -= s.UN @ bc_hi
    x = sla.lu_solve((s.lu, s.piv), rhs.reshape(2 * n_int, -1))
    sol = x.reshape(n_int, 2, -1)
    out = np.empty((2, n_pts, batch))
    out[:, 1:-1, :] = sol.transpose(1, 0, 2)
    out[:, 0, :] = s.bl["M"] @ out[:, 1, :] + bc_lo
    out[:, N, :] = s.br["M"] @ out[:, N - 1, :] + bc_hi
    return _from_lines(out[0], shape, axis), _from_lines(out[1], shape, axis)


def periodic_dense_matrix(N: int, h: float) -> np.ndarray:
    """Block-circulant 2N x 2N system, interleaved [f'_0, f''_0, f'_1, ...]
    (ccd_solver_helpers.py:406-423)."""
    Lb, Ub = lower_block(h), upper_block(h)
    A = np.zeros((2 * N, 2 * N))
    for i in range(N):
        A[2 * i:2 * i + 2, 2 * i:2 * i + 2] += np.eye(2)
        j = (i - 1) % N
        A[2 * i:2 * i + 2, 2 * j:2 * j + 2] += Lb
        j = (i + 1) % N
        A[2 * i:2 * i + 2, 2 * j:2 * j + 2] += Ub
    return A


def differentiate_periodic(data, axis: int, h: float):
    """Periodic CCD along ``axis`` (ccd_solver_helpers.py:426-465): unique nodes
    0..N-1, dense LU solve, image node N <- node 0."""
    f_full, shape = _to_lines(data, axis)
    N = f_full.shape[0] - 1
    if N < 3:
        raise ValueError("periodic CCD needs >= 3 unique nodes")
    fu = f_full[:N]
    fm = np.roll(fu, 1, axis=0)
    fp = np.roll(fu, -1, axis=0)
    rhs = np.empty((2 * N, fu.shape[1]))
    rhs[0::2] = (A1 / h) * (fp - fm)
    rhs[1::2] = (A2 / (h * h)) * (fm - 2.0 * fu + fp)
    lu, piv = sla.lu_factor(periodic_dense_matrix(N, h))
    x = sla.lu_solve((lu, piv), rhs)
    d1 = np.empty_like(f_full)
    d2 = np.empty_like(f_full)
    d1[:N] = x[0::2]
    d2[:N] = x[1::2]
    d1[N] = d1[0]
    d2[N] = d2[0]
    return _from_lines(d1, shape, axis), _from_lines(d2, shape, axis)


def apply_metric(d1_xi, d2_xi, axis: int, J, dJ):
    """Non-uniform map d1_x = J d1_xi, d2_x = J^2 d2_xi + J J' d1_xi
    (ccd_solver_helpers.py:509-519)."""
    ndim = np.ndim(d1_xi)
    shape = [1] * ndim
    shape[axis] = -1
    Jb = np.asarray(J, dtype=np.float64).reshape(shape)
    dJb = np.asarray(dJ, dtype=np.float64).reshape(shape)
    return Jb * d1_xi, Jb * Jb * d2_xi + Jb * dJb * d1_xi


def differentiate(data, axis: int, h: float, bc: str = "wall", bc_left=None,
                  bc_right=None, J=None, dJ=None):
    """Public dispatch of CCDSolver.differentiate (ccd_solver.py:134-172)."""
    if bc == "periodic" and bc_left is None and bc_right is None:
        d1, d2 = differentiate_periodic(data, axis, h)
    else:
        d1, d2 = differentiate_wall(data, axis, h, bc_left, bc_right)
    if J is not None:
        d1, d2 = apply_metric(d1, d2, axis, J, dJ)
    return d1, d2


# ── Unpivoted 2x2 block LU (reference block_tridiag.py:43-164) ─────────────

def block_lu_factor(diag, lower, upper):
    """Block-Thomas factorization; raises on |det| < 1e-300 or non-finite
    pivots (block_tridiag.py:67-104, 167-174)."""
    n = len(diag)
    LU = [None] * n
    Lf = [np.zeros((2, 2)) for _ in range(n)]
    LU[0] = np.array(diag[0], dtype=np.float64)
    _require_pivot(LU[0], 0)
    for i in range(1, n):
        Lf[i] = np.linalg.solve(LU[i - 1].T, np.asarray(lower[i]).T).T
        LU[i] = diag[i] - Lf[i] @ upper[i - 1]
        _require_pivot(LU[i], i)
    return np.stack(LU), np.stack(Lf), np.stack([np.asarray(u) for u in upper])


def block_lu_solve(factors, rhs):
    """Forward/back substitution with Cramer 2x2 solves (block_tridiag.py:108-164).
    rhs: (n, 2, batch)."""
    LU, Lf, U = factors
    n = LU.shape[0]
    y = np.empty_like(rhs)
    y[0] = rhs[0]
    for i in range(1, n):
        y[i] = rhs[i] - Lf[i] @ y[i - 1]
    x = np.empty_like(rhs)
    x[n - 1] = _solve2x2(LU[n - 1], y[n - 1])
    for i in range(n - 2, -1, -1):
        x[i] = _solve2x2(LU[i], y[i] - U[i] @ x[i + 1])
    return x


def _solve2x2(A, b):
    det = A[0, 0] * A[1, 1] - A[0, 1] * A[1, 0]
    inv = 1.0 / det
    x = np.empty_like(b)
    x[0] = inv * (A[1, 1] * b[0] - A[0, 1] * b[1])
    x[1] = inv * (A[0, 0] * b[1] - A[1, 0] * b[0])
    return x


def _require_pivot(A, index):
    det = float(A[0, 0] * A[1, 1] - A[0, 1] * A[1, 0])
    if not np.isfinite(det) or abs(det) < 1e-300:
        raise np.linalg.LinAlgError(
            f"CCD block-tridiagonal factorization encountered a singular pivot at block {index}")
