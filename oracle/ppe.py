"""CPU restatement of the reference variable-density FVM PPE (TEST INFRASTRUCTURE:
the oracle).

Follows ``src/twophase/ppe/fvm_matrixfree.py`` / ``fvm_matrixfree_helpers.py``
(matrix-free operator, Jacobi and shifted line preconditioners, CG on the
control-volume-weighted SPD system, left-preconditioned GMRES),
``src/twophase/linalg_backend.py`` (Thomas on CPU, truncated PCR on GPU),
``src/twophase/ppe/ppe_builder_helpers.py`` + ``fvm_spsolve.py`` (assembled CSR
+ direct solve), ``src/twophase/ppe/ccd_ppe_utils.py`` (CCD variable-density
operator L_H) and ``src/twophase/ppe/defect_correction.py`` (outer DC loop).

The Krylov loops restate SciPy 1.18.1 ``scipy.sparse.linalg.cg`` and ``gmres``
(third-party code the reference calls through ``tp/ppe/gmres_helpers.py:16-80``);
``lartg`` is LAPACK's Givens generator obtained through SciPy, as SciPy does.

Only tests, smoke() and bench.py's CPU-baseline leg may use this module.
"""

from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla
from scipy.linalg import get_lapack_funcs

from . import ccd as occd


def _sl(axis, start, stop, ndim):
    s = [slice(None)] * ndim
    s[axis] = slice(start, stop)
    return tuple(s)


def pin_dof(N) -> int:
    """Wall pin = ravel index of (N//2, ...) (tp/core/boundary.py:182-191)."""
    return int(np.ravel_multi_index(tuple(n // 2 for n in N), tuple(n + 1 for n in N)))


def uniform_coords(N, L):
    """Node coordinates linspace(0, L, N+1) (tp/core/grid.py:62-66)."""
    return [np.linspace(0.0, float(l), int(n) + 1) for n, l in zip(N, L)]


def grid_metrics(coords):
    """h_min, face widths, node control-volume widths
    (fvm_matrixfree_helpers.py:23-43)."""
    ndim = len(coords)
    h_min = min(float(np.min(np.diff(np.asarray(c)))) for c in coords)
    d_face, dv_node = [], []
    for axis in range(ndim):
        c = np.asarray(coords[axis], dtype=np.float64)
        d = c[1:] - c[:-1]
        dv = np.empty_like(c)
        dv[0] = d[0] / 2.0
        dv[-1] = d[-1] / 2.0
        dv[1:-1] = (c[2:] - c[:-2]) / 2.0
        fs = [1] * ndim
        ns = [1] * ndim
        fs[axis] = d.size
        ns[axis] = dv.size
        d_face.append(d.reshape(fs))
        dv_node.append(dv.reshape(ns))
    return h_min, d_face, dv_node


def line_coeffs(rho, axis, d_face, dv_node):
    """(lower, main, upper) of one axis (fvm_matrixfree_helpers.py:46-73)."""
    ndim = rho.ndim
    n_axis = rho.shape[axis] - 1
    lower = np.zeros_like(rho)
    main = np.zeros_like(rho)
    upper = np.zeros_like(rho)
    rho_lo = rho[_sl(axis, 0, n_axis, ndim)]
    rho_hi = rho[_sl(axis, 1, n_axis + 1, ndim)]
    cf = 2.0 / (rho_lo + rho_hi) / d_face[axis]
    upper[_sl(axis, 0, n_axis, ndim)] = cf / dv_node[axis][_sl(axis, 0, n_axis, ndim)]
    lower[_sl(axis, 1, n_axis + 1, ndim)] = cf / dv_node[axis][_sl(axis, 1, n_axis + 1, ndim)]
    main[...] = -(lower + upper)
    return lower, main, upper


def apply(p, coeffs, pin):
    """Pinned matrix-free operator (fvm_matrixfree.py:281-300)."""
    ndim = p.ndim
    out = np.zeros_like(p)
    for axis, (lower, main, upper) in enumerate(coeffs):
        n = p.shape[axis] - 1
        out += main * p
        out[_sl(axis, 1, n + 1, ndim)] += lower[_sl(axis, 1, n + 1, ndim)] * p[_sl(axis, 0, n, ndim)]
        out[_sl(axis, 0, n, ndim)] += upper[_sl(axis, 0, n, ndim)] * p[_sl(axis, 1, n + 1, ndim)]
    out.ravel()[pin] = p.ravel()[pin]
    return out


def jacobi_diag_inv(coeffs, pin):
    """Jacobi state (fvm_matrixfree_helpers.py:95-103)."""
    diag = np.zeros_like(coeffs[0][1])
    for _lo, main, _up in coeffs:
        diag += main
    diag.ravel()[pin] = 1.0
    return 1.0 / np.where(np.abs(diag) > 1e-30, diag, 1.0)


def line_precond_coeffs(coeffs, rho, c_tau, h_min):
    """Shifted line coefficients (-lower, shift - main, -upper) with
    shift = 2/(c_tau rho h_min^2) (fvm_matrixfree_helpers.py:85-94)."""
    shift = 2.0 / (c_tau * rho * (h_min ** 2))
    return [(-lo, shift - m, -up) for lo, m, up in coeffs]


def thomas_variable(lower, diag, upper, rhs, axis):
    """CPU branch of tridiag_variable_batched (linalg_backend.py:444-514)."""
    n = rhs.shape[axis]
    mv = lambda a: np.moveaxis(a, axis, 0).reshape(n, -1)
    lo, d, up, b = mv(lower), mv(diag), mv(upper), mv(rhs)
    dp = np.empty_like(b)
    cp = np.empty_like(up)
    dp[0] = b[0] / d[0]
    if n > 1:
        cp[0] = up[0] / d[0]
    for i in range(1, n):
        den = d[i] - lo[i] * cp[i - 1]
        if i < n - 1:
            cp[i] = up[i] / den
        dp[i] = (b[i] - lo[i] * dp[i - 1]) / den
    x = np.empty_like(b)
    x[n - 1] = dp[n - 1]
    for i in range(n - 2, -1, -1):
        x[i] = dp[i] - cp[i] * x[i + 1]
    moved = np.moveaxis(rhs, axis, 0)
    return np.moveaxis(x.reshape(moved.shape), 0, axis)


def pcr_variable(lower, diag, upper, rhs, axis, max_stages=None):
    """GPU branch: PCR truncated to ``max_stages`` (linalg_backend.py:251-337)."""
    n = rhs.shape[axis]
    mv = lambda a: np.moveaxis(a, axis, 0).reshape(n, -1).copy()
    lo, d, up, b = mv(lower), mv(diag), mv(upper), mv(rhs)
    stages = max(1, math.ceil(math.log2(n)))
    if max_stages is not None:
        stages = min(stages, max(1, int(max_stages)))
    idx = np.arange(n)
    stride = 1
    for _ in range(stages):
        dl = np.roll(d, stride, 0); ul = np.roll(up, stride, 0)
        ll = np.roll(lo, stride, 0); bl = np.roll(b, stride, 0)
        dr = np.roll(d, -stride, 0); lr = np.roll(lo, -stride, 0)
        ur = np.roll(up, -stride, 0); br = np.roll(b, -stride, 0)
        has_l = (idx >= stride)[:, None]
        dls = np.where(np.abs(dl) > 0, dl, 1.0)
        alpha = np.where(has_l, -lo / dls, 0.0)
        has_r = (idx < n - stride)[:, None]
        drs = np.where(np.abs(dr) > 0, dr, 1.0)
        beta = np.where(has_r, -up / drs, 0.0)
        lo = alpha * ll
        d = d + alpha * ul + beta * lr
        up = beta * ur
        b = b + alpha * bl + beta * br
        stride *= 2
    x = b / d
    moved = np.moveaxis(rhs, axis, 0)
    return np.moveaxis(x.reshape(moved.shape), 0, axis)


def line_precond(r, pcoeffs, pin, pcr_stages=None):
    """Additive shifted line preconditioner (fvm_matrixfree.py:302-323).
    ``pcr_stages=None`` is the CPU Thomas path; an int is the GPU PCR path."""
    rw = np.array(r, dtype=np.float64, copy=True)
    rw.ravel()[pin] = 0.0
    z = np.zeros_like(rw)
    for axis, (lo, d, up) in enumerate(pcoeffs):
        if pcr_stages is None:
            z += thomas_variable(lo, d, up, rw, axis)
        else:
            z += pcr_variable(lo, d, up, rw, axis, pcr_stages)
    z /= float(len(pcoeffs))
    z.ravel()[pin] = 0.0
    return z


# ── Krylov loops (SciPy 1.18.1 restated) ────────────────────────────────────

def cg(matvec, psolve, b, x0, rtol, maxiter):
    """scipy.sparse.linalg.cg (1.18.1) with atol=0: stop at ||r|| < rtol ||b||,
    checked at the top of every iteration.  Returns (x, info, iterations)."""
    bnrm2 = np.linalg.norm(b)
    atol = rtol * bnrm2
    if bnrm2 == 0:
        return b.copy(), 0, 0
    x = np.array(x0, dtype=np.float64, copy=True)
    r = b - matvec(x) if x.any() else b.copy()
    rho_prev, p = None, None
    for it in range(maxiter):
        if np.linalg.norm(r) < atol:
            return x, 0, it
        z = psolve(r)
        rho_cur = np.dot(r, z)
        if it > 0:
            p *= rho_cur / rho_prev
            p += z
        else:
            p = z.copy()
        q = matvec(p)
        alpha = rho_cur / np.dot(p, q)
        x += alpha * p
        r -= alpha * q
        rho_prev = rho_cur
    return x, maxiter, maxiter


def gmres(matvec, psolve, b, x0, rtol, restart, maxiter):
    """scipy.sparse.linalg.gmres (1.18.1), left preconditioned, modified
    Gram-Schmidt, LAPACK lartg Givens rotations, gh-8400 inner tolerance
    control; ``maxiter`` counts restart cycles.  Returns
    (x, info, inner_iterations)."""
    n = len(b)
    bnrm2 = np.linalg.norm(b)
    atol = rtol * bnrm2
    if bnrm2 == 0:
        return b.copy(), 0, 0
    x = np.array(x0, dtype=np.float64, copy=True)
    eps = np.finfo(np.float64).eps
    restart = min(restart, n)
    Mb_nrm2 = np.linalg.norm(psolve(b))
    ptol_max_factor = 1.0
    ptol = Mb_nrm2 * min(ptol_max_factor, atol / bnrm2)
    presid = 0.0
    lartg = get_lapack_funcs("lartg", dtype=x.dtype)
    v = np.empty([restart + 1, n])
    h = np.zeros([restart, restart + 1])
    givens = np.zeros([restart, 2])
    inner = 0
    rnorm = np.inf
    for iteration in range(maxiter):
        if iteration == 0:
            r = b - matvec(x) if x.any() else b.copy()
            if np.linalg.norm(r) < atol:
                return x, 0, inner
        v[0] = psolve(r)
        tmp = np.linalg.norm(v[0])
        v[0] *= 1 / tmp
        S = np.zeros(restart + 1)
        S[0] = tmp
        breakdown = False
        for col in range(restart):
            w = psolve(matvec(v[col]))
            h0 = np.linalg.norm(w)
            for k in range(col + 1):
                t = np.dot(v[k], w)
                h[col, k] = t
                w -= t * v[k]
            h1 = np.linalg.norm(w)
            h[col, col + 1] = h1
            v[col + 1] = w
            if h1 <= eps * h0:
                h[col, col + 1] = 0
                breakdown = True
            else:
                v[col + 1] *= 1 / h1
            for k in range(col):
                c, s = givens[k, 0], givens[k, 1]
                n0, n1 = h[col, [k, k + 1]]
                h[col, [k, k + 1]] = [c * n0 + s * n1, -s * n0 + c * n1]
            c, s, mag = lartg(h[col, col], h[col, col + 1])
            givens[col] = [c, s]
            h[col, [col, col + 1]] = mag, 0
            t = -s * S[col]
            S[[col, col + 1]] = [c * S[col], t]
            presid = abs(t)
            inner += 1
            if presid <= ptol or breakdown:
                break
        if h[col, col] == 0:
            S[col] = 0
        y = np.zeros([col + 1])
        y[:] = S[:col + 1]
        for k in range(col, 0, -1):
            if y[k] != 0:
                y[k] /= h[k, k]
                t = y[k]
                y[:k] -= t * h[k, :k]
        if y[0] != 0:
            y[0] /= h[0, 0]
        x += y @ v[:col + 1]
        r = b - matvec(x)
        rnorm = np.linalg.norm(r)
        if rnorm <= atol:
            break
        elif breakdown:
            break
        elif presid <= ptol:
            ptol_max_factor = max(eps, 0.25 * ptol_max_factor)
        else:
            ptol_max_factor = min(1.0, 1.5 * ptol_max_factor)
        ptol = presid * min(ptol_max_factor, atol / rnorm)
    info = 0 if rnorm <= atol else maxiter
    return x, info, inner


class FVMMatrixFree:
    """PPESolverFVMMatrixFree restated (fvm_matrixfree.py:46-363), wall BC."""

    def __init__(self, coords, method="gmres", preconditioner=None, tol=1e-8,
                 maxiter=500, restart=None, c_tau=2.0, pcr_stages=None, pin=None):
        self.coords = [np.asarray(c, dtype=np.float64) for c in coords]
        self.shape = tuple(c.size for c in self.coords)
        self.N = tuple(s - 1 for s in self.shape)
        self.ndim = len(self.shape)
        self.method = {"explicit": "gmres", "gauss_seidel": "gmres", "adi": "gmres"}.get(method, method)
        if self.method not in ("gmres", "cg"):
            raise ValueError(f"unsupported iteration method {method!r}")
        self.preconditioner = preconditioner or ("jacobi" if self.method == "cg" else "line_pcr")
        if self.method == "cg" and self.preconditioner == "line_pcr":
            raise ValueError("line_pcr is a nonsymmetric GMRES preconditioner")
        self.tol, self.maxiter, self.c_tau = float(tol), int(maxiter), float(c_tau)
        self.restart = int(restart) if restart is not None else min(80, max(20, self.maxiter))
        self.pcr_stages = pcr_stages
        self.pin = pin_dof(self.N) if pin is None else int(pin)
        self.h_min, self.d_face, self.dv_node = grid_metrics(self.coords)
        self.coeffs = None
        self.last_iterations = None

    def prepare_operator(self, rho):
        rho = np.asarray(rho, dtype=np.float64)
        self.coeffs = [line_coeffs(rho, a, self.d_face, self.dv_node) for a in range(self.ndim)]

    def apply(self, p):
        return apply(np.asarray(p, dtype=np.float64), self.coeffs, self.pin)

    def cv_weight(self):
        w = np.ones(self.shape)
        for dv in self.dv_node:
            w = w * dv
        return w

    def solve(self, rhs, rho, dt=0.0, p_init=None):
        """fvm_matrixfree.py:150-260."""
        rho = np.asarray(rho, dtype=np.float64)
        rhs = np.asarray(rhs, dtype=np.float64)
        pin, shape = self.pin, self.shape
        rhs_flat = rhs.ravel().copy()
        rhs_flat[pin] = 0.0
        W = self.cv_weight() if self.method == "cg" else None
        solve_rhs = -(rhs * W).ravel().copy() if self.method == "cg" else rhs_flat
        solve_rhs[pin] = 0.0
        self.prepare_operator(rho)
        diag_inv = pco = None
        if self.preconditioner == "jacobi":
            diag_inv = jacobi_diag_inv(self.coeffs, pin)
        elif self.preconditioner == "line_pcr":
            pco = line_precond_coeffs(self.coeffs, rho, self.c_tau, self.h_min)
        x0 = np.zeros_like(rhs_flat) if p_init is None else np.asarray(p_init, dtype=np.float64).ravel().copy()
        x0[pin] = 0.0

        def matvec(pf):
            pv = np.asarray(pf)
            if self.method == "cg":
                pv = pv.copy()
                pinned = pv[pin]
                pv[pin] = 0.0
            out = self.apply(pv.reshape(shape))
            of = out.ravel()
            if self.method == "cg":
                of = -(out * W).ravel()
                of[pin] = pinned
            return of

        def psolve(rf):
            rfield = np.asarray(rf).reshape(shape)
            if self.preconditioner == "jacobi":
                if self.method == "cg":
                    rfield = rfield / W
                z = rfield * diag_inv
                z.ravel()[pin] = 0.0
                if self.method == "cg":
                    z = -z
                    z.ravel()[pin] = np.asarray(rf)[pin]
            elif self.preconditioner == "line_pcr":
                z = line_precond(rfield, pco, pin, self.pcr_stages)
            else:
                z = rfield.copy()
            return z.ravel()

        if self.method == "cg":
            sol, info, its = cg(matvec, psolve, solve_rhs, x0, self.tol, self.maxiter)
        else:
            sol, info, its = gmres(matvec, psolve, solve_rhs, x0, self.tol, self.restart, self.maxiter)
        self.last_iterations = its
        self.last_info = info
        if info != 0:
            raise RuntimeError(f"FVMMatrixFree did not converge cleanly (info={info})")
        sol = sol.reshape(shape).copy()
        sol.ravel()[pin] = 0.0
        return sol


def assemble_csr(rho, coords, pin=None):
    """Assembled FVM matrix for a uniform wall grid (ppe_builder_helpers.py:50-122,
    264-311): face coefficient a_f/h^2, doubled on boundary faces' wall-side
    rows, pin row replaced by identity."""
    rho = np.asarray(rho, dtype=np.float64)
    shape = rho.shape
    ndim = rho.ndim
    N = tuple(s - 1 for s in shape)
    if pin is None:
        pin = pin_dof(N)
    n = rho.size
    idx = np.arange(n).reshape(shape)
    data, rows, cols = [], [], []
    for ax in range(ndim):
        Na = N[ax]
        h = float(coords[ax][-1] - coords[ax][0]) / Na
        iL = idx[_sl(ax, 0, Na, ndim)].ravel()
        iR = idx[_sl(ax, 1, Na + 1, ndim)].ravel()
        a_f = 2.0 / (rho.ravel()[iL] + rho.ravel()[iR])
        coeff = a_f / (h * h)
        axL = np.unravel_index(iL, shape)[ax]
        axR = np.unravel_index(iR, shape)[ax]
        cL = np.where(axL == 0, 2.0 * coeff, coeff)
        cR = np.where(axR == Na, 2.0 * coeff, coeff)
        data += [cL, cR, -cL, -cR]
        rows += [iL, iR, iL, iR]
        cols += [iR, iL, iL, iR]
    data = np.concatenate(data)
    rows = np.concatenate(rows)
    cols = np.concatenate(cols)
    keep = rows != pin
    data = np.concatenate([data[keep], [1.0]])
    rows = np.concatenate([rows[keep], [pin]])
    cols = np.concatenate([cols[keep], [pin]])
    return sp.csr_matrix((data, (rows, cols)), shape=(n, n))


def spsolve_fvm(rhs, rho, coords, pin=None):
    """PPESolverFVMSpsolve.solve (fvm_spsolve.py:117-161), CPU branch."""
    rho = np.asarray(rho, dtype=np.float64)
    N = tuple(s - 1 for s in rho.shape)
    if pin is None:
        pin = pin_dof(N)
    b = np.asarray(rhs, dtype=np.float64).ravel().copy()
    b[pin] = 0.0
    A = assemble_csr(rho, coords, pin)
    return spla.spsolve(A, b).reshape(rho.shape)


# ── CCD variable-density operator and defect correction ────────────────────

def ccd_laplacian(p, rho, drho, h):
    """L_H p = sum_a [D2_a p / rho - (D1_a rho / rho^2) D1_a p], wall CCD
    (ccd_ppe_utils.py:51-82)."""
    Lp = np.zeros(p.shape)
    for ax in range(p.ndim):
        dp, d2p = occd.differentiate_wall(p, ax, h[ax])
        Lp += d2p / rho - (drho[ax] / rho ** 2) * dp
    return Lp


def defect_correction(rhs, rho, base_solve, op_apply, pin, max_corrections=3,
                      tolerance=1e-8, relaxation=1.0):
    """PPESolverDefectCorrection.solve without interface-jump / periodic /
    phase-mean hooks (defect_correction.py:212-371).  Returns (p, history)."""
    rhs = np.array(rhs, dtype=np.float64)
    rhs.ravel()[pin] = 0.0
    p = np.array(base_solve(rhs), dtype=np.float64)
    p.ravel()[pin] = 0.0
    scale = None
    hist = []
    broke = False
    for _ in range(max_corrections):
        res = rhs - op_apply(p)
        res.ravel()[pin] = 0.0
        rn = float(np.linalg.norm(res.ravel()))
        if scale is None:
            scale = max(float(np.linalg.norm(rhs.ravel())), 1.0)
        hist.append(rn)
        if rn <= tolerance * scale:
            broke = True
            break
        corr = np.array(base_solve(res), dtype=np.float64)
        corr.ravel()[pin] = 0.0
        img = op_apply(corr)
        img.ravel()[pin] = 0.0
        rsq = np.sum(res * res)
        num = np.sum(res * img)
        den = np.sum(img * img)
        a_opt = num / (den if den > 0 else 1.0)
        cands = np.concatenate([[a_opt], [relaxation * 0.5 ** k for k in range(12)]])
        trial = rsq - 2.0 * cands * num + cands * cands * den
        valid = (cands > 0) & (trial < rsq)
        if not valid.any():
            break
        p = p + cands[int(np.argmax(valid))] * corr
        p.ravel()[pin] = 0.0
    if not broke:
        res = rhs - op_apply(p)
        res.ravel()[pin] = 0.0
        hist.append(float(np.linalg.norm(res.ravel())))
    return p, hist
