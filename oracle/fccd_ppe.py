"""CPU restatement of the FCCD matrix-free PPE on its default path (TEST
INFRASTRUCTURE: the oracle).

Reference: ``src/twophase/ppe/fccd_matrixfree.py`` (PPESolverFCCDMatrixFree:
constructor :117-215, periodic image rows :310-376, ``apply`` :378-398,
operator core :400-428, ``solve`` :506-611, wall flux divergence :762-829),
``ppe/fccd_matrixfree_helpers.py`` (geometry cache :35-52, phase gauges
:54-85, face inverse density :207-249, Jacobi inverse :251-265, right-hand
side compatibility :337-380) and ``ppe/fccd_matrixfree_lifecycle.py:44-95``;
the face gradient is ``ccd/fccd.py:243-277`` on the oracle's CCD second
derivative.  Default path: ``ppe_coefficient_scheme='phase_density'``, no
interface coupling, ``boundary_face_space='full_face'``, the legacy operator
pairing, SciPy GMRES (``oracle.ppe.gmres``; restart 20 when none is given, as
SciPy defaults) with the Jacobi or no preconditioner.

Pinned against the reference's own outputs in ``tests/golden/fccd_ppe_golden.npz``.
Only tests, smoke() and bench.py's CPU-baseline leg may use this module.
"""

from __future__ import annotations

import numpy as np

from . import ccd as occd
from . import ppe as oppe
from .levelset import axis_kinds


class FCCDPPE:
    def __init__(self, L, N, bc: str = "wall", tol: float = 1e-8, maxiter: int = 500, restart=None,
                 preconditioner: str = "none"):
        self.L = tuple(float(x) for x in L)
        self.N = tuple(int(n) for n in N)
        self.nd = len(self.N)
        self.kinds = axis_kinds(bc, self.nd)
        self.shape = tuple(n + 1 for n in self.N)
        self.tol, self.maxiter = tol, maxiter
        self.restart = 20 if restart is None else int(restart)
        self.preconditioner = preconditioner
        self.pin = int(np.ravel_multi_index(tuple(n // 2 for n in self.N), self.shape))
        self.coords = [np.linspace(0.0, self.L[a], self.N[a] + 1) for a in range(self.nd)]
        self.h = [float(self.L[a] / self.N[a]) for a in range(self.nd)]     # CCD spacing
        self.H = [float(self.coords[a][1] - self.coords[a][0]) for a in range(self.nd)]   # FCCD weights
        # geometry cache (fccd_matrixfree_helpers.py:35-52)
        self.h_min, self.node_width = [], []
        for a in range(self.nd):
            c = self.coords[a]
            fw = c[1:] - c[:-1]
            w = np.empty_like(c)
            w[0] = 0.5 * fw[0]
            w[-1] = 0.5 * fw[-1]
            w[1:-1] = 0.5 * (c[2:] - c[:-2])
            self.h_min.append(float(np.min(fw)))
            self.node_width.append(w)
        self.inv_width = [1.0 / w for w in self.node_width]
        # periodic image -> source map (:310-348): first periodic axis claims a node
        img2src = {}
        for a in range(self.nd):
            if self.kinds[a] != "periodic":
                continue
            ranges = [np.arange(s) for s in self.shape]
            ir = [r.copy() for r in ranges]
            sr = [r.copy() for r in ranges]
            ir[a] = np.array([self.N[a]])
            sr[a] = np.array([0])
            im = np.ravel_multi_index([m.ravel() for m in np.meshgrid(*ir, indexing="ij")], self.shape)
            sm = np.ravel_multi_index([m.ravel() for m in np.meshgrid(*sr, indexing="ij")], self.shape)
            for i, s in zip(im.tolist(), sm.tolist()):
                img2src.setdefault(i, s)
        if img2src:
            self.images = np.array(sorted(img2src), dtype=np.intp)
            self.sources = np.array([img2src[int(i)] for i in self.images], dtype=np.intp)
        else:
            self.images = self.sources = None

    def sync(self, arr):
        if self.images is None:
            return arr
        out = np.array(arr, copy=True)
        f = out.ravel()
        f[self.images] = f[self.sources]
        return out

    def prepare(self, rho):
        """Face inverse densities and the Jacobi inverse diagonal (lifecycle :44-95)."""
        rho = np.asarray(rho, dtype=np.float64)
        self.rho = rho
        self.coeff = []
        for a in range(self.nd):
            ra = np.moveaxis(rho, a, 0)
            n = self.N[a]
            self.coeff.append(np.moveaxis(2.0 / (ra[0:n] + ra[1:n + 1]), 0, a))
        self.diag_inv = None
        if self.preconditioner == "jacobi":
            diag = np.zeros_like(rho)
            for hh in self.h_min:
                diag -= 2.0 / (rho * float(hh) * float(hh))
            diag.ravel()[self.pin] = 1.0
            self.diag_inv = 1.0 / np.where(np.abs(diag) > 1.0e-30, diag, 1.0)

    def face_gradient(self, u, a):
        """(u_hi - u_lo)/H - (H/24)(q_hi - q_lo), q = CCD second derivative (fccd.py:243-277)."""
        q = np.asarray(occd.differentiate(u, a, self.h[a], bc=self.kinds[a])[1])
        ua, qa = np.moveaxis(u, a, 0), np.moveaxis(q, a, 0)
        n = self.N[a]
        if self.kinds[a] == "periodic":
            ulo, uhi = ua[:n], np.roll(ua[:n], -1, axis=0)
            qlo, qhi = qa[:n], np.roll(qa[:n], -1, axis=0)
        else:
            ulo, uhi, qlo, qhi = ua[:-1], ua[1:], qa[:-1], qa[1:]
        H = self.H[a]
        return np.moveaxis((uhi - ulo) * (1.0 / H) - (H / 24.0) * (qhi - qlo), 0, a)

    def core(self, p):
        """sum_a D_a[(1/rho)_f G_a p] without gauge rows (:400-428, :762-829)."""
        out = np.zeros_like(p)
        for a in range(self.nd):
            g = np.moveaxis(self.face_gradient(p, a), a, 0)
            c = np.moveaxis(self.coeff[a], a, 0)
            o = np.moveaxis(out, a, 0)
            n = self.N[a]
            if self.kinds[a] == "periodic":
                F = c * g
                du = (F - np.roll(F, 1, axis=0)) * (1.0 / self.H[a])
                d = np.empty_like(o)
                d[:n] = du
                d[n] = du[0]
                o += d
            else:
                iw = self.inv_width[a].reshape((-1,) + (1,) * (p.ndim - 1))
                o[1:n] += (c[1:] * g[1:] - c[:-1] * g[:-1]) * iw[1:n]
                o[0] += c[0] * g[0] * iw[0]
                o[n] -= c[n - 1] * g[n - 1] * iw[n]
        return out

    def apply(self, p):
        """PPESolverFCCDMatrixFree.apply (:378-398): pin row and image rows."""
        p = np.asarray(p, dtype=np.float64)
        out = self.core(self.sync(p))
        out.ravel()[self.pin] = p.ravel()[self.pin]
        if self.images is not None:
            f, pf = out.ravel(), p.ravel()
            f[self.images] = pf[self.images] - pf[self.sources]
        return out

    def solve(self, rhs, rho):
        """PPESolverFCCDMatrixFree.solve (:506-611): (p, info, inner iterations)."""
        self.prepare(rho)
        r = np.array(rhs, dtype=np.float64, copy=True)
        r.ravel()[self.pin] = 0.0
        if self.images is not None:
            r.ravel()[self.images] = 0.0
        if not np.any(r):
            return np.zeros_like(r), 0, 0
        shape = self.shape
        matvec = lambda x: self.apply(x.reshape(shape)).ravel()
        if self.diag_inv is not None:
            def psolve(v):
                z = v.reshape(shape) * self.diag_inv
                z.ravel()[self.pin] = 0.0
                return z.ravel()
        else:
            psolve = lambda v: v
        x, info, its = oppe.gmres(matvec, psolve, r.ravel(), np.zeros(r.size), self.tol, self.restart, self.maxiter)
        sol = x.reshape(shape).copy()
        sol.ravel()[self.pin] = 0.0
        # synced twice, as the reference does around the (inactive) interface
        # jump (:594-606): a corner image takes its source's synced value
        return self.sync(self.sync(sol)), info, its
