"""CPU restatement of one full two-phase projection step, the reference's
stable quick-start pipeline (TEST INFRASTRUCTURE: the oracle).

Reference: ``src/twophase/simulation/_core.py:126-172`` (``step_forward``) with
``simulation/legacy_flow_helpers.py:23-90`` and the components
``legacy_builder_runtime.py`` builds for a default config with
``extension_method='none'``:

1. FCCD flux-form transport, TVD-RK3, clip, mass correction
   (``oracle.advect.advance`` + ``mass_correction``);
2. split reinitialization, 4 pseudo-steps, Neumann ghost padding, mass
   correction (``oracle.advect.reinitialize``);
3. rho, mu from psi; 4. curvature from psi (DCCD filter 0.05, psi_min 0.01);
5. AB2 + IPC predictor with UCCD6 convection (sigma 1e-3), gravity, CSF and the
   Picard-CN viscous predictor (ccd_bulk), then no-slip on every wall plane
   (``simulation/boundary_condition.py:22-70``);
6. PPE for the pressure increment: Rhie-Chow divergence / dt, FVM matrix-free
   GMRES(80) with the exact line preconditioner (``oracle.ppe.FVMMatrixFree``),
   p += dp; 7. velocity corrector with dp, then no-slip again.

Pinned against the reference's own steps in ``tests/golden/c1_golden.npz``.
Only tests, smoke() and bench.py's CPU-baseline leg may use this module.
"""

from __future__ import annotations

import numpy as np

from . import advect as oa
from . import ccd as occd
from . import levelset as ol
from . import ppe as oppe
from . import step as ostep
from . import viscous as ov


def _no_slip(vel):
    """BoundaryConditionHandler.apply for wall axes: every component zero on
    both planes of every axis."""
    out = [np.array(v, copy=True) for v in vel]
    nd = len(out)
    for ax in range(nd):
        lo = [slice(None)] * nd
        hi = [slice(None)] * nd
        lo[ax] = 0
        hi[ax] = -1
        for c in range(nd):
            out[c][tuple(lo)] = 0.0
            out[c][tuple(hi)] = 0.0
    return out


class QuickStartStep:
    """Wall-bounded uniform grid; liquid rho = mu = 1, gas rho_ratio / mu_ratio."""

    def __init__(self, N, L, psi, Re=100.0, Fr=1.0, We=10.0, rho_ratio=0.1, mu_ratio=0.1, sigma_uccd6=1.0e-3,
                 reinit_steps=4):
        self.N = tuple(int(n) for n in N)
        self.L = tuple(float(x) for x in L)
        self.nd = len(self.N)
        self.h = [float(self.L[a] / self.N[a]) for a in range(self.nd)]
        self.eps = 1.5 * min(self.h)
        self.Re, self.Fr, self.We = Re, Fr, We
        self.rho_l, self.rho_g, self.mu_l, self.mu_g = 1.0, rho_ratio, 1.0, mu_ratio
        self.sigma = sigma_uccd6
        self.reinit_steps = reinit_steps
        shape = tuple(n + 1 for n in self.N)
        self.psi = np.array(psi, dtype=np.float64, copy=True)
        self.vel = [np.zeros(shape) for _ in range(self.nd)]
        self.p = np.zeros(shape)
        self.conv_prev = None
        self.dV = oa.cell_volumes(self.L, self.N, [False] * self.nd)
        coords = [np.linspace(0.0, self.L[a], self.N[a] + 1) for a in range(self.nd)]
        self.ppe = oppe.FVMMatrixFree(coords, method="gmres", tol=1e-8, maxiter=500)

    def _D1(self, f, ax):
        return np.asarray(occd.differentiate(f, ax, self.h[ax], bc="wall")[0])

    def step(self, dt):
        nd, L, N = self.nd, self.L, self.N
        # 1-2 transport (mass-corrected) and reinitialization
        m_old = np.sum(self.psi * self.dV)
        q = oa.advance(self.psi, self.vel, dt, L, N, "wall")
        q = oa.mass_correction(q, self.dV, m_old)
        self.psi = oa.reinitialize(q, L, N, "wall", self.eps, self.reinit_steps, "neumann", 0.05, True)
        # 3-4 properties and curvature
        rho, mu = ol.update_properties(self.psi, self.rho_l, self.rho_g, self.mu_l, self.mu_g)
        kappa = ol.curvature_psi(self.psi, self.h, "wall")
        # 5 predictor: AB2 (UCCD6) + gravity + CSF + IPC, Picard CN viscous
        conv = oa.uccd6(self.vel, L, N, "wall", self.sigma)
        ab2 = conv if self.conv_prev is None else [1.5 * conv[c] - 0.5 * self.conv_prev[c] for c in range(nd)]
        grav = [np.zeros(rho.shape) for _ in range(nd)]
        grav[nd - 1] = -rho / (self.Fr ** 2)
        st = [kappa * self._D1(self.psi, ax) / self.We for ax in range(nd)]
        gp = ostep.pressure_gradient(self.p, self.h, "wall")
        e = [rho * ab2[c] + grav[c] + st[c] + (-gp[c]) for c in range(nd)]
        vel_star = ov.cn_predictor(self.vel, e, mu, rho, self.Re, L, N, "wall", dt, True)
        self.conv_prev = [np.array(c, copy=True) for c in conv]
        vel_star = _no_slip(vel_star)
        # 6 PPE for the pressure increment
        rhs = ostep.rc_divergence(vel_star, self.p, rho, dt, L, N, "wall", "wall") / dt
        dp = self.ppe.solve(rhs, rho, dt)
        self.p = self.p + dp
        # 7 corrector with dp
        self.vel = _no_slip(ostep.correct(vel_star, dp, rho, dt, self.h, "wall"))
        self.rho, self.mu = rho, mu
