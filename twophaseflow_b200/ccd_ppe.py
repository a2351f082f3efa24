"""CCD variable-density operator L_H and the defect-correction PPE loop.

* ``CCDVariableDensityOperator`` -- L_H p = sum_a [D2_a p / rho - (D1_a rho / rho^2) D1_a p]
  (reference src/twophase/ppe/ccd_ppe_utils.py:51-82, density gradients frozen per
  solve as in precompute_density_gradients, :25-48).  ``apply`` runs one fused
  CUDA line solve per axis (tpf_ccd_apply_vd): the variable-density term is
  accumulated in the kernel's output stage, so D1 p and D2 p never reach HBM.
* ``PPESolverDefectCorrection`` -- the outer residual-correction loop of
  src/twophase/ppe/defect_correction.py:212-371 (base solve with a low-order
  L_L solver, residual with L_H, correction with line search), on device
  tensors.  Interface-jump, periodic-image and phase-mean hooks of the
  modern pipeline are not part of this path.
"""

from __future__ import annotations

import numpy as np

from . import _lib
from .arrays import line_split, to_device
from .ccd import CCDSolver


def _torch():
    import torch
    return torch


class CCDVariableDensityOperator:
    """IPPESolver-style operator object for defect correction (prepare_operator / apply)."""

    def __init__(self, grid, ccd: CCDSolver | None = None, bc_spec=None, backend=None):
        self.grid = grid
        self.backend = backend
        self.ccd = ccd if ccd is not None else CCDSolver(grid, backend, bc_type="wall")
        self.ndim = grid.ndim
        if bc_spec is not None:
            self._pin_dof = int(bc_spec.pin_dof)
        else:
            self._pin_dof = int(np.ravel_multi_index(tuple(n // 2 for n in grid.N), tuple(grid.shape)))
        self._rho = None
        self._drho = None
        self.last_diagnostics = {}

    def update_grid(self, grid=None):
        if grid is not None:
            self.grid = grid
        self._rho = None
        self._drho = None

    def invalidate_cache(self):
        self._rho = None
        self._drho = None

    def prepare_operator(self, rho) -> None:
        """Freeze rho and d(rho)/dx_a (CCD first derivatives) for this solve."""
        torch = _torch()
        r = to_device(rho, dtype=torch.float64).tensor
        self._rho = r
        self._drho = [self.ccd.first_derivative(r, ax) for ax in range(self.ndim)]

    def apply(self, p):
        if self._rho is None:
            raise RuntimeError("operator coefficients are not initialised")
        torch = _torch()
        v = to_device(p, dtype=torch.float64)
        t = v.tensor
        out = torch.empty_like(t)
        lib = self.ccd.lib
        for ax in range(self.ndim):
            outer, n, inner = line_split(t.shape, ax)
            plan = self.ccd._plan(ax, self.ccd._axis_periodic(ax))
            flags = 0 if getattr(self.grid, "uniform", True) else _lib.TPF_CCD_APPLY_METRIC
            _lib.check(lib.tpf_ccd_apply_vd(plan, outer, inner, _lib.dptr(t), _lib.dptr(self._rho),
                                            _lib.dptr(self._drho[ax]), _lib.dptr(out), 1 if ax > 0 else 0,
                                            flags, _lib.current_stream_handle()))
        return v.out(out)


class PPESolverDefectCorrection:
    """Defect correction L_H p = rhs with a low-order base solver L_L."""

    def __init__(self, backend, grid, base_solver, operator, *, max_corrections: int = 3,
                 tolerance: float = 1.0e-8, relaxation: float = 1.0, fail_on_nonconvergence: bool = False):
        if max_corrections <= 0:
            raise ValueError("max_corrections must be > 0")
        if tolerance <= 0.0:
            raise ValueError("tolerance must be > 0")
        if relaxation <= 0.0:
            raise ValueError("relaxation must be > 0")
        if not hasattr(operator, "prepare_operator") or not hasattr(operator, "apply"):
            raise TypeError("operator must provide prepare_operator(rho) and apply(p)")
        self.backend = backend
        self.grid = grid
        self.base_solver = base_solver
        self.operator = operator
        self.max_corrections = int(max_corrections)
        self.tolerance = float(tolerance)
        self.relaxation = float(relaxation)
        self.fail_on_nonconvergence = bool(fail_on_nonconvergence)
        self._pin_dof = operator._pin_dof
        self.last_base_pressure = None
        self.last_diagnostics = {}
        self.last_residual_history: list[float] = []
        self.last_stalled = False

    def update_grid(self, grid=None):
        if grid is not None:
            self.grid = grid
        self.base_solver.update_grid(self.grid)
        self.operator.update_grid(self.grid)
        self._pin_dof = self.operator._pin_dof

    def invalidate_cache(self):
        self.base_solver.invalidate_cache()
        self.operator.invalidate_cache()

    def _pinned(self, t):
        t = t.clone()
        t.view(-1)[self._pin_dof] = 0.0
        return t

    def solve(self, rhs, rho, dt: float = 0.0, p_init=None):
        torch = _torch()
        vr = to_device(rhs, dtype=torch.float64)
        rho_t = to_device(rho, dtype=torch.float64).tensor
        self.operator.prepare_operator(rho_t)
        if hasattr(self.base_solver, "prepare_operator"):
            self.base_solver.prepare_operator(rho_t)
        rhs_t = self._pinned(vr.tensor)
        p0 = None if p_init is None else to_device(p_init, dtype=torch.float64).tensor
        pressure = self._pinned(self.base_solver.solve(rhs_t, rho_t, dt=dt, p_init=p0))
        rhs_norm = float(torch.linalg.norm(rhs_t))
        scale = max(rhs_norm, 1.0)
        history: list[float] = []
        broke = False
        applied = 0
        final_residual_norm = 0.0
        final_residual_linf = 0.0
        for _ in range(self.max_corrections):
            residual = self._pinned(rhs_t - self.operator.apply(pressure))
            rn = float(torch.linalg.norm(residual))
            history.append(rn)
            if rn <= self.tolerance * scale:
                broke = True
                final_residual_norm = rn
                final_residual_linf = float(residual.abs().max())
                break
            corr = self._pinned(self.base_solver.solve(residual, rho_t, dt=dt, p_init=None))
            img = self._pinned(self.operator.apply(corr))
            rsq = float(torch.sum(residual * residual))
            num = float(torch.sum(residual * img))
            den = float(torch.sum(img * img))
            a_opt = num / (den if den > 0.0 else 1.0)
            cands = [a_opt] + [self.relaxation * (0.5 ** k) for k in range(12)]
            chosen = None
            for c in cands:
                if c > 0.0 and (rsq - 2.0 * c * num + c * c * den) < rsq:
                    chosen = c
                    break
            if chosen is None:
                final_residual_norm = rn
                final_residual_linf = float(residual.abs().max())
                break
            pressure = self._pinned(pressure + chosen * corr)
            applied += 1
        if not broke:
            fr = self._pinned(rhs_t - self.operator.apply(pressure))
            final_residual_norm = float(torch.linalg.norm(fr))
            final_residual_linf = float(fr.abs().max())
            history.append(final_residual_norm)
            broke = final_residual_norm <= self.tolerance * scale
        self.last_residual_history = history
        self.last_stalled = not broke
        self.last_base_pressure = pressure.clone()
        rel = final_residual_norm / rhs_norm if rhs_norm > 0.0 else final_residual_norm
        self.last_diagnostics = {
            "ppe_dc_iterations": float(applied), "ppe_dc_max_corrections": float(self.max_corrections),
            "ppe_dc_tolerance": self.tolerance, "ppe_dc_relaxation": self.relaxation,
            "ppe_dc_rhs_l2": rhs_norm, "ppe_dc_initial_residual_l2": history[0] if history else 0.0,
            "ppe_dc_final_residual_l2": final_residual_norm, "ppe_dc_final_relative_l2": rel,
            "ppe_dc_final_residual_linf": final_residual_linf, "ppe_dc_converged": float(broke),
            "ppe_dc_stalled": float(not broke)}
        if self.last_stalled and self.fail_on_nonconvergence:
            raise RuntimeError(f"PPESolverDefectCorrection did not converge: relative_l2={final_residual_norm / scale:.3e}, "
                               f"linf={final_residual_linf:.3e}, max_corrections={self.max_corrections}")
        return vr.out(pressure)
