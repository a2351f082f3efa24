"""Steps either side of the PPE on the GPU: the velocity corrector and the CFL
time step, with the reference's classes and signatures.

* ``VelocityCorrector.correct(vel_star, p, rho, dt)`` -- u^{n+1} = u* - (dt/rho)
  D1 p per axis with the wall-normal pressure gradient zeroed on wall planes
  (src/twophase/coupling/velocity_corrector.py:41-89).  Each axis is ONE CCD
  line solve whose epilogue writes the corrected velocity
  (tpf_ccd_apply_corrector): p, u*, rho in, u out, no gradient array.
* ``ccd_pressure_gradient(ccd, p, ndim)`` -- the gradient itself
  (velocity_corrector.py:41-55), for callers that need it (the predictor's
  IPC term).
* ``CFLCalculator.compute(velocity_components, mu, rho)`` -- the CFL-limited
  time step (src/twophase/time_integration/cfl.py:41-137): the maxima come
  from one reduction kernel (tpf_cfl_maxima), the formula is the reference's,
  evaluated on the host in the same order.
* ``RhieChowInterpolator.face_velocity_divergence(vel_star, p, rho, dt, kappa,
  psi, we)`` -- the Rhie-Chow face-velocity divergence, the PPE right-hand side
  (src/twophase/spatial/rhie_chow.py:55-284).
"""

from __future__ import annotations

import ctypes as C
import math
from typing import List, Optional

from . import _lib
from .arrays import line_split, to_device


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("twophaseflow_b200 needs a CUDA device; there is no CPU fallback")
    return torch


def ccd_pressure_gradient(ccd, p, ndim: int) -> List:
    """[dp/dx_0, dp/dx_1, ...] by CCD with the wall-normal components zeroed on
    wall planes (velocity_corrector.py:41-55)."""
    grad = []
    for ax in range(ndim):
        dp_dax, _ = ccd.differentiate(p, ax)
        ccd.enforce_wall_neumann(dp_dax, ax)
        grad.append(dp_dax)
    return grad


class VelocityCorrector:
    """u^{n+1} = u* - (dt / rho) D1 p (velocity_corrector.py:58-89) on the B200
    CCD plans of ``ccd`` (a ``twophaseflow_b200.CCDSolver``)."""

    def __init__(self, backend, grid, ccd):
        self.backend = backend
        self.xp = getattr(backend, "xp", None)
        self.grid = grid
        self.ccd = ccd

    def correct(self, vel_star: List, p, rho, dt: float) -> List:
        """Corrected velocity components; each axis is one fused CCD solve."""
        torch = _torch()
        ccd = self.ccd
        dtype = ccd.dtype
        vp = to_device(p, dtype=dtype)
        pt = vp.tensor
        rt = to_device(rho, dtype=dtype).tensor
        if rt.shape != pt.shape:
            raise ValueError(f"rho shape {tuple(rt.shape)} differs from p shape {tuple(pt.shape)}")
        flags = 0 if getattr(self.grid, "uniform", True) else _lib.TPF_CCD_APPLY_METRIC
        out = []
        for ax in range(len(vel_star)):
            vu = to_device(vel_star[ax], dtype=dtype)
            u = vu.tensor
            if u.shape != pt.shape:
                raise ValueError(f"velocity component {ax} shape {tuple(u.shape)} differs from p")
            outer, n, inner = line_split(u.shape, ax)
            if n != int(self.grid.N[ax]) + 1:
                raise ValueError(f"data has {n} points along axis {ax}, grid has {int(self.grid.N[ax]) + 1}")
            plan = ccd._plan(ax, ccd._axis_periodic(ax))
            un = torch.empty_like(u)
            _lib.check(ccd.lib.tpf_ccd_apply_corrector(plan, outer, inner, _lib.dptr(pt), _lib.dptr(u),
                                                       _lib.dptr(rt), C.c_double(float(dt)), _lib.dptr(un),
                                                       flags, _lib.current_stream_handle()))
            out.append(vu.out(un))
        return out


class CFLCalculator:
    """CFL-limited time step (cfl.py:41-137): advective bound from the sum of the
    per-axis maximum speeds, the viscous bound for explicit viscosity, the
    capillary-wave bound when We is given."""

    def __init__(self, backend, grid, cfl_number: float, We: Optional[float] = None, rho_ratio: float = 0.0,
                 cn_viscous: bool = True):
        self.backend = backend
        self.xp = getattr(backend, "xp", None)
        self.grid = grid
        self.cfl = cfl_number
        self._h_min = min(float(grid.L[ax] / grid.N[ax]) for ax in range(grid.ndim))
        if We is not None and We > 0.0:
            h3 = self._h_min ** 3
            self._dt_sigma = math.sqrt((1.0 + rho_ratio) * We * h3 / (2.0 * math.pi))
        else:
            self._dt_sigma = None
        self._cn_viscous = cn_viscous
        self.lib = _lib.load()

    def maxima(self, velocity_components: List, mu=None, rho=None):
        """(max |u_i| per component, max mu/rho or None) from one reduction kernel."""
        torch = _torch()
        comps = [to_device(v).tensor for v in velocity_components]
        if not 1 <= len(comps) <= 3:
            raise ValueError("1..3 velocity components")
        dtype = comps[0].dtype
        if dtype not in (torch.float64, torch.float32):
            raise ValueError("velocity components must be float64 or float32")
        comps = [c.to(dtype).contiguous() for c in comps]
        n = comps[0].numel()
        if any(c.numel() != n for c in comps):
            raise ValueError("velocity components differ in size")
        mt = rt = None
        if mu is not None and rho is not None:
            mt = to_device(mu, dtype=dtype).tensor
            rt = to_device(rho, dtype=dtype).tensor
            if mt.numel() != n or rt.numel() != n:
                raise ValueError("mu / rho differ in size from the velocity")
        out = torch.empty(4, dtype=torch.float64, device=comps[0].device)
        ptrs = (C.c_void_p * len(comps))(*[_lib.dptr(c) for c in comps])
        _lib.check(self.lib.tpf_cfl_maxima(n, len(comps), ptrs, _lib.dptr(mt) if mt is not None else None,
                                           _lib.dptr(rt) if rt is not None else None,
                                           _lib.TPF_F64 if dtype == torch.float64 else _lib.TPF_F32,
                                           _lib.dptr(out), _lib.current_stream_handle()))
        host = out.cpu().tolist()
        return host[:len(comps)], (host[3] if mt is not None else None)

    def compute(self, velocity_components: List, mu, rho) -> float:
        """The time step dt > 0 (cfl.py:85-137)."""
        h = self._h_min
        cfl = self.cfl
        speeds, nu_max = self.maxima(velocity_components, None if self._cn_viscous else mu,
                                     None if self._cn_viscous else rho)
        u_sum = 0.0
        for v in speeds:
            u_sum = u_sum + v
        dt_conv = cfl * h / max(u_sum, 1.0e-14)
        dt_candidates = [dt_conv]
        if not self._cn_viscous:
            dt_visc = cfl * h * h / (4.0 * max(nu_max, 1.0e-14))
            dt_candidates.append(dt_visc)
        if self._dt_sigma is not None:
            dt_candidates.append(cfl * self._dt_sigma)
        return max(min(dt_candidates), 1.0e-8)


class RhieChowInterpolator:
    """Rhie-Chow face velocities and their divergence, the PPE right-hand side
    (src/twophase/spatial/rhie_chow.py:38-284).

    Per axis: one CCD line solve for the cell pressure gradient (and for
    D1 psi when the balanced-force terms are on), then one kernel
    (tpf_rc_divergence_axis) that forms both faces of every node and adds the
    axis' flux divergence into the result.  ``bc_type`` picks the face-0 and
    node-N rules per axis, independently of the CCD's boundary type, as in the
    reference."""

    def __init__(self, backend, grid, ccd, bc_type: str = "wall"):
        from .grid import boundary_axes
        self.backend = backend
        self.xp = getattr(backend, "xp", None)
        self.grid = grid
        self.ndim = grid.ndim
        self.ccd = ccd
        self.bc_type = bc_type
        self._axes = boundary_axes(bc_type, self.ndim)
        self.lib = _lib.load()

    def face_velocity_divergence(self, vel_star: List, p, rho, dt: float, kappa=None, psi=None, we: float = None):
        """div u_RC (rhie_chow.py:55-115); the balanced-force form when kappa,
        psi and we are all given."""
        torch = _torch()
        dtype = getattr(self.ccd, "dtype", torch.float64)
        vp = to_device(p, dtype=dtype)
        pt = vp.tensor
        rt = to_device(rho, dtype=dtype).tensor
        bf = kappa is not None and psi is not None and we is not None
        kt = to_device(kappa, dtype=dtype).tensor if bf else None
        st = to_device(psi, dtype=dtype).tensor if bf else None
        div = torch.empty_like(pt)
        shape = (C.c_int64 * pt.dim())(*[int(s) for s in pt.shape])
        tdt = _lib.TPF_F64 if dtype == torch.float64 else _lib.TPF_F32
        for ax in range(self.ndim):
            h = float(self.grid.L[ax] / self.grid.N[ax])
            ut = to_device(vel_star[ax], dtype=dtype).tensor
            if ut.shape != pt.shape or rt.shape != pt.shape:
                raise ValueError("u*, p and rho must have the grid's shape")
            dp = self.ccd.first_derivative(pt, ax)
            dpsi = self.ccd.first_derivative(st, ax) if bf else None
            _lib.check(self.lib.tpf_rc_divergence_axis(
                pt.dim(), shape, ax, 1 if self._axes[ax] == "periodic" else 0, h, float(dt),
                _lib.dptr(ut), _lib.dptr(pt), _lib.dptr(rt), _lib.dptr(dp),
                _lib.dptr(kt) if bf else None, _lib.dptr(st) if bf else None, _lib.dptr(dpsi) if bf else None,
                float(we) if bf else 0.0, 1 if ax > 0 else 0, _lib.dptr(div), tdt, _lib.current_stream_handle()))
        return vp.out(div)
