"""CLS transport on the GPU: the FCCD flux-form advection right-hand side and
the TVD-RK3 level-set step, with the reference's classes and signatures.

* ``FCCDSolver(grid, backend, bc_type="wall", ccd_solver=None)`` -- the
  face-centred compact operator (src/twophase/ccd/fccd.py:139-200), uniform
  grids: ``advection_rhs(velocity_components, scalar=None, mode="flux")``
  returns -div(P_f(u_k phi)) summed over the axes for the scalar (level set)
  or for every velocity component (momentum), as
  ccd/fccd_advection_helpers.py:16-72 composes it.  Per axis: one product
  kernel, one CCD line solve for the second derivative of the product (the
  B200 CCD kernels), one face-value + divergence kernel that accumulates.
* ``FCCDLevelSetAdvection(backend, grid, fccd, mode="flux",
  mass_correction=False).advance(psi, velocity_components, dt,
  clip_bounds=(0, 1))`` -- one TVD-RK3 step (levelset/fccd_advection.py:86-129,
  time_integration/tvd_rk3.py:26-48): three right-hand sides and three stage
  kernels, each stage clipped and its periodic image nodes synchronised.
"""

from __future__ import annotations

import ctypes as C
from typing import List

from . import _lib
from .arrays import to_device
from .grid import boundary_axes


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("twophaseflow_b200 needs a CUDA device; there is no CPU fallback")
    return torch


class FCCDSolver:
    """Face-centred compact operator on a B200 ``CCDSolver`` (uniform grids)."""

    def __init__(self, grid, backend=None, bc_type: str = "wall", ccd_solver=None):
        from .ccd import CCDSolver
        self.grid = grid
        self.backend = backend
        self.xp = getattr(backend, "xp", None)
        self.ndim = grid.ndim
        self.bc_type = bc_type
        self._axes = boundary_axes(bc_type, self.ndim)
        if ccd_solver is not None and boundary_axes(getattr(ccd_solver, "bc_type", bc_type), self.ndim) != self._axes:
            raise ValueError("FCCD and CCD solvers must share the same boundary topology")
        if not getattr(grid, "uniform", True):
            raise NotImplementedError("the B200 FCCD operator covers uniform grids")
        self._ccd = ccd_solver if ccd_solver is not None else CCDSolver(grid, backend, bc_type=bc_type)
        # H = x_1 - x_0 of the node coordinates, as the reference's weights take it
        self._H = [float(grid.coords[ax][1] - grid.coords[ax][0]) for ax in range(self.ndim)]
        self.lib = _lib.load()

    @property
    def dtype(self):
        return self._ccd.dtype

    def _tdt(self, t):
        torch = _torch()
        return _lib.TPF_F64 if t.dtype == torch.float64 else _lib.TPF_F32

    def _shape(self, t):
        return (C.c_int64 * t.dim())(*[int(s) for s in t.shape])

    def periodic_flags(self):
        return (C.c_int * self.ndim)(*[1 if a == "periodic" else 0 for a in self._axes])

    def _flux_into(self, acc, u_k, phi, axis: int, accumulate: bool, prod=None):
        """acc (+)= -div(P_f(u_k phi)) along ``axis`` (fccd_advection_helpers.py:8-13)."""
        torch = _torch()
        prod = torch.empty_like(phi) if prod is None else prod
        st = _lib.current_stream_handle()
        _lib.check(self.lib.tpf_fccd_product(phi.numel(), _lib.dptr(u_k), _lib.dptr(phi), _lib.dptr(prod),
                                             self._tdt(phi), st))
        q = self._ccd.second_derivative(prod, axis)
        _lib.check(self.lib.tpf_fccd_flux_divergence_axis(
            phi.dim(), self._shape(phi), axis, 1 if self._axes[axis] == "periodic" else 0, self._H[axis],
            _lib.dptr(prod), _lib.dptr(q), 1 if accumulate else 0, _lib.dptr(acc), self._tdt(phi), st))

    def _rhs_tensors(self, vel: List, scalar=None):
        torch = _torch()
        ndim = len(vel)
        prod = torch.empty_like(vel[0])
        if scalar is not None:
            acc = torch.empty_like(scalar)
            for k in range(ndim):
                self._flux_into(acc, vel[k], scalar, k, k > 0, prod)
            return [acc]
        out = []
        for j in range(ndim):
            acc = torch.empty_like(vel[j])
            for k in range(ndim):
                self._flux_into(acc, vel[k], vel[j], k, k > 0, prod)
            out.append(acc)
        return out

    def advection_rhs(self, velocity_components: List, scalar=None, mode: str = "flux", *,
                      skip_zero_check: bool = False) -> List:
        """-(u.grad) u per component (scalar None) or [-u.grad psi] (fccd.py:523-563)."""
        if mode not in ("node", "flux"):
            raise ValueError(f"mode must be 'node' or 'flux', got {mode!r}")
        if mode == "node":
            raise NotImplementedError("the B200 FCCD operator implements the flux form (Option B)")
        vs = [to_device(v, dtype=self.dtype) for v in velocity_components]
        vel = [v.tensor for v in vs]
        if scalar is not None:
            sv = to_device(scalar, dtype=self.dtype)
            return [sv.out(t) for t in self._rhs_tensors(vel, sv.tensor)]
        return [vs[j].out(t) for j, t in enumerate(self._rhs_tensors(vel))]


class FCCDLevelSetAdvection:
    """TVD-RK3 transport of psi with the FCCD flux-form right-hand side
    (levelset/fccd_advection.py:55-129)."""

    def __init__(self, backend, grid, fccd: FCCDSolver, mode: str = "flux", mass_correction: bool = False):
        if mode not in ("node", "flux"):
            raise ValueError(f"mode must be 'node' or 'flux', got {mode!r}")
        if mode == "node":
            raise NotImplementedError("the B200 FCCD transport implements the flux form (Option B)")
        if mass_correction:
            raise NotImplementedError("mass_correction is not implemented on the B200 path")
        self._backend = backend
        self.xp = getattr(backend, "xp", None)
        self._grid = grid
        self._fccd = fccd
        self._mode = mode
        self._mass_correction = mass_correction

    def advance(self, psi, velocity_components: List, dt: float, clip_bounds=(0.0, 1.0)):
        """psi after one RK3 step; psi's periodic image nodes are synchronised in
        place first, as the reference does."""
        import numpy as np
        torch = _torch()
        fccd = self._fccd
        lib = fccd.lib
        per = fccd.periodic_flags()
        if isinstance(psi, np.ndarray) and any(a == "periodic" for a in fccd._axes):
            for ax, kind in enumerate(fccd._axes):   # the caller's array, as the reference mutates it
                if kind == "periodic":
                    src = [slice(None)] * psi.ndim
                    img = [slice(None)] * psi.ndim
                    src[ax] = 0
                    img[ax] = -1
                    psi[tuple(img)] = psi[tuple(src)]
        v = to_device(psi, dtype=fccd.dtype)
        q0 = v.tensor
        shape = fccd._shape(q0)
        tdt = fccd._tdt(q0)
        st = _lib.current_stream_handle()
        _lib.check(lib.tpf_sync_periodic_images(q0.dim(), shape, per, _lib.dptr(q0), tdt, st))
        vel = [to_device(u, dtype=fccd.dtype).tensor for u in velocity_components]
        clip = clip_bounds is not None
        lo, hi = (float(clip_bounds[0]), float(clip_bounds[1])) if clip else (0.0, 0.0)
        coeffs = ((1, 0.0, 0.0), (2, 0.75, 0.25), (3, 1.0 / 3.0, 2.0 / 3.0))
        q = q0
        for stage, ca, cb in coeffs:
            L = fccd._rhs_tensors(vel, q)[0]
            nxt = torch.empty_like(q0)
            _lib.check(lib.tpf_tvd_rk3_stage(q0.dim(), shape, per, stage, ca, cb, float(dt), _lib.dptr(q0),
                                             _lib.dptr(q), _lib.dptr(L), 1 if clip else 0, lo, hi, _lib.dptr(nxt),
                                             tdt, st))
            q = nxt
        return v.out(q)
