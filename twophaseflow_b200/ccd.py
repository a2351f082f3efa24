"""CCDSolver: drop-in for ``twophase.ccd.ccd_solver.CCDSolver`` on a B200.

Same constructor and methods as the reference (src/twophase/ccd/ccd_solver.py:
79-281): ``differentiate``, ``first_derivative``, ``second_derivative``,
``differentiate_raw``, ``enforce_wall_neumann`` and the attributes ``grid``,
``backend``, ``xp``, ``ndim``, ``bc_type``.  Every derivative is computed by the
CUDA line kernels of ``libtpf.so`` (include/tpf.h: tpf_ccd_*).

Arrays: torch CUDA tensors and ``__cuda_array_interface__`` objects are used in
place; NumPy inputs are copied to the device and results come back as NumPy.
``dtype`` selects FP64 (default, the reference's precision) or FP32 line
solves (the boundary closures stay FP64 inside the kernel).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .arrays import line_split, to_device
from .grid import boundary_axes


class CCDSolver:
    def __init__(self, grid, backend=None, bc_type: str = "wall", dtype=None):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("CCDSolver (B200) needs a CUDA device; there is no CPU fallback")
        self.lib = _lib.load()
        self.grid = grid
        self.backend = backend
        self.xp = getattr(backend, "xp", np)
        self.ndim = grid.ndim
        self.bc_type = bc_type
        self.dtype = dtype if dtype is not None else torch.float64
        if self.dtype not in (torch.float64, torch.float32):
            raise ValueError("CCDSolver dtype must be float64 or float32")
        self._tpf_dtype = _lib.TPF_F64 if self.dtype == torch.float64 else _lib.TPF_F32
        if hasattr(grid, "set_boundary_type"):
            grid.set_boundary_type(bc_type)
        self._axes = boundary_axes(bc_type, self.ndim)
        self._plans = {}          # (axis, periodic) -> plan handle
        # periodic plans are built eagerly, wall plans lazily (ccd_solver.py:108-120)
        for ax in range(self.ndim):
            if self._axis_periodic(ax):
                self._plan(ax, True)

    # -- plans -------------------------------------------------------------------
    def _axis_periodic(self, axis: int) -> bool:
        return self._axes[axis] == "periodic"

    def _axis_solver_spacing(self, axis: int) -> float:
        """L/N on uniform grids, 1/N in xi-space (ccd_solver.py:126-130)."""
        if getattr(self.grid, "uniform", True):
            return float(self.grid.L[axis]) / float(self.grid.N[axis])
        return 1.0 / float(self.grid.N[axis])

    def _plan(self, axis: int, periodic: bool):
        key = (axis, periodic)
        p = self._plans.get(key)
        if p is None:
            h = C.c_void_p()
            n_pts = int(self.grid.N[axis]) + 1
            st = self.lib.tpf_ccd_plan_create(C.byref(h), n_pts, self._axis_solver_spacing(axis),
                                              _lib.TPF_BC_PERIODIC if periodic else _lib.TPF_BC_WALL,
                                              self._tpf_dtype)
            _lib.check(st)
            if not getattr(self.grid, "uniform", True):
                J = np.ascontiguousarray(np.asarray(self.grid.J[axis], dtype=np.float64))
                dJ = np.ascontiguousarray(np.asarray(self.grid.dJ_dxi[axis], dtype=np.float64))
                _lib.check(self.lib.tpf_ccd_plan_set_metric(
                    h, J.ctypes.data_as(C.POINTER(C.c_double)), dJ.ctypes.data_as(C.POINTER(C.c_double))))
            self._plans[key] = h
            p = h
        return p

    def __del__(self):
        lib = getattr(self, "lib", None)
        for h in getattr(self, "_plans", {}).values():
            try:
                lib.tpf_ccd_plan_destroy(h)
            except Exception:
                pass

    # -- core call ---------------------------------------------------------------
    def _run(self, data, axis, bc_left, bc_right, apply_metric, need1, need2):
        import torch
        if not 0 <= axis < self.ndim:
            raise ValueError(f"axis {axis} out of range for ndim={self.ndim}")
        v = to_device(data, dtype=self.dtype)
        f = v.tensor
        periodic = self._axis_periodic(axis) and bc_left is None and bc_right is None
        plan = self._plan(axis, periodic)
        outer, n, inner = line_split(f.shape, axis)
        if n != int(self.grid.N[axis]) + 1:
            raise ValueError(f"data has {n} points along axis {axis}, grid has {int(self.grid.N[axis]) + 1}")
        d1 = torch.empty_like(f) if need1 else None
        d2 = torch.empty_like(f) if need2 else None
        bl = (C.c_double * 2)(*bc_left) if bc_left is not None else None
        br = (C.c_double * 2)(*bc_right) if bc_right is not None else None
        flags = _lib.TPF_CCD_APPLY_METRIC if (apply_metric and not getattr(self.grid, "uniform", True)) else 0
        st = self.lib.tpf_ccd_apply(plan, outer, inner, _lib.dptr(f),
                                    _lib.dptr(d1) if d1 is not None else None,
                                    _lib.dptr(d2) if d2 is not None else None,
                                    bl, br, flags, _lib.current_stream_handle())
        _lib.check(st)
        return v, d1, d2

    # -- public API (ccd_solver.py:134-281) ---------------------------------------
    def differentiate(self, data, axis: int, bc_left=None, bc_right=None, apply_metric: bool = True):
        v, d1, d2 = self._run(data, axis, bc_left, bc_right, apply_metric, True, True)
        return v.out(d1), v.out(d2)

    def first_derivative(self, data, axis: int, bc_left=None, bc_right=None, apply_metric: bool = True):
        v, d1, _ = self._run(data, axis, bc_left, bc_right, apply_metric, True, False)
        return v.out(d1)

    def second_derivative(self, data, axis: int, bc_left=None, bc_right=None, apply_metric: bool = True):
        v, _, d2 = self._run(data, axis, bc_left, bc_right, apply_metric, False, True)
        return v.out(d2)

    def differentiate_refined(self, data, axis: int, refinements: int = 2):
        """(d1, d2) of FP64 data from FP32 line solves under FP64 iterative
        refinement (no counterpart in the reference, whose CCD is FP64): the
        FP32 solve of the FP32-rounded field, then ``refinements`` times the
        residual of the full CCD system (interior rows and the one-sided wall
        closures) in FP64 and an FP32 correction solve added in FP64.  Wall
        axes of a uniform grid; FP64 solver only."""
        import torch
        if self.dtype != torch.float64:
            raise ValueError("differentiate_refined needs an FP64 CCDSolver")
        if self._axis_periodic(axis):
            raise NotImplementedError("iterative refinement of the CCD line solves covers wall axes")
        if not getattr(self.grid, "uniform", True):
            raise NotImplementedError("iterative refinement of the CCD line solves covers uniform grids")
        v = to_device(data, dtype=torch.float64)
        f = v.tensor
        outer, n, inner = line_split(f.shape, axis)
        if n != int(self.grid.N[axis]) + 1:
            raise ValueError(f"data has {n} points along axis {axis}, grid has {int(self.grid.N[axis]) + 1}")
        p64 = self._plan(axis, False)
        key = (axis, "f32")
        p32 = self._plans.get(key)
        if p32 is None:
            h = C.c_void_p()
            _lib.check(self.lib.tpf_ccd_plan_create(C.byref(h), n, self._axis_solver_spacing(axis), _lib.TPF_BC_WALL,
                                                    _lib.TPF_F32))
            self._plans[key] = h
            p32 = h
        d1 = torch.empty_like(f)
        d2 = torch.empty_like(f)
        work = torch.empty(5 * f.numel(), dtype=torch.float32, device=f.device)
        _lib.check(self.lib.tpf_ccd_apply_refined(p64, p32, outer, inner, _lib.dptr(f), _lib.dptr(d1), _lib.dptr(d2),
                                                  int(refinements), _lib.dptr(work), _lib.current_stream_handle()))
        self._work_keep = work
        return v.out(d1), v.out(d2)

    def differentiate_raw(self, data, axis: int):
        """xi-space derivatives of a 1-D array of N[axis]+1 values (wall closure),
        ccd_solver.py:174-203."""
        v = to_device(data, dtype=self.dtype)
        f = v.tensor.reshape(-1)
        plan = self._plan(axis, False)
        d1 = f.new_empty(f.shape)
        d2 = f.new_empty(f.shape)
        _lib.check(self.lib.tpf_ccd_apply(plan, 1, 1, _lib.dptr(f), _lib.dptr(d1), _lib.dptr(d2),
                                          None, None, 0, _lib.current_stream_handle()))
        return v.out(d1), v.out(d2)

    def enforce_wall_neumann(self, grad, ax: int) -> None:
        """Zero the gradient on both wall planes of axis ``ax`` in place
        (ccd_solver.py:264-281).  No-op on periodic axes."""
        import torch
        if self._axis_periodic(ax):
            return
        if isinstance(grad, torch.Tensor) and grad.is_cuda and grad.is_contiguous() and grad.dtype == self.dtype:
            outer, n, inner = line_split(grad.shape, ax)
            plan = self._plan(ax, False)
            _lib.check(self.lib.tpf_ccd_enforce_wall_neumann(plan, outer, inner, _lib.dptr(grad),
                                                             _lib.current_stream_handle()))
            return
        # host / foreign arrays: plain indexing keeps the in-place contract
        sl_lo = [slice(None)] * grad.ndim
        sl_hi = [slice(None)] * grad.ndim
        sl_lo[ax] = 0
        sl_hi[ax] = -1
        grad[tuple(sl_lo)] = 0.0
        grad[tuple(sl_hi)] = 0.0
