"""PPESolverFVMMatrixFree: drop-in for the reference's matrix-free FVM PPE solver.

Mirrors ``twophase.ppe.fvm_matrixfree.PPESolverFVMMatrixFree``
(src/twophase/ppe/fvm_matrixfree.py:46-363) and the ``IPPESolver`` contract
(src/twophase/ppe/interfaces.py:28-86): same constructor, same configuration
attributes read with ``getattr`` (``pseudo_tol``, ``pseudo_maxiter``,
``pseudo_c_tau``, ``ppe_iteration_method``, ``ppe_restart``,
``ppe_preconditioner``, ``ppe_pcr_stages``), same pinned gauge, same
exceptions (ValueError for unsupported boundary/options, RuntimeError on
non-convergence).  All arithmetic runs in ``libtpf.so`` (tpf_ppe_*).

B200 additions, read the same way from the solver config:
``ppe_precision`` ('fp64' | 'mixed': FP32 inner CG under FP64 iterative
refinement), ``ppe_inner_tol``, ``ppe_max_refine`` and ``ppe_line_solver``
('thomas': exact line solves as the reference's CPU backend; 'pcr': PCR
truncated to ``ppe_pcr_stages`` as the reference's GPU backend).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .arrays import to_device


class MatrixAssemblyUnavailable(RuntimeError):
    """Raised by get_matrix: this solver is matrix-free (interfaces.py:24-25)."""


_METHOD = {"gmres": _lib.TPF_PPE_GMRES, "cg": _lib.TPF_PPE_CG}
_PRECOND = {"none": _lib.TPF_PRECOND_NONE, "jacobi": _lib.TPF_PRECOND_JACOBI, "line_pcr": _lib.TPF_PRECOND_LINE}


class PPESolverFVMMatrixFree:
    scheme_names = ("fvm_iterative",)

    def __init__(self, backend, config, grid, bc_type: str = "wall", bc_spec=None):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("PPESolverFVMMatrixFree (B200) needs a CUDA device; there is no CPU fallback")
        self.lib = _lib.load()
        self.backend = backend
        self.xp = getattr(backend, "xp", np)
        self.grid = grid
        self.ndim = grid.ndim
        self.bc_type = bc_type
        self.bc_spec = bc_spec
        solver_cfg = getattr(config, "solver", config)
        if str(getattr(bc_type, "value", bc_type)).strip().lower() != "wall":
            raise ValueError(
                "PPESolverFVMMatrixFree supports bc_type='wall' only; "
                f"got {bc_type!r}. Select ppe_solver_type='fvm_direct' "
                "explicitly if sparse FVM is intended for this boundary condition.")
        self.tol = float(getattr(solver_cfg, "pseudo_tol", 1e-8))
        self.maxiter = int(getattr(solver_cfg, "pseudo_maxiter", 500))
        self.c_tau = float(getattr(solver_cfg, "pseudo_c_tau", 2.0))
        method = str(getattr(solver_cfg, "ppe_iteration_method", "gmres")).strip().lower()
        if method in {"explicit", "gauss_seidel", "adi"}:
            method = "gmres"
        if method not in _METHOD:
            raise ValueError("PPESolverFVMMatrixFree supports ppe_iteration_method='gmres' or 'cg' "
                             f"today, got {method!r}")
        self.iteration_method = method
        restart = getattr(solver_cfg, "ppe_restart", None)
        self.restart = int(restart) if restart is not None else min(80, max(20, self.maxiter))
        default_pc = "jacobi" if method == "cg" else "line_pcr"
        self.preconditioner = str(getattr(solver_cfg, "ppe_preconditioner", default_pc)).strip().lower()
        if self.preconditioner not in _PRECOND:
            raise ValueError("ppe_preconditioner must be 'jacobi', 'line_pcr', or 'none', "
                             f"got {self.preconditioner!r}")
        if method == "cg" and self.preconditioner == "line_pcr":
            raise ValueError("ppe_iteration_method='cg' supports preconditioner='jacobi' or 'none'; "
                             "line_pcr is a nonsymmetric GMRES preconditioner.")
        pcr = getattr(solver_cfg, "ppe_pcr_stages", 4)
        self.precond_pcr_stages = int(pcr if pcr is not None else 4)
        # the reference solves the shifted line systems exactly (Thomas) on the
        # CPU backend and by PCR truncated to ppe_pcr_stages on its GPU backend
        self.line_solver = str(getattr(solver_cfg, "ppe_line_solver", "thomas")).strip().lower()
        if self.line_solver not in ("thomas", "pcr"):
            raise ValueError(f"ppe_line_solver must be 'thomas' or 'pcr', got {self.line_solver!r}")
        self.precision = str(getattr(solver_cfg, "ppe_precision", "fp64")).strip().lower()
        if self.precision not in ("fp64", "mixed"):
            raise ValueError(f"ppe_precision must be 'fp64' or 'mixed', got {self.precision!r}")
        if self.precision == "mixed" and method != "cg":
            raise ValueError("ppe_precision='mixed' runs the CG route (ppe_iteration_method='cg')")
        self.inner_tol = float(getattr(solver_cfg, "ppe_inner_tol", 1e-3))
        self.max_refine = int(getattr(solver_cfg, "ppe_max_refine", 60))
        if bc_spec is not None:
            self._pin_dof = int(bc_spec.pin_dof)
        else:
            self._pin_dof = int(np.ravel_multi_index(tuple(n // 2 for n in grid.N), tuple(grid.shape)))
        self.last_diagnostics = {}
        self._handle = None
        self._prepared = False
        self._create()

    # -- handle -------------------------------------------------------------------
    def _options(self):
        o = _lib.tpf_ppe_options()
        self.lib.tpf_ppe_default_options(C.byref(o))
        o.method = _METHOD[self.iteration_method]
        o.precond = _PRECOND[self.preconditioner]
        if o.precond == _lib.TPF_PRECOND_LINE and self.line_solver == "pcr":
            o.precond = _lib.TPF_PRECOND_LINE_PCR
        o.precision = _lib.TPF_PREC_MIXED if self.precision == "mixed" else _lib.TPF_PREC_F64
        o.tol = self.tol
        o.maxiter = self.maxiter
        o.restart = self.restart
        o.c_tau = self.c_tau
        o.pcr_stages = self.precond_pcr_stages
        o.inner_tol = self.inner_tol
        o.max_refine = self.max_refine
        return o

    def _create(self):
        if self._handle is not None:
            self.lib.tpf_ppe_destroy(self._handle)
            self._handle = None
        N = (C.c_int64 * self.ndim)(*[int(n) for n in self.grid.N])
        self._coords = [np.ascontiguousarray(np.asarray(c, dtype=np.float64)) for c in self.grid.coords]
        cptr = (C.POINTER(C.c_double) * self.ndim)(
            *[c.ctypes.data_as(C.POINTER(C.c_double)) for c in self._coords])
        h = C.c_void_p()
        o = self._options()
        _lib.check(self.lib.tpf_ppe_create(C.byref(h), self.ndim, N, cptr, self._pin_dof, C.byref(o)))
        self._handle = h
        self._prepared = False
        self._h_min = min(float(np.min(np.diff(c))) for c in self._coords)

    def _sync_options(self):
        o = self._options()
        _lib.check(self.lib.tpf_ppe_set_options(self._handle, C.byref(o)))

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None:
            try:
                self.lib.tpf_ppe_destroy(h)
            except Exception:
                pass

    # -- IPPESolver ----------------------------------------------------------------
    def update_grid(self, grid=None) -> None:
        """Refresh metric caches after a grid rebuild (fvm_matrixfree.py:140-148)."""
        if grid is not None:
            self.grid = grid
            self.ndim = grid.ndim
        self._create()

    def invalidate_cache(self) -> None:
        self._prepared = False

    def clear_interface_jump_context(self) -> None:
        return None

    def get_matrix(self, rho):
        raise MatrixAssemblyUnavailable(f"{type(self).__name__} does not provide an assembled PPE matrix")

    def prepare_operator(self, rho) -> None:
        """Face coefficients and preconditioner state for ``rho``."""
        self._sync_options()
        v = to_device(rho, dtype=_torch().float64)
        self._check_shape(v.tensor)
        _lib.check(self.lib.tpf_ppe_prepare(self._handle, _lib.dptr(v.tensor), _lib.current_stream_handle()))
        self._rho_keep = v.tensor
        self._prepared = True

    def apply(self, p):
        """Pinned matrix-free operator (fvm_matrixfree.py:281-300)."""
        if not self._prepared:
            raise RuntimeError("operator coefficients are not initialised")
        v = to_device(p, dtype=_torch().float64)
        self._check_shape(v.tensor)
        out = _torch().empty_like(v.tensor)
        _lib.check(self.lib.tpf_ppe_apply(self._handle, _lib.dptr(v.tensor), _lib.dptr(out),
                                          _lib.current_stream_handle()))
        return v.out(out)

    def _precondition(self, r, kind):
        if not self._prepared:
            raise RuntimeError(f"{kind} preconditioner state is not initialised")
        v = to_device(r, dtype=_torch().float64)
        z = _torch().empty_like(v.tensor)
        _lib.check(self.lib.tpf_ppe_precondition(self._handle, _lib.dptr(v.tensor), _lib.dptr(z),
                                                 _lib.current_stream_handle()))
        return v.out(z)

    def apply_line_preconditioner(self, r):
        """Shifted additive line preconditioner (fvm_matrixfree.py:302-323)."""
        if self.preconditioner != "line_pcr":
            raise RuntimeError("line preconditioner coefficients are not initialised")
        return self._precondition(r, "line")

    def apply_jacobi_preconditioner(self, r):
        """Diagonal Jacobi preconditioner (fvm_matrixfree.py:325-331)."""
        if self.preconditioner != "jacobi":
            raise RuntimeError("Jacobi preconditioner diagonal is not initialised")
        return self._precondition(r, "Jacobi")

    def solve(self, rhs, rho, dt: float = 0.0, p_init=None):
        """Solve the FVM PPE (fvm_matrixfree.py:150-260); returns p with p[pin] = 0."""
        torch = _torch()
        self._sync_options()
        vr = to_device(rhs, dtype=torch.float64)
        vrho = to_device(rho, dtype=torch.float64)
        self._check_shape(vr.tensor)
        self._check_shape(vrho.tensor)
        p0 = None
        if p_init is not None:
            p0 = to_device(p_init, dtype=torch.float64).tensor
            self._check_shape(p0)
        p = torch.empty_like(vr.tensor)
        res = _lib.tpf_ppe_result()
        st = self.lib.tpf_ppe_solve(self._handle, _lib.dptr(vr.tensor), _lib.dptr(vrho.tensor), _lib.dptr(p),
                                    _lib.dptr(p0) if p0 is not None else None,
                                    _lib.current_stream_handle(), C.byref(res))
        self._prepared = True
        self._rho_keep = vrho.tensor
        self._fill_diagnostics(res)
        if st == _lib.TPF_ENOCONV:
            raise RuntimeError(
                f"{type(self).__name__} did not converge cleanly (info={res.info}); "
                "no alternate PPE solver was applied. Increase the matrix-free "
                "iteration budget/tolerance or select ppe_solver_type='fvm_direct' "
                "explicitly if sparse FVM is intended.")
        _lib.check(st)
        return vr.out(p)

    def read_result(self):
        """Result of the last replay of a solve captured into a CUDA graph
        (the CG route records its whole solve when called under stream
        capture; nothing is read back then).  Synchronizes the current stream,
        fills ``last_diagnostics`` and raises RuntimeError like ``solve`` when
        that replay did not converge."""
        res = _lib.tpf_ppe_result()
        st = self.lib.tpf_ppe_read_result(self._handle, _lib.current_stream_handle(), C.byref(res))
        if st not in (_lib.TPF_OK, _lib.TPF_ENOCONV):
            _lib.check(st)
        self._fill_diagnostics(res)
        if st == _lib.TPF_ENOCONV:
            raise RuntimeError(
                f"{type(self).__name__} did not converge cleanly (info={res.info}); "
                "no alternate PPE solver was applied. Increase the matrix-free "
                "iteration budget/tolerance or select ppe_solver_type='fvm_direct' "
                "explicitly if sparse FVM is intended.")
        return dict(self.last_diagnostics)

    def _fill_diagnostics(self, res):
        key = f"ppe_low_order_{self.iteration_method}"
        self.last_diagnostics = {
            f"{key}_info": int(res.info),
            f"{key}_tol": float(self.tol),
            f"{key}_maxiter": int(self.maxiter),
            f"{key}_iterations": int(res.iterations),
            f"{key}_applies": int(res.applies),
            f"{key}_refinements": int(res.refinements),
            f"{key}_relative_residual": float(res.rel_residual),
        }

    def _check_shape(self, t):
        if tuple(t.shape) != tuple(self.grid.shape):
            raise ValueError(f"array shape {tuple(t.shape)} does not match grid shape {tuple(self.grid.shape)}")


def _torch():
    import torch
    return torch


def create_fvm_matrixfree(config, backend, grid, ccd=None, bc_spec=None):
    """Factory with the reference registry signature
    ``factory_fn(config, backend, grid, ccd, bc_spec)`` (tp/ppe/factory.py:31-39)."""
    bc_type = getattr(getattr(config, "numerics", None), "bc_type", "wall")
    return PPESolverFVMMatrixFree(backend, config, grid, bc_type=bc_type, bc_spec=bc_spec)


def register_with_reference(register_ppe_solver, names=("fvm_iterative", "fvm_matrixfree")):
    """Install this solver under the reference's registry keys, e.g.
    ``register_with_reference(twophase.ppe.factory.register_ppe_solver)``."""
    for n in names:
        register_ppe_solver(n, create_fvm_matrixfree)


def solve_batched(solvers, rhs_list, rho_list=None):
    """Solve many independent PPE systems in ONE persistent launch
    (tpf_ppe_solve_batched): ``solvers`` are CG-route PPESolverFVMMatrixFree
    instances (each with its own grid), ``rhs_list`` / ``rho_list`` their
    fields.  Returns the list of pressures (p[pin] = 0); each solver's
    ``last_diagnostics`` is filled as by its own solve."""
    torch = _torch()
    n = len(solvers)
    if n == 0:
        return []
    if len(rhs_list) != n or (rho_list is not None and len(rho_list) != n):
        raise ValueError("one rhs (and rho) per solver")
    lib = solvers[0].lib
    keep, outs, views = [], [], []
    for k, s in enumerate(solvers):
        if s.iteration_method != "cg":
            raise ValueError("batched solves run the CG route (ppe_iteration_method='cg')")
        s._sync_options()
        vr = to_device(rhs_list[k], dtype=torch.float64)
        s._check_shape(vr.tensor)
        views.append(vr)
        keep.append(vr.tensor)
        if rho_list is not None:
            vrho = to_device(rho_list[k], dtype=torch.float64)
            s._check_shape(vrho.tensor)
            keep.append(vrho.tensor)
            s._rho_keep = vrho.tensor
        outs.append(torch.empty_like(vr.tensor))
    H = (C.c_void_p * n)(*[s._handle.value for s in solvers])
    R = (C.c_void_p * n)(*[int(v.tensor.data_ptr()) for v in views])
    P = (C.c_void_p * n)(*[int(o.data_ptr()) for o in outs])
    RHO = None
    if rho_list is not None:
        RHO = (C.c_void_p * n)(*[int(t.data_ptr()) for t in keep[1::2]])
    res = (_lib.tpf_ppe_result * n)()
    st = lib.tpf_ppe_solve_batched(H, n, R, RHO, P, _lib.current_stream_handle(), res)
    for k, s in enumerate(solvers):
        s._prepared = True
        key = "ppe_low_order_cg"
        s.last_diagnostics = {
            f"{key}_info": int(res[k].info),
            f"{key}_iterations": int(res[k].iterations),
            f"{key}_applies": int(res[k].applies),
            f"{key}_refinements": int(res[k].refinements),
            f"{key}_relative_residual": float(res[k].rel_residual),
        }
    if st == _lib.TPF_ENOCONV:
        raise RuntimeError(_lib.last_error())
    _lib.check(st)
    return [v.out(o) for v, o in zip(views, outs)]
