"""PPESolverFCCDMatrixFree: drop-in for the reference's FCCD matrix-free PPE.

Mirrors ``twophase.ppe.fccd_matrixfree.PPESolverFCCDMatrixFree``
(src/twophase/ppe/fccd_matrixfree.py:105-611) on its default path: the
constructor reads ``pseudo_tol`` (1e-8), ``pseudo_maxiter`` (500),
``ppe_restart`` (None: SciPy's 20), ``ppe_preconditioner`` ('none' |
'jacobi'), ``ppe_coefficient_scheme`` ('phase_density'),
``ppe_interface_coupling_scheme`` ('none') and ``boundary_face_space``
('full_face') from the solver config; the pin is ``bc_spec.pin_dof`` or the
centre node.  ``solve(rhs, rho, dt, p_init)``, ``apply(p)``,
``prepare_operator(rho)`` and the ``IPPESolver`` surface keep their
signatures and exceptions (ValueError for unsupported options, RuntimeError
for non-convergence and for ``apply`` before ``prepare_operator``).

All arithmetic runs in ``libtpf.so`` (tpf_fccd_ppe_*): the CCD line solves for
the second derivative, one fused face-gradient / face-coefficient / weighted
divergence kernel, and device GMRES.  Variants the reference offers beyond the
default path (phase-separated coefficients, interface jump couplings, reduced
boundary face spaces, the variational operator pairing, non-uniform grids)
raise NotImplementedError.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .arrays import to_device
from .grid import boundary_axes
from .ppe import MatrixAssemblyUnavailable


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("PPESolverFCCDMatrixFree (B200) needs a CUDA device; there is no CPU fallback")
    return torch


class PPESolverFCCDMatrixFree:
    scheme_names = ("fccd_iterative",)

    def __init__(self, backend, config, grid, fccd, *, bc_spec=None):
        _torch()
        self.lib = _lib.load()
        self.backend = backend
        self.xp = getattr(backend, "xp", np)
        self.grid = grid
        self.ndim = grid.ndim
        self.fccd = fccd
        solver_cfg = getattr(config, "solver", config)
        self.tol = float(getattr(solver_cfg, "pseudo_tol", 1.0e-8))
        self.maxiter = int(getattr(solver_cfg, "pseudo_maxiter", 500))
        restart = getattr(solver_cfg, "ppe_restart", None)
        self.restart = int(restart) if restart is not None else None
        self.preconditioner = str(getattr(solver_cfg, "ppe_preconditioner", "none")).strip().lower()
        self.coefficient_scheme = str(getattr(solver_cfg, "ppe_coefficient_scheme", "phase_density")).strip().lower()
        self.interface_coupling_scheme = str(getattr(solver_cfg, "ppe_interface_coupling_scheme",
                                                     "none")).strip().lower()
        self.boundary_face_space = str(getattr(solver_cfg, "boundary_face_space", "full_face")).strip().lower()
        pairing = getattr(solver_cfg, "scalar_operator_pairing", None)
        if self.coefficient_scheme not in {"phase_density", "phase_separated"}:
            raise ValueError("FCCD PPE supports ppe_coefficient_scheme='phase_density'|'phase_separated'")
        if self.interface_coupling_scheme not in {"none", "jump_decomposition", "affine_jump"}:
            raise ValueError("FCCD PPE supports ppe_interface_coupling_scheme='none'|'jump_decomposition'|'affine_jump'")
        if self.coefficient_scheme == "phase_density" and self.interface_coupling_scheme != "none":
            raise ValueError("phase_density PPE requires interface_coupling='none'")
        if self.preconditioner not in {"jacobi", "none"}:
            raise ValueError("FCCD PPE supports preconditioner='jacobi'|'none'")
        if self.coefficient_scheme != "phase_density":
            raise NotImplementedError("the B200 FCCD PPE implements ppe_coefficient_scheme='phase_density'")
        if self.boundary_face_space != "full_face":
            raise NotImplementedError("the B200 FCCD PPE implements boundary_face_space='full_face'")
        if pairing is not None and str(pairing).strip().lower() not in ("", "legacy", "none", "legacy_operator"):
            raise NotImplementedError("the B200 FCCD PPE implements the legacy operator pairing")
        if not getattr(grid, "uniform", True):
            raise NotImplementedError("the B200 FCCD PPE covers uniform grids")
        bc = getattr(fccd, "bc_type", "wall")
        self._axes = boundary_axes(bc, self.ndim)
        if bc_spec is not None:
            self._pin_dof = int(bc_spec.pin_dof)
        else:
            self._pin_dof = int(np.ravel_multi_index(tuple(n // 2 for n in grid.N), tuple(grid.shape)))
        self._pin_dofs = (self._pin_dof,)
        self.last_diagnostics = {}
        self.last_base_pressure = None
        self._handle = None
        self._prepared = False
        self._create()

    # -- handle -----------------------------------------------------------------
    def _options(self):
        o = _lib.tpf_fccd_ppe_options()
        self.lib.tpf_fccd_ppe_default_options(C.byref(o))
        o.tol = self.tol
        o.maxiter = self.maxiter
        o.restart = 20 if self.restart is None else self.restart
        o.precond = _lib.TPF_PRECOND_JACOBI if self.preconditioner == "jacobi" else _lib.TPF_PRECOND_NONE
        return o

    def _create(self):
        if self._handle is not None:
            self.lib.tpf_fccd_ppe_destroy(self._handle)
            self._handle = None
        nd = self.ndim
        N = (C.c_int64 * nd)(*[int(n) for n in self.grid.N])
        self._coords = [np.ascontiguousarray(np.asarray(c, dtype=np.float64)) for c in self.grid.coords]
        cptr = (C.POINTER(C.c_double) * nd)(*[c.ctypes.data_as(C.POINTER(C.c_double)) for c in self._coords])
        hccd = (C.c_double * nd)(*[float(self.grid.L[a]) / float(self.grid.N[a]) for a in range(nd)])
        per = (C.c_int * nd)(*[1 if a == "periodic" else 0 for a in self._axes])
        h = C.c_void_p()
        o = self._options()
        _lib.check(self.lib.tpf_fccd_ppe_create(C.byref(h), nd, N, cptr, hccd, per, self._pin_dof, C.byref(o)))
        self._handle = h
        self._prepared = False

    def _sync_options(self):
        o = self._options()
        _lib.check(self.lib.tpf_fccd_ppe_set_options(self._handle, C.byref(o)))

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None:
            try:
                self.lib.tpf_fccd_ppe_destroy(h)
            except Exception:
                pass

    def _check_shape(self, t):
        if tuple(t.shape) != tuple(self.grid.shape):
            raise ValueError(f"array shape {tuple(t.shape)} does not match grid shape {tuple(self.grid.shape)}")

    # -- IPPESolver ----------------------------------------------------------------
    def update_grid(self, grid=None) -> None:
        """Refresh grid-dependent FCCD weights after a mesh rebuild (:217-221)."""
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
        """Face inverse densities and the Jacobi inverse diagonal for ``rho``
        (fccd_matrixfree_lifecycle.py:44-95)."""
        self._sync_options()
        v = to_device(rho, dtype=_torch().float64)
        self._check_shape(v.tensor)
        _lib.check(self.lib.tpf_fccd_ppe_prepare(self._handle, _lib.dptr(v.tensor), _lib.current_stream_handle()))
        self._rho_keep = v.tensor
        self._prepared = True

    def apply(self, p):
        """The FCCD PPE operator with its pinned and periodic-image rows (:378-398)."""
        if not self._prepared:
            raise RuntimeError("prepare_operator(rho) must be called before apply(p)")
        v = to_device(p, dtype=_torch().float64)
        self._check_shape(v.tensor)
        out = _torch().empty_like(v.tensor)
        _lib.check(self.lib.tpf_fccd_ppe_apply(self._handle, _lib.dptr(v.tensor), _lib.dptr(out),
                                               _lib.current_stream_handle()))
        return v.out(out)

    def jacobi_inverse_diagonal(self):
        """The Jacobi inverse diagonal of the last ``prepare_operator`` (the
        reference's ``_diag_inv``), as a device tensor."""
        if not self._prepared:
            raise RuntimeError("Jacobi preconditioner is not initialised")
        out = _torch().empty(tuple(self.grid.shape), dtype=_torch().float64, device=self._rho_keep.device)
        _lib.check(self.lib.tpf_fccd_ppe_diag_inv(self._handle, _lib.dptr(out), _lib.current_stream_handle()))
        return out

    def solve(self, rhs, rho, dt: float = 0.0, p_init=None):
        """Solve the FCCD PPE with device GMRES (:506-611); p[pin] = 0 and the
        periodic image nodes synchronised."""
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
        st = self.lib.tpf_fccd_ppe_solve(self._handle, _lib.dptr(vr.tensor), _lib.dptr(vrho.tensor), _lib.dptr(p),
                                         _lib.dptr(p0) if p0 is not None else None,
                                         _lib.current_stream_handle(), C.byref(res))
        self._prepared = True
        self._rho_keep = vrho.tensor
        self.last_diagnostics = {
            "ppe_linear_info": int(res.info),
            "ppe_gmres_iterations": int(res.iterations),
            "ppe_operator_applies": int(res.applies),
            "ppe_gmres_relative_residual": float(res.rel_residual),
        }
        if st == _lib.TPF_ENOCONV:
            raise RuntimeError(f"PPESolverFCCDMatrixFree did not converge: info={res.info}, maxiter={self.maxiter}")
        _lib.check(st)
        self.last_base_pressure = p.clone()
        return vr.out(p)
