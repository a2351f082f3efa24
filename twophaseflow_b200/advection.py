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
  ``mode="node"`` (Option C) is -sum_k u_k (R_4 grad_k phi) instead: per axis
  one CCD second derivative of phi and one kernel that forms the face
  gradients, the Hermite node gradient and the accumulation;
  ``node_gradient(u, axis, q=None)`` is that gradient alone (fccd.py:392-462).
* ``FCCDLevelSetAdvection(backend, grid, fccd, mode="flux",
  mass_correction=False).advance(psi, velocity_components, dt,
  clip_bounds=(0, 1))`` -- one TVD-RK3 step (levelset/fccd_advection.py:86-129,
  time_integration/tvd_rk3.py:26-48): three right-hand sides and three stage
  kernels, each stage clipped and its periodic image nodes synchronised,
  then (mass_correction) the interface-weighted mass correction.
* ``SplitReinitializer(backend, grid, ccd, eps, n_steps=4, bc="zero",
  eps_d_comp=0.05, mass_correction=True).reinitialize(psi)`` -- compression
  (forward Euler on the filtered CCD divergence of psi(1-psi) n) and CN-ADI
  diffusion line solves per pseudo-step, then the interface-weighted mass
  correction (levelset/reinit_split.py:22-102, reinit_ops.py:34-204,
  heaviside.py:118-149).
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
    """Face-centred compact operator on a B200 ``CCDSolver`` (uniform grids,
    and non-uniform grids with wall axes: the reference's per-face and
    per-node weights, the CCD derivatives with the grid metric)."""

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
        self._uniform = bool(getattr(grid, "uniform", True))
        if not self._uniform and any(a == "periodic" for a in self._axes):
            raise NotImplementedError("the B200 FCCD operator covers non-uniform grids on wall axes")
        self._ccd = ccd_solver if ccd_solver is not None else CCDSolver(grid, backend, bc_type=bc_type)
        # H = x_1 - x_0 of the node coordinates, as the reference's weights take it
        self._H = [float(grid.coords[ax][1] - grid.coords[ax][0]) for ax in range(self.ndim)]
        self._w = [self._nonuniform_weights(ax) for ax in range(self.ndim)] if not self._uniform else None
        self.lib = _lib.load()

    def _nonuniform_weights(self, ax: int):
        """The reference's array weights of a non-uniform wall axis
        (fccd_helpers.py:8-52), computed on the host in the same order:
        H_f^2/16, 1/H_node (interior nodes), 1/H_f, H_f/24, H_node/16."""
        import numpy as np
        torch = _torch()
        H = np.asarray(self.grid.coords[ax], dtype=np.float64)
        H = H[1:] - H[:-1]
        node = np.zeros(len(H) + 1)
        node[1:-1] = 0.5 * (H[:-1] + H[1:])
        node[0] = H[0]
        node[-1] = H[-1]
        arrays = {"face_h2_16": H * H / 16.0, "node_inv_width": 1.0 / (0.5 * (H[:-1] + H[1:])),
                  "face_inv_h": 1.0 / H, "face_h_24": H / 24.0, "node_h_16": node / 16.0}
        dev = torch.device("cuda", torch.cuda.current_device())
        return {k: torch.from_numpy(np.ascontiguousarray(v)).to(dev) for k, v in arrays.items()}

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
        per = 1 if self._axes[axis] == "periodic" else 0
        if self._w is not None:
            w = self._w[axis]
            _lib.check(self.lib.tpf_fccd_flux_divergence_axis_nonuniform(
                phi.dim(), self._shape(phi), axis, per, _lib.dptr(w["face_h2_16"]), _lib.dptr(w["node_inv_width"]),
                _lib.dptr(prod), _lib.dptr(q), 1 if accumulate else 0, _lib.dptr(acc), self._tdt(phi), st))
            return
        _lib.check(self.lib.tpf_fccd_flux_divergence_axis(
            phi.dim(), self._shape(phi), axis, per, self._H[axis],
            _lib.dptr(prod), _lib.dptr(q), 1 if accumulate else 0, _lib.dptr(acc), self._tdt(phi), st))

    def _node_into(self, out, phi, axis: int, mode: int, u_k=None, q=None):
        """Option C: out = the R_4 node gradient of phi (mode 0), or
        out (=, -=) u_k * gradient (modes 1, 2) (fccd.py:392-462)."""
        if q is None:
            q = self._ccd.second_derivative(phi, axis)
        per = 1 if self._axes[axis] == "periodic" else 0
        uk = _lib.dptr(u_k) if u_k is not None else None
        st = _lib.current_stream_handle()
        if self._w is not None:
            w = self._w[axis]
            _lib.check(self.lib.tpf_fccd_node_gradient_axis_nonuniform(
                phi.dim(), self._shape(phi), axis, per, _lib.dptr(w["face_inv_h"]), _lib.dptr(w["face_h_24"]),
                _lib.dptr(w["node_h_16"]), _lib.dptr(phi), _lib.dptr(q), uk, mode, _lib.dptr(out), self._tdt(phi), st))
            return
        _lib.check(self.lib.tpf_fccd_node_gradient_axis(
            phi.dim(), self._shape(phi), axis, per, self._H[axis], _lib.dptr(phi), _lib.dptr(q), uk, mode,
            _lib.dptr(out), self._tdt(phi), st))

    def _rhs_tensors(self, vel: List, scalar=None, mode: str = "flux"):
        torch = _torch()
        ndim = len(vel)
        prod = torch.empty_like(vel[0])
        fields = [scalar] if scalar is not None else vel
        out = []
        for phi in fields:
            acc = torch.empty_like(phi)
            for k in range(ndim):
                if mode == "node":   # acc -= u_k * R_4 grad_k phi (fccd_advection_helpers.py:53-69)
                    self._node_into(acc, phi, k, 1 if k == 0 else 2, u_k=vel[k])
                else:
                    self._flux_into(acc, vel[k], phi, k, k > 0, prod)
            out.append(acc)
        return out

    def node_gradient(self, u, axis: int, q=None):
        """4th-order node gradient by R_4 Hermite reconstruction of the FCCD
        face gradients (fccd.py:392-462): O(H^4) inside, the one-sided face
        gradient on wall nodes; ``q`` the CCD second derivative if known."""
        torch = _torch()
        v = to_device(u, dtype=self.dtype)
        qt = to_device(q, dtype=self.dtype).tensor if q is not None else None
        out = torch.empty_like(v.tensor)
        self._node_into(out, v.tensor, axis, 0, q=qt)
        return v.out(out)

    def advection_rhs(self, velocity_components: List, scalar=None, mode: str = "flux", *,
                      skip_zero_check: bool = False) -> List:
        """-(u.grad) u per component (scalar None) or [-u.grad psi] (fccd.py:523-563)."""
        if mode not in ("node", "flux"):
            raise ValueError(f"mode must be 'node' or 'flux', got {mode!r}")
        vs = [to_device(v, dtype=self.dtype) for v in velocity_components]
        vel = [v.tensor for v in vs]
        if scalar is not None:
            sv = to_device(scalar, dtype=self.dtype)
            return [sv.out(t) for t in self._rhs_tensors(vel, sv.tensor, mode)]
        return [vs[j].out(t) for j, t in enumerate(self._rhs_tensors(vel, None, mode))]


class FCCDLevelSetAdvection:
    """TVD-RK3 transport of psi with the FCCD flux-form right-hand side
    (levelset/fccd_advection.py:55-129)."""

    def __init__(self, backend, grid, fccd: FCCDSolver, mode: str = "flux", mass_correction: bool = False):
        if mode not in ("node", "flux"):
            raise ValueError(f"mode must be 'node' or 'flux', got {mode!r}")
        self._backend = backend
        self.xp = getattr(backend, "xp", None)
        self._grid = grid
        self._fccd = fccd
        self._mode = mode
        self._mass_correction = mass_correction
        self._dV = None
        if mass_correction:   # grid.cell_volumes(bc_type=fccd.bc_type), uploaded once
            import numpy as np
            torch = _torch()
            per = _periodic_flags(fccd.bc_type, grid.ndim)
            vol = _control_widths(grid, 0, per[0])
            for ax in range(1, grid.ndim):
                vol = np.expand_dims(vol, axis=ax) * _control_widths(grid, ax, per[ax])
            dev = torch.device("cuda", torch.cuda.current_device())
            self._dV = torch.from_numpy(np.ascontiguousarray(vol, dtype=np.float64)).to(dev)
            self._partials = torch.empty(2048, dtype=torch.float64, device=dev)

    def advance(self, psi, velocity_components: List, dt: float, clip_bounds=(0.0, 1.0), velocity_is_zero=False):
        """psi after one RK3 step; psi's periodic image nodes are synchronised in
        place first, as the reference does.

        ``velocity_is_zero=True`` is the caller's statement that every velocity
        component is exactly zero.  The reference's CPU backend tests this
        itself and then skips the RK3 stages, returning the clipped (and
        mass-corrected) psi (fccd_advection.py:99-110); its GPU backend has
        no such shortcut.  The stages would leave psi within an ulp, but not
        bit-equal (0.75 q + 0.25 q), so callers that compare with the CPU
        reference pass the flag when they know the velocity is zero."""
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
        if self._mass_correction:
            m_old = torch.empty(2, dtype=torch.float64, device=q0.device)
            _lib.check(lib.tpf_mass_sums(q0.numel(), _lib.dptr(q0), _lib.dptr(self._dV), _lib.dptr(self._partials),
                                         _lib.dptr(m_old), tdt, st))
        clip = clip_bounds is not None
        lo, hi = (float(clip_bounds[0]), float(clip_bounds[1])) if clip else (0.0, 0.0)
        coeffs = ((1, 0.0, 0.0), (2, 0.75, 0.25), (3, 1.0 / 3.0, 2.0 / 3.0))
        if velocity_is_zero:
            coeffs = ()   # stage 0 below: q0 copied through the clip and the image sync
            nxt = torch.empty_like(q0)
            _lib.check(lib.tpf_tvd_rk3_stage(q0.dim(), shape, per, 0, 0.0, 0.0, 0.0, None, _lib.dptr(q0), None,
                                             1 if clip else 0, lo, hi, _lib.dptr(nxt), tdt, st))
            q = nxt
        else:
            q = q0
        for stage, ca, cb in coeffs:
            L = fccd._rhs_tensors(vel, q, self._mode)[0]
            nxt = torch.empty_like(q0)
            _lib.check(lib.tpf_tvd_rk3_stage(q0.dim(), shape, per, stage, ca, cb, float(dt), _lib.dptr(q0),
                                             _lib.dptr(q), _lib.dptr(L), 1 if clip else 0, lo, hi, _lib.dptr(nxt),
                                             tdt, st))
            q = nxt
        if self._mass_correction:
            sums = torch.empty(2, dtype=torch.float64, device=q.device)
            _lib.check(lib.tpf_mass_sums(q.numel(), _lib.dptr(q), _lib.dptr(self._dV), _lib.dptr(self._partials),
                                         _lib.dptr(sums), tdt, st))
            out = torch.empty_like(q)
            _lib.check(lib.tpf_mass_correction_apply(q.numel(), _lib.dptr(q), _lib.dptr(m_old), _lib.dptr(sums),
                                                     _lib.dptr(out), tdt, st))
            _lib.check(lib.tpf_sync_periodic_images(q.dim(), shape, per, _lib.dptr(out), tdt, st))
            q = out
        return v.out(q)


_BETA2 = -1.0 / 8.0   # CCD Eq-II off-diagonal (reinit_ops.py:19)


def _periodic_flags(bc, ndim: int):
    """periodic_axis_flags (core/boundary.py:94-113): only axes labelled periodic."""
    if isinstance(bc, (tuple, list)):
        return tuple(str(v).strip().lower() == "periodic" for v in bc)
    value = str(getattr(bc, "value", bc)).strip().lower()
    if value in ("zero", "neumann", "outflow"):
        return tuple(False for _ in range(ndim))
    return tuple(a == "periodic" for a in boundary_axes(bc, ndim))


def _pad_kind(bc, axis: int) -> int:
    """Ghost padding of the filtered divergence (pad_ghost_cells): 1 periodic,
    2 neumann / outflow (the end node), 0 otherwise (zeros)."""
    label = str(bc[axis] if isinstance(bc, (tuple, list)) else bc).strip().lower()
    return {"periodic": 1, "neumann": 2, "outflow": 2}.get(label, 0)


def _control_widths(grid, axis: int, periodic: bool):
    """Grid._axis_control_widths (core/grid.py:1158-1170): half-cell sums on
    periodic axes, the node metric spacing ``grid.h`` on wall axes (L/N on a
    uniform grid without ``h``)."""
    import numpy as np
    coords = np.asarray(grid.coords[axis], dtype=float)
    if periodic:
        cw = np.diff(coords)
        w = np.empty_like(coords)
        w[:-1] = 0.5 * (np.roll(cw, 1) + cw)
        w[-1] = 0.0
        return w
    if getattr(grid, "h", None) is not None:
        return np.asarray(grid.h[axis], dtype=float)
    return np.full(grid.N[axis] + 1, grid.L[axis] / grid.N[axis])


class SplitReinitializer:
    """Operator-split reinitialization, compression (forward Euler) + CN-ADI
    diffusion (levelset/reinit_split.py:22-102).  On non-uniform grids (as
    the reference): dtau and the CN factors from the smallest node spacing
    ``grid.h``, the filtered divergence in xi-space times the metric J, the
    mass correction over the grid's control volumes."""

    def __init__(self, backend, grid, ccd, eps: float, n_steps: int = 4, bc: str = "zero",
                 eps_d_comp: float = 0.05, mass_correction: bool = True):
        import numpy as np
        torch = _torch()
        self.xp = getattr(backend, "xp", None)
        self.grid = grid
        self.ccd = ccd
        self.eps = eps
        self.n_steps = n_steps
        self._bc = bc
        self._eps_d_comp = float(eps_d_comp)
        self._mass_correction = mass_correction
        nd = grid.ndim
        # smallest node spacing per axis (reinit_split.py:64-66); L/N on a uniform grid
        hs = getattr(grid, "h", None)
        self._h = [float(np.min(hs[ax])) if hs is not None else float(grid.L[ax] / grid.N[ax]) for ax in range(nd)]
        self._J = None
        if not getattr(grid, "uniform", True):
            dev0 = torch.device("cuda", torch.cuda.current_device())
            self._J = [torch.from_numpy(np.ascontiguousarray(np.asarray(grid.J[ax], dtype=np.float64))).to(dev0)
                       for ax in range(nd)]
        # compute_dtau (reinit_ops.py:34-54)
        dx_min = min(self._h)
        eps_min = float(np.min(eps))
        self.dtau = min(0.5 * dx_min ** 2 / (2.0 * nd * eps_min), 0.5 * dx_min)
        dev = torch.device("cuda", torch.cuda.current_device())
        self._cn = []
        for ax in range(nd):   # build_cn_factors (reinit_ops.py:117-166), same host arithmetic
            h = self._h[ax]
            mu = eps * self.dtau / (2.0 * h ** 2)
            n = grid.N[ax] + 1
            d_L = 1.0 + 6.0 * mu
            c_L = _BETA2 - 3.0 * mu
            main = np.full(n, d_L)
            sup = np.full(n - 1, c_L)
            sub = np.full(n - 1, c_L)
            sup[0] = 2.0 * c_L
            sub[-1] = 2.0 * c_L
            m = main.copy()
            f = np.empty(n - 1)
            for i in range(1, n):
                f[i - 1] = sub[i - 1] / m[i - 1]
                m[i] -= f[i - 1] * sup[i - 1]
            mu_r = eps * self.dtau / (2.0 * h ** 2)
            cR = _BETA2 + 3.0 * mu_r
            dR = 1.0 - 6.0 * mu_r
            self._cn.append((cR, dR, torch.from_numpy(f).to(dev), torch.from_numpy(m).to(dev),
                             torch.from_numpy(sup).to(dev)))
        self._per = _periodic_flags(bc, nd)
        vol = _control_widths(grid, 0, self._per[0])
        for ax in range(1, nd):
            vol = np.expand_dims(vol, axis=ax) * _control_widths(grid, ax, self._per[ax])
        self._dV = torch.from_numpy(np.ascontiguousarray(vol, dtype=np.float64)).to(dev)
        self._partials = torch.empty(2048, dtype=torch.float64, device=dev)
        self.lib = _lib.load()

    def reinitialize(self, psi):
        torch = _torch()
        lib = self.lib
        nd = self.grid.ndim
        v = to_device(psi, dtype=self.ccd.dtype)
        q = v.tensor.clone()
        shape = (C.c_int64 * nd)(*[int(s) for s in q.shape])
        per = (C.c_int * nd)(*[1 if f else 0 for f in self._per])
        tdt = _lib.TPF_F64 if q.dtype == torch.float64 else _lib.TPF_F32
        st = _lib.current_stream_handle()
        n = q.numel()
        _lib.check(lib.tpf_sync_periodic_images(nd, shape, per, _lib.dptr(q), tdt, st))
        if self._mass_correction:
            m_old = torch.empty(2, dtype=torch.float64, device=q.device)
            _lib.check(lib.tpf_mass_sums(n, _lib.dptr(q), _lib.dptr(self._dV), _lib.dptr(self._partials),
                                         _lib.dptr(m_old), tdt, st))
        P = C.c_void_p * nd
        for _ in range(self.n_steps):
            d1 = [self.ccd.first_derivative(q, ax) for ax in range(nd)]
            flux = [torch.empty_like(q) for _ in range(nd)]
            _lib.check(lib.tpf_reinit_compression_flux(nd, n, _lib.dptr(q), P(*[_lib.dptr(t) for t in d1]),
                                                       P(*[_lib.dptr(t) for t in flux]), tdt, st))
            div = torch.empty_like(q)
            for ax in range(nd):
                if self._J is None:
                    g = self.ccd.first_derivative(flux[ax], ax)
                    _lib.check(lib.tpf_reinit_filtered_divergence_axis(nd, shape, ax, _pad_kind(self._bc, ax),
                                                                       self._eps_d_comp, _lib.dptr(g), 1 if ax else 0,
                                                                       _lib.dptr(div), tdt, st))
                else:   # xi-space derivative and filter, then J (reinit_ops.py:95-105)
                    g = self.ccd.first_derivative(flux[ax], ax, apply_metric=False)
                    _lib.check(lib.tpf_reinit_filtered_divergence_axis_metric(
                        nd, shape, ax, _pad_kind(self._bc, ax), self._eps_d_comp, _lib.dptr(self._J[ax]),
                        _lib.dptr(g), 1 if ax else 0, _lib.dptr(div), tdt, st))
            # q* = clip(q - dtau div, 0, 1) with the image nodes synchronised
            q_new = torch.empty_like(q)
            _lib.check(lib.tpf_tvd_rk3_stage(nd, shape, per, 1, 0.0, 0.0, -self.dtau, None, _lib.dptr(q),
                                             _lib.dptr(div), 1, 0.0, 1.0, _lib.dptr(q_new), tdt, st))
            for ax in range(nd):
                cR, dR, f, m, sup = self._cn[ax]
                out = torch.empty_like(q)
                _lib.check(lib.tpf_reinit_cn_axis(nd, shape, ax, cR, dR, _lib.dptr(f), _lib.dptr(m), _lib.dptr(sup),
                                                  _lib.dptr(q_new), _lib.dptr(out), tdt, st))
                _lib.check(lib.tpf_sync_periodic_images(nd, shape, per, _lib.dptr(out), tdt, st))
                q_new = out
            q = torch.empty_like(q_new)
            _lib.check(lib.tpf_tvd_rk3_stage(nd, shape, per, 0, 0.0, 0.0, 0.0, None, _lib.dptr(q_new), None, 1, 0.0,
                                             1.0, _lib.dptr(q), tdt, st))
        if self._mass_correction:
            sums = torch.empty(2, dtype=torch.float64, device=q.device)
            _lib.check(lib.tpf_mass_sums(n, _lib.dptr(q), _lib.dptr(self._dV), _lib.dptr(self._partials),
                                         _lib.dptr(sums), tdt, st))
            out = torch.empty_like(q)
            _lib.check(lib.tpf_mass_correction_apply(n, _lib.dptr(q), _lib.dptr(m_old), _lib.dptr(sums),
                                                     _lib.dptr(out), tdt, st))
            _lib.check(lib.tpf_sync_periodic_images(nd, shape, per, _lib.dptr(out), tdt, st))
            q = out
        return v.out(q)


class UCCD6ConvectionTerm:
    """Skew-symmetric CCD convection with sixth-order-scaled hyperviscosity
    (src/twophase/ns_terms/uccd6_convection.py:31-128):
    -0.5 [(u.grad) u_j + div(u_j u)] - sigma max|u_k| h_k^7 (D2_k)^4 u_j.
    Per (j, k): CCD solves for D1/D2 of u_j, D1 of u_k u_j and the three further
    second derivatives, max|u_k| by the CFL reduction kernel (kept on the
    device), one accumulation kernel."""

    scheme_names = ("uccd6",)

    def __init__(self, backend, grid, ccd, sigma: float = 1.0e-3):
        if sigma <= 0.0:
            raise ValueError(f"sigma must be > 0, got {sigma}")
        self._backend = backend
        self.xp = getattr(backend, "xp", None)
        self._ccd = ccd
        self._grid = grid
        self._sigma = float(sigma)
        self._h7 = [(float(grid.L[ax]) / int(grid.N[ax])) ** 7 for ax in range(grid.ndim)]
        self.lib = _lib.load()

    def compute(self, ctx_or_velocity, ccd=None) -> List:
        torch = _torch()
        comps = ctx_or_velocity if isinstance(ctx_or_velocity, list) else ctx_or_velocity.velocity
        cc = self._ccd
        vs = [to_device(v, dtype=cc.dtype) for v in comps]
        vel = [v.tensor for v in vs]
        nd = len(vel)
        n = vel[0].numel()
        tdt = _lib.TPF_F64 if vel[0].dtype == torch.float64 else _lib.TPF_F32
        st = _lib.current_stream_handle()
        lib = self.lib
        # max |u_k| of every component in one reduction, kept on the device
        uref = torch.empty(4, dtype=torch.float64, device=vel[0].device)
        ptrs = (C.c_void_p * nd)(*[_lib.dptr(v) for v in vel])
        _lib.check(lib.tpf_cfl_maxima(n, nd, ptrs, None, None, tdt, _lib.dptr(uref), st))
        prod = torch.empty_like(vel[0])
        out = []
        for j in range(nd):
            acc = torch.empty_like(vel[j])
            for k in range(nd):
                d1, d2 = cc.differentiate(vel[j], k)
                _lib.check(lib.tpf_fccd_product(n, _lib.dptr(vel[k]), _lib.dptr(vel[j]), _lib.dptr(prod), tdt, st))
                cons = cc.first_derivative(prod, k)
                d8 = cc.second_derivative(cc.second_derivative(cc.second_derivative(d2, k), k), k)
                ur = uref[k:k + 1]
                _lib.check(lib.tpf_uccd6_accumulate(n, 1 if k == 0 else 0, _lib.dptr(vel[k]), _lib.dptr(d1),
                                                    _lib.dptr(cons), _lib.dptr(d8), self._sigma * self._h7[k],
                                                    _lib.dptr(ur), _lib.dptr(acc), tdt, st))
            out.append(vs[j].out(acc))
        return out
