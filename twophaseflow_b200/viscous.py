"""Viscous stress divergence on the GPU with the reference's class and
signature: ``ViscousTerm(backend, Re, cn_viscous=True,
spatial_scheme="ccd_bulk").compute_explicit(velocity_components, mu, rho, ccd)``
returns V_a = (1/Re) sum_b d/dx_b [mu (du_a/dx_b + du_b/dx_a)] / rho
(src/twophase/ns_terms/viscous.py:50-133, viscous_spatial.py:28-153) for the
three spatial schemes:

* ``ccd_bulk`` (default): CCD velocity derivatives, low-order stress derivative;
* ``conservative_stress``: low-order everywhere;
* ``ccd_stress_legacy``: CCD everywhere.

The CCD derivatives run on the CCD line kernels, each of the ndim^2
velocity gradients once (the reference forms each twice); the stress
mu (a + b) is formed inside the low-order derivative kernel, which also
accumulates over b and divides by Re rho on the last axis.  ``apply_cn_predictor`` runs the
explicit Euler branch or ``PicardCNAdvance`` (Heun: two viscous evaluations,
two combination kernels).  The interface-band variant (``psi`` given with
``ccd_bulk``) is not built.
"""

from __future__ import annotations

import ctypes as C
from typing import List

from . import _lib
from .arrays import to_device


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("twophaseflow_b200 needs a CUDA device; there is no CPU fallback")
    return torch


_ALIASES = {"stress_divergence": "conservative_stress", "low_order_conservative": "conservative_stress",
            "ccd": "ccd_bulk", "ccd_legacy": "ccd_stress_legacy"}


def canonical_viscous_spatial_scheme(name: str) -> str:
    """viscous_spatial.py:9-25."""
    c = _ALIASES.get(str(name).strip().lower(), str(name).strip().lower())
    if c not in ("conservative_stress", "ccd_bulk", "ccd_stress_legacy"):
        raise ValueError("viscous spatial scheme must be one of 'conservative_stress', 'ccd_bulk', or "
                         f"'ccd_stress_legacy', got {name!r}")
    return c


class ViscousTerm:
    """(1/Re) div[mu (grad u + grad u^T)] / rho (viscous.py:50-133)."""

    def __init__(self, backend, Re: float, cn_viscous: bool = True, spatial_scheme: str = "ccd_bulk",
                 cn_advance=None):
        self.backend = backend
        self.xp = getattr(backend, "xp", None)
        self.Re = Re
        self.cn_viscous = cn_viscous
        self.spatial_scheme = canonical_viscous_spatial_scheme(spatial_scheme)
        self.cn_advance = cn_advance
        self._coef = {}
        self.lib = _lib.load()

    def _coefficients(self, grid, axis: int):
        """Interior three-point coefficients of _low_order_derivative from the
        node coordinates, as the reference evaluates them (viscous_spatial.py:70-104)."""
        import numpy as np
        torch = _torch()
        coords = np.asarray(grid.coords[axis], dtype=float)
        key = (axis, coords.tobytes())   # the coordinates themselves: non-uniform grids of equal N, L differ
        if key not in self._coef:
            dx = coords[1:] - coords[:-1]
            h_l, h_r = dx[:-1], dx[1:]
            cl = -(h_r / (h_l * (h_l + h_r)))
            cc = (h_r - h_l) / (h_l * h_r)
            cr = h_l / (h_r * (h_l + h_r))
            dev = torch.device("cuda", torch.cuda.current_device())
            self._coef[key] = ([torch.from_numpy(np.ascontiguousarray(c)).to(dev) for c in (cl, cc, cr)],
                               float(dx[0]), float(dx[-1]))
        return self._coef[key]

    def compute(self, ctx) -> List:
        return self.compute_explicit(ctx.velocity, ctx.mu, ctx.rho, ctx.ccd)

    def compute_explicit(self, velocity_components: List, mu, rho, ccd, psi=None) -> List:
        torch = _torch()
        dtype = getattr(ccd, "dtype", torch.float64)
        vs = [to_device(v, dtype=dtype) for v in velocity_components]
        vel = [v.tensor for v in vs]
        mt = to_device(mu, dtype=dtype).tensor
        rt = to_device(rho, dtype=dtype).tensor
        nd = len(vel)
        shape = (C.c_int64 * nd)(*[int(s) for s in vel[0].shape])
        tdt = _lib.TPF_F64 if dtype == torch.float64 else _lib.TPF_F32
        st = _lib.current_stream_handle()
        lib = self.lib
        grid = ccd.grid

        def lowfd(total, ax, a, b=None, m=None, accumulate=False, finalize=False):
            (cl, cc, cr), dx0, dxl = self._coefficients(grid, ax)
            _lib.check(lib.tpf_visc_lowfd_axis(nd, shape, ax, _lib.dptr(cl), _lib.dptr(cc), _lib.dptr(cr), dx0, dxl,
                                               _lib.dptr(a), _lib.dptr(b) if b is not None else None,
                                               _lib.dptr(m) if m is not None else None, 1 if accumulate else 0,
                                               1 if finalize else 0, _lib.dptr(rt), float(self.Re), _lib.dptr(total),
                                               tdt, st))

        if psi is not None and self.spatial_scheme == "ccd_bulk":
            return [vs[c].out(v) for c, v in enumerate(self._band_evaluate(vel, mt, rt, psi, ccd, lowfd, dtype))]

        # each velocity gradient du_i/dx_j is needed twice (as du_a/dx_b for
        # component a and as du_b/dx_a for component b): computed once
        grads = {}

        def grad(i, j):
            if (i, j) not in grads:
                if self.spatial_scheme == "conservative_stress":
                    g = torch.empty_like(vel[i])
                    lowfd(g, j, vel[i])
                else:
                    g = ccd.first_derivative(vel[i], j)
                grads[(i, j)] = g
            return grads[(i, j)]

        out = []
        for al in range(nd):
            total = torch.empty_like(vel[al])
            for be in range(nd):
                last = be == nd - 1
                a = grad(al, be)
                b = grad(be, al)
                if self.spatial_scheme == "ccd_stress_legacy":
                    stress = torch.empty_like(a)
                    _lib.check(lib.tpf_visc_stress(a.numel(), _lib.dptr(mt), _lib.dptr(a), _lib.dptr(b),
                                                   _lib.dptr(stress), tdt, st))
                    g = ccd.first_derivative(stress, be)
                    _lib.check(lib.tpf_visc_accumulate(g.numel(), _lib.dptr(g), 1 if be else 0, 1 if last else 0,
                                                       _lib.dptr(rt), float(self.Re), _lib.dptr(total), tdt, st))
                else:
                    lowfd(total, be, a, b, mt, accumulate=be > 0, finalize=last)
            out.append(vs[al].out(total))
        return out

    def _band_evaluate(self, vel, mt, rt, psi, ccd, lowfd, dtype) -> List:
        """ccd_bulk with psi (viscous_spatial.py:50-64,158-221): inside the
        interface band the stress divergence whose derivatives are low-order
        along each node's normal axis and CCD along the others; outside it
        mu times the CCD Laplacian; both / (Re rho)."""
        torch = _torch()
        lib = self.lib
        st = _lib.current_stream_handle()
        tdt = _lib.TPF_F64 if dtype == torch.float64 else _lib.TPF_F32
        nd = len(vel)
        n = vel[0].numel()
        p = to_device(psi, dtype=dtype).tensor

        def low(arr, ax):
            out = torch.empty_like(arr)
            lowfd(out, ax, arr)
            return out

        def select(mask, lo, hi, mode, out):
            _lib.check(lib.tpf_visc_select(n, _lib.dptr(mask) if mask is not None else None, _lib.dptr(lo),
                                           _lib.dptr(hi) if hi is not None else None, mode, _lib.dptr(out), tdt, st))

        gpsi = [low(p, a) for a in range(nd)]
        band = torch.empty(p.shape, dtype=torch.uint8, device=p.device)
        normal = [torch.empty_like(band) for _ in range(nd)]
        shape = (C.c_int64 * nd)(*[int(x) for x in p.shape])
        _lib.check(lib.tpf_visc_band_masks(nd, shape, _lib.dptr(p), (C.c_void_p * nd)(*[_lib.dptr(g) for g in gpsi]),
                                           _lib.dptr(band), (C.c_void_p * nd)(*[_lib.dptr(m) for m in normal]),
                                           tdt, st))

        def switch(data, ax):
            out = torch.empty_like(data)
            select(normal[ax], low(data, ax), ccd.first_derivative(data, ax), 0, out)
            return out

        outs = []
        for al in range(nd):
            nt = torch.empty_like(vel[al])
            for be in range(nd):
                stress = torch.empty_like(vel[al])
                # both gradients held by name until the stress kernel is queued (a temporary
                # freed after dptr() would hand its memory to the second one)
                ga, gb = switch(vel[al], be), switch(vel[be], al)
                _lib.check(lib.tpf_visc_stress(n, _lib.dptr(mt), _lib.dptr(ga), _lib.dptr(gb), _lib.dptr(stress),
                                               tdt, st))
                select(normal[be], low(stress, be), ccd.first_derivative(stress, be), 2 if be == 0 else 1, nt)
            lap = torch.empty_like(vel[al])
            for ax in range(nd):
                select(None, ccd.second_derivative(vel[al], ax), None, 2 if ax == 0 else 1, lap)
            out = torch.empty_like(vel[al])
            _lib.check(lib.tpf_visc_band_finalize(n, _lib.dptr(band), _lib.dptr(nt), _lib.dptr(lap), _lib.dptr(mt),
                                                  _lib.dptr(rt), float(self.Re), _lib.dptr(out), tdt, st))
            outs.append(out)
        return outs

    def _evaluate(self, vel: List, mu, rho, ccd, psi=None) -> List:
        return self.compute_explicit(vel, mu, rho, ccd, psi=psi)

    def _combine(self, mode, dt, u, e, rho, vn, vs=None):
        torch = _torch()
        out = torch.empty_like(u)
        _lib.check(self.lib.tpf_cn_predictor_combine(
            u.numel(), mode, float(dt), _lib.dptr(u), _lib.dptr(e), _lib.dptr(rho), _lib.dptr(vn),
            _lib.dptr(vs) if vs is not None else None, _lib.dptr(out),
            _lib.TPF_F64 if u.dtype == torch.float64 else _lib.TPF_F32, _lib.current_stream_handle()))
        return out

    def apply_cn_predictor(self, u_old: List, explicit_rhs: List, mu, rho, ccd, dt: float, psi=None,
                           intermediate_velocity_operator_transform=None, predictor_state_assembly=None,
                           convective_rhs=None, buoyancy_rhs=None) -> List:
        """The viscous predictor step (viscous.py:135-181): forward Euler when
        cn_viscous is False, else the CN strategy (PicardCNAdvance by default)."""
        torch = _torch()
        dtype = getattr(ccd, "dtype", torch.float64)
        vs = [to_device(u, dtype=dtype) for u in u_old]
        u = [v.tensor for v in vs]
        e = [to_device(x, dtype=dtype).tensor for x in explicit_rhs]
        rt = to_device(rho, dtype=dtype).tensor
        if not self.cn_viscous:
            visc_n = self.compute_explicit(u, mu, rt, ccd)
            return [vs[c].out(self._combine(0, dt, u[c], e[c], rt, visc_n[c])) for c in range(len(u))]
        adv = self.cn_advance if self.cn_advance is not None else PicardCNAdvance(self.backend)
        out = adv.advance(u, e, mu, rt, self, ccd, dt, psi=psi,
                          intermediate_velocity_operator_transform=intermediate_velocity_operator_transform,
                          predictor_state_assembly=predictor_state_assembly, convective_rhs=convective_rhs,
                          buoyancy_rhs=buoyancy_rhs)
        return [vs[c].out(out[c]) for c in range(len(out))]


class RichardsonCNAdvance:
    """Richardson extrapolation around a base CN strategy
    (src/twophase/time_integration/cn_advance/richardson_cn.py:62-109): one
    base step of dt, two of dt/2 from the same frozen explicit right-hand
    side, combined as (4 u_{dt/2,2} - u_dt) / 3 by one kernel."""

    def __init__(self, base):
        self.base = base

    def advance(self, u_old: List, explicit_rhs: List, mu, rho, viscous_op: ViscousTerm, ccd, dt: float, psi=None,
                intermediate_velocity_operator_transform=None, predictor_state_assembly=None, convective_rhs=None,
                buoyancy_rhs=None) -> List:
        torch = _torch()
        kw = dict(psi=psi, intermediate_velocity_operator_transform=intermediate_velocity_operator_transform,
                  predictor_state_assembly=predictor_state_assembly, convective_rhs=convective_rhs,
                  buoyancy_rhs=buoyancy_rhs)
        u1 = self.base.advance(u_old, explicit_rhs, mu, rho, viscous_op, ccd, dt, **kw)
        half = 0.5 * dt
        uh = self.base.advance(u_old, explicit_rhs, mu, rho, viscous_op, ccd, half, **kw)
        u2 = self.base.advance(uh, explicit_rhs, mu, rho, viscous_op, ccd, half, **kw)
        out = []
        lib = viscous_op.lib
        for c in range(len(u_old)):
            o = torch.empty_like(u2[c])
            _lib.check(lib.tpf_cn_predictor_combine(
                o.numel(), 3, 0.0, _lib.dptr(u2[c]), None, None, _lib.dptr(u1[c]), None, _lib.dptr(o),
                _lib.TPF_F64 if o.dtype == torch.float64 else _lib.TPF_F32, _lib.current_stream_handle()))
            out.append(o)
        return out


def make_cn_advance(backend, mode: str = "picard"):
    """``numerics.cn_mode`` -> CN strategy (cn_advance/__init__.py:25-55):
    'picard' or 'richardson_picard'; anything else is a ValueError."""
    if mode == "picard":
        return PicardCNAdvance(backend)
    if mode == "richardson_picard":
        return RichardsonCNAdvance(PicardCNAdvance(backend))
    raise ValueError(f"Unknown cn_mode={mode!r}; supported in this build: 'picard', 'richardson_picard'.")


class PicardCNAdvance:
    """One Picard step on the CN equation, i.e. Heun's predictor-corrector
    (src/twophase/time_integration/cn_advance/picard_cn.py:31-96):
    u_pred = u + dt (e/rho + V(u)); u* = u + dt (e/rho + V(u)/2 + V(u_pred)/2).
    Two viscous evaluations and two combination kernels; the optional
    predictor-assembly and operator-transform hooks are called like the
    reference calls them (with device tensors)."""

    def __init__(self, backend=None):
        self.backend = backend
        self.xp = getattr(backend, "xp", None)

    def advance(self, u_old: List, explicit_rhs: List, mu, rho, viscous_op: ViscousTerm, ccd, dt: float, psi=None,
                intermediate_velocity_operator_transform=None, predictor_state_assembly=None, convective_rhs=None,
                buoyancy_rhs=None) -> List:
        nd = len(u_old)
        visc_n = viscous_op._evaluate(u_old, mu, rho, ccd, psi=psi)
        if predictor_state_assembly is not None:
            u_pred = predictor_state_assembly(u_old=u_old, explicit_rhs=explicit_rhs, convective_rhs=convective_rhs,
                                              buoyancy_rhs=buoyancy_rhs, visc_n=visc_n, rho=rho, dt=dt, xp=self.xp)
        else:
            u_pred = [viscous_op._combine(0, dt, u_old[c], explicit_rhs[c], rho, visc_n[c]) for c in range(nd)]
        u_eval = u_pred
        if intermediate_velocity_operator_transform is not None:
            u_eval = [c.clone() for c in u_pred]
            intermediate_velocity_operator_transform(u_eval)
        visc_star = viscous_op._evaluate(u_eval, mu, rho, ccd, psi=psi)
        return [viscous_op._combine(1, dt, u_old[c], explicit_rhs[c], rho, visc_n[c], visc_star[c])
                for c in range(nd)]
