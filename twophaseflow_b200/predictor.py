"""AB2 + IPC momentum predictor on the GPU with the reference's classes and
signatures (src/twophase/time_integration/ab2_predictor.py:53-209):

* ``ConvectionTerm(backend).compute(ctx_or_velocity, ccd=None)`` -- -(u.grad) u
  with CCD first derivatives (ns_terms/convection.py:23-82);
* ``GravityTerm(backend, Fr, ndim).compute(ctx_or_rho, vel_shape=None)`` --
  -rho/Fr^2 on the last axis (ns_terms/gravity.py:33-86);
* ``SurfaceTensionTerm(backend, We).compute(ctx_or_kappa, psi=None, ...)`` --
  CSF kappa grad(psi) / We with CCD gradients (ns_terms/surface_tension.py:11-96);
* ``Predictor(backend, config, ccd, convection=None, viscous=None,
  gravity=None, surface_tension=None, use_gfm=False).compute(state, dt)`` --
  u* from AB2 convection (forward Euler on the first call), gravity, CSF,
  the IPC term -grad p^n and the viscous predictor (Picard CN, or explicit).

Each term is CCD line solves plus one small kernel; the explicit right-hand
side is one fused kernel per component.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import List, Optional

from . import _lib
from .arrays import to_device
from .step import ccd_pressure_gradient
from .viscous import ViscousTerm, make_cn_advance


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("twophaseflow_b200 needs a CUDA device; there is no CPU fallback")
    return torch


def _tdt(t):
    torch = _torch()
    return _lib.TPF_F64 if t.dtype == torch.float64 else _lib.TPF_F32


@dataclass
class NSComputeContext:
    """Fields the NS terms read (ns_terms/context.py)."""

    velocity: List
    ccd: object
    rho: object = None
    mu: object = None
    kappa: object = None
    psi: object = None


@dataclass
class FlowState:
    """One time level's fields (core/flow_state.py:35-60)."""

    velocity: List
    psi: object
    rho: object
    mu: object
    kappa: object
    pressure: object


class ConvectionTerm:
    """-(u.grad) u_c with CCD first derivatives (ns_terms/convection.py:23-82)."""

    def __init__(self, backend=None):
        self.backend = backend
        self.xp = getattr(backend, "xp", None)
        self.lib = _lib.load()

    def compute(self, ctx_or_velocity, ccd=None) -> List:
        torch = _torch()
        if ccd is None:
            vel_in, ccd = ctx_or_velocity.velocity, ctx_or_velocity.ccd
        else:
            vel_in = ctx_or_velocity
        vs = [to_device(v, dtype=ccd.dtype) for v in vel_in]
        vel = [v.tensor for v in vs]
        st = _lib.current_stream_handle()
        out = []
        for c in range(len(vel)):
            acc = torch.empty_like(vel[c])
            for ax in range(len(vel)):
                du = ccd.first_derivative(vel[c], ax)
                _lib.check(self.lib.tpf_ns_conv_accumulate(acc.numel(), 1 if ax == 0 else 0, _lib.dptr(vel[ax]),
                                                           _lib.dptr(du), _lib.dptr(acc), _tdt(acc), st))
            out.append(vs[c].out(acc))
        return out


class GravityTerm:
    """Body force -rho/Fr^2 on the last axis, zeros elsewhere (ns_terms/gravity.py:33-86)."""

    def __init__(self, backend, Fr: float, ndim: int):
        self.backend = backend
        self.xp = getattr(backend, "xp", None)
        self.Fr = Fr
        self.ndim = ndim
        self.grav_axis = ndim - 1
        self.lib = _lib.load()

    def compute(self, ctx_or_rho, vel_shape=None) -> List:
        torch = _torch()
        rho_in = ctx_or_rho if vel_shape is not None else ctx_or_rho.rho
        v = to_device(rho_in)
        rho = v.tensor
        out = [torch.zeros_like(rho) for _ in range(self.ndim)]
        _lib.check(self.lib.tpf_ns_scaled(rho.numel(), 0, _lib.dptr(rho), None, float(self.Fr ** 2),
                                          _lib.dptr(out[self.grav_axis]), _tdt(rho), _lib.current_stream_handle()))
        return [v.out(t) for t in out]


class SurfaceTensionTerm:
    """CSF force kappa dpsi/dx_a / We with CCD gradients (ns_terms/surface_tension.py:11-96)."""

    def __init__(self, backend, We: float):
        self.backend = backend
        self.xp = getattr(backend, "xp", None)
        self.We = We
        self.lib = _lib.load()

    def compute(self, ctx_or_kappa, psi=None, sigma=None, ccd=None, grad_op=None) -> List:
        torch = _torch()
        if psi is not None and ccd is not None:
            kappa_in = ctx_or_kappa
        else:
            ctx = ctx_or_kappa
            kappa_in, psi, ccd = ctx.kappa, ctx.psi, ctx.ccd
        if grad_op is not None:
            raise NotImplementedError("a custom gradient operator is not supported on the B200 path")
        v = to_device(kappa_in, dtype=ccd.dtype)
        kappa = v.tensor
        p = to_device(psi, dtype=ccd.dtype).tensor
        out = []
        for ax in range(ccd.ndim):
            d = ccd.first_derivative(p, ax)
            f = torch.empty_like(kappa)
            _lib.check(self.lib.tpf_ns_scaled(f.numel(), 1, _lib.dptr(kappa), _lib.dptr(d), float(self.We),
                                              _lib.dptr(f), _tdt(f), _lib.current_stream_handle()))
            out.append(v.out(f))
        return out


class Predictor:
    """u* by AB2 + IPC (time_integration/ab2_predictor.py:53-209)."""

    def __init__(self, backend, config, ccd, convection=None, viscous=None, gravity=None, surface_tension=None,
                 use_gfm: bool = False):
        self.backend = backend
        self.xp = getattr(backend, "xp", None)
        self.config = config
        self.ccd = ccd
        self.use_gfm = use_gfm
        fluid, numerics = config.fluid, config.numerics
        ndim = config.grid.ndim
        cn_mode = str(getattr(numerics, "cn_mode", "picard")).strip().lower()
        self.convection = convection or ConvectionTerm(backend)
        self.viscous = viscous or ViscousTerm(backend, fluid.Re, getattr(numerics, "cn_viscous", True),
                                              cn_advance=make_cn_advance(backend, cn_mode))
        self.gravity = gravity or GravityTerm(backend, fluid.Fr, ndim)
        self.surface_tens = surface_tension or SurfaceTensionTerm(backend, fluid.We)
        self._conv_prev: Optional[List] = None
        self._ab2_ready = False
        self.lib = _lib.load()

    def compute(self, state, dt: float) -> List:
        torch = _torch()
        ccd = self.ccd
        ndim = self.config.grid.ndim
        dtype = ccd.dtype
        vs = [to_device(v, dtype=dtype) for v in state.velocity]
        vel = [v.tensor for v in vs]
        rho = to_device(state.rho, dtype=dtype).tensor
        mu = to_device(state.mu, dtype=dtype).tensor
        kappa = to_device(state.kappa, dtype=dtype).tensor if state.kappa is not None else None
        psi = to_device(state.psi, dtype=dtype).tensor if state.psi is not None else None
        ctx = NSComputeContext(velocity=vel, ccd=ccd, rho=rho, mu=mu, kappa=kappa, psi=psi)
        conv_n = [to_device(c, dtype=dtype).tensor for c in self.convection.compute(ctx)]
        grav = [to_device(g, dtype=dtype).tensor for g in self.gravity.compute(ctx)]
        st_f = None if self.use_gfm else [to_device(f, dtype=dtype).tensor for f in self.surface_tens.compute(ctx)]
        gradp = ccd_pressure_gradient(ccd, to_device(state.pressure, dtype=dtype).tensor, ndim)
        ab2 = self._ab2_ready and self._conv_prev is not None
        st = _lib.current_stream_handle()
        explicit_rhs = []
        for c in range(ndim):
            e = torch.empty_like(vel[c])
            _lib.check(self.lib.tpf_ns_explicit_rhs(
                e.numel(), 1 if ab2 else 0, _lib.dptr(conv_n[c]), _lib.dptr(self._conv_prev[c]) if ab2 else None,
                _lib.dptr(rho), _lib.dptr(grav[c]), _lib.dptr(st_f[c]) if st_f is not None else None,
                _lib.dptr(gradp[c]), _lib.dptr(e), _tdt(e), st))
            explicit_rhs.append(e)
        if getattr(self.config.numerics, "cn_viscous", True):
            vel_star = self.viscous.apply_cn_predictor(vel, explicit_rhs, mu, rho, ccd, dt)
            vel_star = [to_device(u, dtype=dtype).tensor for u in vel_star]
        else:
            visc = [to_device(x, dtype=dtype).tensor for x in self.viscous.compute_explicit(vel, mu, rho, ccd)]
            vel_star = []
            for c in range(ndim):
                u = torch.empty_like(vel[c])
                _lib.check(self.lib.tpf_cn_predictor_combine(u.numel(), 2, float(dt), _lib.dptr(vel[c]),
                                                             _lib.dptr(explicit_rhs[c]), _lib.dptr(rho),
                                                             _lib.dptr(visc[c]), None, _lib.dptr(u), _tdt(u), st))
                vel_star.append(u)
        # the stored convection is updated in place once it exists, so a CUDA
        # graph that captured this call keeps reading and writing the same buffers
        if self._conv_prev is None:
            self._conv_prev = [c.clone() for c in conv_n]
        else:
            for c in range(ndim):
                self._conv_prev[c].copy_(conv_n[c])
        self._ab2_ready = True
        return [vs[c].out(vel_star[c]) for c in range(ndim)]
