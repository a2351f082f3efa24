"""Interface geometry and material properties from the CLS field psi on the GPU,
with the reference's classes and signatures.

* ``CurvatureCalculatorPsi(backend, ccd, psi_min=0.01, gaussian_filter=False,
  dccd_eps=0.05).compute(psi)`` -- curvature straight from psi
  (src/twophase/levelset/curvature_psi.py:55-173): CCD first / second
  derivatives (the B200 CCD kernels), the DCCD dissipative filter weighted by
  (2 psi - 1)^2 (curvature.py:60-127), the mixed derivatives by sequential
  CCD, the 2-D / 3-D curvature formula with the far-field mask, optional 3x3
  Gaussian (2-D).
* ``dccd_filter_nd(f, grid, eps_d, bc_type, switch)`` -- that filter alone.
* ``update_properties(xp, psi, rho_l, rho_g, mu_l, mu_g)`` -- rho and mu
  (heaviside.py:167-187) in one kernel.
"""

from __future__ import annotations

import ctypes as C

from . import _lib
from .arrays import to_device
from .grid import boundary_axes

DCCD_EPS_D = 0.05   # curvature.py:43


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("twophaseflow_b200 needs a CUDA device; there is no CPU fallback")
    return torch


def _tdtype(t):
    torch = _torch()
    if t.dtype == torch.float64:
        return _lib.TPF_F64
    if t.dtype == torch.float32:
        return _lib.TPF_F32
    raise ValueError("fields must be float64 or float32")


def _filter_tensor(f, grid, eps_d: float, bc_type: str, switch=None):
    torch = _torch()
    nd = f.dim()
    if nd not in (2, 3):
        raise ValueError("the DCCD filter is 2-D or 3-D")
    axes = boundary_axes(bc_type, nd)
    shape = (C.c_int64 * nd)(*[int(s) for s in f.shape])
    per = (C.c_int * nd)(*[1 if axes[a] == "periodic" else 0 for a in range(nd)])
    out = torch.empty_like(f)
    tmp = torch.empty_like(f) if nd == 3 else None
    sw = switch.contiguous() if switch is not None else None
    _lib.check(_lib.load().tpf_dccd_filter(nd, shape, per, float(eps_d), _lib.dptr(sw) if sw is not None else None,
                                           _lib.dptr(f), _lib.dptr(out), _lib.dptr(tmp) if tmp is not None else None,
                                           _tdtype(f), _lib.current_stream_handle()))
    return out


def dccd_filter_nd(f, grid, eps_d: float, *, bc_type: str = "wall", switch=None):
    """DCCD filter along every axis, wall planes restored (curvature.py:105-127)."""
    v = to_device(f)
    sw = to_device(switch, dtype=v.tensor.dtype).tensor if switch is not None else None
    return v.out(_filter_tensor(v.tensor, grid, eps_d, bc_type, sw))


class CurvatureCalculatorPsi:
    """kappa from psi (curvature_psi.py:55-173) on a ``twophaseflow_b200.CCDSolver``."""

    def __init__(self, backend, ccd, psi_min: float = 0.01, gaussian_filter: bool = False,
                 dccd_eps: float = DCCD_EPS_D):
        self.backend = backend
        self.xp = getattr(backend, "xp", None)
        self.ccd = ccd
        self.psi_min = psi_min
        self.gaussian_filter = gaussian_filter
        self.dccd_eps = dccd_eps

    def compute(self, psi):
        torch = _torch()
        ccd = self.ccd
        ndim = ccd.ndim
        if ndim not in (2, 3):
            raise ValueError("curvature is 2-D or 3-D")
        v = to_device(psi, dtype=ccd.dtype)
        p = v.tensor
        filt = self.dccd_eps > 0
        switch = (2.0 * p - 1.0) ** 2 if filt else None

        def F(g):
            return _filter_tensor(g, ccd.grid, self.dccd_eps, ccd.bc_type, switch) if filt else g

        d1, d2 = [], []
        for ax in range(ndim):
            g1, g2 = ccd.differentiate(p, ax)
            d1.append(F(g1))
            d2.append(F(g2))
        # mixed derivatives by sequential CCD, first derivative only (the same
        # line solve; the unused second derivative is not written)
        if ndim == 2:
            mixed = [F(ccd.first_derivative(d1[0], 1))]
        else:   # the 3-D formula uses them unfiltered (curvature_psi.py:153-162)
            mixed = [ccd.first_derivative(d1[i], j) for i in range(3) for j in range(i + 1, 3)]
        kappa = torch.empty_like(p)
        P = C.c_void_p * 3
        pd1 = P(*([_lib.dptr(t) for t in d1] + [None] * (3 - ndim)))
        pd2 = P(*([_lib.dptr(t) for t in d2] + [None] * (3 - ndim)))
        pmx = P(*([_lib.dptr(t) for t in mixed] + [None] * (3 - len(mixed))))
        _lib.check(_lib.load().tpf_curvature_psi(ndim, p.numel(), _lib.dptr(p), pd1, pd2, pmx, float(self.psi_min),
                                                 _lib.dptr(kappa), _tdtype(p), _lib.current_stream_handle()))
        if self.gaussian_filter and ndim == 2:
            sm = torch.empty_like(kappa)
            _lib.check(_lib.load().tpf_gaussian3x3(int(kappa.shape[0]), int(kappa.shape[1]), _lib.dptr(kappa),
                                                   _lib.dptr(sm), _tdtype(kappa), _lib.current_stream_handle()))
            kappa = sm
        return v.out(kappa)


def update_properties(xp, psi, rho_l: float, rho_g: float, mu_l: float, mu_g: float):
    """(rho, mu) = (rho_g + (rho_l - rho_g) psi, mu_g + (mu_l - mu_g) psi) (heaviside.py:167-187)."""
    torch = _torch()
    v = to_device(psi)
    p = v.tensor
    if p.dtype not in (torch.float64, torch.float32):
        p = p.to(torch.float64)
    rho = torch.empty_like(p)
    mu = torch.empty_like(p)
    _lib.check(_lib.load().tpf_update_properties(p.numel(), _lib.dptr(p), float(rho_l), float(rho_g), float(mu_l),
                                                 float(mu_g), _lib.dptr(rho), _lib.dptr(mu), _tdtype(p),
                                                 _lib.current_stream_handle()))
    return v.out(rho), v.out(mu)
