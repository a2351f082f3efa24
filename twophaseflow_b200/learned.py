"""Learned PPE preconditioner: U-Net network, training, and the flexible Krylov solver.

The reference has no learned component (its PPE Krylov loops are SciPy's
``cg`` / ``gmres``, src/twophase/ppe/gmres_helpers.py:16-80).  This module is
the B200 addition built on top of the plain method:

* ``UNet`` -- the 4-level U-Net (3x3 convolutions, channels 16-32-64-128,
  BF16 weights and activations, FP32 accumulation) whose forward, backward
  and Adam kernels run in ``libtpf.so`` (tpf_unet_*; tcgen05 tensor cores).
* ``generate_pairs`` -- (residual, correction) training pairs produced by the
  plain PPE solver itself: for seeded droplet/bubble densities it solves the
  PPE with Jacobi PCG and takes the CG iterates x_k along the way; each pair
  is (r_k = S e_k, e_k = x* - x_k) in the Jacobi-scaled, normalised form the
  network sees (tpf_lppe_pair).
* ``train`` -- Adam on the relative squared error of the scaled correction.
* ``PPESolverLearned`` -- an ``IPPESolver`` with the reference's
  ``solve(rhs, rho, dt, p_init)`` contract whose solve is flexible GMRES (or
  flexible CG) preconditioned by the network (tpf_lppe_solve), checked on the
  true residual, falling back to plain Jacobi PCG when the residual stalls.

All arithmetic runs on the GPU in the CUDA library; PyTorch only holds device
memory.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib
from .arrays import to_device
from .ppe import PPESolverFVMMatrixFree

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_WEIGHTS = os.path.join(HERE, "weights", "unet_ppe.npz")

# (cin, cout) of the 14 convolutions, then the 16 -> 1 output layer; the 4 input
# channels are the scaled residual, the density feature and the two scaled
# couplings of the (fine or coarse) operator to the next row / column
IN_CHANNELS = 4
LAYERS = [(4, 16), (16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (64, 128), (128, 128),
          (128, 64), (64, 64), (64, 32), (32, 32), (32, 16), (16, 16)]


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("the learned preconditioner needs a CUDA device; there is no CPU fallback")
    return torch


def round8(n: int) -> int:
    return (int(n) + 7) // 8 * 8


def net_image(shape, coarsen: int):
    """Network image for a 2-D node grid: nodes (coarsen = 1) or b x b aggregates,
    rounded up to multiples of 8."""
    b = int(coarsen)
    return round8((int(shape[0]) + b - 1) // b), round8((int(shape[1]) + b - 1) // b)


def num_params() -> int:
    return int(_lib.load().tpf_unet_num_params())


def he_init(seed: int = 0) -> np.ndarray:
    """He-normal convolution weights, zero biases, flat FP32 in the library's layout."""
    rng = np.random.default_rng(seed)
    out = []
    for cin, cout in LAYERS:
        out.append(rng.standard_normal(cout * cin * 9) * np.sqrt(2.0 / (9 * cin)))
        out.append(np.zeros(cout))
    out.append(rng.standard_normal(16) * np.sqrt(1.0 / 16))
    out.append(np.zeros(1))
    p = np.concatenate(out).astype(np.float32)
    assert p.size == num_params()
    return p


class UNet:
    """Device workspace + parameters of the preconditioner network (tpf_unet)."""

    def __init__(self, H: int, W: int, max_batch: int = 1, params=None, seed: int = 0):
        self.lib = _lib.load()
        _torch()
        self.H, self.W, self.max_batch = int(H), int(W), int(max_batch)
        h = C.c_void_p()
        _lib.check(self.lib.tpf_unet_create(C.byref(h), self.H, self.W, self.max_batch))
        self.handle = h
        self.set_params(he_init(seed) if params is None else params)

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None:
            try:
                self.lib.tpf_unet_destroy(h)
            except Exception:
                pass

    def set_params(self, params):
        torch = _torch()
        if isinstance(params, torch.Tensor) and params.is_cuda:
            t = params.detach().to(torch.float32).contiguous()
            _lib.check(self.lib.tpf_unet_set_params(self.handle, _lib.dptr(t), 1))
        else:
            a = np.ascontiguousarray(np.asarray(params, dtype=np.float32))
            if a.size != num_params():
                raise ValueError(f"expected {num_params()} parameters, got {a.size}")
            _lib.check(self.lib.tpf_unet_set_params(self.handle, a.ctypes.data_as(C.c_void_p), 0))

    def get_params(self) -> np.ndarray:
        a = np.empty(num_params(), np.float32)
        _lib.check(self.lib.tpf_unet_get_params(self.handle, a.ctypes.data_as(C.c_void_p), 0))
        return a

    def set_forward_mode(self, mode: int) -> None:
        """0 (default, also -1): one launch per layer; 1: the whole network in one persistent launch."""
        _lib.check(self.lib.tpf_unet_set_forward_mode(self.handle, int(mode)))

    def forward(self, in2):
        """y[B,H,W] for in2[B,H,W,IN_CHANNELS] (FP32 CUDA tensor)."""
        torch = _torch()
        x = in2.to(torch.float32).contiguous()
        B = int(x.shape[0])
        y = torch.empty((B, self.H, self.W), dtype=torch.float32, device=x.device)
        _lib.check(self.lib.tpf_unet_forward(self.handle, B, _lib.dptr(x), _lib.dptr(y),
                                             _lib.current_stream_handle()))
        return y

    def backward(self, dy):
        """Parameter gradient of sum(dy * y) for the last forward (FP32 CUDA tensor)."""
        torch = _torch()
        d = dy.to(torch.float32).contiguous()
        g = torch.empty(num_params(), dtype=torch.float32, device=d.device)
        _lib.check(self.lib.tpf_unet_backward(self.handle, int(d.shape[0]), _lib.dptr(d), _lib.dptr(g),
                                              _lib.current_stream_handle()))
        return g

    def train_step(self, in2, target, lr: float, weight_decay: float = 0.0) -> float:
        loss = C.c_double()
        _lib.check(self.lib.tpf_unet_train_step(self.handle, int(in2.shape[0]), _lib.dptr(in2), _lib.dptr(target),
                                                float(lr), float(weight_decay), C.byref(loss),
                                                _lib.current_stream_handle()))
        return float(loss.value)

    def train_step_energy(self, in2, coupl, escale, nc0: int, nc1: int, lr: float, weight_decay: float = 0.0) -> float:
        """Adam step on the energy loss of a coarse-grid correction (tpf_unet_train_step_energy)."""
        loss = C.c_double()
        _lib.check(self.lib.tpf_unet_train_step_energy(self.handle, int(in2.shape[0]), _lib.dptr(in2), _lib.dptr(coupl),
                                                       _lib.dptr(escale), int(nc0), int(nc1), float(lr),
                                                       float(weight_decay), C.byref(loss),
                                                       _lib.current_stream_handle()))
        return float(loss.value)

    def save(self, path: str, **meta):
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        np.savez(path, params=self.get_params(), **meta)


def load_meta(path: str = DEFAULT_WEIGHTS) -> dict:
    """Training metadata stored beside the parameters ({} when absent)."""
    import json
    with np.load(path) as d:
        if "meta" not in d.files:
            return {}
        return json.loads(str(d["meta"]))


def default_coarsen(shape, meta=None) -> int:
    """Aggregation that puts the network's coarse grid nearest the size it was
    trained on (grid / coarsen of the training run, 512 / 4 = 128 cells for the
    shipped weights): 4, or 8 once the grid has more than ~5.7x that many
    cells per axis.  Both were validated on held-out fields (4 at 512^2, 8 at
    1024^2); with 4 at 1024^2 the coarse problem outgrows the network's
    receptive field and the flexible iteration stalls."""
    meta = meta or {}
    c_train = float(meta.get("grid", 512)) / float(meta.get("coarsen", 4))
    cells = max(int(n) - 1 for n in shape)
    return 8 if cells / c_train > 4 * np.sqrt(2.0) else 4


def load_params(path: str = DEFAULT_WEIGHTS) -> np.ndarray:
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"no trained preconditioner parameters at {path}: train them with "
            "`python -m twophaseflow_b200.train_preconditioner --out <path>` and pass "
            "ppe_learned_weights=<path> (or params=...)")
    with np.load(path) as d:
        return np.asarray(d["params"], np.float32)


# ---------------------------------------------------------------------------------------------
class PPESolverLearned(PPESolverFVMMatrixFree):
    """IPPESolver: flexible GMRES / CG preconditioned by the trained U-Net (2-D, wall).

    Options are read from the solver config like the reference's own
    (``pseudo_tol``, ``pseudo_maxiter``) plus ``ppe_learned_coarsen`` (b > 1:
    the network solves the problem aggregated over b x b node blocks inside a
    two-grid cycle; 1: the network reads the fine residual; default: 4 or 8,
    whichever puts the coarse grid nearest the training size, see
    ``default_coarsen``),
    ``ppe_learned_smooth`` (damped Jacobi sweeps after the network, default 16),
    ``ppe_learned_omega`` (0.8), ``ppe_learned_weights`` (path of the trained
    parameters), ``ppe_learned_fallback`` (finish with plain Jacobi PCG on a
    stall, True) and ``ppe_learned_outer``: 'fgmres' (flexible GMRES with
    restart ``ppe_learned_restart``, default 60: each basis vector
    preconditioned by the network, the solution built from the preconditioned
    basis; the default) or 'fcg' (truncated flexible CG with
    ``ppe_learned_window`` stored directions).  The defaults (FGMRES(60), 16
    sweeps, omega 0.8) were chosen on validation density fields (seeds 21-30
    at 512^2, 21-24 at 1024^2) that neither training nor the benchmark use.
    """

    scheme_names = ("fvm_learned",)

    def __init__(self, backend, config, grid, bc_type: str = "wall", bc_spec=None, params=None):
        super().__init__(backend, config, grid, bc_type=bc_type, bc_spec=bc_spec)
        # the plain route of this solver (stall fallback) is Jacobi PCG
        self.iteration_method = "cg"
        self.preconditioner = "jacobi"
        self.precision = "fp64"
        self._sync_options()
        if self.ndim != 2:
            raise ValueError("the learned preconditioner is two-dimensional")
        solver_cfg = getattr(config, "solver", config)
        self.smooth = int(getattr(solver_cfg, "ppe_learned_smooth", 16))
        self.omega = float(getattr(solver_cfg, "ppe_learned_omega", 0.8))
        self.fallback = bool(getattr(solver_cfg, "ppe_learned_fallback", True))
        self.learned_maxiter = int(getattr(solver_cfg, "ppe_learned_maxiter", max(self.maxiter, 2000)))
        self.window = int(getattr(solver_cfg, "ppe_learned_window", 8))
        outer = str(getattr(solver_cfg, "ppe_learned_outer", "fgmres")).strip().lower()
        if outer not in ("fcg", "fgmres"):
            raise ValueError("ppe_learned_outer must be 'fcg' (flexible CG) or 'fgmres' (flexible GMRES)")
        self.outer = outer
        self.restart = int(getattr(solver_cfg, "ppe_learned_restart", 60))
        meta = {}
        if params is None:
            wpath = str(getattr(solver_cfg, "ppe_learned_weights", DEFAULT_WEIGHTS))
            params = load_params(wpath)
            meta = load_meta(wpath)
        coarsen = getattr(solver_cfg, "ppe_learned_coarsen", None)
        self.coarsen = int(coarsen) if coarsen is not None else default_coarsen(self.grid.shape, meta)
        H, W = net_image(self.grid.shape, self.coarsen)
        self.net = UNet(H, W, 1, params=params)
        self._lp = None
        self._make_lp()

    def _make_lp(self):
        if self._lp is not None:
            self.lib.tpf_lppe_destroy(self._lp)
            self._lp = None
        h = C.c_void_p()
        _lib.check(self.lib.tpf_lppe_create(C.byref(h), self._handle, self.net.handle, self.coarsen))
        self._lp = h

    def __del__(self):
        lp = getattr(self, "_lp", None)
        if lp is not None:
            try:
                self.lib.tpf_lppe_destroy(lp)
            except Exception:
                pass
        super().__del__()

    def update_grid(self, grid=None) -> None:
        super().update_grid(grid)
        self._make_lp()

    def learned_options(self):
        o = _lib.tpf_learned_options()
        self.lib.tpf_lppe_default_options(C.byref(o))
        o.tol = self.tol
        o.maxiter = self.learned_maxiter
        o.smooth = self.smooth
        o.omega = self.omega
        o.fallback = 1 if self.fallback else 0
        o.window = self.window
        o.outer = 1 if self.outer == "fgmres" else 0
        o.restart = self.restart
        return o

    def prepare_operator(self, rho) -> None:
        torch = _torch()
        v = to_device(rho, dtype=torch.float64)
        self._check_shape(v.tensor)
        _lib.check(self.lib.tpf_lppe_prepare(self._lp, _lib.dptr(v.tensor), _lib.current_stream_handle()))
        self._rho_keep = v.tensor
        self._prepared = True

    def precondition(self, r):
        """z = B(r): the network preconditioner (+ smoothing) alone."""
        torch = _torch()
        v = to_device(r, dtype=torch.float64)
        z = torch.empty_like(v.tensor)
        _lib.check(self.lib.tpf_lppe_precondition(self._lp, _lib.dptr(v.tensor), _lib.dptr(z), self.smooth,
                                                  self.omega, _lib.current_stream_handle()))
        return v.out(z)

    def solve(self, rhs, rho, dt: float = 0.0, p_init=None):
        torch = _torch()
        vr = to_device(rhs, dtype=torch.float64)
        vrho = to_device(rho, dtype=torch.float64)
        self._check_shape(vr.tensor)
        self._check_shape(vrho.tensor)
        p0 = None
        if p_init is not None:
            p0 = to_device(p_init, dtype=torch.float64).tensor
            self._check_shape(p0)
        p = torch.empty_like(vr.tensor)
        res = _lib.tpf_lppe_result()
        o = self.learned_options()
        st = self.lib.tpf_lppe_solve(self._lp, _lib.dptr(vr.tensor), _lib.dptr(vrho.tensor), _lib.dptr(p),
                                     _lib.dptr(p0) if p0 is not None else None, C.byref(o),
                                     _lib.current_stream_handle(), C.byref(res))
        self._prepared = True
        self._rho_keep = vrho.tensor
        self.last_diagnostics = {
            "ppe_learned_info": int(res.info),
            "ppe_learned_tol": float(self.tol),
            "ppe_learned_iterations": int(res.iterations),
            "ppe_learned_fallback_iterations": int(res.fallback_iterations),
            "ppe_learned_restarts": int(res.restarts),
            "ppe_learned_fell_back": bool(res.fell_back),
            "ppe_learned_relative_residual": float(res.rel_residual),
        }
        if st == _lib.TPF_ENOCONV:
            raise RuntimeError(f"{type(self).__name__} did not converge cleanly (info={res.info})")
        _lib.check(st)
        return vr.out(p)


# ---------------------------------------------------------------------------------------------
# training data and training
def random_case(N, rng):
    """Seeded density (droplets or a bubble, density ratio 10..1000) and a divergence RHS."""
    from .workloads import bubble_density, divergence_rhs, droplet_density
    ratio = float(10.0 ** rng.uniform(1.0, 3.0))
    seed = int(rng.integers(0, 2**31 - 1))
    if rng.uniform() < 0.75:
        n = int(rng.integers(4, 17))
        rho = droplet_density(N, n_drops=n, rho_l=1.0, rho_g=1.0 / ratio, seed=seed)
    else:
        c = tuple(rng.uniform(0.3, 0.7, size=len(N)))
        rho = bubble_density(N, centre=c, radius=float(rng.uniform(0.1, 0.3)), rho_l=1.0, rho_g=1.0 / ratio)
    rhs = divergence_rhs(N, n_modes=int(rng.integers(4, 13)), seed=seed + 1)
    return rho, rhs


class _Cfg:
    def __init__(self, **kw):
        self.__dict__.update(kw)


def generate_pairs(N=(256, 256), n_cases: int = 64, snapshots=(0, 3, 10, 30, 80, 200, 500, 1000),
                   seed: int = 0, coarsen: int = 4, omega: float = 0.8, energy: bool = False, log=None):
    """Training pairs from plain-PCG runs on the network image of ``coarsen``
    (M = n_cases x len(snapshots)):
    energy=False: (in2 [M,H,W,2], target [M,H,W]) (tpf_lppe_pair);
    energy=True (two-level mode): (in2, coupl [M,H,W,2], escale [M]) for the
    energy loss (tpf_lppe_pair_energy)."""
    torch = _torch()
    from .grid import UniformGrid
    rng = np.random.default_rng(seed)
    grid = UniformGrid(N)
    cfg = _Cfg(pseudo_tol=1e-12, pseudo_maxiter=100000, ppe_iteration_method="cg", ppe_preconditioner="jacobi")
    ppe = PPESolverFVMMatrixFree(None, cfg, grid)
    lib = ppe.lib
    H, W = net_image(grid.shape, coarsen)
    net = UNet(H, W, 1)
    lp = C.c_void_p()
    _lib.check(lib.tpf_lppe_create(C.byref(lp), ppe._handle, net.handle, int(coarsen)))
    M = n_cases * len(snapshots)
    dev = torch.device("cuda")
    in2 = torch.empty((M, H, W, IN_CHANNELS), dtype=torch.float32, device=dev)
    if energy:
        tgt = torch.empty((M, H, W, 2), dtype=torch.float32, device=dev)
        esc = torch.empty((M,), dtype=torch.float64, device=dev)
    else:
        tgt = torch.empty((M, H, W), dtype=torch.float32, device=dev)
    s = _lib.current_stream_handle()
    m = 0
    try:
        for c in range(n_cases):
            rho, rhs = random_case(N, rng)
            rho_t = torch.from_numpy(rho).to(dev)
            rhs_t = torch.from_numpy(rhs).to(dev)
            _lib.check(lib.tpf_lppe_prepare(lp, _lib.dptr(rho_t), s))
            xs = torch.empty_like(rhs_t)
            res = _lib.tpf_ppe_result()
            _lib.check(lib.tpf_ppe_solve(ppe._handle, _lib.dptr(rhs_t), None, _lib.dptr(xs), None, s, C.byref(res)))
            xk = torch.empty_like(rhs_t)
            o = ppe._options()
            for k in snapshots:
                if k == 0:
                    xk.zero_()
                else:
                    o.maxiter = int(k)
                    _lib.check(lib.tpf_ppe_set_options(ppe._handle, C.byref(o)))
                    st = lib.tpf_ppe_solve(ppe._handle, _lib.dptr(rhs_t), None, _lib.dptr(xk), None, s,
                                           C.byref(_lib.tpf_ppe_result()))
                    if st not in (_lib.TPF_OK, _lib.TPF_ENOCONV):
                        _lib.check(st)
                e = (xs - xk).contiguous()
                if energy:
                    _lib.check(lib.tpf_lppe_pair_energy(lp, _lib.dptr(e), _lib.dptr(in2[m]), _lib.dptr(tgt[m]),
                                                        _lib.dptr(esc[m:m + 1]), float(omega), s))
                else:
                    _lib.check(lib.tpf_lppe_pair(lp, _lib.dptr(e), _lib.dptr(in2[m]), _lib.dptr(tgt[m]), float(omega),
                                                 s))
                m += 1
            o.maxiter = 100000
            _lib.check(lib.tpf_ppe_set_options(ppe._handle, C.byref(o)))
            if log and (c + 1) % max(1, n_cases // 8) == 0:
                log(f"pairs: case {c + 1}/{n_cases} ({res.iterations} CG iterations)")
    finally:
        lib.tpf_lppe_destroy(lp)
    torch.cuda.synchronize()
    if energy:
        return in2[:m], tgt[:m], esc[:m]
    return in2[:m], tgt[:m]


def train(net: UNet, in2, target, epochs: int = 10, batch: int = 16, lr: float = 1e-3, weight_decay: float = 0.0,
          seed: int = 0, log=None, escale=None, coarse=None):
    """Adam over shuffled mini-batches with a cosine learning-rate decay; returns per-epoch mean losses.
    With ``escale`` (and ``coarse`` = (nc0, nc1)) ``target`` holds the coarse
    couplings and the energy loss is used."""
    torch = _torch()
    M = int(in2.shape[0])
    g = torch.Generator(device="cpu")
    g.manual_seed(seed)
    steps = epochs * max(1, M // batch)
    step = 0
    history = []
    for ep in range(epochs):
        perm = torch.randperm(M, generator=g)
        losses = []
        for i in range(0, M - batch + 1, batch):
            idx = perm[i:i + batch].to(in2.device)
            xb = in2.index_select(0, idx).contiguous()
            tb = target.index_select(0, idx).contiguous()
            cur = lr * 0.5 * (1.0 + np.cos(np.pi * step / max(1, steps)))
            if escale is not None:
                eb = escale.index_select(0, idx).contiguous()
                losses.append(net.train_step_energy(xb, tb, eb, coarse[0], coarse[1], cur, weight_decay))
            else:
                losses.append(net.train_step(xb, tb, cur, weight_decay))
            step += 1
        history.append(float(np.mean(losses)) if losses else float("nan"))
        if log:
            log(f"epoch {ep + 1}/{epochs}: loss {history[-1]:.4f}")
    return history
