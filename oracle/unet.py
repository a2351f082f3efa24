"""CPU oracle of the learned PPE preconditioner network (TEST INFRASTRUCTURE ONLY).

The reference has no learned component (its PPE Krylov loops are SciPy's
``cg`` / ``gmres``, src/twophase/ppe/gmres_helpers.py:16-80), so this module
restates the library's own network definition in NumPy: the 4-level U-Net
(3x3 convolutions, channels 16-32-64-128, 2x2 average pooling, 2x nearest
upsampling, additive skips, ReLU, 1x1 output), its backward pass, and the
training loss (relative squared error).

``precision="bf16"`` rounds at the same points as the CUDA kernels: weights
of the 3x3 convolutions, the packed input and every stored activation /
activation gradient are rounded to BF16 (round to nearest even); sums are
carried in float64 here (FP32 on the GPU).  ``precision="fp64"`` rounds
nowhere; it is the version the finite-difference check runs on.

Parameter layout (flat FP32, identical to the library's): for each of the 14
convolutions W[cout][cin][3][3] then b[cout]; then w_out[16], b_out.
Arrays are [B, H, W, C] (unpadded; zero padding is applied per convolution).
"""

from __future__ import annotations

import numpy as np

LAYERS = [(4, 16, 0, 1), (16, 16, 0, 1), (16, 32, 1, 1), (32, 32, 1, 1),
          (32, 64, 2, 1), (64, 64, 2, 1), (64, 128, 3, 1), (128, 128, 3, 1),
          (128, 64, 3, 0), (64, 64, 2, 1), (64, 32, 2, 0), (32, 32, 1, 1),
          (32, 16, 1, 0), (16, 16, 0, 1)]
OUT_C = 16


def param_layout():
    offs = []
    o = 0
    for cin, cout, _lvl, _relu in LAYERS:
        w = o
        o += cout * cin * 9
        b = o
        o += cout
        offs.append((w, b))
    wo = o
    o += OUT_C
    bo = o
    o += 1
    return offs, wo, bo, o


def num_params() -> int:
    return param_layout()[3]


def init_params(seed: int = 0, out_scale: float = 1.0) -> np.ndarray:
    """He-normal weights, zero biases (float32)."""
    rng = np.random.default_rng(seed)
    offs, wo, bo, n = param_layout()
    p = np.zeros(n, np.float32)
    for (cin, cout, _l, _r), (w, _b) in zip(LAYERS, offs):
        std = np.sqrt(2.0 / (cin * 9))
        p[w:w + cout * cin * 9] = (rng.standard_normal(cout * cin * 9) * std).astype(np.float32)
    p[wo:wo + OUT_C] = (rng.standard_normal(OUT_C) * np.sqrt(1.0 / OUT_C) * out_scale).astype(np.float32)
    return p


def bf16(x):
    """Round float32 values to the nearest BF16 (ties to even), returned as float32."""
    x = np.ascontiguousarray(np.asarray(x, np.float32))
    b = x.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32)


class _Net:
    def __init__(self, params, precision):
        self.lowp = precision == "bf16"
        self.p = np.asarray(params, np.float32 if self.lowp else np.float64)
        offs, wo, bo, _ = param_layout()
        self.W, self.b = [], []
        for (cin, cout, _l, _r), (w, b) in zip(LAYERS, offs):
            Wl = self.p[w:w + cout * cin * 9].reshape(cout, cin, 3, 3).astype(np.float64)
            if self.lowp:
                Wl = bf16(Wl).astype(np.float64)
            self.W.append(Wl)
            self.b.append(self.p[b:b + cout].astype(np.float64))
        self.wo = self.p[wo:wo + OUT_C].astype(np.float64)
        self.bo = float(self.p[bo])

    def r(self, x):
        """Storage rounding of an activation (or activation gradient)."""
        return bf16(x).astype(np.float64) if self.lowp else x


def _pad(x):
    return np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))


def conv3x3(x, W):
    """y[b,h,w,o] = sum_{ky,kx,c} xpad[b,h+ky,w+kx,c] W[o,c,ky,kx]."""
    B, H, Wd, _ = x.shape
    xp = _pad(x)
    y = np.zeros((B, H, Wd, W.shape[0]))
    for ky in range(3):
        for kx in range(3):
            y += np.einsum("bhwc,oc->bhwo", xp[:, ky:ky + H, kx:kx + Wd, :], W[:, :, ky, kx], optimize=True)
    return y


def conv3x3_bwd_data(dz, W):
    B, H, Wd, _ = dz.shape
    dp = _pad(dz)
    dx = np.zeros((B, H, Wd, W.shape[1]))
    for ky in range(3):
        for kx in range(3):
            dx += np.einsum("bhwo,oc->bhwc", dp[:, 2 - ky:2 - ky + H, 2 - kx:2 - kx + Wd, :], W[:, :, ky, kx],
                            optimize=True)
    return dx


def conv3x3_bwd_weight(x, dz):
    B, H, Wd, _ = x.shape
    xp = _pad(x)
    gW = np.zeros((dz.shape[3], x.shape[3], 3, 3))
    for ky in range(3):
        for kx in range(3):
            gW[:, :, ky, kx] = np.einsum("bhwo,bhwc->oc", dz, xp[:, ky:ky + H, kx:kx + Wd, :], optimize=True)
    return gW, dz.sum(axis=(0, 1, 2))


def pool(x):
    B, H, W, C = x.shape
    return x.reshape(B, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4))


def up(x):
    return x.repeat(2, axis=1).repeat(2, axis=2)


def downsum(x):
    B, H, W, C = x.shape
    return x.reshape(B, H // 2, 2, W // 2, 2, C).sum(axis=(2, 4))


def forward(params, in2, precision="bf16"):
    """y[B,H,W] of the network for in2[B,H,W,4]; returns (y, activations)."""
    n = _Net(params, precision)
    x = np.asarray(in2, np.float64)
    x = n.r(x)
    A = {"xin": x}

    def c(l, inp):
        z = conv3x3(inp, n.W[l]) + n.b[l]
        if LAYERS[l][3]:
            z = np.maximum(z, 0.0)
        return n.r(z)

    A["e0a"] = c(0, x)
    A["e0"] = c(1, A["e0a"])
    A["p0"] = n.r(pool(A["e0"]))
    A["e1a"] = c(2, A["p0"])
    A["e1"] = c(3, A["e1a"])
    A["p1"] = n.r(pool(A["e1"]))
    A["e2a"] = c(4, A["p1"])
    A["e2"] = c(5, A["e2a"])
    A["p2"] = n.r(pool(A["e2"]))
    A["e3a"] = c(6, A["p2"])
    A["e3"] = c(7, A["e3a"])
    A["t2"] = c(8, A["e3"])
    A["d2a"] = n.r(np.maximum(up(A["t2"]) + A["e2"], 0.0))
    A["d2"] = c(9, A["d2a"])
    A["t1"] = c(10, A["d2"])
    A["d1a"] = n.r(np.maximum(up(A["t1"]) + A["e1"], 0.0))
    A["d1"] = c(11, A["d1a"])
    A["t0"] = c(12, A["d1"])
    A["d0a"] = n.r(np.maximum(up(A["t0"]) + A["e0"], 0.0))
    A["d0"] = c(13, A["d0a"])
    y = A["d0"] @ n.wo + n.bo
    return y, A


def backward(params, A, dy, precision="bf16"):
    """Flat parameter gradient of sum(dy * y) for the activations A of forward()."""
    n = _Net(params, precision)
    offs, wo, bo, total = param_layout()
    g = np.zeros(total)
    dy = np.asarray(dy, np.float64)
    g[wo:wo + OUT_C] = np.einsum("bhw,bhwc->c", dy, A["d0"])
    g[bo] = dy.sum()

    def mask(t, act):
        return t * (act > 0)

    def wg(l, x, dz):
        gW, gb = conv3x3_bwd_weight(x, dz)
        w, b = offs[l]
        g[w:w + gW.size] = gW.ravel()
        g[b:b + gb.size] = gb

    def bd(l, dz, act=None):
        t = conv3x3_bwd_data(dz, n.W[l])
        if act is not None:
            t = mask(t, act)
        return n.r(t)

    g_d0 = n.r(mask(dy[..., None] * n.wo, A["d0"]))
    wg(13, A["d0a"], g_d0)
    g_d0a = bd(13, g_d0, A["d0a"])
    g_t0 = n.r(downsum(g_d0a))
    wg(12, A["d1"], g_t0)
    g_d1 = bd(12, g_t0, A["d1"])
    wg(11, A["d1a"], g_d1)
    g_d1a = bd(11, g_d1, A["d1a"])
    g_t1 = n.r(downsum(g_d1a))
    wg(10, A["d2"], g_t1)
    g_d2 = bd(10, g_t1, A["d2"])
    wg(9, A["d2a"], g_d2)
    g_d2a = bd(9, g_d2, A["d2a"])
    g_t2 = n.r(downsum(g_d2a))
    wg(8, A["e3"], g_t2)
    g_e3 = bd(8, g_t2, A["e3"])
    wg(7, A["e3a"], g_e3)
    g_e3a = bd(7, g_e3, A["e3a"])
    wg(6, A["p2"], g_e3a)
    g_p2 = bd(6, g_e3a)
    g_e2 = n.r(mask(0.25 * up(g_p2) + g_d2a, A["e2"]))
    wg(5, A["e2a"], g_e2)
    g_e2a = bd(5, g_e2, A["e2a"])
    wg(4, A["p1"], g_e2a)
    g_p1 = bd(4, g_e2a)
    g_e1 = n.r(mask(0.25 * up(g_p1) + g_d1a, A["e1"]))
    wg(3, A["e1a"], g_e1)
    g_e1a = bd(3, g_e1, A["e1a"])
    wg(2, A["p0"], g_e1a)
    g_p0 = bd(2, g_e1a)
    g_e0 = n.r(mask(0.25 * up(g_p0) + g_d0a, A["e0"]))
    wg(1, A["e0a"], g_e0)
    g_e0a = bd(1, g_e0, A["e0a"])
    wg(0, A["xin"], g_e0a)
    return g


def loss(y, target):
    """Mean over the batch of sum (y - t)^2 / sum t^2, and dL/dy."""
    y = np.asarray(y, np.float64)
    t = np.asarray(target, np.float64)
    B = y.shape[0]
    s = np.maximum((t * t).reshape(B, -1).sum(axis=1), 1e-300)
    e = ((y - t) ** 2).reshape(B, -1).sum(axis=1)
    dy = 2.0 * (y - t) / (B * s[:, None, None])
    return float(np.mean(e / s)), dy
