"""CPU checks of the U-Net oracle: its backward pass against finite differences
(FP64 mode) and the BF16 rounding helper."""

from __future__ import annotations

import numpy as np

from oracle import unet as ou


def test_bf16_rounding_ties_to_even():
    x = np.array([1.0, 1.0 + 2**-8, 1.0 + 3 * 2**-8, -2.5, 3.140625], np.float32)
    r = ou.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                  # tie -> even mantissa
    assert r[2] == np.float32(1.0 + 4 * 2**-8)
    assert r[3] == -2.5 and r[4] == np.float32(3.140625)


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(3)
    p = ou.init_params(seed=1)
    B, H, W = 2, 16, 16
    x = rng.standard_normal((B, H, W, 4))
    dy = rng.standard_normal((B, H, W))
    y, A = ou.forward(p, x, precision="fp64")
    g = ou.backward(p, A, dy, precision="fp64")
    offs, wo, bo, total = ou.param_layout()
    picks = [wo + 3, bo]
    for (w, b) in offs:
        picks += [w + 5, w + 17, b]
    h = 1e-6  # ReLU kinks make larger steps inexact
    for i in picks:
        pp, pm = p.astype(np.float64).copy(), p.astype(np.float64).copy()
        pp[i] += h
        pm[i] -= h
        fp = float(np.sum(dy * ou.forward(pp, x, precision="fp64")[0]))
        fm = float(np.sum(dy * ou.forward(pm, x, precision="fp64")[0]))
        num = (fp - fm) / (2 * h)
        assert abs(num - g[i]) <= 1e-5 * max(1.0, abs(num)), (i, num, g[i])


def test_loss_gradient():
    rng = np.random.default_rng(0)
    y = rng.standard_normal((2, 4, 4))
    t = rng.standard_normal((2, 4, 4))
    L, dy = ou.loss(y, t)
    h = 1e-6
    y2 = y.copy()
    y2[1, 2, 3] += h
    L2, _ = ou.loss(y2, t)
    assert abs((L2 - L) / h - dy[1, 2, 3]) < 1e-4


def test_default_aggregation_matches_training_coarse_size():
    """The learned solver aggregates so that the network's coarse grid is
    nearest the size it was trained on (grid / coarsen of the training run,
    read from the weights' metadata): 4 x 4 up to ~720 cells per axis for the
    shipped 512 / 4 training, 8 x 8 beyond."""
    from twophaseflow_b200.learned import default_coarsen, load_meta
    meta = load_meta()
    assert meta["grid"] == 512 and meta["coarsen"] == 4
    assert [default_coarsen((n + 1, n + 1), meta) for n in (64, 256, 512, 700)] == [4, 4, 4, 4]
    assert [default_coarsen((n + 1, n + 1), meta) for n in (1024, 2048)] == [8, 8]
    assert default_coarsen((1025, 257), meta) == 8          # the longest axis decides
    assert default_coarsen((1025, 1025), {"grid": 1024, "coarsen": 4}) == 4   # other training sizes
    assert default_coarsen((513, 513), {}) == 4              # no metadata: the shipped training size


def test_shipped_weights_metadata():
    """The shipped parameters come from the project's own GPU training: 20 000
    (residual, correction) pairs of plain-PCG runs on 2 500 seeded 512^2
    droplet / bubble densities, energy loss, two-level mode (4x4 aggregates)."""
    from twophaseflow_b200.learned import load_meta, load_params, num_params
    meta = load_meta()
    assert meta["pairs"] == 20000 and meta["cases"] == 2500 and meta["grid"] == 512
    assert meta["loss"] == "energy" and meta["coarsen"] == 4
    hist = meta["loss_history"]
    assert len(hist) == meta["epochs"] and hist[-1] < hist[0]
    p = load_params()
    assert p.shape == (num_params(),) and np.all(np.isfinite(p))
