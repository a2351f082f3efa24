"""Train the learned PPE preconditioner on the GPU.

    python -m twophaseflow_b200.train_preconditioner [--grid 256] [--cases 400]
        [--epochs 8] [--batch 16] [--lr 1e-3] [--seed 0] [--out PATH]

1. Pairs: for ``--cases`` seeded densities (4..16 droplets or one bubble,
   density ratio 10..1000) on a ``--grid``^2 box, the plain Jacobi PCG solver
   runs to convergence and its iterates x_k at several k give pairs
   (S e_k, e_k), e_k = x* - x_k, stored in the Jacobi-scaled normalised form
   the network reads (tpf_lppe_pair).
2. Training: Adam (cosine-decayed learning rate) on the relative squared
   error, forward/backward/update all in libtpf.so.
3. The parameters are written to ``--out`` (default: the package's weights
   file) with the loss history.
"""

from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from .learned import DEFAULT_WEIGHTS, UNet, generate_pairs, net_image, train


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--grid", type=int, default=256)
    ap.add_argument("--cases", type=int, default=400)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--weight-decay", type=float, default=0.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--coarsen", type=int, default=4, help="aggregate size of the two-level mode (1: fine-grid network)")
    ap.add_argument("--omega", type=float, default=0.8, help="damping of the pre-smoothing sweep")
    ap.add_argument("--loss", choices=["energy", "l2"], default="energy",
                    help="energy: A-norm error left by the coarse correction (two-level mode); l2: squared error")
    ap.add_argument("--init", default=None, help="start from these parameters (.npz)")
    ap.add_argument("--out", default=DEFAULT_WEIGHTS)
    a = ap.parse_args(argv)

    import torch
    t0 = time.perf_counter()
    N = (a.grid, a.grid)
    energy = a.loss == "energy" and a.coarsen > 1
    data = generate_pairs(N=N, n_cases=a.cases, seed=a.seed, coarsen=a.coarsen, omega=a.omega, energy=energy,
                          log=print)
    in2, tgt = data[0], data[1]
    esc = data[2] if energy else None
    torch.cuda.synchronize()
    t_pairs = time.perf_counter() - t0
    print(f"{in2.shape[0]} pairs in {t_pairs:.1f} s", flush=True)
    params = None
    if a.init:
        with np.load(a.init) as d:
            params = d["params"]
    H, W = net_image((a.grid + 1, a.grid + 1), a.coarsen)
    net = UNet(H, W, a.batch, params=params, seed=a.seed)
    t1 = time.perf_counter()
    nc = (-(-(a.grid + 1) // a.coarsen), -(-(a.grid + 1) // a.coarsen))
    hist = train(net, in2, tgt, epochs=a.epochs, batch=a.batch, lr=a.lr, weight_decay=a.weight_decay, seed=a.seed,
                 log=lambda m: print(m, flush=True), escale=esc, coarse=nc)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t1
    meta = {"grid": a.grid, "coarsen": a.coarsen, "omega": a.omega, "loss": "energy" if energy else "l2",
            "cases": a.cases, "pairs": int(in2.shape[0]), "epochs": a.epochs, "batch": a.batch,
            "lr": a.lr, "seed": a.seed, "loss_history": hist, "pair_seconds": t_pairs, "train_seconds": t_train}
    net.save(a.out, meta=json.dumps(meta))
    print(json.dumps(meta))
    return 0


if __name__ == "__main__":
    sys.exit(main())
