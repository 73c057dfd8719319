"""Train the warm-start network on the GPU and save it.

    python -m mrtrix3_b200.train_warmstart [--n 32000000] [--epochs 60]
        [--lr 4e-3] [--batch 4096] [--seed 11] [--workers <host cores>]
        [--out mrtrix3_b200/data/warmstart_c5.npz]

Signals: seeded synthetic voxels on the 6 b=0 + 60 b=3000 Fibonacci scheme
(1-3 fibres, SNR U[15,40]), generated in blocks of 2^20 voxels on the host
cores; labels: the converged negative sets of the plain GPU CSD.  The
committed data/warmstart_c5.npz was produced by this command with its
defaults (about 2 minutes of generation and 2 minutes of training on one
B200).  The wrong first-set bits per voxel of a fresh volume fall with the
training set: 9.7 (2M voxels), 8.5 (8M), 8.3 (16M), 8.2 (32M).
"""
import argparse
import os

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=32_000_000)
    ap.add_argument("--epochs", type=int, default=60)
    ap.add_argument("--lr", type=float, default=4e-3)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--workers", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "data",
                                                  "warmstart_c5.npz"))
    a = ap.parse_args()
    from . import synth
    from .warmstart import train_warm_start
    grad = synth.config5_scheme()
    sig = synth.voxel_signals_parallel(grad, a.n, (15.0, 40.0), a.seed, workers=a.workers)
    net, losses = train_warm_start(grad, n_train=a.n, epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed,
                                   verbose=True, signals=sig)
    net.save(a.out)
    print(f"saved {a.out}: final BCE {losses[-1]:.5f}")


if __name__ == "__main__":
    main()
