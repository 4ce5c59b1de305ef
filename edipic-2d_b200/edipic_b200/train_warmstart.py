"""Trains the learned warm start on the device and writes its parameters.

    python -m edipic_b200.train_warmstart --out edipic-2d_b200/weights/warmstart_cfg3.npz

Samples are the potential updates of plain runs (multigrid-preconditioned CG from the previous potential, 1e-10) on
512 x 512-cell walled domains with a 64 x 32-cell metal rectangle whose centre is jittered by +-64 cells around
(256, 128) and whose bias is uniform in [-200, 0] V, 100 electrons and 100 Ar+ per cell with the full collision set
(the learned-warm-start configuration, reduced in sample count: --decks x --steps samples instead of 50,000).
"""
import argparse
import json
import os
import sys
import tempfile
import time

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import numpy as np  # noqa: E402

from edipic_b200 import decks, warmstart  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--decks", type=int, default=12)
    ap.add_argument("--steps", type=int, default=32, help="samples per deck")
    ap.add_argument("--warmup", type=int, default=8)
    ap.add_argument("--cells", type=int, default=512)
    ap.add_argument("--ppc", type=int, default=100)
    ap.add_argument("--train-steps", type=int, default=1500)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    import torch
    torch.cuda.set_device(0)
    t0 = time.time()
    geo = warmstart.cfg3_geometries(args.decks, seed=args.seed, ncx=args.cells, ncy=args.cells)
    with tempfile.TemporaryDirectory() as tmp:
        dirs = [decks.write_deck(os.path.join(tmp, f"d{k}"), "cfg2", ncx=args.cells, ncy=args.cells, ppc=args.ppc,
                                 inner=g, seed=args.seed + k) for k, g in enumerate(geo)]
        dphi, unk = warmstart.generate_samples(dirs, args.steps, warmup=args.warmup)
    t1 = time.time()
    # how white the residuals are: relative residual after one Jacobi step u = r0 / 4 (0.25 for white noise, near 1
    # for fields smooth on the grid scale), on the first samples
    with torch.no_grad():
        x, rhat, t = warmstart.make_batch(dphi[:8], unk[:8])
        jac = warmstart.stencil(rhat / 4.0, unk[:8])
        jr = ((rhat - jac) ** 2).sum(dim=(1, 2)) / (rhat ** 2).sum(dim=(1, 2))
        print("jacobi residual ratio of the samples:", [round(float(v), 4) for v in jr], flush=True)
    K = warmstart.k_factor(args.cells, args.cells)
    net = warmstart.WarmStartNet(seed=args.seed)
    hist = warmstart.train(net, dphi, unk, K, steps=args.train_steps, batch=args.batch, lr=args.lr,
                           seed=args.seed, log=lambda m: print(m, flush=True))
    torch.cuda.synchronize()
    t2 = time.time()
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    warmstart.save_blob(args.out, net.blob())
    info = {"samples": int(dphi.shape[0]), "decks": args.decks, "cells": args.cells, "train_steps": args.train_steps,
            "batch": args.batch, "lr": args.lr, "sample_s": t1 - t0, "train_s": t2 - t1, "history": hist}
    with open(os.path.splitext(args.out)[0] + ".json", "w") as f:
        json.dump(info, f, indent=1)
    print(json.dumps({k: v for k, v in info.items() if k != "history"}))


if __name__ == "__main__":
    main()
