"""Training and use of the learned error-bound proposer (2D).

Training data: seeded 2048 x 2048 fields of the cfg0 generator (Gaussian-
windowed linear flows, sigma 40); per field a sample of vertices with
 * features: the vertex's 7 x 7 (u, v) neighbourhood normalised by its largest
   |value|, plus log2 of the analytic bound / 32 (99 values, BF16);
 * label: the largest log2 multiplier of the analytic bound (16-step bisection
   over [0, 16]) under which moving the vertex alone to any corner of its bound
   box keeps the exact CP codes of its incident triangles.
The MLP (99 -> 128 -> 128 -> 1, ReLU) trains with Adam on mean squared error,
forward / backward on the tensor cores.  The saved parameters are flat float32
(``models/eb_mlp_2d.f32``); ``margin`` is subtracted from the output bias so the
proposals err on the safe side (the fallback loop repairs the rest).

    python -m cpsz_b200.learned train [--fields 64] [--side 2048] [--out PATH]
"""
from __future__ import annotations

import argparse
import os
import time

import numpy as np

from . import Context, Mlp, compress_2d_learned, debug_eb2d, learned_labels_2d, mlp_features_2d
from . import workloads as W

DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "models", "eb_mlp_2d.f32")


def training_set(ctx, n_fields=64, side=2048, samples=16384, eb=0.1, seed=0):
    rng = np.random.default_rng(seed)
    Xs, ts = [], []
    for k in range(n_fields):
        U, V = W.cfg0_like(1000 + seed + k, side, side)
        eb_a, _ = debug_eb2d(U, V, eb, ctx=ctx)
        idx = rng.integers(0, side * side, samples).astype(np.int32)
        Xs.append(mlp_features_2d(U, V, eb_a.ravel(), idx, ctx=ctx))
        ts.append(learned_labels_2d(U, V, eb_a.ravel(), idx, ctx=ctx))
    return np.concatenate(Xs), np.concatenate(ts)


def train(ctx, X, t, epochs=100, batch=65536, lr=2e-3, seed=0, margin=1.0, log=print):
    mlp = Mlp(ctx, seed=seed)
    rng = np.random.default_rng(seed)
    n = X.shape[0]
    for ep in range(epochs):
        order = rng.permutation(n)
        losses = []
        # cosine decay of the learning rate over the epochs
        lr_ep = lr * 0.5 * (1 + np.cos(np.pi * ep / epochs))
        for s in range(0, n, batch):
            sel = order[s:s + batch]
            loss, _ = mlp.train_step(X[sel], t[sel], lr=lr_ep)
            losses.append(loss)
        log(f"epoch {ep}: mse {np.mean(losses):.4f}")
    p = mlp.params()
    p[-1] -= margin
    mlp.set_params(p)
    return mlp


def load(ctx, path: str = DEFAULT_WEIGHTS) -> Mlp:
    p = np.fromfile(path, np.float32)
    return Mlp(ctx, params=p)


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    tr = sub.add_parser("train")
    tr.add_argument("--fields", type=int, default=64)
    tr.add_argument("--side", type=int, default=2048)
    tr.add_argument("--samples", type=int, default=16384)
    tr.add_argument("--epochs", type=int, default=100)
    tr.add_argument("--margin", type=float, default=1.0)
    tr.add_argument("--out", default=DEFAULT_WEIGHTS)
    tr.add_argument("--eval-side", type=int, default=2048)
    args = ap.parse_args()
    ctx = Context(0)
    t0 = time.time()
    X, t = training_set(ctx, args.fields, args.side, args.samples)
    print(f"training set: {X.shape[0]} samples in {time.time() - t0:.1f} s; label mean {t.mean():.3f} "
          f"quantiles {np.quantile(t, [0.1, 0.5, 0.9]).round(3).tolist()}")
    t0 = time.time()
    mlp = train(ctx, X, t, epochs=args.epochs, margin=args.margin)
    print(f"trained in {time.time() - t0:.1f} s")
    # held-out check: a fresh field at the evaluation size, a few output margins;
    # the margin with the smallest blob is saved
    U, V = W.cfg0_like(99991, args.eval_side, args.eval_side)
    from . import sz_compress_cp_preserve_2d_offline as plain
    base = len(plain(U, V, max_pwr_eb=0.1, ctx=ctx))
    p = mlp.params()
    best = None
    for extra in (-1.0, -0.5, 0.0, 0.5, 1.0, 1.5):
        q = p.copy()
        q[-1] -= extra
        probe = Mlp(ctx, params=q)
        t0 = time.time()
        blob, st = compress_2d_learned(U, V, 0.1, mlp=probe, ctx=ctx)
        dt = time.time() - t0
        print(f"held-out {args.eval_side}^2, margin {args.margin + extra}: plain {base} B, learned {len(blob)} B "
              f"({base / len(blob):.3f}x) in {dt * 1e3:.0f} ms, {st}")
        probe.close()
        if best is None or len(blob) < best[0]:
            best = (len(blob), q, args.margin + extra)
    os.makedirs(os.path.dirname(args.out), exist_ok=True)
    best[1].tofile(args.out)
    print(f"saved margin {best[2]} to {args.out}")


if __name__ == "__main__":
    main()
