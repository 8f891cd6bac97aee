"""Trains the learned preconditioner on the GPU and writes its weights.

    python npb-gpu_b200/npbcg/train_lp.py [--small] [--out PATH]

Training data (the generator's matrices at seeds the NPB classes never
use): 128 matrices at n=14000, nonzer=11, shift=20 and 128 at n=75000,
nonzer=13, shift=60, each seen once, 16 Adam steps per matrix on 32 probe
vectors: residual histories (the residuals after 0, 2, 4 or 8 batched CG
steps on the scaled matrix, one of the starting vectors all ones like the
benchmark's first x) and plain normal vectors.  Forward, backward and the
optimiser run in libcgb's CUDA kernels (cgb_gnn_train_step).  --small trains
on 16 + 4 matrices for a quick check.  Prints one JSON line per matrix
block and a final summary; writes float32 weights (little endian).
"""
import argparse
import json
import os
import sys
import time

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import npbcg  # noqa: E402

SETS = [dict(n=14000, nonzer=11, shift=20.0), dict(n=75000, nonzer=13, shift=60.0)]


def train_seeds(count, base):
    """Odd LCG seeds in (1, 2^46), distinct from the NPB seed 314159265."""
    return [float(base + 2 * 7919 * k) for k in range(count)]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--small", action="store_true")
    ap.add_argument("--out", default=npbcg.WEIGHTS_PATH)
    ap.add_argument("--steps-per-matrix", type=int, default=16)
    ap.add_argument("--lr", type=float, default=2e-3)
    a = ap.parse_args()
    counts = (16, 4) if a.small else (128, 128)
    model = npbcg.Gnn(seed=20241203)
    plan = []
    for cfg, cnt, base in zip(SETS, counts, (1000003, 3000017)):
        plan += [(cfg, s) for s in train_seeds(cnt, base)]
    # interleave the two sizes
    small = [p for p in plan if p[0]["n"] == 14000]
    large = [p for p in plan if p[0]["n"] == 75000]
    order = []
    for i in range(max(len(small), len(large))):
        if i < len(small):
            order.append(small[i])
        if i < len(large):
            order.append(large[i])
    t0 = time.time()
    total_steps = len(order) * a.steps_per_matrix
    step = 0
    history = []
    for mi, (cfg, seed) in enumerate(order):
        rs, ci, av = npbcg.makea(cfg["n"], cfg["nonzer"], npbcg.RCOND, cfg["shift"], seed)
        with model.graph(rs, ci, av) as g:
            for k in range(a.steps_per_matrix):
                # cosine decay of the step size over the run
                import math
                lr = a.lr * 0.5 * (1.0 + math.cos(math.pi * step / total_steps))
                cg_steps = (0, 2, 4, 8)[k % 4]
                loss = model.train_step(g, seed=int(seed) % 1000003 * 31 + k, cg_steps=cg_steps, lr=lr)
                history.append(loss)
                step += 1
        if mi % 16 == 15 or mi == len(order) - 1:
            recent = history[-16 * a.steps_per_matrix:]
            print(json.dumps({"matrices": mi + 1, "steps": step, "loss_mean_recent": sum(recent) / len(recent),
                              "seconds": round(time.time() - t0, 1)}), flush=True)
    model.save(a.out)
    first = history[: 4 * a.steps_per_matrix]
    last = history[-4 * a.steps_per_matrix:]
    print(json.dumps({"done": True, "matrices": len(order), "steps": step,
                      "loss_first": sum(first) / len(first), "loss_last": sum(last) / len(last),
                      "seconds": round(time.time() - t0, 1), "weights": a.out}), flush=True)


if __name__ == "__main__":
    main()
