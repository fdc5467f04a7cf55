"""Trains the pruner and chooses its thresholds; writes weights.npz and report.json.

    python -m celv2_b200.pruner.train [--out DIR] [--clips 200] [--test-clips 20] [--steps N]

1. Seeded synthetic 1080p 10-bit clips (the workload's generator, seeds apart from the bench's):
   `--clips` of 17 frames (one mini-GOP each) for training, qindex cycling through 100 / 130 / 160 /
   190 (200 clips: about 1.6M inter superblock records); 4 of 17 frames for choosing the thresholds
   (one per qindex); `--test-clips` held-out clips of 33 frames (two mini-GOPs), each evaluated at
   all four qindex values.
2. Labels: per superblock the options the exhaustive decision's chosen partition uses (references,
   intra, block levels, intra modes; data.labels). Masks of exactly those options lose nothing.
   (`--weights`: thresholds for weights trained before; steps 1-3 are skipped.)
3. Adam on the weighted cross-entropy, with the library's own forward, backward, loss and Adam
   kernels.
4. Thresholds: on the validation clips, the fastest setting (device time of the clips through the
   engine) whose summed chosen-partition cost rises by at most `--max-loss` (1 %) over the
   exhaustive search, by a coordinate search over the four thresholds; then the confidence band
   (the fallback to the full search) widened as far as the budget allows.
5. Report: per qindex on the held-out clips, the cost increase and speed-up of the network, of the
   used-option masks (the ceiling: perfect masks, no loss) and of rules without the network (keep
   the k nearest references, intra or not, every level or only the small ones), and the fallback
   rate.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import time

import numpy as np

from . import THRESHOLDS, WEIGHTS
from . import data as D
from . import evaluate as V
from . import net as N

QS = [100, 130, 160, 190]
TRAIN_SEED0, VAL_SEEDS, TEST_SEED0 = 1001, [2001, 2002, 2003, 2004], 3001


def _clip(args):
    from .. import synth

    seed, frames = args
    return [f.hy for f in synth.hd_clip(seed, frames)]


def clips_in_chunks(pool, seeds, frames, chunk):
    """Yields (seed, 10-bit planes) of seeded 1080p clips, made `chunk` at a time in the pool."""
    for i in range(0, len(seeds), chunk):
        part = seeds[i:i + chunk]
        for s, c in zip(part, pool.map(_clip, [(s, frames) for s in part])):
            yield s, c


def train_network(eng, pool, seeds, args, t0):
    """1-3: the records of the training clips and the network trained on them; returns (params,
    the samples, the loss curve, the positive share per output)."""
    import torch

    from .. import gop

    plan17 = gop.stream_plan(17)
    xs, ys, ws = [], [], []
    for k, (seed, clip) in enumerate(clips_in_chunks(pool, seeds, 17, 2 * args.workers)):
        (x, y, w, _), _, _ = D.collect(eng, clip, QS[k % 4], plan17)
        xs.append(x), ys.append(y), ws.append(w)
        if (k + 1) % 20 == 0:
            print(f"records: {k + 1} clips, {time.time() - t0:.0f}s", flush=True)
    X, Y, Wt = np.concatenate(xs), np.concatenate(ys), np.concatenate(ws)
    del xs, ys, ws
    positives = (Y * (Wt > 0)).sum(0) / np.maximum((Wt > 0).sum(0), 1)
    print(f"samples {X.shape[0]}, positive share per output {np.round(positives, 3).tolist()}", flush=True)

    # 3. training
    dev = torch.device("cuda:0")
    x, y, w = (torch.from_numpy(a).to(dev) for a in (X, Y, Wt))
    tr = N.Trainer(args.batch, lr=2e-3)
    g = torch.Generator(device=dev)
    g.manual_seed(0)
    losses = []
    for step in range(args.steps):
        if step == int(args.steps * 0.75):
            tr.lr *= 0.1
        idx = torch.randint(0, x.shape[0], (args.batch,), device=dev, generator=g)
        tr.step(x[idx].contiguous(), y[idx].contiguous(), w[idx].contiguous())
        if (step + 1) % 500 == 0:
            losses.append(tr.take_loss() / 500)
            print(f"step {step + 1} loss {losses[-1]:.4f}", flush=True)
    params = tr.params()
    del x, y, w
    torch.cuda.empty_cache()
    return params, X, losses, positives


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.dirname(WEIGHTS))
    ap.add_argument("--clips", type=int, default=200)
    ap.add_argument("--test-clips", type=int, default=20)
    ap.add_argument("--steps", type=int, default=8000)
    ap.add_argument("--batch", type=int, default=2048)
    ap.add_argument("--max-loss", type=float, default=0.01)
    ap.add_argument("--workers", type=int, default=max(1, min(16, (os.cpu_count() or 2) // 2)))
    ap.add_argument("--weights", default=None,
                    help="trained weights to choose thresholds for (skips the records and the training)")
    args = ap.parse_args()
    t0 = time.time()
    pool = mp.get_context("spawn").Pool(args.workers)  # spawned workers: no CUDA state inherited

    from .. import engine as E
    from .. import gop

    eng = E.CudaEngine(1920, 1080)
    eng.reserve_group(10)
    eng.set_config(E.CFG_GRAPHS, 1)
    plan17, plan33 = gop.stream_plan(17), gop.stream_plan(33)

    seeds = list(range(TRAIN_SEED0, TRAIN_SEED0 + args.clips))
    if args.weights:
        prev = json.load(open(os.path.join(os.path.dirname(args.weights), "report.json")))
        params, X, losses, positives = np.load(args.weights)["params"], None, prev["loss_curve"], \
            np.array(prev["positive_share"])
    else:
        params, X, losses, positives = train_network(eng, pool, seeds, args, t0)
    samples = int(X.shape[0]) if X is not None else prev["samples"]
    del X

    # 4. thresholds on the validation clips (each at one qindex)
    val = [(c, QS[i]) for i, (_, c) in enumerate(clips_in_chunks(pool, VAL_SEEDS, 17, len(VAL_SEEDS)))]

    def measure(clips_q, plan, setting, reps=1):
        """Summed cost increase, speed-up and kept work of a setting over (clip, qindex) pairs."""
        pruned_cost = full_cost = ms = ms_full = 0.0
        kept_all = []
        for clip, q, full, t_full in clips_q:
            V.upload(eng, clip)
            if setting[0] == "net":
                eng.set_pruner(params, *setting[1:])
                costs, t, kept = V.run(eng, plan, q, reps=reps)
                eng.set_pruner(None)
            elif setting[0] == "used":
                costs, t, kept = V.run(eng, plan, q, masks=lambda f, n, nsb, u=setting[1][id(clip), q]: u[f], reps=reps)
            else:
                costs, t, kept = V.run(eng, plan, q, masks=V.nearest(*setting[1:]), reps=reps)
            pruned_cost += sum(float(v.sum()) for v in costs.values())
            full_cost += sum(float(full[k].sum()) for k in costs)
            ms += t
            ms_full += t_full
            kept_all.append(V.kept_work(kept, plan))
        out = {"loss": pruned_cost / full_cost - 1.0, "speedup": ms_full / ms, "ms": ms / len(clips_q),
               "ms_full": ms_full / len(clips_q)}
        for key in kept_all[0]:
            out[key] = float(np.mean([k[key] for k in kept_all]))
        return out

    def baseline(clips_q, plan, reps=1):
        """(clip, qindex, exhaustive costs, exhaustive ms) per pair, and the used-option words."""
        rows, used = [], {}
        for clip, q in clips_q:
            (_, _, _, _), costs, words = D.collect(eng, clip, q, plan)
            V.upload(eng, clip)
            _, t, _ = V.run(eng, plan, q, reps=reps)
            rows.append((clip, q, costs, t))
            used[id(clip), q] = words
        return rows, used

    val_rows, val_used = baseline(val, plan17)
    # coordinate search from a middle setting: each threshold over its range in turn, keeping the
    # fastest setting within the budget (the least costly one while none is within it), two rounds
    ranges = [(0.3, 0.5, 0.65, 0.8, 0.9, 0.95, 0.98), (0.3, 0.5, 0.7, 0.9, 0.95, 0.99),
              (0.1, 0.2, 0.35, 0.5, 0.7, 0.85), (0.1, 0.2, 0.3, 0.5, 0.7)]
    cur = [0.5, 0.5, 0.35, 0.3]
    sweep, seen = [], {}

    def score(th):
        key = tuple(th)
        if key not in seen:
            r = {"setting": ["net", *th, 0.0], **measure(val_rows, plan17, ("net", *th, 0.0))}
            seen[key] = r
            sweep.append(r)
        return seen[key]

    def better(a, b):
        fa, fb = a["loss"] <= args.max_loss, b["loss"] <= args.max_loss
        if fa != fb:
            return fa
        return a["speedup"] > b["speedup"] if fa else a["loss"] < b["loss"]

    best = score(cur)
    for _ in range(2):
        for i, rng in enumerate(ranges):
            for v in rng:
                th = list(cur)
                th[i] = v
                r = score(th)
                if better(r, best):
                    best, cur = r, th
    for band in (0.01, 0.02, 0.05):  # the fallback band: widest that keeps the budget and some speed
        s = tuple(best["setting"][:5]) + (band,)
        r = {"setting": list(s), **measure(val_rows, plan17, s)}
        sweep.append(r)
        if r["loss"] <= args.max_loss and r["speedup"] >= 0.97 * best["speedup"]:
            best = r
    chosen = dict(zip(THRESHOLDS, best["setting"][1:]))
    print("chosen", best, flush=True)

    # 5. the held-out clips at every qindex
    test_seeds = list(range(TEST_SEED0, TEST_SEED0 + args.test_clips))
    rules = [("nearest", k, intra, small) for k in (2, 3, 4) for intra in (True, False) for small in (False, True)]
    per_q = {q: {} for q in QS}
    net_setting = ("net",) + tuple(best["setting"][1:])
    for _, clip in clips_in_chunks(pool, test_seeds, 33, args.workers):
        for q in QS:
            rows, used = baseline([(clip, q)], plan33, reps=2)
            for name, s in [("net", net_setting), ("used_options", ("used", used))] + [("-".join(map(str, r)), r)
                                                                                   for r in rules]:
                per_q[q].setdefault(name, []).append(measure(rows, plan33, s, reps=2))
    test = {}
    for q in QS:
        test[q] = {name: {k: float(np.mean([r[k] for r in rs])) for k in rs[0]} for name, rs in per_q[q].items()}
    pool.close()
    os.makedirs(args.out, exist_ok=True)
    np.savez(os.path.join(args.out, "weights.npz"), params=params,
             **{k: np.float32(v) for k, v in chosen.items()})
    report = {"samples": samples, "clips": args.clips, "steps": args.steps, "batch": args.batch,
              "loss_curve": losses, "positive_share": positives.tolist(), "max_loss": args.max_loss,
              "chosen": best, "thresholds": chosen, "validation": sweep, "test_per_qindex": test,
              "seeds": {"train": [seeds[0], seeds[-1]], "val": VAL_SEEDS, "test": [test_seeds[0], test_seeds[-1]]},
              "seconds": time.time() - t0}
    with open(os.path.join(args.out, "report.json"), "w") as fh:
        json.dump(report, fh, indent=1)
    print(json.dumps({q: {k: {"loss": v["loss"], "speedup": v["speedup"]} for k, v in t.items()}
                      for q, t in test.items()}, indent=1))
    eng.close()


if __name__ == "__main__":
    main()
