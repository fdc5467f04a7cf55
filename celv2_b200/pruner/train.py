"""Trains the pruner and chooses its thresholds; writes weights.npz and report.json.

    python -m celv2_b200.pruner.train [--out DIR] [--clips 200] [--test-clips 20] [--steps N]

1. Seeded synthetic 1080p 10-bit clips of two kinds of content, seeds apart from the bench's:
   natural-like (the workload's sinusoid generator) and animation-like (flat colours, 1-px hard
   edges, piecewise motion up to +-24 or +-48 px: `synth.animation_clip`). `--clips` of 17 frames
   (one mini-GOP each) for training, a share `--anime-share` of them animation-like, qindex cycling
   through 100 / 130 / 160 / 190 within each kind (200 clips: about 1.6M inter superblock records);
   for choosing the thresholds 4 natural-like and 12 animation-like clips of `--val-frames` (33)
   frames (qindex cycling); held out,
   `--test-clips` natural-like and `--test-anime-clips` animation-like clips of 33 frames (two
   mini-GOPs), each evaluated at all four qindex values.
2. Labels: per superblock the options the exhaustive decision's chosen partition uses (references,
   intra, block levels, intra modes; data.labels). Masks of exactly those options lose nothing. A
   needed reference's, intra's or block level's weight grows with its regret: the cost increase
   when that option alone is pruned (one more decision of each group per option), relative to the
   frame's mean superblock cost.
   (`--weights`: thresholds for weights trained before; steps 1-3 are skipped.)
3. Adam on the weighted cross-entropy, with the library's own forward, backward, loss and Adam
   kernels.
4. Thresholds: on the validation clips, the fastest setting (device time of the clips through the
   engine) whose summed chosen-partition cost rises by at most `--val-margin` x `--max-loss`
   (0.7 %, headroom for the held-out clips) over the exhaustive search on each kind of content (the summed costs of flat content are small beside
   natural content's, so one sum over both would let the flat clips lose anything), by a
   coordinate search over the four thresholds; then the confidence band (the fallback to the full
   search) widened as far as the budget allows.
5. Report: per qindex on the held-out clips of each kind, the cost increase and speed-up of the
   network and of the used-option masks (the ceiling: perfect masks, no loss), on the natural-like
   clips also of rules without the network (keep the k nearest references, intra or not, every
   level or only the small ones), and the fallback rate.
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
# animation-like clips: seeds of their own (the generator differs, so equal seeds would not repeat
# content either, but separate ranges keep the kinds apart in the report)
ANIME_TRAIN_SEED0, ANIME_VAL_SEEDS, ANIME_TEST_SEED0 = 5001, list(range(6001, 6013)), 7001
SINUSOID, ANIME = "sinusoid", "animation"


def _clip(args):
    from .. import synth

    seed, frames, kind = args
    if kind == ANIME:  # half the clips at the 4K content's +-48 px motion, half at +-24
        clip = synth.animation_clip(1920, 1080, frames, seed, colours=(8, 24), motion=48.0 if seed % 2 else 24.0)
    else:
        clip = synth.hd_clip(seed, frames)
    return [f.hy for f in clip]


def clips_in_chunks(pool, seeds, frames, chunk):
    """Yields (seed, kind, 10-bit planes) of seeded 1080p clips, made `chunk` at a time in the pool;
    `seeds` holds (seed, kind) pairs."""
    for i in range(0, len(seeds), chunk):
        part = seeds[i:i + chunk]
        for (s, kind), c in zip(part, pool.map(_clip, [(s, frames, kind) for s, kind in part])):
            yield s, kind, c


def training_seeds(n: int, anime_share: float):
    """(seed, kind) of the n training clips: the animation-like ones spread evenly among them, the
    qindex of clip k being QS[k % 4] within its kind (data is collected in this order)."""
    na = int(round(n * anime_share))
    kinds = [ANIME if na and (k * na) // n != ((k + 1) * na) // n else SINUSOID for k in range(n)]
    out, counts = [], {SINUSOID: 0, ANIME: 0}
    for kind in kinds:
        seed0 = ANIME_TRAIN_SEED0 if kind == ANIME else TRAIN_SEED0
        out.append((seed0 + counts[kind], kind))
        counts[kind] += 1
    return out


def train_network(eng, pool, seeds, args, t0):
    """1-3: the records of the training clips and the network trained on them; returns (params,
    the samples, the loss curve, the positive share per output)."""
    import torch

    from .. import gop

    plan17 = gop.stream_plan(17)
    xs, ys, ws = [], [], []
    seen = {SINUSOID: 0, ANIME: 0}
    for k, (seed, kind, clip) in enumerate(clips_in_chunks(pool, seeds, 17, 2 * args.workers)):
        q = QS[seen[kind] % 4]
        seen[kind] += 1
        (x, y, w, _), _, _ = D.collect(eng, clip, q, plan17, regrets=True)
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
    ap.add_argument("--val-frames", type=int, default=33, help="frames per validation clip (33: two mini-GOPs)")
    ap.add_argument("--val-margin", type=float, default=0.7,
                    help="thresholds are chosen within this share of --max-loss on the validation clips")
    ap.add_argument("--anime-share", type=float, default=0.3, help="share of animation-like training clips")
    ap.add_argument("--test-anime-clips", type=int, default=8)
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
    plan33 = gop.stream_plan(33)

    seeds = training_seeds(args.clips, args.anime_share)
    if args.weights:
        prev = json.load(open(os.path.join(os.path.dirname(args.weights), "report.json")))
        params, X, losses, positives = np.load(args.weights)["params"], None, prev["loss_curve"], \
            np.array(prev["positive_share"])
    else:
        params, X, losses, positives = train_network(eng, pool, seeds, args, t0)
    samples = int(X.shape[0]) if X is not None else prev["samples"]
    del X

    # 4. thresholds on the validation clips (each at one qindex, four of each kind)
    val_seeds = [(s, SINUSOID) for s in VAL_SEEDS] + [(s, ANIME) for s in ANIME_VAL_SEEDS]
    plan_val = gop.stream_plan(args.val_frames)
    val = [(c, QS[i % 4], kind)
           for i, (_, kind, c) in enumerate(clips_in_chunks(pool, val_seeds, args.val_frames, args.workers))]

    def measure(clips_q, plan, setting, reps=1):
        """Cost increase, speed-up and kept work of a setting over (clip, qindex, ...) rows: `loss` is
        the largest of the kinds' summed cost increases (`loss_by_kind`), the speed-up the summed
        exhaustive time over the summed pruned time."""
        pruned_cost, full_cost = {}, {}
        ms = ms_full = 0.0
        kept_all = []
        for clip, q, full, t_full, kind in clips_q:
            V.upload(eng, clip)
            if setting[0] == "net":
                eng.set_pruner(params, *setting[1:])
                costs, t, kept = V.run(eng, plan, q, reps=reps)
                eng.set_pruner(None)
            elif setting[0] == "used":
                costs, t, kept = V.run(eng, plan, q, masks=lambda f, n, nsb, u=setting[1][id(clip), q]: u[f], reps=reps)
            else:
                costs, t, kept = V.run(eng, plan, q, masks=V.nearest(*setting[1:]), reps=reps)
            pruned_cost[kind] = pruned_cost.get(kind, 0.0) + sum(float(v.sum()) for v in costs.values())
            full_cost[kind] = full_cost.get(kind, 0.0) + sum(float(full[k].sum()) for k in costs)
            ms += t
            ms_full += t_full
            kept_all.append(V.kept_work(kept, plan))
        by_kind = {k: pruned_cost[k] / full_cost[k] - 1.0 for k in pruned_cost}
        out = {"loss": max(by_kind.values()), "loss_by_kind": by_kind, "speedup": ms_full / ms,
               "ms": ms / len(clips_q), "ms_full": ms_full / len(clips_q)}
        for key in kept_all[0]:
            out[key] = float(np.mean([k[key] for k in kept_all]))
        return out

    def baseline(clips_q, plan, reps=1):
        """(clip, qindex, exhaustive costs, exhaustive ms, kind) per (clip, qindex, kind), and the
        used-option words."""
        rows, used = [], {}
        for clip, q, kind in clips_q:
            (_, _, _, _), costs, words = D.collect(eng, clip, q, plan)
            V.upload(eng, clip)
            _, t, _ = V.run(eng, plan, q, reps=reps)
            rows.append((clip, q, costs, t, kind))
            used[id(clip), q] = words
        return rows, used

    val_rows, val_used = baseline(val, plan_val)
    # coordinate search from a middle setting: each threshold over its range in turn, keeping the
    # fastest setting within the budget (the least costly one while none is within it), two rounds
    ranges = [(0.05, 0.1, 0.2, 0.3, 0.5, 0.65, 0.8, 0.9, 0.95, 0.98), (0.02, 0.05, 0.1, 0.2, 0.3, 0.5, 0.7, 0.9, 0.95, 0.99),
              (0.02, 0.05, 0.1, 0.2, 0.35, 0.5, 0.7, 0.85), (0.02, 0.05, 0.1, 0.2, 0.3, 0.5, 0.7)]
    cur = [0.5, 0.5, 0.35, 0.3]
    sweep, seen = [], {}

    def score(th):
        key = tuple(th)
        if key not in seen:
            r = {"setting": ["net", *th, 0.0], **measure(val_rows, plan_val, ("net", *th, 0.0))}
            seen[key] = r
            sweep.append(r)
        return seen[key]

    budget = args.max_loss * args.val_margin  # headroom for the held-out clips

    def better(a, b):
        fa, fb = a["loss"] <= budget, b["loss"] <= budget
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
        r = {"setting": list(s), **measure(val_rows, plan_val, s)}
        sweep.append(r)
        if r["loss"] <= budget and r["speedup"] >= 0.97 * best["speedup"]:
            best = r
    chosen = dict(zip(THRESHOLDS, best["setting"][1:]))
    print("chosen", best, flush=True)

    # 5. the held-out clips of each kind at every qindex
    test_seeds = [(s, SINUSOID) for s in range(TEST_SEED0, TEST_SEED0 + args.test_clips)]
    anime_seeds = [(s, ANIME) for s in range(ANIME_TEST_SEED0, ANIME_TEST_SEED0 + args.test_anime_clips)]
    rules = [("nearest", k, intra, small) for k in (2, 3, 4) for intra in (True, False) for small in (False, True)]
    per_q = {SINUSOID: {q: {} for q in QS}, ANIME: {q: {} for q in QS}}
    net_setting = ("net",) + tuple(best["setting"][1:])
    for _, kind, clip in clips_in_chunks(pool, test_seeds + anime_seeds, 33, args.workers):
        for q in QS:
            rows, used = baseline([(clip, q, kind)], plan33, reps=2)
            settings = [("net", net_setting), ("used_options", ("used", used))]
            if kind == SINUSOID:
                settings += [("-".join(map(str, r)), r) for r in rules]
            for name, s in settings:
                per_q[kind][q].setdefault(name, []).append(measure(rows, plan33, s, reps=2))

    def mean_rows(rs):
        return {k: float(np.mean([r[k] for r in rs])) for k in rs[0] if k != "loss_by_kind"}

    test = {kind: {q: {name: mean_rows(rs) for name, rs in per_q[kind][q].items()} for q in QS} for kind in per_q}
    pool.close()
    os.makedirs(args.out, exist_ok=True)
    np.savez(os.path.join(args.out, "weights.npz"), params=params,
             **{k: np.float32(v) for k, v in chosen.items()})

    def span(ss, kind):
        ks = [s for s, k in ss if k == kind]
        return [ks[0], ks[-1]] if ks else []

    report = {"samples": samples, "clips": args.clips, "anime_share": args.anime_share, "steps": args.steps,
              "batch": args.batch, "loss_curve": losses, "positive_share": positives.tolist(),
              "max_loss": args.max_loss, "val_margin": args.val_margin, "chosen": best, "thresholds": chosen, "validation": sweep,
              "test_per_qindex": test[SINUSOID], "test_animation_per_qindex": test[ANIME],
              "seeds": {"train": span(seeds, SINUSOID), "train_animation": span(seeds, ANIME), "val": VAL_SEEDS,
                        "val_animation": ANIME_VAL_SEEDS, "test": span(test_seeds, SINUSOID),
                        "test_animation": span(anime_seeds, ANIME)},
              "seconds": time.time() - t0}
    with open(os.path.join(args.out, "report.json"), "w") as fh:
        json.dump(report, fh, indent=1)
    print(json.dumps({kind: {q: {k: {"loss": v["loss"], "speedup": v["speedup"]} for k, v in t.items()}
                             for q, t in test[kind].items()} for kind in test}, indent=1))
    eng.close()


if __name__ == "__main__":
    main()
