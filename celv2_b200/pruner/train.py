"""Trains the pruner and chooses its thresholds; writes weights.npz and a JSON report.

    python -m celv2_b200.pruner.train [--out DIR] [--steps N]

1. seeded synthetic 1080p clips (the workload's generator, other seeds): 24 for training, 2 for
   choosing the thresholds, 2 held out for the report; qindex 100 / 130 / 160 / 190 in training,
   130 for validation and test (the benchmark's);
2. for every inter frame, every superblock's chosen cost under every mask (data.mask_costs: a
   superblock's decision depends only on its own mask);
3. the targets: per superblock the mask minimising work + mu * cost increase (data.policy), mu set
   so that this exact policy loses `--target` (0.4 %) of the summed cost on the training clips
   (`--weighting regret`: each bit weighted by the regret of getting it wrong; on these clips it
   did not beat uniform weights);
4. Adam on the weighted cross-entropy of the mask bits, with the library's own kernels;
5. thresholds: on the validation clips, the fastest setting (device time of the mini-GOP through
   the engine) whose cost rises by at most `--max-loss` (1 %) over the exhaustive search;
6. the report: on the held-out clips, cost increase and speed-up of the network, of the exact
   policy it imitates, and of the heuristic without the network (keep the k nearest references).
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import WEIGHTS
from . import data as D
from . import evaluate as V
from . import net as N

TRAIN_SEEDS = list(range(101, 125))
VAL_SEEDS = [201, 202]
TEST_SEEDS = [301, 302]
QS = [100, 130, 160, 190]


def find_mu(tables, target):
    """The mu whose policy loses `target` of the summed cost over the clips (bisection in log mu)."""
    lo, hi = 1e-2, 1e7
    for _ in range(40):
        mid = float(np.sqrt(lo * hi))
        dj = sum(D.policy(c, n, mid)[2] * w for c, n, w in tables)
        if dj > target:
            lo = mid
        else:
            hi = mid
    return hi


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.dirname(WEIGHTS))
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=1024)
    ap.add_argument("--target", type=float, default=0.004)
    ap.add_argument("--max-loss", type=float, default=0.01)
    ap.add_argument("--workers", type=int, default=6)
    ap.add_argument("--weighting", choices=["uniform", "regret"], default="uniform",
                    help="per-output weights: 1, or the regret of a wrong bit (data.regret_targets)")
    args = ap.parse_args()
    t0 = time.time()
    clips = D.make_clips(TRAIN_SEEDS + VAL_SEEDS + TEST_SEEDS, workers=args.workers)  # before any CUDA use
    print(f"clips {time.time() - t0:.1f}s", flush=True)

    import torch

    from .. import engine as E

    eng = E.CudaEngine(1920, 1080)
    eng.reserve_group(10)
    eng.set_config(E.CFG_GRAPHS, 1)
    plan = V.default_plan()
    nt = len(TRAIN_SEEDS)
    qs = [QS[i % 4] for i in range(nt)] + [130] * 4
    tables = [D.mask_costs(eng, c, q, plan) for c, q in zip(clips, qs)]
    print(f"mask costs {time.time() - t0:.1f}s", flush=True)
    train_t = tables[:nt]
    # mu on the training clips: each clip's loss weighs by its share of the summed cost
    tot = [sum(float(c[:, -1].sum()) for c in t[1].values()) for t in train_t]
    mu = find_mu([(t[1], t[2], tc / sum(tot)) for t, tc in zip(train_t, tot)], args.target)
    xs, ys, ws, oracle_work = [], [], [], []
    for feats, costs, nrefs in train_t:
        keeps, work, _ = D.policy(costs, nrefs, mu)
        y, w = D.regret_targets(costs, nrefs, mu) if args.weighting == "regret" else D.policy_labels(keeps, nrefs)
        xs.append(np.concatenate([feats[s] for s in keeps])), ys.append(y), ws.append(w)
        oracle_work.append(work)
    X, Y, Wt = np.concatenate(xs), np.concatenate(ys), np.concatenate(ws)
    print(f"mu {mu:.4g}: exact policy keeps {np.mean(oracle_work):.3f} of the prunable work; samples {X.shape[0]}, "
          f"targets {Y.sum(0) / np.maximum(Wt.astype(bool).sum(0), 1)}", flush=True)
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
        if (step + 1) % 250 == 0:
            losses.append(tr.take_loss() / 250)
            print(f"step {step + 1} loss {losses[-1]:.4f}", flush=True)
    params = tr.params()

    def sweep(idx, settings):
        rows = []
        for i in idx:
            V.upload(eng, clips[i])
            eng.set_pruner(None)
            full, ms_full, _ = V.run(eng, plan, 130, reps=3)
            for s in settings:
                if s[0] == "net":
                    eng.set_pruner(params, s[1], s[2], s[3])
                    costs, ms, kept = V.run(eng, plan, 130, reps=3)
                    eng.set_pruner(None)
                elif s[0] == "exact":
                    keeps, _, predicted = D.policy(tables[i][1], tables[i][2], mu)
                    costs, ms, kept = V.run(eng, plan, 130, masks=lambda f, n, nsb, k=keeps: k[f], reps=3)
                    rows.append({"setting": ["exact-predicted"], "loss": predicted, "speedup": 0.0, "ms": 0.0,
                                 "ms_full": ms_full, "refs_kept": 0.0, "intra_kept": 0.0})
                else:
                    costs, ms, kept = V.run(eng, plan, 130, masks=V.nearest(s[1], s[2]), reps=3)
                rows.append({"setting": list(s), "loss": V.cost_increase(costs, full), "speedup": ms_full / ms,
                             "ms": ms, "ms_full": ms_full, **V.kept_work(kept, plan)})
        agg = {}
        for r in rows:
            agg.setdefault(tuple(r["setting"]), []).append(r)
        return [{"setting": list(k), "loss": float(np.mean([r["loss"] for r in v])),
                 "speedup": float(np.mean([r["speedup"] for r in v])),
                 "ms": float(np.mean([r["ms"] for r in v])), "ms_full": float(np.mean([r["ms_full"] for r in v])),
                 "refs_kept": float(np.mean([r["refs_kept"] for r in v])),
                 "intra_kept": float(np.mean([r["intra_kept"] for r in v]))} for k, v in agg.items()]

    net_settings = [("net", a, b, 0.0) for a in (0.3, 0.5, 0.6, 0.7, 0.8, 0.85, 0.9, 0.95)
                    for b in (0.3, 0.5, 0.7, 0.8, 0.9)]
    val = sweep([nt, nt + 1], net_settings + [("exact",)])
    ok = [r for r in val if r["setting"][0] == "net" and r["loss"] <= args.max_loss]
    best = max(ok, key=lambda r: r["speedup"]) if ok else min((r for r in val if r["setting"][0] == "net"),
                                                              key=lambda r: r["loss"])
    _, tr_, ti, band = best["setting"]
    print("chosen", best, flush=True)
    heur = [("nearest", k, intra) for k in (1, 2, 3, 4) for intra in (True, False)]
    test = sweep([nt + 2, nt + 3], [("net", tr_, ti, band), ("exact",)] + heur)
    # the exact policy's trade-off on the held-out clips (no network: what perfect masks would give)
    curve = []
    for f in (0.25, 0.5, 1.0, 2.0, 4.0, 8.0):
        pts = [D.policy(tables[i][1], tables[i][2], mu * f) for i in (nt + 2, nt + 3)]
        curve.append({"mu": mu * f, "loss": float(np.mean([p[2] for p in pts])),
                      "work_kept": float(np.mean([p[1] for p in pts]))})
    os.makedirs(args.out, exist_ok=True)
    np.savez(os.path.join(args.out, "weights.npz"), params=params, ref_threshold=np.float32(tr_),
             intra_threshold=np.float32(ti), band=np.float32(band))
    report = {"samples": int(X.shape[0]), "steps": args.steps, "weighting": args.weighting, "batch": args.batch, "loss_curve": losses,
              "mu": mu, "target": args.target, "exact_policy_work": float(np.mean(oracle_work)),
              "targets_positive": (Y.sum(0) / np.maximum(Wt.astype(bool).sum(0), 1)).tolist(),
              "validation": val, "chosen": best, "test": test, "exact_policy_curve": curve,
              "seeds": {"train": TRAIN_SEEDS, "val": VAL_SEEDS, "test": TEST_SEEDS}, "seconds": time.time() - t0}
    with open(os.path.join(args.out, "report.json"), "w") as fh:
        json.dump(report, fh, indent=1)
    print(json.dumps(test, indent=1))
    eng.close()


if __name__ == "__main__":
    main()
