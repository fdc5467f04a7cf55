"""Training records for the pruner: the exhaustive CUDA engine's decisions on seeded synthetic
clips, with the features the engine computes for every inter frame (CELV2_CFG_FEATURES).

Labels per superblock: reference r is needed where a leaf of the chosen partition predicts from it
(its reference or its compound's second); the intra modes are needed where a leaf is intra.
"""
from __future__ import annotations

import multiprocessing as mp

import numpy as np

from .. import engine as E
from .. import gop, synth

INTER = 13  # the record's mode of an inter leaf


def labels(records: np.ndarray, nrefs: int, pos_weight: float = 2.0):
    """(labels, weights), each nsb x 8, from one frame's records: outputs 0..6 the references, 7
    intra; absent references weigh 0, needed ones `pos_weight` (missing a needed option costs more
    than keeping an unneeded one)."""
    nsb = records.size
    mode = records["mode"].astype(np.int64)
    ref = records["ref"].astype(np.int64)
    ref2 = records["ref2"].astype(np.int64)
    leaf = np.arange(mode.shape[1])[None, :] < records["nblocks"].astype(np.int64)[:, None]
    y = np.zeros((nsb, 8), np.float32)
    inter = leaf & (mode == INTER)
    for r in range(nrefs):
        y[:, r] = (inter & ((ref == r) | (ref2 == r))).any(axis=1)
    y[:, 7] = (leaf & (mode != INTER)).any(axis=1)
    w = np.zeros((nsb, 8), np.float32)
    w[:, :nrefs] = 1.0
    w[:, 7] = 1.0
    w = np.where(y > 0, w * pos_weight, w)
    return y, w


def _clip(args):
    seed, frames = args
    return [f.hy for f in synth.hd_clip(seed, frames)]


def make_clips(seeds, frames: int = 17, workers: int = 4):
    """10-bit luma planes of seeded 1080p clips, made in worker processes (spawned: no CUDA state
    is inherited)."""
    with mp.get_context("spawn").Pool(workers) as pool:
        return pool.map(_clip, [(s, frames) for s in seeds])


def collect(eng: E.CudaEngine, clip, qindex: int, plan=None):
    """Features, labels, weights and (frame, nrefs) of every inter superblock of one mini-GOP of
    `clip` (10-bit planes) decided exhaustively, plus each inter frame's exhaustive costs."""
    plan = plan or gop.mini_gop_plan(len(clip))
    eng.clear_store()
    eng.set_config(E.CFG_FEATURES, 1)
    for i, f in enumerate(clip):
        eng.upload(f, i)
    xs, ys, ws, meta, costs = [], [], [], [], {}
    for group in plan:
        eng.launch_group([s for s, _ in group], [r for _, r in group], qindex, to_host=True)
        for j, (s, refs) in enumerate(group):
            if not refs:
                continue
            x = eng.features(j)
            y, w = labels(eng.group_records(j), len(refs))
            xs.append(x), ys.append(y), ws.append(w)
            meta.append(np.tile([s, len(refs), qindex], (x.shape[0], 1)))
            costs[s] = eng.sb_costs(j)
    eng.set_config(E.CFG_FEATURES, 0)
    return (np.concatenate(xs), np.concatenate(ys), np.concatenate(ws), np.concatenate(meta)), costs


def mask_costs(eng: E.CudaEngine, clip, qindex: int, plan=None):
    """Every superblock's chosen cost under every mask, for every inter frame of one mini-GOP.

    A superblock's decision depends only on its own mask (the level-0 cells a kept reference reads
    are searched exactly as without pruning), so deciding each frame once per mask -- the same mask
    for all its superblocks -- gives every superblock's cost for every mask. Returns
    (features {frame: nsb x FEATURES}, costs {frame: nsb x 2^(nrefs + 1) int64}, nrefs {frame}); mask
    index m keeps the references of its low nrefs bits (none named: all of them, as celv2_set_keep
    reads it) and intra if bit nrefs is set."""
    plan = plan or gop.mini_gop_plan(len(clip))
    eng.clear_store()
    for i, f in enumerate(clip):
        eng.upload(f, i)
    nsb = eng.sb_cols * eng.sb_rows
    feats, costs, nrefs = {}, {}, {}
    for group in plan:
        jobs = [(s, refs) for s, refs in group if refs]
        if not jobs:
            continue
        eng.set_config(E.CFG_FEATURES, 1)
        eng.launch_group([s for s, _ in jobs], [r for _, r in jobs], qindex)
        for j, (s, refs) in enumerate(jobs):
            feats[s] = eng.features(j)
            nrefs[s] = len(refs)
            costs[s] = np.zeros((nsb, 2 ** (len(refs) + 1)), np.int64)
            costs[s][:, -1] = eng.sb_costs(j)  # all references and intra
        eng.set_config(E.CFG_FEATURES, 0)
        top = max(2 ** (len(r) + 1) for _, r in jobs)
        for m in range(top - 1):
            # m == 2^n names no reference and keeps intra: the full search, measured above
            live = [(j, s, refs) for j, (s, refs) in enumerate(jobs)
                    if m < 2 ** (len(refs) + 1) - 1 and m != 2 ** len(refs)]
            if not live:
                continue
            for k, (_, s, refs) in enumerate(live):
                n = len(refs)
                eng.set_keep(k, np.full(nsb, (m & ((1 << n) - 1)) | (0x80 if m >> n & 1 else 0), np.uint8))
            eng.launch_group([s for _, s, _ in live], [refs for _, _, refs in live], qindex)
            for k, (_, s, _) in enumerate(live):
                costs[s][:, m] = eng.sb_costs(k)
        for s, refs in jobs:
            costs[s][:, 2 ** len(refs)] = costs[s][:, -1]
    return feats, costs, nrefs


def policy(costs: dict, nrefs: dict, mu: float, c_ref: float = 1.0, c_intra: float = 1.48):
    """The per-superblock masks minimising work + mu * (cost increase / total exhaustive cost), as
    keep bytes {frame: nsb}, with their work share and cost increase. Work: c_ref per kept reference,
    c_intra for intra (the measured per-superblock times of a reference's motion search and inter
    scoring, and of the intra scoring)."""
    total = sum(float(c[:, -1].sum()) for c in costs.values())
    keeps, work, full_work, dj = {}, 0.0, 0.0, 0.0
    for s, c in costs.items():
        n = nrefs[s]
        ms = np.arange(c.shape[1])
        refbits = ms & ((1 << n) - 1)
        cnt = np.array([bin(int(r)).count("1") if r else n for r in refbits], np.float64)
        w = c_ref * cnt + c_intra * ((ms >> n) & 1)
        delta = (c - c[:, -1:]).astype(np.float64) / total
        best = np.argmin(w[None, :] + mu * delta, axis=1)
        keeps[s] = (refbits[best] | np.where((best >> n) & 1, 0x80, 0)).astype(np.uint8)
        work += float(w[best].sum())
        full_work += float(w[-1]) * c.shape[0]
        dj += float(delta[np.arange(c.shape[0]), best].sum())
    return keeps, work / full_work, dj


def policy_labels(keeps: dict, nrefs: dict):
    """BCE targets from policy masks: bit r of the mask for reference r, bit 7 for intra; absent
    references weigh 0."""
    ys, ws = [], []
    for s, k in keeps.items():
        n = nrefs[s]
        bits = np.unpackbits(k[:, None], axis=1, bitorder="little").astype(np.float32)
        bits[bits[:, :n].sum(1) == 0, :n] = 1.0  # no reference named: all of them
        y = np.zeros((k.size, 8), np.float32)
        y[:, :n] = bits[:, :n]
        y[:, 7] = bits[:, 7]
        w = np.zeros((k.size, 8), np.float32)
        w[:, :n] = 1.0
        w[:, 7] = 1.0
        ys.append(y), ws.append(w)
    return np.concatenate(ys), np.concatenate(ws)


def regret_targets(costs: dict, nrefs: dict, mu: float, c_ref: float = 1.0, c_intra: float = 1.48,
                   floor: float = 0.05):
    """Cost-sensitive targets: the policy's mask bits, each weighted by the regret of flipping it --
    how much work + mu * cost increase the superblock loses if that one bit of its optimal mask is
    wrong -- so the network learns hardest where a mistake is expensive. Weights are scaled to mean
    1 over the present outputs, plus `floor`; absent references weigh 0."""
    total = sum(float(c[:, -1].sum()) for c in costs.values())
    ys, ws = [], []
    for s, c in costs.items():
        n = nrefs[s]
        ms = np.arange(c.shape[1])
        refbits = ms & ((1 << n) - 1)
        cnt = np.array([bin(int(r)).count("1") if r else n for r in refbits], np.float64)
        w = c_ref * cnt + c_intra * ((ms >> n) & 1)
        obj = w[None, :] + mu * (c - c[:, -1:]).astype(np.float64) / total
        best = np.argmin(obj, axis=1)
        rows = np.arange(c.shape[0])
        y = np.zeros((c.shape[0], 8), np.float32)
        wt = np.zeros((c.shape[0], 8), np.float32)
        rb = refbits[best]
        all_refs = rb == 0  # no reference named: all of them
        for r in range(n):
            y[:, r] = np.where(all_refs, 1.0, (rb >> r) & 1)
            flip = best ^ (1 << r)
            flip = np.where((flip & ((1 << n) - 1)) == 0, best, flip)  # dropping the last one: no change
            wt[:, r] = obj[rows, flip] - obj[rows, best]
        y[:, 7] = (best >> n) & 1
        wt[:, 7] = obj[rows, best ^ (1 << n)] - obj[rows, best]
        ys.append(y), ws.append(wt)
    Y, W = np.concatenate(ys), np.concatenate(ws)
    present = np.zeros_like(W, dtype=bool)
    k = 0
    for s in costs:
        present[k:k + costs[s].shape[0], :nrefs[s]] = True
        present[k:k + costs[s].shape[0], 7] = True
        k += costs[s].shape[0]
    W = np.where(present, np.maximum(W, 0.0), 0.0)
    W = np.where(present, W / max(W[present].mean(), 1e-12) + floor, 0.0).astype(np.float32)
    return Y, W
