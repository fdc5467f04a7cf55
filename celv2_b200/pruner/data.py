"""Training records for the pruner: the exhaustive CUDA engine's decisions on seeded synthetic
clips, with the features the engine computes for every inter frame (CELV2_CFG_FEATURES).

Labels per superblock (the network's 24 outputs): the options its chosen partition uses --
reference r where a leaf predicts from it (its reference or its compound's second), intra where a
leaf is intra, block level l where a leaf is of that level, intra mode m (3..12) where an intra
leaf uses it. Keeping exactly these options loses nothing (used_options), so the network learns
which options the exhaustive search would have needed, and its thresholds trade speed for cost.
"""
from __future__ import annotations

import multiprocessing as mp

import numpy as np

from .. import engine as E
from .. import gop, synth

INTER = 13  # the record's mode of an inter leaf
OUT = E.PRUNER_OUTPUTS
MODE0 = 12  # output of intra mode 3; modes 3..12 at outputs 12..21


def block_level(w4: np.ndarray, h4: np.ndarray) -> np.ndarray:
    """The square level of leaves of w4 x h4 (4-sample units): 0 for 64x64 / 64x32 / 32x64, 1 for
    32x32 / 32x16 / 16x32, 2 for 16-, 3 for 8-sample squares and their halves."""
    side = np.maximum(w4, h4).astype(np.int64) * 4
    return np.select([side >= 64, side >= 32, side >= 16], [0, 1, 2], 3)


def used_options(records: np.ndarray, nrefs: int) -> np.ndarray:
    """Per superblock the keep word (include/celv2_decision.h) of exactly the options its chosen
    partition uses: the references of its inter leaves (a compound's second too), intra and the
    modes of its intra leaves, the levels of its leaves. These masks keep every block of the chosen
    partition with its choice at its cost (a block's best reference stays the best of the kept
    ones, a used compound's two references stay its best two), so the pruned search's cost is at
    most the exhaustive one -- lower where pruning a reference lets a block try its compound with
    another second reference, which the exhaustive search never tries."""
    nsb = records.size
    mode = records["mode"].astype(np.int64)
    leaf = np.arange(mode.shape[1])[None, :] < records["nblocks"].astype(np.int64)[:, None]
    inter = leaf & (mode == INTER)
    intra = leaf & (mode != INTER)
    words = np.zeros(nsb, np.uint64)
    for r in range(nrefs):
        used = (inter & ((records["ref"] == r) | (records["ref2"] == r))).any(axis=1)
        words |= np.where(used, np.uint64(1 << r), np.uint64(0))
    words |= np.where(intra.any(axis=1), np.uint64(0x80), np.uint64(0))
    lvl = block_level(records["w4"], records["h4"])
    for l in range(4):
        words |= np.where((leaf & (lvl == l)).any(axis=1), np.uint64(0x100 << l), np.uint64(0))
    for m in range(13):
        words |= np.where((intra & (mode == m)).any(axis=1), np.uint64(0x10000 << m), np.uint64(0))
    return words.astype(np.uint32)


def _clip(args):
    seed, frames = args
    return [f.hy for f in synth.hd_clip(seed, frames)]


def make_clips(seeds, frames: int = 17, workers: int = 4):
    """10-bit luma planes of seeded 1080p clips, made in worker processes (spawned: no CUDA state
    is inherited)."""
    with mp.get_context("spawn").Pool(workers) as pool:
        return pool.map(_clip, [(s, frames) for s in seeds])


def labels(words: np.ndarray, nrefs: int, pos_weight: float = 2.0, regret=None, cost=None,
           cap: float = 20.0):
    """(labels, weights), each nsb x OUTPUTS, from keep words of the used options: outputs 0..6 the
    references, 7 intra, 8..11 the levels, 12..21 intra modes 3..12 (weighed only where the chosen
    partition has intra leaves: the modes matter only when intra is kept). Absent references and
    the unused outputs weigh 0; needed options weigh `pos_weight` (missing one costs more than
    keeping one that is not needed). `regret` ({output: per superblock the cost increase of pruning
    that option alone}) and `cost` (the exhaustive costs) scale a needed option's weight by
    1 + regret / (the frame's mean superblock cost), at most `cap`: where the summed cost is small
    (flat content) a missed option costs a large share of it, which the plain labels do not show."""
    words = words.astype(np.int64)
    nsb = words.size
    y = np.zeros((nsb, OUT), np.float32)
    w = np.zeros((nsb, OUT), np.float32)
    for r in range(nrefs):
        y[:, r] = (words >> r) & 1
    w[:, :nrefs] = 1.0
    y[:, 7] = (words >> 7) & 1
    w[:, 7] = 1.0
    for l in range(4):
        y[:, 8 + l] = (words >> (8 + l)) & 1
    w[:, 8:12] = 1.0
    has_intra = y[:, 7] > 0
    for m in range(3, 13):
        y[:, MODE0 + m - 3] = (words >> (16 + m)) & 1
        w[:, MODE0 + m - 3] = has_intra
    w = np.where(y > 0, w * pos_weight, w)
    if regret:
        scale = max(float(np.mean(cost)), 1.0)
        for o, reg in regret.items():
            f = np.minimum(cap, 1.0 + np.maximum(reg.astype(np.float64), 0.0) / scale).astype(np.float32)
            w[:, o] = np.where(y[:, o] > 0, w[:, o] * f, w[:, o])
    return y, w


# The options whose training weight is scaled by their regret (collect(regrets=True)): output ->
# the keep word without that option alone, for a frame of n references (None: nothing to prune --
# a frame's only reference is always kept).
def _without_ref(r):
    return lambda n: None if n < 2 or r >= n else (((1 << n) - 1) & ~(1 << r)) | 0x80 | 0xF00 | 0x1FFF0000


def _without_level(l):
    return lambda n: ((1 << n) - 1) | 0x80 | (0xF00 & ~(0x100 << l)) | 0x1FFF0000


REGRET_OUTPUTS = {**{r: _without_ref(r) for r in range(7)},
                  7: lambda n: ((1 << n) - 1) | 0xF00 | 0x1FFF0000,
                  **{8 + l: _without_level(l) for l in range(4)}}


def collect(eng: E.CudaEngine, clip, qindex: int, plan=None, regrets: bool = False):
    """Features, labels, weights and (frame, nrefs, qindex) of every inter superblock of `clip`
    (10-bit planes, coded by `plan`) decided exhaustively, with each inter frame's exhaustive
    superblock costs and used-option keep words. regrets: each group is decided again once per
    REGRET_OUTPUTS option (each reference, intra, each block level), with that option alone pruned
    everywhere, and the cost increase per superblock scales the option's weight (labels)."""
    plan = plan or gop.mini_gop_plan(len(clip))
    nsb = eng.sb_cols * eng.sb_rows
    eng.clear_store()
    eng.set_config(E.CFG_FEATURES, 1)
    for i, f in enumerate(clip):
        eng.upload(f, i)
    xs, ys, ws, meta, costs, used = [], [], [], [], {}, {}
    for group in plan:
        srcs, refl = [s for s, _ in group], [r for _, r in group]
        eng.launch_group(srcs, refl, qindex, to_host=True)
        feats, words = {}, {}
        for j, (s, refs) in enumerate(group):
            if refs:
                feats[j] = eng.features(j)
                words[j] = used_options(eng.group_records(j), len(refs))
                costs[s] = eng.sb_costs(j)
        reg = {j: {} for j in feats}
        if regrets and feats:
            for o, word in REGRET_OUTPUTS.items():
                ks = {j: word(len(group[j][1])) for j in feats}
                if all(k is None for k in ks.values()):
                    continue
                for j, k in ks.items():
                    # a job with nothing to prune here is decided with all of it (its regret is 0)
                    eng.set_keep(j, np.full(nsb, 0xFFFFFFFF if k is None else k, np.uint32))
                eng.launch_group(srcs, refl, qindex)
                for j, k in ks.items():
                    if k is not None:
                        reg[j][o] = eng.sb_costs(j) - costs[group[j][0]]
        for j, x in feats.items():
            s, refs = group[j]
            y, w = labels(words[j], len(refs), regret=reg[j], cost=costs[s])
            xs.append(x), ys.append(y), ws.append(w)
            meta.append(np.tile([s, len(refs), qindex], (x.shape[0], 1)))
            used[s] = words[j]
    eng.set_config(E.CFG_FEATURES, 0)
    return (np.concatenate(xs), np.concatenate(ys), np.concatenate(ws), np.concatenate(meta)), costs, used
