"""What pruning costs and saves on a mini-GOP: the chosen partitions' total cost against the
exhaustive search's (the engine's own rate-distortion measure, lambda-weighted SATD plus rate; the
BD-rate needs AVM), and the device time of the mini-GOP's decisions."""
from __future__ import annotations

import numpy as np

from .. import engine as E
from .. import gop


def upload(eng: E.CudaEngine, clip) -> None:
    eng.clear_store()
    for i, f in enumerate(clip):
        eng.upload(f, i)


def run(eng: E.CudaEngine, plan, qindex: int, masks=None, reps: int = 1):
    """(per inter frame: its superblock costs, ms per mini-GOP, per inter frame: its masks) for the
    frames already in the store. masks: None (the engine's own setting: exhaustive, or the pruner
    if one is set), or a function (frame, nrefs, nsb) -> keep words (or bytes) given through
    celv2_set_keep_words."""
    import torch

    stream = torch.cuda.ExternalStream(eng.stream())
    nsb = eng.sb_cols * eng.sb_rows

    def once(collect: bool):
        costs, kept = {}, {}
        for group in plan:
            if masks is not None:
                for j, (s, refs) in enumerate(group):
                    if refs:
                        eng.set_keep(j, masks(s, len(refs), nsb))
            eng.launch_group([s for s, _ in group], [r for _, r in group], qindex)
            if collect:
                for j, (s, refs) in enumerate(group):
                    if refs:
                        costs[s] = eng.sb_costs(j)
                        kept[s] = eng.pruner_masks(j) if masks is None else masks(s, len(refs), nsb)
        return costs, kept

    costs, kept = once(True)
    once(False)  # warm: graphs, caches
    eng.finish()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        once(False)
    b.record(stream)
    b.synchronize()
    return costs, a.elapsed_time(b) / reps, kept


def cost_increase(pruned: dict, full: dict) -> float:
    """Relative increase of the summed chosen cost over the inter frames."""
    p = sum(float(v.sum()) for v in pruned.values())
    f = sum(float(full[k].sum()) for k in pruned)
    return p / f - 1.0


def kept_work(kept: dict, plan) -> dict:
    """What the keep words left to score, over the inter superblocks: the share of the frame's
    references kept, the share that keeps intra, the share of block levels kept, the share of the
    superblocks where the inter stage ran on 16x16 regions (no 64- or 32-level blocks), and the
    share that fell back to the full search (every bit set)."""
    nrefs = {s: len(r) for g in plan for s, r in g}
    refs = total = intra = n = lv = r16 = full = 0
    for s, k in kept.items():
        k = k.astype(np.int64)
        bits = (k[:, None] >> np.arange(7)[None, :]) & 1
        live = bits[:, :nrefs[s]].sum(1)
        live = np.where(live == 0, nrefs[s], live)  # none named keeps them all
        levels = (k >> 8) & 0xF
        levels = np.where(levels == 0, 0xF, levels)
        refs += int(live.sum())
        total += nrefs[s] * k.size
        intra += int(((k >> 7) & 1).sum())
        lv += int(sum(((levels >> l) & 1).sum() for l in range(4)))
        r16 += int(((levels & 3) == 0).sum())
        full += int((k == 0xFFFFFFFF).sum())
        n += k.size
    n = max(1, n)
    return {"refs_kept": refs / max(1, total), "intra_kept": intra / n, "levels_kept": lv / (4 * n),
            "regions16": r16 / n, "fallback": full / n}


def nearest(k: int, intra: bool, small_only: bool = False):
    """The rule without the network: keep the k nearest references, intra or not, and every block
    level or (small_only) only the 16- and 8-sample levels."""
    def f(_frame, nrefs, nsb):
        bits = (1 << min(k, nrefs)) - 1
        levels = 0xC00 if small_only else 0xF00
        return np.full(nsb, bits | (0x80 if intra else 0) | levels, np.uint32)
    return f


def default_plan(frames: int = 17):
    return gop.stream_plan(frames)
