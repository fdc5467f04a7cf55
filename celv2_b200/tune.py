"""Autotuner of the engine's launch configuration, per frame size.

The decisions never depend on these knobs (the tests check every one against the oracle); only the
speed does. For one resolution it times the stage kernels under every combination of
  - motion-search cells per CTA (15 or 30),
  - persistent queue-draining grid or one CTA per unit,
  - inter MV chunk (32 or 64),
on a representative job (a frame and its references already in the engine's store), with the
engine's CUDA-event stage timing, and keeps for each stage its fastest setting: the cells per
pyramid level, the persistent mask per stage, the inter chunk. Results can be cached in a JSON file
keyed by device name and frame size.
"""
from __future__ import annotations

import itertools
import json
import os

from . import engine as E

STAGES_ME = ["me_l0", "me_l1", "me_l2", "me_l3", "me_l4"]


def _measure(eng: E.CudaEngine, run, reps: int) -> dict:
    eng.stage_times()
    for _ in range(reps):
        run()
    return eng.stage_times()


def autotune(eng: E.CudaEngine, src_key: int, ref_keys, qindex: int = 130, reps: int = 3) -> dict:
    """Times every combination on the job (src_key, ref_keys) and sets the fastest per stage."""
    return autotune_run(eng, lambda: eng.launch_group([src_key], [list(ref_keys)], qindex), reps)


def autotune_run(eng: E.CudaEngine, run, reps: int = 3) -> dict:
    """Times every combination on the work `run` launches -- a group of eng's, or a batch of several
    engines whose first job is eng's (celv2_launch_multi runs the stages with its first engine's
    configuration) -- and sets eng's fastest per stage."""
    eng.set_config(E.CFG_GRAPHS, 0)
    eng.set_config(E.CFG_PERSISTENT, 1)
    eng.stage_timing(True)
    run()  # warm-up
    results = []
    try:
        for cells, persistent, chunk in itertools.product((15, 30), (0, 1), (32, 64)):
            for l in range(5):
                eng.set_config(E.CFG_ME_CELLS_L0 + l, cells)
            eng.set_config(E.CFG_PERSISTENT_OFF, 0 if persistent else 0x1FF)
            eng.set_config(E.CFG_INTER_CHUNK, chunk)
            results.append(((cells, persistent, chunk), _measure(eng, run, reps)))
    finally:
        eng.stage_timing(False)

    def best(stage, key):
        # the fastest setting of this stage's own knobs
        return min(results, key=lambda r: (r[1][stage][0], r[0]))[0] if any(r[1][stage][1] for r in results) else None

    chosen = {"me_cells": [], "persistent_off": 0, "inter_chunk": 64, "stage_ms": {}}
    for l in range(5):
        b = best(f"me_l{l}", None)
        cells, persistent = (b[0], b[1]) if b else (30, 1)
        chosen["me_cells"].append(cells)
        if not persistent:
            chosen["persistent_off"] |= 1 << l
    for bit, stage in ((5, "intra"), (6, "inter"), (7, "finalize"), (8, "me_refine")):
        b = best(stage, None)
        if b and not b[1]:
            chosen["persistent_off"] |= 1 << bit
        if stage == "inter" and b:
            chosen["inter_chunk"] = b[2]
    for stage in STAGES_ME + ["me_refine", "intra", "inter", "finalize"]:
        chosen["stage_ms"][stage] = min(r[1][stage][0] for r in results) / reps
    apply(eng, chosen)
    return chosen


def apply(eng: E.CudaEngine, chosen: dict) -> None:
    for l, cells in enumerate(chosen["me_cells"]):
        eng.set_config(E.CFG_ME_CELLS_L0 + l, cells)
    eng.set_config(E.CFG_PERSISTENT, 1)
    eng.set_config(E.CFG_PERSISTENT_OFF, chosen["persistent_off"])
    eng.set_config(E.CFG_INTER_CHUNK, chosen["inter_chunk"])


def cache_path() -> str:
    return os.environ.get("CELV2_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "celv2_b200", "tune.json"))


def cached(eng: E.CudaEngine, device_name: str, src_key: int, ref_keys, qindex: int = 130) -> dict:
    """The cached choice for this device and frame size, tuned and stored when absent."""
    key = f"{device_name}:{eng.width}x{eng.height}:refs{len(ref_keys)}"
    path = cache_path()
    table = {}
    if os.path.exists(path):
        try:
            table = json.load(open(path))
        except (OSError, ValueError):
            table = {}
    if key in table:
        apply(eng, table[key])
        return table[key]
    chosen = autotune(eng, src_key, ref_keys, qindex)
    table[key] = chosen
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as fh:
            json.dump(table, fh, indent=1)
    except OSError:
        pass
    return chosen
