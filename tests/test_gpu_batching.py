"""Batching changes the launch structure, not the decisions: persistent queue-draining stage
kernels, CUDA-graph replay of a batch, and one batch over streams of different frame sizes must
all give the oracle's records byte for byte."""
import json

import pytest

from celv2_b200 import lam, synth
from celv2_b200 import engine as E
from celv2_b200.records import first_difference, records_equal

pytestmark = pytest.mark.gpu


def check(oracle, w, h, clip, src, refs, q, got, what):
    want = oracle.decide(w, h, clip[src].y, [clip[r].y for r in refs], lam.lambda_q8(q))
    assert records_equal(got, want), f"{what}: {first_difference(got, want)}"


@pytest.mark.parametrize("persistent", [0, 1])
@pytest.mark.parametrize("graphs", [0, 1])
def test_group_modes_match_oracle(oracle, persistent, graphs):
    w, h = 416, 240
    clip = synth.small_clip(seed=21, frames=8)
    with E.CudaEngine(w, h) as e:
        e.set_config(E.CFG_PERSISTENT, persistent)
        e.set_config(E.CFG_GRAPHS, graphs)
        for i, f in enumerate(clip):
            e.upload(f.hy, i)
        batches = [[(7, [6, 5, 4])], [(3, [2, 1, 0]), (4, [3, 2]), (5, [4]), (6, [])]]
        for rep in range(2):  # a graph is captured on the first pass and replayed on the second
            for batch in batches:
                e.launch_group([s for s, _ in batch], [r for _, r in batch], 120, to_host=True)
                for j, (s, refs) in enumerate(batch):
                    check(oracle, w, h, clip, s, refs, 120, e.group_records(j), f"rep {rep} job {s}")


def test_multi_resolution_batch_matches_oracle(oracle):
    sizes = [(416, 240), (320, 192), (640, 360), (202, 122)]
    clips = [synth.sinusoid_clip(w, h, 4, 30 + k, noise_sigma=3.0) for k, (w, h) in enumerate(sizes)]
    engines = [E.CudaEngine(w, h) for w, h in sizes]
    try:
        for e, clip in zip(engines, clips):
            for i, f in enumerate(clip):
                e.upload(f.hy, i)
        jobs = [(engines[0], 3, [2, 1, 0]), (engines[1], 3, [2, 1]), (engines[2], 2, [1, 0]),
                (engines[0], 2, [1]), (engines[3], 3, [2, 1, 0]), (engines[2], 1, []), (engines[1], 2, [1, 0])]
        E.launch_multi(jobs, 130, to_host=True)
        seen = {}
        for e, src, refs in jobs:
            k = seen.get(id(e), 0)
            seen[id(e)] = k + 1
            i = engines.index(e)
            w, h = sizes[i]
            check(oracle, w, h, clips[i], src, refs, 130, e.group_records(k), f"{w}x{h} frame {src}")
    finally:
        for e in engines:
            e.close()


@pytest.mark.parametrize("cells,chunk,off", [(16, 32, 0), (16, 64, 0xFF), (32, 32, 0x55)])
def test_tuning_knobs_match_oracle(oracle, cells, chunk, off):
    w, h = 416, 240
    clip = synth.small_clip(seed=23, frames=8)
    with E.CudaEngine(w, h) as e:
        for l in range(5):
            e.set_config(E.CFG_ME_CELLS_L0 + l, cells)
        e.set_config(E.CFG_INTER_CHUNK, chunk)
        e.set_config(E.CFG_PERSISTENT_OFF, off)
        for i, f in enumerate(clip):
            e.upload(f.hy, i)
        e.launch_group([7, 6], [[6, 5, 4, 3, 2, 1, 0], [5, 4]], 120, to_host=True)
        check(oracle, w, h, clip, 7, [6, 5, 4, 3, 2, 1, 0], 120, e.group_records(0), "7 refs")
        check(oracle, w, h, clip, 6, [5, 4], 120, e.group_records(1), "2 refs")


def test_autotuner_sets_a_valid_config(tmp_path, monkeypatch):
    from celv2_b200 import tune

    monkeypatch.setenv("CELV2_TUNE_CACHE", str(tmp_path / "tune.json"))
    clip = synth.small_clip(seed=25, frames=8)
    with E.CudaEngine(416, 240) as e:
        for i, f in enumerate(clip):
            e.upload(f.hy, i)
        chosen = tune.cached(e, "test-gpu", 7, [6, 5, 4, 3, 2, 1, 0])
        assert len(chosen["me_cells"]) == 5 and all(c in (16, 32) for c in chosen["me_cells"])
        assert chosen["inter_chunk"] in (32, 64)
        assert [e.get_config(E.CFG_ME_CELLS_L0 + l) for l in range(5)] == chosen["me_cells"]
        again = tune.cached(e, "test-gpu", 7, [6, 5, 4, 3, 2, 1, 0])  # from the cache file
        assert again == json.loads(json.dumps(chosen))
