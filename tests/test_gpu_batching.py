"""Batching changes the launch structure, not the decisions: persistent queue-draining stage
kernels, CUDA-graph replay of a batch, and one batch over streams of different frame sizes must
all give the oracle's records byte for byte."""
import ctypes as C
import json

import numpy as np
import pytest

from celv2_b200 import lam, synth
from celv2_b200 import engine as E
from celv2_b200.records import SB_OUT_DTYPE, DecisionMap, first_difference, records_equal

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


@pytest.mark.parametrize("cells,chunk,off", [(15, 32, 0), (15, 64, 0x1FF), (30, 32, 0x155)])
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
        assert len(chosen["me_cells"]) == 5 and all(c in (15, 30) for c in chosen["me_cells"])
        assert chosen["inter_chunk"] in (32, 64)
        assert [e.get_config(E.CFG_ME_CELLS_L0 + l) for l in range(5)] == chosen["me_cells"]
        again = tune.cached(e, "test-gpu", 7, [6, 5, 4, 3, 2, 1, 0])  # from the cache file
        assert again == json.loads(json.dumps(chosen))


def test_records_land_in_caller_memory(oracle):
    w, h = 416, 240
    clip = synth.small_clip(seed=4, frames=3)
    with E.CudaEngine(w, h) as e:
        bad = np.zeros(e.sb_cols * e.sb_rows, dtype=SB_OUT_DTYPE)  # pageable memory is refused
        with pytest.raises(RuntimeError):
            e.set_output(0, bad.ctypes.data)
        dm, gate = DecisionMap(), E.RowGate()
        e.launch(clip[2].hy, [clip[1].hy, clip[0].hy], 120, dm)
        e.collect(dm, gate)
        ptr = C.c_void_p()
        assert E.library().celv2_wait_row(e._h, 0, C.byref(ptr)) == 0
        assert ptr.value == dm.records.ctypes.data  # the rows were copied into dm itself
        check(oracle, w, h, clip, 2, [1, 0], 120, dm.records, "launch into caller memory")
        keep = dm.records.copy()
        dm2 = e.decide_inter(clip[1].hy, [clip[0].hy], 120)  # a later launch leaves dm alone
        assert records_equal(dm.records, keep)
        check(oracle, w, h, clip, 1, [0], 120, dm2.records, "second launch")


@pytest.mark.parametrize("graphs", [0, 1])
def test_decide_group_pipelined_matches_oracle(oracle, graphs):
    """The mini-GOP through decide_group with every group in flight before the first is read:
    double-buffered device records, copies overlapping the next group, keyed references reused."""
    w, h = 416, 240
    clip = synth.small_clip(seed=9, frames=9)
    plan = [[(0, [])], [(8, [0])], [(4, [0, 8])], [(2, [0, 4, 8]), (6, [4, 8, 0])],
            [(1, [0, 2, 4]), (3, [2, 4, 0]), (5, [4, 6, 2]), (7, [6, 8, 4])]]
    with E.CudaEngine(w, h) as e:
        e.set_config(E.CFG_GRAPHS, graphs)
        for rep in range(2):
            out = []
            for group in plan:
                dms = e.decide_group([clip[s].hy for s, _ in group], [[clip[r].hy for r in refs] for _, refs in group],
                                     120, ref_keys=[list(refs) for _, refs in group], wait=False)
                out.append(dms)
            e.finish()
            for group, dms in zip(plan, out):
                for (s, refs), dm in zip(group, dms):
                    check(oracle, w, h, clip, s, refs, 120, dm.records, f"rep {rep} frame {s}")


def test_launch_multi_into_maps(oracle):
    sizes = [(416, 240), (202, 122)]
    clips = [synth.sinusoid_clip(w, h, 3, 50 + k, noise_sigma=3.0) for k, (w, h) in enumerate(sizes)]
    engines = [E.CudaEngine(w, h) for w, h in sizes]
    try:
        for e, clip in zip(engines, clips):
            for i, f in enumerate(clip):
                e.upload(f.hy, i)
        jobs = [(engines[0], 2, [1, 0]), (engines[1], 2, [1]), (engines[0], 1, [0])]
        for rep in range(3):  # alternating device record buffers
            dms = [DecisionMap() for _ in jobs]
            E.launch_multi(jobs, 130, dms=dms)
            for e in engines:
                e.finish()
            for (e, src, refs), dm in zip(jobs, dms):
                i = engines.index(e)
                check(oracle, *sizes[i], clips[i], src, refs, 130, dm.records, f"rep {rep} {sizes[i]} frame {src}")
    finally:
        for e in engines:
            e.close()


def test_pinned_uploads_match_oracle(oracle):
    """celv2_upload_pinned: planes in page-locked memory go to the device by DMA after the call;
    the decisions are the oracle's; pageable planes are refused."""
    w, h = 416, 240
    clip = synth.small_clip(seed=23, frames=4)
    pool = []
    for f in clip:
        a = E.host_array(f.hy.shape, np.uint16)
        a[...] = f.hy
        pool.append(a)
    with E.CudaEngine(w, h) as e:
        with pytest.raises(RuntimeError):
            e.upload(clip[0].hy.copy(), 0, pinned=True)
        groups = [[(0, [])], [(3, [0])], [(1, [0, 3]), (2, [3, 0])]]
        out = []
        for g in groups:
            out.append(e.decide_group([pool[s] for s, _ in g], [[pool[r] for r in refs] for _, refs in g], 120,
                                      ref_keys=[list(refs) for _, refs in g], wait=False, pinned=True))
        e.finish()
        for g, dms in zip(groups, out):
            for (s, refs), dm in zip(g, dms):
                check(oracle, w, h, clip, s, refs, 120, dm.records, f"frame {s}")


def test_records_left_on_the_device_are_not_returned(oracle):
    """A group launched with to_host 0 leaves its records on the device: group_records refuses it
    (rather than returning an older group's records), and set_output is refused for such a launch."""
    w, h = 416, 240
    clip = synth.small_clip(seed=27, frames=4)
    with E.CudaEngine(w, h) as e:
        for i, f in enumerate(clip):
            e.upload(f.hy, i)
        e.launch_group([3], [[2, 1]], 120, to_host=True)
        check(oracle, w, h, clip, 3, [2, 1], 120, e.group_records(0), "to_host group")
        e.launch_group([2], [[1]], 120, to_host=False)
        with pytest.raises(RuntimeError, match="on the device"):
            e.group_records(0)
        out = E.host_array((e.sb_cols * e.sb_rows * SB_OUT_DTYPE.itemsize,), np.uint8)
        e.set_output(0, out.ctypes.data)
        with pytest.raises(RuntimeError, match="to_host 0"):
            e.launch_group([2], [[1]], 120, to_host=False)
        e.launch_group([2], [[1]], 120, to_host=True)
        check(oracle, w, h, clip, 2, [1], 120, e.group_records(0), "after the refused launch")


def test_rejected_multi_batch_leaves_the_engines_as_they_were(oracle):
    """A batch with a missing reference key is rejected before it changes any engine's state; the
    next two batches, both in flight before either is read, still give the oracle's records."""
    sizes = [(416, 240), (202, 122)]
    clips = [synth.sinusoid_clip(w, h, 3, 60 + k, noise_sigma=3.0) for k, (w, h) in enumerate(sizes)]
    engines = [E.CudaEngine(w, h) for w, h in sizes]
    try:
        for e, clip in zip(engines, clips):
            for i, f in enumerate(clip):
                e.upload(f.hy, i)
        with pytest.raises(RuntimeError, match="reference key"):
            E.launch_multi([(engines[0], 2, [1, 0]), (engines[1], 2, [99])], 130, to_host=True)
        batches = [[(engines[0], 2, [1, 0]), (engines[1], 2, [1])], [(engines[1], 1, [0]), (engines[0], 1, [0])]]
        maps = []
        for jobs in batches:
            dms = [DecisionMap() for _ in jobs]
            E.launch_multi(jobs, 130, dms=dms)
            maps.append(dms)
        for e in engines:
            e.finish()
        for jobs, dms in zip(batches, maps):
            for (e, src, refs), dm in zip(jobs, dms):
                i = engines.index(e)
                check(oracle, *sizes[i], clips[i], src, refs, 130, dm.records, f"{sizes[i]} frame {src}")
    finally:
        for e in engines:
            e.close()
