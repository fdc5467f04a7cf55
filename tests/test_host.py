"""Host-side logic without a GPU: the RowGate mirror (tests/test_row_gate.cpp), the mini-GOP plan
of the benchmark (src/chunk_coder.cpp:213-225), the record conversion, and the multi-rank timing
path as world-size-2 gloo ranks."""
import os
import threading
import time

import numpy as np
import pytest

import bench
from celv2_b200.engine import RowGate
from celv2_b200.records import SB_OUT_DTYPE, to_decision


def test_publish_releases_waiters():
    g = RowGate()
    done = []
    t = threading.Thread(target=lambda: (g.wait_row(2, timeout=10), done.append(1)))
    t.start()
    time.sleep(0.05)
    assert not done
    g.publish(2)
    t.join(5)
    assert done and g.ready_rows() == 3


def test_publish_out_of_order_is_monotonic():
    g = RowGate()
    g.publish_one(1)
    assert g.ready_rows() == 0
    g.wait_row(1, timeout=1)  # row 1 itself is ready
    g.publish_one(0)
    assert g.ready_rows() == 2
    g.publish(0)  # smaller values are ignored
    assert g.ready_rows() == 2


def test_fail_wakes_and_rethrows():
    g = RowGate()
    errs = []

    def waiter():
        try:
            g.wait_row(4, timeout=10)
        except RuntimeError as e:
            errs.append(str(e))

    ts = [threading.Thread(target=waiter) for _ in range(3)]
    for t in ts:
        t.start()
    time.sleep(0.05)
    g.fail(RuntimeError("boom"))
    g.fail(RuntimeError("second"))  # the first failure is kept
    for t in ts:
        t.join(5)
    assert errs == ["boom"] * 3


def test_mini_gop_plan():
    plan = bench.mini_gop_plan()
    order = [s for g in plan for s, _ in g]
    assert order[:7] == [0, 16, 8, 4, 2, 6, 12]
    assert sorted(order) == list(range(17))
    assert [s for s, _ in plan[-1]] == [1, 3, 5, 7, 9, 10, 11, 13, 14, 15]
    refs_done = set()
    for group in plan:
        for s, refs in group:
            assert len(refs) <= 7 and set(refs) <= refs_done | {0} - {s}
            dist = [abs(r - s) for r in refs]
            assert dist == sorted(dist)
        refs_done |= {s for s, _ in group if s in (0, 16, 8, 4, 2, 6, 12)}
    assert all(len(refs) == 7 for _, refs in plan[-1])


def test_record_conversion_doubles_mvs():
    r = np.zeros(1, SB_OUT_DTYPE)[0]
    r["ntree"], r["nblocks"] = 1, 1
    r["w4"][0], r["h4"][0], r["mode"][0], r["mvx"][0], r["mvy"][0], r["ref"][0] = 16, 16, 13, 5, -3, 2
    r["ref2"][0] = 255
    r["c_ref2"][:] = 255
    d = to_decision(r)
    assert d.tree == [0]
    b = d.blocks[0]
    assert (b.inter, b.mv_col, b.mv_row, b.ref, b.ref2) == (True, 10, -6, 2, 255)
    assert len(d.cands) == 425


def _rank(rank, world, port, out):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench.barrier(dist, 0)
        v = bench.max_over_ranks(10.0 * (rank + 1), dist, 0)
        out.put((rank, v))
    finally:
        dist.destroy_process_group()


def test_two_rank_max_over_ranks_gloo():
    import multiprocessing as mp
    import socket

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(60)
    assert got == [(0, 20.0), (1, 20.0)]


def _stream_rank(rank, world, port, out):
    import torch
    import torch.distributed as dist

    from celv2_b200 import gop

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sizes = [(3840, 2160), (1920, 1080), (1920, 1080), (1280, 720), (960, 540), (640, 360)]
        mine = gop.assign_streams(sizes, [33] * 6, world)[rank]
        sbs = sum(((w + 63) // 64) * ((h + 63) // 64) * 33 for w, h in (sizes[i] for i in mine))
        t = torch.tensor([sbs], dtype=torch.float64)
        dist.all_reduce(t)  # the aggregate superblocks of the multi-stream configuration
        out.put((rank, mine, int(t.item())))
    finally:
        dist.destroy_process_group()


def test_streams_shard_across_two_ranks_gloo():
    """Whole streams to ranks (the multi-stream configuration on 2 GPUs): each stream on exactly
    one rank, the 4K stream alone on one, and the ranks' superblocks sum to the whole workload."""
    import multiprocessing as mp
    import socket

    from celv2_b200 import gop

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_stream_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(60)
    assert sorted(got[0][1] + got[1][1]) == list(range(6))
    assert got[0][1] == [0] and got[1][1] == [1, 2, 3, 4, 5]  # 2040 x 33 against 2070 x 33 superblocks
    assert got[0][2] == got[1][2] == 33 * (2040 + 510 + 510 + 240 + 135 + 60)
    assert gop.assign_streams([(640, 360)] * 3, [33] * 3, 4) == [[0], [1], [2], []]


def test_stream_plan_chains_mini_gops_and_cuts():
    """gop.stream_plan: 17 frames are the mini-GOP plan; 33 frames two mini-GOPs whose second takes
    its references from an 8-slot buffer (at most 7, nearest display distance first); a scene cut
    starts over with a KEY frame and no reference from before it."""
    from celv2_b200 import gop

    assert gop.stream_plan(17) == gop.mini_gop_plan(17)
    plan = gop.stream_plan(33)
    frames = [s for g in plan for s, _ in g]
    assert sorted(frames) == list(range(33))
    coded = []
    for g in plan:
        for s, refs in g:
            assert len(refs) <= 7 and all(r in coded for r in refs)
            assert refs == sorted(refs, key=lambda r: (abs(r - s), r))
        coded += [s for s, _ in g]
    assert [len(g) for g in plan].count(10) == 2  # two leaf groups
    cut = gop.stream_plan(65, cuts=[33])
    assert sorted(s for g in cut for s, _ in g) == list(range(65))
    for g in cut:
        for s, refs in g:
            assert all((r >= 33) == (s >= 33) for r in refs)
    assert (33, []) in [x for g in cut for x in g]


def test_animation_generator():
    """The animation-like content: flat colours (few distinct values), the scene cut a new picture,
    deterministic per seed."""
    from celv2_b200 import synth

    clip = synth.animation_clip(320, 192, 6, seed=4, scene_cut=3)
    again = synth.animation_clip(320, 192, 6, seed=4, scene_cut=3)
    assert all(np.array_equal(a.hy, b.hy) for a, b in zip(clip, again))
    assert len(np.unique(clip[1].y)) < 64
    step = np.abs(clip[2].y.astype(int) - clip[1].y).mean()
    cut = np.abs(clip[3].y.astype(int) - clip[2].y).mean()
    assert cut > step
