"""The benchmarked configurations decided exactly as bench.py decides them, against the oracle.

- The 1080p 10-bit mini-GOP (17 frames, hidden anchor and pyramid, refs 7, qindex 130, the bench
  clip): the coding groups of the bench's step, the ten leaves as one batch, CUDA graphs captured
  and replayed, the launch knobs the autotuner picks at 1080p, records double-buffered into host
  maps while the next group runs -- every frame's records byte-identical to the oracle's.
- 3840x2160: one frame against 7 references, through the per-frame launch and a group launch.
- Six streams of uneven size (640x360, 960x540, 1280x720, 1920x1080 twice, 3840x2160), each tuned
  for its size, decided in one multi-resolution batch (celv2_launch_multi).
- Animation-like content (flat colours, hard edges, sparse noise, piecewise motion, a scene cut),
  where equal costs are everywhere and the first-strict-minimum rules of the motion search, the
  candidate scan and the partition choice decide (reference src/gpu/inter_common.h:108-119,
  src/gpu/kernels_ref.cpp:145-149,174-178): 640x360 per frame and as a group, and one 4K frame.
The oracle runs on every host core.
"""
import numpy as np
import pytest

from celv2_b200 import engine as E
from celv2_b200 import lam, synth, tune
from celv2_b200.records import DecisionMap, first_difference, records_equal

pytestmark = pytest.mark.gpu

Q = 130


def check(oracle, w, h, cur, refs, q, got, what):
    want = oracle.decide(w, h, cur, refs, lam.lambda_q8(q))
    assert records_equal(got, want), f"{what}: {first_difference(got, want)}"


@pytest.fixture(scope="module")
def clip_4k():
    """Eight 3840x2160 frames of the sinusoid workload (8 sinusoids, 12 rectangles, per-region
    affine motion, noise sigma 4)."""
    return synth.hd_clip(seed=41, frames=8, width=3840, height=2160)


def test_headline_mini_gop_as_benched(oracle):
    import bench

    clip = bench.make_clip(bench.SEED)
    plan = bench.mini_gop_plan()
    w, h = bench.W, bench.H
    with E.CudaEngine(w, h) as e:
        e.reserve_group(max(len(g) for g in plan))
        for i, f in enumerate(clip):
            e.upload(f.hy, i)
        leaf_src, leaf_refs = plan[-1][0]
        tune.autotune(e, leaf_src, leaf_refs, Q)
        e.set_config(E.CFG_GRAPHS, 1)
        for _ in range(2):  # the bench's warm-up steps: graphs captured, then replayed
            for group in plan:
                e.launch_group([s for s, _ in group], [r for _, r in group], Q)
        maps = []
        for group in plan:  # a replayed step, records into host maps while the next group runs
            dms = [DecisionMap() for _ in group]
            e.launch_group([s for s, _ in group], [r for _, r in group], Q, dms=dms)
            maps.append(dms)
        e.finish()
    for group, dms in zip(plan, maps):
        for (s, refs), dm in zip(group, dms):
            check(oracle, w, h, clip[s].y, [clip[r].y for r in refs], Q, dm.records, f"frame {s} ({len(refs)} refs)")


def test_4k_seven_references(oracle, clip_4k):
    w, h = 3840, 2160
    src, refs = 7, [6, 5, 4, 3, 2, 1, 0]
    want = oracle.decide(w, h, clip_4k[src].y, [clip_4k[r].y for r in refs], lam.lambda_q8(Q))
    with E.CudaEngine(w, h) as e:
        got = e.decide_inter(clip_4k[src].hy, [clip_4k[r].hy for r in refs], Q).records
        assert records_equal(got, want), f"launch: {first_difference(got, want)}"
        for i in range(8):
            e.upload(clip_4k[i].hy, i)
        e.set_config(E.CFG_GRAPHS, 1)
        for _ in range(2):
            e.launch_group([src, 3], [refs, [2, 1, 0]], Q, to_host=True)
            got = e.group_records(0)
            assert records_equal(got, want), f"group: {first_difference(got, want)}"
        check(oracle, w, h, clip_4k[3].y, [clip_4k[r].y for r in (2, 1, 0)], Q, e.group_records(1), "group, 3 refs")


C3_SIZES = [(640, 360), (960, 540), (1280, 720), (1920, 1080), (1920, 1080), (3840, 2160)]


def test_six_uneven_streams_one_batch(oracle, clip_4k):
    """The multi-stream configuration's sizes in one launch_multi batch, each engine tuned for its
    frame size, two frames per stream (a 3-reference and a 7-reference one)."""
    clips = [synth.hd_clip(seed=k, frames=8, width=w, height=h) if w < 3840 else clip_4k
             for k, (w, h) in enumerate(C3_SIZES)]
    engines = [E.CudaEngine(w, h) for w, h in C3_SIZES]
    try:
        for e, clip in zip(engines, clips):
            e.reserve_group(2)
            for i, f in enumerate(clip):
                e.upload(f.hy, i)
            tune.autotune(e, 7, [6, 5, 4, 3, 2, 1, 0], Q, reps=1)
        jobs = []
        for e in engines:
            jobs += [(e, 3, [2, 1, 0]), (e, 7, [6, 5, 4, 3, 2, 1, 0])]
        wants = {}
        for rep in range(3):  # each batch in its own device record buffer set (three in turn)
            dms = [DecisionMap() for _ in jobs]
            E.launch_multi(jobs, Q, dms=dms)
            for e in engines:
                e.finish()
            for (e, src, refs), dm in zip(jobs, dms):
                i = engines.index(e)
                w, h = C3_SIZES[i]
                if (i, src) not in wants:
                    wants[i, src] = oracle.decide(w, h, clips[i][src].y, [clips[i][r].y for r in refs],
                                                  lam.lambda_q8(Q))
                want = wants[i, src]
                assert records_equal(dm.records, want), \
                    f"rep {rep} stream {i} ({w}x{h}) frame {src}: {first_difference(dm.records, want)}"
    finally:
        for e in engines:
            e.close()


def test_animation_scene_cut_per_frame_and_group(oracle):
    w, h = 640, 360
    clip = synth.animation_clip(w, h, 12, seed=5, scene_cut=6)
    plan = [(k, [k - d for d in range(1, 8) if k - d >= 0]) for k in range(1, 12)]
    with E.CudaEngine(w, h) as e:
        want = {}
        for src, refs in plan:  # per frame: the reference's launch / collect
            want[src] = oracle.decide(w, h, clip[src].y, [clip[r].y for r in refs], lam.lambda_q8(Q))
            got = e.decide_inter(clip[src].hy, [clip[r].hy for r in refs], Q).records
            assert records_equal(got, want[src]), f"launch frame {src}: {first_difference(got, want[src])}"
        got = e.decide_intra(clip[6].hy, Q).records  # the cut frame as a KEY frame
        check(oracle, w, h, clip[6].y, [], Q, got, "KEY at the cut")
        for i, f in enumerate(clip):
            e.upload(f.hy, i)
        e.set_config(E.CFG_GRAPHS, 1)
        for rep in range(2):
            e.launch_group([s for s, _ in plan], [r for _, r in plan], Q, to_host=True)
            for j, (s, _) in enumerate(plan):
                got = e.group_records(j)
                assert records_equal(got, want[s]), f"rep {rep} group frame {s}: {first_difference(got, want[s])}"


def test_animation_4k_frame(oracle):
    w, h = 3840, 2160
    clip = synth.anime_clip(seed=3, frames=9, scene_cut=7)
    # frame 8 (after the cut at 7) against the cut frame and six frames of the previous scene
    src, refs = 8, [7, 6, 5, 4, 3, 2, 1]
    want = oracle.decide(w, h, clip[src].y, [clip[r].y for r in refs], lam.lambda_q8(Q))
    with E.CudaEngine(w, h) as e:
        got = e.decide_inter(clip[src].hy, [clip[r].hy for r in refs], Q).records
        assert records_equal(got, want), f"launch: {first_difference(got, want)}"
        for i in refs + [src, 0]:
            e.upload(clip[i].hy, i)
        e.launch_group([src, 1], [refs, [0]], Q, to_host=True)
        got = e.group_records(0)
        assert records_equal(got, want), f"group: {first_difference(got, want)}"
        check(oracle, w, h, clip[1].y, [clip[0].y], Q, e.group_records(1), "group, frame 1")
    assert len(np.unique(clip[src].y)) < 64  # flat content: the tie rules decide
