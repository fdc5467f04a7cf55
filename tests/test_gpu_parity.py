"""CUDA engine against the oracle: byte-identical decision records, motion fields and intra SATDs.

Mirrors the reference's engine parity tests (tests/test_gpu_intra.cpp, tests/test_gpu_me.cpp,
tests/test_vk_kernels.cpp), with the C restatement of the reference rules as the oracle.
"""
import threading

import numpy as np
import pytest

import frames as F
from celv2_b200 import lam, synth
from celv2_b200.engine import CudaEngine, RowGate, unpack_field
from celv2_b200.records import DecisionMap, first_difference, records_equal

pytestmark = pytest.mark.gpu


def oracle_decide(oracle, w, h, src, refs, q):
    return oracle.decide(w, h, src, refs, lam.lambda_q8(q))


def assert_same(got, want, what=""):
    assert records_equal(got, want), f"{what}: first difference {first_difference(got, want)}"


CASES = [
    ("scene-202x122", 202, 122, lambda: (F.scene_frame(202, 122, 3, -2), [F.scene_frame(202, 122)])),
    ("scene-640x360", 640, 360, lambda: (F.scene_frame(640, 360, 3, -2), [F.scene_frame(640, 360)])),
    ("scene-32", 32, 32, lambda: (F.scene_frame(32, 32, 1, 1), [F.scene_frame(32, 32)])),
    ("scene-16", 16, 16, lambda: (F.scene_frame(16, 16, 1, 1), [F.scene_frame(16, 16)])),
    ("odd-72x40", 72, 40, lambda: (F.scene_frame(72, 40, 2, 1), [F.scene_frame(72, 40)])),
    ("multi3-202x122", 202, 122, lambda: (F.scene_frame(202, 122, 6, -3),
                                           [F.scene_frame(202, 122, 40, 30, 5), F.scene_frame(202, 122, 6, -3),
                                            F.scene_frame(202, 122, 3, -1)])),
    ("textured-640x360", 640, 360, lambda: (F.textured(640, 360, 5, -3), [F.textured(640, 360, 0, 0)])),
    ("glyph", 200, 120, lambda: (F.glyph_frame(200, 120, 3), [F.glyph_frame(200, 120, 0)])),
    ("noise7", 130, 90, lambda: (F.noise(130, 90, 1), [F.noise(130, 90, k + 2) for k in range(7)])),
    ("flat", 640, 360, lambda: (np.full((360, 640), 128, np.uint8), [np.full((360, 640), 128, np.uint8)])),
    ("smooth7", 320, 192, lambda: (F.smooth(320, 192, 0, 0), [F.smooth(320, 192, 1.25 * i, -0.75 * i)
                                                              for i in range(1, 8)])),
]


@pytest.mark.parametrize("name,w,h,make", CASES, ids=[c[0] for c in CASES])
def test_decisions_match_oracle(oracle, name, w, h, make):
    src, refs = make()
    with CudaEngine(w, h) as e:
        for q in (40, 120, 220):
            for key in (True, False):
                rr = [] if key else refs
                got = e.decide_inter(src, rr, q).records
                want = oracle_decide(oracle, w, h, src, rr, q)
                assert_same(got, want, f"{name} q{q} {'key' if key else 'inter'}")


@pytest.mark.parametrize("w,h", [(202, 122), (640, 360), (16, 16)])
def test_fields_match_oracle(oracle, w, h):
    cur, prev = F.scene_frame(w, h, 5, 3), F.scene_frame(w, h)
    want = oracle.me_fields(cur, prev)
    with CudaEngine(w, h) as e:
        e.decide_inter(cur, [prev], 120)
        for l in range(5):
            gx, gy = unpack_field(e.debug_field(0, l))
            assert np.array_equal(gx, want[l][0]) and np.array_equal(gy, want[l][1]), f"level {l}"


def test_intra_matches_oracle(oracle):
    w, h = 202, 122
    src = F.test_frame(w, h)
    with CudaEngine(w, h) as e:
        e.decide_intra(src, 120)
        got = e.debug_intra()
    for sb in range(got.shape[0]):
        want = oracle.intra_satd_sb(src, sb % 4, sb // 4)
        assert np.array_equal(got[sb][5:], want[5:]), f"superblock {sb}"


def test_synthetic_416x240_3refs(oracle):
    clip = synth.small_clip(seed=7)
    w, h = 416, 240
    with CudaEngine(w, h) as e:
        for i in range(3, 8):
            refs = [clip[i - k].y for k in range(1, 4)]
            got = e.decide_inter(clip[i].y, refs, 120).records
            assert_same(got, oracle_decide(oracle, w, h, clip[i].y, refs, 120), f"frame {i}")


def test_launch_copies_inputs(oracle):
    """launch must not read the caller's frames after it returns (test_gpu_intra.cpp:95-114)."""
    for w, h in ((202, 122), (640, 360)):
        src, prev = F.test_frame(w, h), F.scene_frame(w, h)
        want = oracle_decide(oracle, w, h, src, [prev], 120)
        with CudaEngine(w, h) as e:
            s, p = src.copy(), prev.copy()
            dm, gate = DecisionMap(), RowGate()
            e.launch(s, [p], 120, dm)
            s[:] = 0
            p[:] = 255
            e.collect(dm, gate)
            assert_same(dm.records, want)
            assert gate.ready_rows() == dm.sb_rows


def test_ten_bit_ingest(oracle):
    """10-bit planes rounded on the device decide exactly as their 8-bit rounding (y4m.cpp:28-34)."""
    clip = synth.small_clip(seed=3, frames=4)
    w, h = 416, 240
    with CudaEngine(w, h) as e:
        a = e.decide_inter(clip[3].hy, [clip[2].hy, clip[1].hy], 130).records
        b = e.decide_inter(clip[3].y, [clip[2].y, clip[1].y], 130).records
    assert_same(a, b, "10-bit vs 8-bit input")
    assert_same(a, oracle_decide(oracle, w, h, clip[3].y, [clip[2].y, clip[1].y], 130))


def test_seven_refs_key_reuse(oracle):
    """Seven references, then again with one new to the store and six reused (test_gpu_me.cpp:167-194)."""
    w, h = 320, 192
    pics = [F.smooth(w, h, 1.25 * i, -0.75 * i) for i in range(9)]
    with CudaEngine(w, h) as e:
        for first in (1, 2):
            refs = [pics[i] for i in range(first, first + 7)]
            keys = list(range(first, first + 7))
            dm, gate = DecisionMap(), RowGate()
            e.launch(pics[0], refs, 90, dm, keys)
            e.collect(dm, gate)
            assert_same(dm.records, oracle_decide(oracle, w, h, pics[0], refs, 90), f"refs from {first}")


def test_prepare_and_keys_sequence(oracle):
    """engine_bench's protocol (tools/engine_bench.cpp:44-57): refs nearest first by key, next prepared."""
    clip = synth.small_clip(seed=11)
    w, h, nr = 416, 240, 3
    with CudaEngine(w, h) as e:
        for i in range(nr, len(clip)):
            refs = [clip[i - k].y for k in range(1, nr + 1)]
            keys = [i - k for k in range(1, nr + 1)]
            dm, gate = DecisionMap(), RowGate()
            e.launch(clip[i].y, refs, 120, dm, keys, i)
            if i + 1 < len(clip):
                e.prepare(clip[i + 1].y, i + 1)
            e.collect(dm, gate)
            assert_same(dm.records, oracle_decide(oracle, w, h, clip[i].y, refs, 120), f"frame {i}")


def test_row_streams_order_and_gate():
    w, h = 640, 360
    src, prev = F.scene_frame(w, h, 3, -2), F.scene_frame(w, h)
    with CudaEngine(w, h) as e:
        base = e.decide_inter(src, [prev], 120).records
        e.set_row_streams(2)
        dm, gate = DecisionMap(), RowGate()
        e.launch(src, [prev], 120, dm)
        assert e.row_order() == [0, 3, 1, 4, 2, 5]
        seen = []
        e.row_hook = seen.append
        e.collect(dm, gate)
        assert seen == [0, 3, 1, 4, 2, 5]
        assert gate.ready_rows() == 6
        assert_same(dm.records, base)


def test_collect_failure_reaches_gate():
    """A failure during collect fails the gate and is raised (test_cpu_engine.cpp:90-116), host side."""
    w, h = 640, 360
    src, prev = F.scene_frame(w, h, 3, -2), F.scene_frame(w, h)
    with CudaEngine(w, h) as e:
        def hook(row):
            if row == 2:
                raise RuntimeError("hook")
        e.row_hook = hook
        dm, gate = DecisionMap(), RowGate()
        e.launch(src, [prev], 120, dm)
        with pytest.raises(RuntimeError, match="hook"):
            e.collect(dm, gate)
        with pytest.raises(RuntimeError, match="hook"):
            gate.wait_row(5, timeout=5)
        e.row_hook = None
        assert_same(e.decide_inter(src, [prev], 120).records, e.decide_inter(src, [prev], 120).records)


def test_errors_match_reference_contract():
    with pytest.raises(RuntimeError):
        CudaEngine(0, 0)
    with pytest.raises(RuntimeError):
        CudaEngine(64, 64, sb_size=128)
    with CudaEngine(64, 64) as e:
        src = F.scene_frame(64, 64)
        with pytest.raises(RuntimeError):
            e.decide_inter(src, [src] * 8, 120)
        with pytest.raises(ValueError):
            e.launch(src, [src, src], 120, DecisionMap(), ref_keys=[1])
        with pytest.raises(RuntimeError):
            e.decide_inter(F.scene_frame(32, 32), [], 120)


def test_group_matches_single(oracle):
    clip = synth.small_clip(seed=5)
    w, h = 416, 240
    with CudaEngine(w, h) as e:
        for i, f in enumerate(clip):
            e.upload(f.y, i)
        srcs = [3, 4, 5, 6, 7]
        refs = [[i - 1, i - 2, i - 3] for i in srcs]
        e.launch_group(srcs, refs, 120, to_host=True)
        for j, i in enumerate(srcs):
            got = e.group_records(j)
            want = oracle_decide(oracle, w, h, clip[i].y, [clip[k].y for k in refs[j]], 120)
            assert_same(got, want, f"job {j}")


def test_three_engines_on_threads(oracle):
    """Several engines on one GPU from different threads (test_gpu_me.cpp:201-257)."""
    w, h = 320, 192
    pics = [F.smooth(w, h, 1.25 * i, -0.75 * i) for i in range(9)]
    refs = pics[1:8]
    want = [oracle_decide(oracle, w, h, pics[0], refs, 90), oracle_decide(oracle, w, h, pics[8], refs, 90)]
    assert not records_equal(want[0], want[1])
    bad, errors = [], []

    def run(t):
        try:
            with CudaEngine(w, h) as e:
                for i in range(6):
                    s = (i + t) % 2
                    got = e.decide_inter(pics[8 if s else 0], refs, 90, ref_keys=list(range(1, 8))).records
                    if not records_equal(got, want[s]):
                        bad.append((t, i))
        except Exception as ex:  # reported below
            errors.append(repr(ex))

    ts = [threading.Thread(target=run, args=(t,)) for t in range(3)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert not errors and not bad, (errors, bad)


def test_full_size_1080p_seven_refs(oracle):
    """The bench's workload at full size: a 1080p 10-bit leaf frame against its 7 references
    (the mini-GOP's reference lists), byte-identical records; the oracle runs on every host core."""
    from bench import mini_gop_plan

    clip = synth.hd_clip(seed=1, frames=17)
    w, h = 1920, 1080
    src, refs = mini_gop_plan()[-1][0]
    with CudaEngine(w, h) as e:
        got = e.decide_inter(clip[src].hy, [clip[r].hy for r in refs], 130).records
    want = oracle.decide(w, h, clip[src].y, [clip[r].y for r in refs], lam.lambda_q8(130))
    assert_same(got, want, "1080p leaf, 7 references")


def test_batched_leaves_match_single_launches():
    """A mini-GOP's leaves decided as one batch equal the same frames decided one at a time."""
    from bench import mini_gop_plan

    clip = synth.sinusoid_clip(640, 360, 17, 4, sinusoids=8, rects=12, affine_regions=(4, 3), noise_sigma=4.0)
    leaves = mini_gop_plan()[-1]
    with CudaEngine(640, 360) as e:
        for i, f in enumerate(clip):
            e.upload(f.hy, i)
        e.launch_group([s for s, _ in leaves], [r for _, r in leaves], 130, to_host=True)
        batched = [e.group_records(j) for j in range(len(leaves))]
        for j, (s, refs) in enumerate(leaves):
            single = e.decide_inter(clip[s].y, [clip[r].y for r in refs], 130).records
            assert_same(batched[j], single, f"leaf {s}")


def leaves_of(rec, sb_cols, sb_rows):
    out = []
    for sr in range(sb_rows):
        for sc in range(sb_cols):
            r = rec[sr * sb_cols + sc]
            tree = list(r["tree"][: int(r["ntree"])])
            pos, blocks = [0], []

            def walk(x, y, bw, bh):
                p = tree[pos[0]]
                pos[0] += 1
                if p == 0:
                    blocks.append((x, y, bw, bh))
                elif p == 1:
                    walk(x, y, bw, bh // 2), walk(x, y + bh // 2, bw, bh // 2)
                elif p == 2:
                    walk(x, y, bw // 2, bh), walk(x + bw // 2, y, bw // 2, bh)
                else:
                    for q in range(4):
                        walk(x + (q & 1) * bw // 2, y + (q >> 1) * bh // 2, bw // 2, bh // 2)

            walk(sc * 64, sr * 64, 64, 64)
            out += [(*b, r, k) for k, b in enumerate(blocks)]
    return out


def test_cuda_finds_integer_and_quarter_pel_motion():
    """Known answers of tests/test_gpu_me.cpp:71-163 on the CUDA engine: (5, -3) px on >= 90% of
    the interior, (2.5, -1.25) px on >= 75% of the inter area."""
    w, h = 640, 360
    with CudaEngine(w, h) as e:
        rec = e.decide_inter(F.textured(w, h, 5, -3), [F.textured(w, h, 0, 0)], 120).records
    interior = hit = 0
    for x, y, bw, bh, r, k in leaves_of(rec, 10, 6):
        if x < 16 or y < 16 or x + bw > w - 16 or y + bh > h - 16:
            continue
        interior += bw * bh
        hit += bw * bh if (r["mode"][k] == 13 and r["mvx"][k] == 20 and r["mvy"][k] == -12) else 0
    assert interior > 0 and hit * 10 >= interior * 9
    w, h = 320, 192
    with CudaEngine(w, h) as e:
        rec = e.decide_inter(F.smooth(w, h, 2.5, -1.25), [F.smooth(w, h, 0, 0)], 60).records
    inter = hit = 0
    for r in rec:
        for k in range(int(r["nblocks"])):
            if r["mode"][k] == 13:
                a = int(r["w4"][k]) * int(r["h4"][k])
                inter += a
                hit += a if (r["mvx"][k], r["mvy"][k]) == (10, -5) else 0
    assert inter > 0 and hit * 4 >= inter * 3


def test_cuda_finds_large_motion():
    """tests/test_gpu_me.cpp:293-308 on the CUDA engine's level-0 field: (96, 24) px."""
    with CudaEngine(640, 360) as e:
        e.decide_inter(F.scene_frame(640, 360, 96, 24), [F.scene_frame(640, 360, 0, 0)], 120)
        fx, fy = unpack_field(e.debug_field(0, 0))
    sub = (fx[4:, 13:] == -96 * 4) & (fy[4:, 13:] == -24 * 4)
    assert sub.sum() * 4 >= sub.size * 3
