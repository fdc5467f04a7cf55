"""The oracle (C restatement of the reference rules) pinned to the reference: against the golden
digests the reference produced (tests/golden), against the reference compiled here when it is,
and on the reference's known-answer tests (tests/test_gpu_me.cpp, tests/test_gpu_intra.cpp)."""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

import frames as F
from celv2_b200 import lam, synth

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import make_golden  # noqa: E402

GOLD = json.load(open(os.path.join(HERE, "golden", "golden.json")))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_lambda_table_is_the_golden_one():
    assert sha(np.array(lam.table(), np.int64)) == GOLD["lambda_table_sha256"]


@pytest.mark.parametrize("case", make_golden.cases(), ids=[c[0] for c in make_golden.cases()])
def test_oracle_matches_reference_digests(oracle, case):
    name, w, h, src, refs, q = case
    got = oracle.decide(w, h, src, refs, lam.lambda_q8(q))
    assert sha(got) == GOLD["decide"][name]["sha256"], name


def test_oracle_matches_full_golden_records(oracle):
    want = np.load(os.path.join(HERE, "golden", "scene32_inter_q120.npy"))
    got = oracle.decide(32, 32, F.scene_frame(32, 32, 1, 1), [F.scene_frame(32, 32)], lam.lambda_q8(120))
    assert got.tobytes() == want.tobytes()


@pytest.mark.parametrize("wh", [(202, 122), (16, 16), (416, 240)])
def test_oracle_pyramid_and_fields_match_reference_digests(oracle, wh):
    w, h = wh
    cur, prev = F.scene_frame(w, h, 5, 3), F.scene_frame(w, h)
    g = GOLD["pyramid"][f"{w}x{h}"]
    assert sha(oracle.pyramid(cur, False)) == g["cur"]
    assert sha(oracle.pyramid(prev, True)) == g["ref"]
    fields = oracle.me_fields(cur, prev)
    assert [sha(np.stack([fx, fy])) for fx, fy in fields] == GOLD["fields"][f"{w}x{h}"]


def test_round_to_8bit_matches_reference_digest(oracle):
    hy = synth.small_clip(seed=2, frames=1)[0].hy
    g = GOLD["round_to_8bit"]["synth416"]
    assert sha(hy) == g["input_sha256"]
    assert sha(oracle.round_to_8bit(hy)) == g["sha256"]
    assert sha(synth.round_to_8bit(hy)) == g["sha256"]


def test_oracle_matches_reference_engine_live(oracle, reference):
    """Where the reference compiled here: its threaded CpuEngine on a synthetic clip."""
    clip = synth.small_clip(seed=9, frames=6)
    eng = reference.engine(416, 240, 4)
    for i in (3, 5):
        refs = [clip[i - k].y for k in range(1, 4)]
        a = eng.decide(clip[i].y, refs, 130)
        b = oracle.decide(416, 240, clip[i].y, refs, lam.lambda_q8(130))
        assert a.tobytes() == b.tobytes()
    eng.close()


def test_me_cell_searches_two_centres(oracle):
    """tests/test_gpu_me.cpp:312-332: the second centre (the coarser level's 26, 0) is searched
    and finds the exact match at (20, 0) past a dead-end first centre."""
    import ctypes as C

    w, h, bx, by = 128, 64, 4, 2
    v = 7
    cur = np.zeros(w * h, np.uint8)
    ref = np.zeros(w * h, np.uint8)

    def rnd():
        nonlocal v
        v = (v * 1664525 + 1013904223) & 0xFFFFFFFF
        return v >> 24

    for i in range(w * h):
        cur[i] = rnd()
    for i in range(w * h):
        ref[i] = rnd()
    for y in range(by * 8, by * 8 + 8):
        for x in range(bx * 8, bx * 8 + 8):
            ref[y * w + x + 20] = cur[y * w + x]
            ref[y * w + x] = (int(cur[y * w + x]) + 3) & 255
    pcols, prows = w // 16, h // 16
    pmx = np.full(pcols * prows, 13, np.int32)
    pmy = np.zeros(pcols * prows, np.int32)
    mx, my = C.c_int32(), C.c_int32()
    P = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint8))  # noqa: E731
    Q = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))  # noqa: E731
    oracle.lib.oro_me_cell(P(cur), P(ref), w, w, h, bx, by, Q(pmx), Q(pmy), pcols, prows, 0, C.byref(mx), C.byref(my))
    assert (mx.value, my.value) == (20, 0)


def leaves_of(rec, sb_cols, sb_rows):
    """(x, y, w, h, block) of every leaf from the preorder tree (tests/test_gpu_me.cpp:85-98)."""
    out = []
    for sr in range(sb_rows):
        for sc in range(sb_cols):
            r = rec[sr * sb_cols + sc]
            tree = list(r["tree"][: int(r["ntree"])])
            pos = [0]
            blocks = []

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
            for k, b in enumerate(blocks):
                out.append((*b, r, k))
    return out


def test_integer_motion_found(oracle):
    """tests/test_gpu_me.cpp:71-112: content moved (5, -3) px; >= 90% of the interior area takes
    that MV."""
    w, h = 640, 360
    rec = oracle.decide(w, h, F.textured(w, h, 5, -3), [F.textured(w, h, 0, 0)], lam.lambda_q8(120))
    interior = hit = 0
    for x, y, bw, bh, r, k in leaves_of(rec, 10, 6):
        if x < 16 or y < 16 or x + bw > w - 16 or y + bh > h - 16:
            continue
        interior += bw * bh
        if r["mode"][k] == 13 and r["mvx"][k] * 2 == 40 and r["mvy"][k] * 2 == -24:
            hit += bw * bh
    assert interior > 0 and hit * 10 >= interior * 9


def test_quarter_pel_motion_found(oracle):
    """tests/test_gpu_me.cpp:141-163: a (2.5, -1.25) px shift is found at quarter pel on >= 75%
    of the inter area."""
    w, h = 320, 192
    rec = oracle.decide(w, h, F.smooth(w, h, 2.5, -1.25), [F.smooth(w, h, 0, 0)], lam.lambda_q8(60))
    inter = hit = 0
    for r in rec:
        for k in range(int(r["nblocks"])):
            if r["mode"][k] == 13:
                a = int(r["w4"][k]) * int(r["h4"][k])
                inter += a
                hit += a if (r["mvx"][k] * 2, r["mvy"][k] * 2) == (20, -10) else 0
    assert inter > 0 and hit * 4 >= inter * 3


def test_large_motion_found(oracle):
    """tests/test_gpu_me.cpp:293-308: (96, 24) px, beyond a 3-level pyramid, is found by >= 75% of
    the level-0 cells where the earlier frame has the content."""
    fields = oracle.me_fields(F.scene_frame(640, 360, 96, 24), F.scene_frame(640, 360, 0, 0))
    fx, fy = fields[0]
    sub = (fx[4:, 13:] == -96 * 4) & (fy[4:, 13:] == -24 * 4)
    assert sub.sum() * 4 >= sub.size * 3


def test_no_intra_block_wider_than_32(oracle):
    """tests/test_gpu_intra.cpp:248-262."""
    for w, h in ((640, 360), (202, 122)):
        flat = np.full(((h + 7) & ~7, (w + 7) & ~7), 128, np.uint8)
        for refs in ([], [flat]):
            rec = oracle.decide(w, h, flat, refs, lam.lambda_q8(120))
            for r in rec:
                for k in range(int(r["nblocks"])):
                    lim = 16 if r["mode"][k] == 13 else 8
                    assert r["w4"][k] <= lim and r["h4"][k] <= lim


def test_block_geometry(oracle):
    """sb_blocks.h: 85 squares x 5 kinds, each inside the 64x64 superblock."""
    seen = set()
    for b in range(425):
        x, y, w, h = oracle.block_geom(b)
        assert 0 <= x and x + w <= 64 and 0 <= y and y + h <= 64
        seen.add((x, y, w, h))
    assert len(seen) == 425


def test_hadamard_known_values(oracle):
    assert oracle.hadamard4x4([0] * 16) == 0
    assert oracle.hadamard4x4([1] * 16) == 16
    assert oracle.hadamard4x4([255] * 16) == 16 * 255
    d = [(-1) ** (i + j) * 255 for i in range(4) for j in range(4)]
    assert oracle.hadamard4x4(d) == 16 * 255
