"""Generates tests/golden/golden.json from the REFERENCE's own code (oracle/_ref, compiled from the
reference sources by oracle/Makefile): SHA-256 digests of the decision records, pyramids and
motion fields the reference produces on seeded inputs, plus one full small record set.

The reference has no golden vectors of its own; these pin the oracle restatement (and through it
the CUDA engine) to the reference run here. Run from the repository root:
    make -C oracle && python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import frames as F  # noqa: E402
from celv2_b200 import lam, synth  # noqa: E402


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def cases():
    """(name, width, height, src plane, [ref planes], qindex) -- small enough for the CPU suite."""
    out = []
    for w, h in ((202, 122), (64, 64), (32, 32), (16, 16), (72, 40)):
        out.append((f"scene-{w}x{h}-inter", w, h, F.scene_frame(w, h, 3, -2), [F.scene_frame(w, h)], 120))
        out.append((f"scene-{w}x{h}-key", w, h, F.scene_frame(w, h, 3, -2), [], 120))
    w, h = 202, 122
    out.append(("multi3", w, h, F.scene_frame(w, h, 6, -3),
                [F.scene_frame(w, h, 40, 30, 5), F.scene_frame(w, h, 6, -3), F.scene_frame(w, h, 3, -1)], 120))
    for q in (40, 220):
        out.append((f"testframe-q{q}-key", 200, 120, F.test_frame(200, 120), [], q))
    out.append(("smooth7", 160, 96, F.smooth(160, 96, 0, 0), [F.smooth(160, 96, 1.25 * i, -0.75 * i) for i in range(1, 8)],
                90))
    out.append(("textured", 200, 120, F.textured(200, 120, 5, -3), [F.textured(200, 120, 0, 0)], 120))
    out.append(("glyph", 200, 120, F.glyph_frame(200, 120, 3), [F.glyph_frame(200, 120, 0)], 120))
    out.append(("noise7", 130, 90, F.noise(130, 90, 1), [F.noise(130, 90, k + 2) for k in range(7)], 160))
    clip = synth.small_clip(seed=1, frames=4)
    out.append(("synth416-3refs", 416, 240, clip[3].y, [clip[2].y, clip[1].y, clip[0].y], 120))
    return out


def main():
    from oracle import Reference, reference_available

    if not reference_available():
        sys.exit("oracle/_ref/libcelv2ref.so is missing: build it with make -C oracle where the reference is")
    ref = Reference(lam.table())
    gold = {"lambda_table_sha256": sha(np.array(lam.table(), np.int64)), "decide": {}, "pyramid": {}, "fields": {},
            "round_to_8bit": {}}
    for name, w, h, src, refs, q in cases():
        rec = ref.decide_ref(w, h, src, refs, q)
        gold["decide"][name] = {"w": w, "h": h, "q": q, "nrefs": len(refs), "sha256": sha(rec)}
    for w, h in ((202, 122), (16, 16), (416, 240)):
        cur, prev = F.scene_frame(w, h, 5, 3), F.scene_frame(w, h)
        gold["pyramid"][f"{w}x{h}"] = {"cur": sha(ref.pyramid(w, h, cur, False)), "ref": sha(ref.pyramid(w, h, prev, True))}
        fields = ref.me_fields(w, h, cur, prev)
        gold["fields"][f"{w}x{h}"] = [sha(np.stack([fx, fy])) for fx, fy in fields]
    hy = synth.small_clip(seed=2, frames=1)[0].hy
    y = np.zeros(hy.shape, np.uint8)
    import ctypes as C

    ref.lib.refx_round_to_8bit(416, 240, hy.ctypes.data_as(C.POINTER(C.c_uint16)), y.ctypes.data_as(C.POINTER(C.c_uint8)))
    gold["round_to_8bit"]["synth416"] = {"input_sha256": sha(hy), "sha256": sha(y)}
    # one full record set for a 32x32 inter frame (readable when a digest test fails)
    src, prev = F.scene_frame(32, 32, 1, 1), F.scene_frame(32, 32)
    np.save(os.path.join(HERE, "scene32_inter_q120.npy"), ref.decide_ref(32, 32, src, [prev], 120))
    with open(os.path.join(HERE, "golden.json"), "w") as fh:
        json.dump(gold, fh, indent=1, sort_keys=True)
    print(f"wrote {len(gold['decide'])} decision digests")


if __name__ == "__main__":
    main()
