"""The decision record (include/celv2_decision.h) as a numpy dtype, and its DecisionMap view.

``SB_OUT_DTYPE`` is byte-for-byte the C struct ``celv2_sb_out`` (the reference's ``SbOut``,
src/gpu/sb_out.h:13-31). ``to_decision`` restates the reference's ``sb_out_to_decision``
(src/gpu/decision_map.cpp:65-105): MVs doubled from quarter pels to 1/8 pel, mode 13 = inter.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

SB_OUT_BYTES = 38872
NUM_MODES = 13
SINGLE_REF = 255
SB_BLOCKS = 425

SB_OUT_DTYPE = np.dtype(
    [
        ("ntree", "<i4"), ("nblocks", "<i4"),
        ("tree", "u1", 256), ("w4", "u1", 256), ("h4", "u1", 256), ("mode", "u1", 256),
        ("mvx", "<i2", 256), ("mvy", "<i2", 256),
        ("ref", "u1", 256), ("ref2", "u1", 256),
        ("mv2x", "<i2", 256), ("mv2y", "<i2", 256),
        ("c_inter_cost", "<i8", 425), ("c_intra_cost", "<i8", 425),
        ("c_mvx", "<i2", 425), ("c_mvy", "<i2", 425), ("c_mv2x", "<i2", 425), ("c_mv2y", "<i2", 425),
        ("c_ref", "u1", 425), ("c_ref2", "u1", 425), ("c_intra", "u1", 425),
        ("_pad", "u1", 1),
        ("c_rcost", "<u4", (7, 425)),
        ("c_rmvx", "<i2", (7, 425)), ("c_rmvy", "<i2", (7, 425)),
        ("_tail", "u1", 4),
    ]
)
assert SB_OUT_DTYPE.itemsize == SB_OUT_BYTES


@dataclass
class BlockDecision:
    """The reference's BlockDecision (src/gpu/decision_map.h:22-36)."""

    w4: int = 0
    h4: int = 0
    inter: bool = False
    intra: int = 0
    mv_row: int = 0
    mv_col: int = 0
    ref: int = 0
    ref2: int = SINGLE_REF
    mv2_row: int = 0
    mv2_col: int = 0


@dataclass
class BlockCandidates:
    """The reference's BlockCandidates (src/gpu/decision_map.h:41-50)."""

    inter_cost: int
    intra_cost: int
    inter: BlockDecision
    intra: int
    ref_cost: list
    ref_mv_col: list
    ref_mv_row: list


@dataclass
class SbDecision:
    tree: list = field(default_factory=list)
    blocks: list = field(default_factory=list)
    cands: list = field(default_factory=list)


@dataclass
class DecisionMap:
    """One frame's decisions: ``records`` (raster order) and, on demand, their SbDecision view."""

    sb_size: int = 0
    sb_cols: int = 0
    sb_rows: int = 0
    records: np.ndarray | None = None

    def sbs(self) -> list:
        return [to_decision(r) for r in self.records]


def _geom(b: int):
    sq, kind = divmod(b, 5)
    level = 3 if sq >= 21 else 2 if sq >= 5 else 1 if sq >= 1 else 0
    idx = sq - ((1 << (2 * level)) - 1) // 3
    n, size = 1 << level, 64 >> level
    sx, sy, half = (idx % n) * size, (idx // n) * size, size // 2
    x, y, w, h = sx, sy, size, size
    if kind in (1, 2):
        h, y = half, sy + (half if kind == 2 else 0)
    if kind in (3, 4):
        w, x = half, sx + (half if kind == 4 else 0)
    return x, y, w, h


def to_decision(o) -> SbDecision:
    """sb_out_to_decision (src/gpu/decision_map.cpp:65-105)."""
    d = SbDecision()
    d.tree = [int(v) for v in o["tree"][: int(o["ntree"])]]
    for k in range(int(o["nblocks"])):
        inter = int(o["mode"][k]) == NUM_MODES
        b = BlockDecision(int(o["w4"][k]), int(o["h4"][k]), inter, 0 if inter else int(o["mode"][k]),
                          int(o["mvy"][k]) * 2, int(o["mvx"][k]) * 2, int(o["ref"][k]))
        if inter and int(o["ref2"][k]) != SINGLE_REF:
            b.ref2, b.mv2_col, b.mv2_row = int(o["ref2"][k]), int(o["mv2x"][k]) * 2, int(o["mv2y"][k]) * 2
        d.blocks.append(b)
    for k in range(SB_BLOCKS):
        x, y, w, h = _geom(k)
        inter = BlockDecision(w // 4, h // 4, True, 0, int(o["c_mvy"][k]) * 2, int(o["c_mvx"][k]) * 2,
                              int(o["c_ref"][k]))
        if int(o["c_ref2"][k]) != SINGLE_REF:
            inter.ref2, inter.mv2_col, inter.mv2_row = (int(o["c_ref2"][k]), int(o["c_mv2x"][k]) * 2,
                                                        int(o["c_mv2y"][k]) * 2)
        d.cands.append(BlockCandidates(int(o["c_inter_cost"][k]), int(o["c_intra_cost"][k]), inter,
                                       int(o["c_intra"][k]), [int(v) for v in o["c_rcost"][:, k]],
                                       [int(v) * 2 for v in o["c_rmvx"][:, k]],
                                       [int(v) * 2 for v in o["c_rmvy"][:, k]]))
    return d


def records_equal(a: np.ndarray, b: np.ndarray) -> bool:
    return a.shape == b.shape and a.tobytes() == b.tobytes()


def first_difference(a: np.ndarray, b: np.ndarray):
    """(superblock, field, index, a value, b value) of the first difference, or None."""
    if a.shape != b.shape:
        return ("shape", a.shape, b.shape)
    for i in range(a.shape[0]):
        if a[i].tobytes() == b[i].tobytes():
            continue
        for name in SB_OUT_DTYPE.names:
            x, y = np.asarray(a[i][name]), np.asarray(b[i][name])
            if not np.array_equal(x, y):
                idx = tuple(int(v) for v in np.argwhere(x != y)[0])
                return (i, name, idx, x[idx].item(), y[idx].item())
        return (i, "padding", None)
    return None
