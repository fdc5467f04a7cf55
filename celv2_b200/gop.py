"""The coding order of a mini-GOP, as the reference encoder lays it out.

src/chunk_coder.cpp:213-225,340-430: the KEY frame, the hidden anchor (the last frame), the pyramid
mids (each a reference for what follows), then the non-reference leaves, which depend on none of
each other. Each frame's references are the reference frames coded before it, nearest display
distance first, at most `refs`.
"""
from __future__ import annotations


def mids_of(m: int, refs: int):
    """The pyramid mids of an m-frame mini-GOP (src/chunk_coder.cpp:213-225): positions, coded order."""
    mids = []

    def split(lo, hi, level):
        if hi - lo - 1 < 3 or refs < 3 or len(mids) + 2 >= refs:
            return
        mid = (lo + hi) // 2
        mids.append(mid)
        split(lo, mid, level + 1)
        split(mid, hi, level + 1)

    split(-1, m - 1, 1)
    return mids


def mini_gop_plan(nframes: int = 17, refs: int = 7):
    """[(group of (src, [refs nearest first]))] in coding order: KEY, anchor, mids, then the leaves
    as one group. Frame numbers are display order; frame 0 is the KEY frame."""
    m = nframes - 1
    mids = [1 + p for p in mids_of(m, refs)]
    anchor = m
    leaves = [d for d in range(1, m) if d not in mids]
    coded_refs = [0]
    groups = [[(0, [])]]

    def refs_of(d):
        order = sorted(coded_refs, key=lambda r: (abs(r - d), r))
        return order[:refs]

    for d in [anchor] + mids:
        groups.append([(d, refs_of(d))])
        coded_refs.append(d)
    groups.append([(d, refs_of(d)) for d in leaves])
    return groups
