"""The coding order of a mini-GOP, as the reference encoder lays it out.

src/chunk_coder.cpp:213-225,340-430: the KEY frame, the hidden anchor (the last frame), the pyramid
mids (each a reference for what follows), then the non-reference leaves, which depend on none of
each other. Each frame's references are the reference frames coded before it, nearest display
distance first, at most `refs`. Longer streams (stream_plan) chain mini-GOPs: each one's anchor is
16 frames on, and the reference frames kept are the last refs + 1 coded ones (a buffer of that
many slots refreshed in coding order); a scene cut starts a new chunk with a KEY frame and an empty
buffer, as the reference's scene chunks do. The reference lists are a harness choice: any list
given to two engines must give both the same decisions.
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


def stream_plan(nframes: int, gop: int = 16, refs: int = 7, cuts=()):
    """[(group of (src, [refs nearest first]))] in coding order for a stream of nframes frames:
    per scene chunk (a KEY frame at 0 and at every cut) mini-GOPs of `gop` frames (the last one
    shorter), each its anchor, its mids, then its leaves as one group. Frame numbers are display
    order."""
    starts = sorted({0, *[c for c in cuts if 0 < c < nframes]})
    groups = []
    for ci, first in enumerate(starts):
        end = starts[ci + 1] if ci + 1 < len(starts) else nframes
        kept = [first]  # reference frames in the buffer, oldest first
        groups.append([(first, [])])

        def refs_of(d):
            return sorted(kept, key=lambda r: (abs(r - d), r))[:refs]

        def keep(d):
            kept.append(d)
            del kept[: max(0, len(kept) - (refs + 1))]

        lo = first
        while lo + 1 < end:
            m = min(gop, end - 1 - lo)
            mids = [lo + 1 + p for p in mids_of(m, refs)]
            anchor = lo + m
            for d in [anchor] + mids:
                groups.append([(d, refs_of(d))])
                keep(d)
            leaves = [d for d in range(lo + 1, anchor) if d not in mids]
            if leaves:
                groups.append([(d, refs_of(d)) for d in leaves])
            lo = anchor
    return groups


def assign_streams(sizes, frames, world: int):
    """Whole streams to GPUs (ranks) for several concurrent streams: stream i (width, height) with
    frames[i] frames goes to one rank, largest first onto the least loaded rank (work = superblocks
    x frames; ties to the lower rank). Streams are independent, so no data crosses between GPUs.
    Returns each rank's stream indices (ascending). Every rank computes the same assignment."""
    work = [((w + 63) // 64) * ((h + 63) // 64) * f for (w, h), f in zip(sizes, frames)]
    load = [0] * world
    out = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda i: (-work[i], i)):
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += work[i]
        out[r].append(i)
    return [sorted(o) for o in out]
