"""The pruned search on the GPU against the oracle with the same masks: records and per-superblock
costs byte for byte (the kept options are scored exactly; the level-0 motion search skips only
cells no kept reference reads; with the 64- or 32-level blocks pruned the inter stage scores
32x32 or 16x16 regions on their own MVs; the intra stage skips pruned levels and modes)."""
import numpy as np
import pytest

import frames as F
from celv2_b200 import lam, synth
from celv2_b200 import engine as E
from celv2_b200.records import first_difference, records_equal

pytestmark = pytest.mark.gpu


def masks(nsb, seed, nrefs):
    rng = np.random.default_rng(seed)
    k = rng.integers(0, 1 << nrefs, nsb) | (rng.integers(0, 2, nsb) << 7)
    return k.astype(np.uint8)


def words(nsb, seed, nrefs):
    """Keep words: random references and intra, block levels (a third with no 64-level blocks, a
    third with neither 64- nor 32-level ones, the rest random) and intra modes."""
    rng = np.random.default_rng(seed)
    k = rng.integers(0, 1 << nrefs, nsb) | (rng.integers(0, 2, nsb) << 7)
    kind = rng.integers(0, 3, nsb)
    levels = np.where(kind == 0, rng.integers(0, 8, nsb) << 1, np.where(kind == 1, rng.integers(1, 4, nsb) << 2,
                                                                         rng.integers(0, 16, nsb)))
    modes = np.where(rng.random(nsb) < 0.5, rng.integers(0, 1 << 13, nsb), 0)
    return (k | levels << 8 | modes << 16).astype(np.uint32)


@pytest.mark.parametrize("w,h,nrefs", [(202, 122, 3), (640, 360, 7), (72, 40, 2)])
def test_masked_launch_matches_oracle(oracle, w, h, nrefs):
    src = F.textured(w, h, 5, -3)
    refs = [F.textured(w, h, i, -(i // 2)) for i in range(nrefs)]
    with E.CudaEngine(w, h) as e:
        nsb = e.sb_cols * e.sb_rows
        for seed in range(6):
            keep = masks(nsb, seed, nrefs) if seed < 2 else words(nsb, seed, nrefs)
            want, want_cost = oracle.decide_masked(w, h, src, refs, lam.lambda_q8(120), keep)
            e.set_keep(0, keep)
            got = e.decide_inter(src, refs, 120)
            assert records_equal(got.records, want), f"seed {seed}: {first_difference(got.records, want)}"
            assert (e.sb_costs() == want_cost).all()
        # no masks: the exhaustive search, and its costs
        want, want_cost = oracle.decide_masked(w, h, src, refs, lam.lambda_q8(120))
        got = e.decide_inter(src, refs, 120)
        assert records_equal(got.records, want)
        assert (e.sb_costs() == want_cost).all()


def test_masked_group_matches_oracle(oracle):
    w, h = 416, 240
    clip = synth.small_clip(seed=13, frames=6)
    jobs = [(5, [4, 3, 2, 1]), (4, [3, 2]), (3, []), (2, [1, 0])]
    with E.CudaEngine(w, h) as e:
        for i, f in enumerate(clip):
            e.upload(f.hy, i)
        nsb = e.sb_cols * e.sb_rows
        keeps = [words(nsb, 10 + j, max(1, len(refs))) for j, (_, refs) in enumerate(jobs)]
        for j, k in enumerate(keeps):
            e.set_keep(j, k)
        e.launch_group([s for s, _ in jobs], [r for _, r in jobs], 130, to_host=True)
        for j, (s, refs) in enumerate(jobs):
            want, want_cost = oracle.decide_masked(w, h, clip[s].y, [clip[r].y for r in refs], lam.lambda_q8(130),
                                                   keeps[j])
            got = e.group_records(j)
            assert records_equal(got, want), f"job {j}: {first_difference(got, want)}"
            assert (e.sb_costs(j) == want_cost).all()


@pytest.mark.parametrize("graphs", [0, 1])
def test_region_scoring_at_1080p(oracle, graphs):
    """A 1080p frame against 4 references with the used options of its exhaustive decision (no loss:
    the same chosen costs) and with the large levels pruned everywhere: the 16x16- and 32x32-region
    inter paths over a whole frame, through a group launch."""
    from celv2_b200.pruner.data import used_options

    clip = synth.hd_clip(seed=77, frames=5)
    w, h = 1920, 1080
    refs = [3, 2, 1, 0]
    with E.CudaEngine(w, h) as e:
        e.set_config(E.CFG_GRAPHS, graphs)
        for i, f in enumerate(clip):
            e.upload(f.hy, i)
        nsb = e.sb_cols * e.sb_rows
        e.launch_group([4], [refs], 130, to_host=True)
        full_rec, full_cost = e.group_records(0), e.sb_costs(0)
        used = used_options(full_rec, len(refs))
        small = np.full(nsb, 0x8F | 0xC00, np.uint32)  # 16- and 8-sample levels only
        mid = np.full(nsb, 0x0F | 0xE00, np.uint32)    # no 64-level blocks, no intra
        for keep in (used, small, mid):
            e.set_keep(0, keep)
            e.launch_group([4], [refs], 130, to_host=True)
            got, cost = e.group_records(0), e.sb_costs(0)
            want, want_cost = oracle.decide_masked(w, h, clip[4].y, [clip[r].y for r in refs], lam.lambda_q8(130), keep)
            assert records_equal(got, want), first_difference(got, want)
            assert (cost == want_cost).all()
        e.set_keep(0, used)
        e.launch_group([4], [refs], 130, to_host=True)
        # the used options lose nothing (a block of the chosen partition keeps its choice; a pruned
        # reference can only change which second reference a compound tries, never raise a cost)
        assert (e.sb_costs(0) <= full_cost).all()


def test_masked_replay_after_an_exhaustive_capture(oracle):
    """With CUDA graphs, a batch of one shape first decided exhaustively (its graph captured with no
    keep words, so without the region pass of the inter stage) and then, on another frame, with
    keep words that prune the 64-level blocks: the masked batch must not replay the exhaustive
    graph, whose inter stage would leave the region units unscored."""
    w, h = 416, 240
    clip = synth.small_clip(seed=21, frames=6)
    with E.CudaEngine(w, h) as e:
        e.set_config(E.CFG_GRAPHS, 1)
        for i, f in enumerate(clip):
            e.upload(f.hy, i)
        nsb = e.sb_cols * e.sb_rows
        for _ in range(2):  # captured, then replayed
            e.launch_group([5], [[4, 3, 2, 1]], 130, to_host=True)
        want, _ = oracle.decide_masked(w, h, clip[5].y, [clip[r].y for r in (4, 3, 2, 1)], lam.lambda_q8(130))
        assert records_equal(e.group_records(0), want)
        keep = np.full(nsb, 0x0F | 0x80 | 0xE00, np.uint32)  # every reference and intra, no 64-level blocks
        for _ in range(2):
            e.set_keep(0, keep)
            e.launch_group([4], [[3, 2, 1, 0]], 130, to_host=True)
            want, want_cost = oracle.decide_masked(w, h, clip[4].y, [clip[r].y for r in (3, 2, 1, 0)],
                                                   lam.lambda_q8(130), keep)
            got = e.group_records(0)
            assert records_equal(got, want), first_difference(got, want)
            assert (e.sb_costs(0) == want_cost).all()
