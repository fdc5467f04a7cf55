"""The pruned search's semantics on the oracle (CPU): masks that keep everything change nothing,
a pruned option is never chosen, and keeping the options the exhaustive partition uses never raises
a superblock's cost. (Pruning is not monotone in general: the exhaustive search tries a block's
compound only with its second-best reference, so pruning another reference can make a compound
with a different second reference available, which may be cheaper.)"""
import numpy as np

import frames as F
from celv2_b200 import lam
from celv2_b200.records import records_equal

NO_REF_COST = 0xFFFFFFFF


def case(w=202, h=122, nrefs=3):
    src = F.scene_frame(w, h, 6, -3)
    refs = [F.scene_frame(w, h, 40, 30, 5), F.scene_frame(w, h, 6, -3), F.scene_frame(w, h, 3, -1)][:nrefs]
    return w, h, src, refs


def test_full_masks_change_nothing(oracle):
    w, h, src, refs = case()
    want = oracle.decide(w, h, src, refs, lam.lambda_q8(120))
    nsb = want.size
    for keep in (None, np.full(nsb, 0xFF, np.uint8), np.full(nsb, 0x80, np.uint8)):  # 0x80: no ref named = all
        got, cost = oracle.decide_masked(w, h, src, refs, lam.lambda_q8(120), keep)
        assert records_equal(got, want)
        assert (cost > 0).all()


def test_pruned_options_are_never_chosen(oracle):
    w, h, src, refs = case()
    rng = np.random.default_rng(3)
    nsb = ((w + 63) // 64) * ((h + 63) // 64)
    keep = rng.integers(0, 256, nsb).astype(np.uint8)
    _, full = oracle.decide_masked(w, h, src, refs, lam.lambda_q8(120))
    got, cost = oracle.decide_masked(w, h, src, refs, lam.lambda_q8(120), keep)
    for i, o in enumerate(got):
        k = int(keep[i])
        refs_kept = (k & 7) or 7
        for b in range(int(o["nblocks"])):
            if int(o["mode"][b]) == 13:  # inter
                assert refs_kept >> int(o["ref"][b]) & 1
                if int(o["ref2"][b]) != 255:
                    assert refs_kept >> int(o["ref2"][b]) & 1
            else:
                assert k & 0x80, "an intra leaf where intra was pruned"
        for r in range(3):
            if not refs_kept >> r & 1:
                assert (o["c_rcost"][r] == NO_REF_COST).all()


def test_key_frames_ignore_masks(oracle):
    w, h, src, _ = case()
    want = oracle.decide(w, h, src, [], lam.lambda_q8(120))
    got, _ = oracle.decide_masked(w, h, src, [], lam.lambda_q8(120), np.zeros(want.size, np.uint8))
    assert records_equal(got, want)


def test_keeping_the_used_options_loses_nothing(oracle):
    """Masks of exactly the options each superblock's chosen partition uses (references, intra
    modes, block levels) never raise a superblock's cost above the exhaustive one."""
    from celv2_b200.pruner.data import used_options

    for w, h, src, refs in (case(), case(416, 240, 3), case(202, 122, 2)):
        q = lam.lambda_q8(120)
        full_rec, full = oracle.decide_masked(w, h, src, refs, q)
        keep = used_options(full_rec, len(refs))
        assert (keep & 0xF00).all() and (keep & 0x7F).all()
        got, cost = oracle.decide_masked(w, h, src, refs, q, keep)
        assert (cost <= full).all()


def test_pruned_levels_and_modes_are_never_chosen(oracle):
    """Random level and intra-mode masks: the chosen leaves use only kept levels and modes, the
    records of pruned-level blocks read as blocks with no choice, and no superblock gets cheaper."""
    from celv2_b200.pruner.data import block_level

    w, h, src, refs = case()
    nsb = ((w + 63) // 64) * ((h + 63) // 64)
    rng = np.random.default_rng(11)
    q = lam.lambda_q8(120)
    _, full = oracle.decide_masked(w, h, src, refs, q)
    for trial in range(6):
        levels = rng.integers(1, 16, nsb).astype(np.uint32)
        modes = rng.integers(1, 1 << 13, nsb).astype(np.uint32)
        keep = 0x87 | levels << 8 | modes << 16
        got, cost = oracle.decide_masked(w, h, src, refs, q, keep)
        assert (cost < 1 << 56).all()  # a complete partition of kept blocks
        for i, o in enumerate(got):
            n = int(o["nblocks"])
            lv = block_level(o["w4"][:n], o["h4"][:n])
            assert all(levels[i] >> int(l) & 1 for l in lv), (trial, i)
            for k in range(n):
                m = int(o["mode"][k])
                if m != 13:
                    assert modes[i] >> m & 1
            for b in range(425):
                sq = b // 5
                level = 3 if sq >= 21 else 2 if sq >= 5 else 1 if sq >= 1 else 0
                if not levels[i] >> level & 1:
                    assert o["c_inter_cost"][b] == np.iinfo(np.int64).max
                    assert o["c_intra_cost"][b] == np.iinfo(np.int64).max
                    assert (o["c_rcost"][:, b] == NO_REF_COST).all()
