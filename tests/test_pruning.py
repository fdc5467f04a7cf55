"""The pruned search's semantics on the oracle (CPU): masks that keep everything change nothing,
a pruned option is never chosen, and pruning never lowers a superblock's cost."""
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
    assert (cost >= full).all()  # a subset of the options: never cheaper
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
