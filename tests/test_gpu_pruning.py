"""The pruned search on the GPU against the oracle with the same masks: records and per-superblock
costs byte for byte (the kept options are scored exactly; the level-0 motion search skips only
cells no kept reference reads)."""
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


@pytest.mark.parametrize("w,h,nrefs", [(202, 122, 3), (640, 360, 7), (72, 40, 2)])
def test_masked_launch_matches_oracle(oracle, w, h, nrefs):
    src = F.textured(w, h, 5, -3)
    refs = [F.textured(w, h, i, -(i // 2)) for i in range(nrefs)]
    with E.CudaEngine(w, h) as e:
        nsb = e.sb_cols * e.sb_rows
        for seed in range(3):
            keep = masks(nsb, seed, nrefs)
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
        keeps = [masks(nsb, 10 + j, max(1, len(refs))) for j, (_, refs) in enumerate(jobs)]
        for j, k in enumerate(keeps):
            e.set_keep(j, k)
        e.launch_group([s for s, _ in jobs], [r for _, r in jobs], 130, to_host=True)
        for j, (s, refs) in enumerate(jobs):
            want, want_cost = oracle.decide_masked(w, h, clip[s].y, [clip[r].y for r in refs], lam.lambda_q8(130),
                                                   keeps[j])
            got = e.group_records(j)
            assert records_equal(got, want), f"job {j}: {first_difference(got, want)}"
            assert (e.sb_costs(j) == want_cost).all()
