"""The pruner's training data on the host (no GPU): the mix of content kinds, the keep words of the
regret decisions, and the regret-weighted labels."""
import numpy as np

from celv2_b200.pruner import data as D
from celv2_b200.pruner import train as T


def test_training_seeds_mix_the_kinds_evenly():
    seeds = T.training_seeds(200, 0.3)
    kinds = [k for _, k in seeds]
    assert kinds.count(T.ANIME) == 60 and kinds.count(T.SINUSOID) == 140
    # spread: every run of 10 consecutive clips holds 3 animation-like ones
    for i in range(0, 200, 10):
        assert kinds[i:i + 10].count(T.ANIME) == 3
    anime = [s for s, k in seeds if k == T.ANIME]
    natural = [s for s, k in seeds if k == T.SINUSOID]
    assert anime == list(range(T.ANIME_TRAIN_SEED0, T.ANIME_TRAIN_SEED0 + 60))
    assert natural == list(range(T.TRAIN_SEED0, T.TRAIN_SEED0 + 140))
    # held-out and validation seeds are none of the training ones
    held = set(T.VAL_SEEDS) | set(T.ANIME_VAL_SEEDS) | set(range(T.TEST_SEED0, T.TEST_SEED0 + 20)) | \
        set(range(T.ANIME_TEST_SEED0, T.ANIME_TEST_SEED0 + 8))
    assert not held & (set(anime) | set(natural))
    assert T.training_seeds(8, 0.0) == [(T.TRAIN_SEED0 + k, T.SINUSOID) for k in range(8)]


def test_regret_words_prune_one_option_each():
    allm = 0x1FFF0000
    for n in range(1, 8):
        refs = (1 << n) - 1
        assert D.REGRET_OUTPUTS[7](n) == refs | 0xF00 | allm  # every option but intra
        for r in range(7):
            w = D.REGRET_OUTPUTS[r](n)
            if n < 2 or r >= n:
                assert w is None  # a frame's only reference is always kept; absent ones are not pruned
            else:
                assert w == (refs & ~(1 << r)) | 0x80 | 0xF00 | allm
        for l in range(4):
            assert D.REGRET_OUTPUTS[8 + l](n) == refs | 0x80 | (0xF00 & ~(0x100 << l)) | allm


def test_regret_scales_only_needed_options():
    nsb, nrefs = 6, 3
    words = np.array([0x183, 0x101, 0x282, 0x800 | 0x1, 0x181, 0x401], np.uint32)
    y0, w0 = D.labels(words, nrefs)
    cost = np.full(nsb, 1000, np.int64)
    reg = {7: np.array([0, 0, 5000, 50000, 50000, 0], np.int64),  # intra: needed in sb 0, 2 and 4
           8: np.array([2000, 100, 0, 0, 0, 0], np.int64),     # the 64 level: needed in sb 0, 1, 4
           1: np.array([9000, 0, 9000, 0, 0, 0], np.int64)}    # reference 1: needed in sb 0 and 2
    y, w = D.labels(words, nrefs, regret=reg, cost=cost)
    assert (y == y0).all()
    f = np.ones_like(w0)
    f[0, 8] = 1 + 2000 / 1000
    f[1, 8] = 1 + 100 / 1000
    f[2, 7] = 1 + 5000 / 1000
    f[4, 7] = 20.0  # capped
    f[0, 1] = f[2, 1] = 10.0
    # sb 3 has no intra leaf: its intra regret does not count; unused options keep their weights
    np.testing.assert_allclose(w, w0 * f, rtol=1e-6)
    # a negative cost change (pruning can lower a cost) never lowers a weight
    _, wn = D.labels(words, nrefs, regret={7: np.full(nsb, -500, np.int64)}, cost=cost)
    np.testing.assert_allclose(wn, w0)
