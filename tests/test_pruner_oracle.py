"""The pruner network's CPU restatement (oracle/pruner_ref.py), checked before it checks the CUDA
kernels: its backward pass against finite differences of its forward pass (FP64, no rounding),
and the BF16 rounding it mirrors."""
import numpy as np

from oracle import pruner_ref as R


def init(rng):
    p = rng.normal(0, 0.2, R.PARAMS)
    return p


def loss_of(p, x, y, w):
    z, _ = R.forward(p, x, bf=False)
    return R.bce(z, y, w)[0]


def test_parameter_count():
    assert R.PARAMS == 56120


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = init(rng)
    x = rng.normal(0, 1, (3, R.FEATURES))
    y = (rng.random((3, R.OUTPUTS)) < 0.5).astype(np.float64)
    w = np.ones((3, R.OUTPUTS))
    z, cache = R.forward(p, x, bf=False)
    _, dz = R.bce(z, y, w)
    g = R.backward(p, cache, dz.astype(np.float64), bf=False)
    offsets = np.cumsum([0] + [int(np.prod(s)) for _, s in R.SHAPES])
    eps = 1e-6
    for t in range(len(R.SHAPES)):
        for i in rng.integers(offsets[t], offsets[t + 1], 4):
            q = p.copy()
            q[i] += eps
            up = loss_of(q, x, y, w)
            q[i] -= 2 * eps
            down = loss_of(q, x, y, w)
            fd = (up - down) / (2 * eps)
            assert abs(fd - g[i]) <= 1e-4 + 1e-3 * abs(fd), (R.SHAPES[t][0], i, fd, g[i])


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0, 1e-3], np.float32)
    r = R.bf16(v)
    assert r[0] == 1.0
    assert r[1] == 1.0                  # halfway between 1 and 1 + 2^-7: ties to even
    assert r[2] == np.float32(1.0078125)
    assert abs(r[3] + 3.140625) < 1e-6
    assert (r.view(np.uint32) & 0xFFFF == 0).all()
