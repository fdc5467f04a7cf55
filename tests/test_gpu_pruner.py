"""The learned pruner's CUDA kernels against their CPU restatement (oracle/pruner_ref.py): the
tensor-core forward pass, every parameter's gradient, the loss, the Adam step and the features;
then the engine running the network: its masks are the network's, applied exactly."""
import ctypes as C

import numpy as np
import pytest

import frames as F
from celv2_b200 import engine as E
from celv2_b200 import lam
from celv2_b200.pruner import net as N
from celv2_b200.records import first_difference, records_equal
from oracle import pruner_ref as R
from oracle.binding import field_dims

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def ptr(t):
    return C.c_void_p(t.data_ptr())


def case(batch, seed=0):
    rng = np.random.default_rng(seed)
    p = N.init_params(seed) + rng.normal(0, 0.02, E.PRUNER_PARAMS).astype(np.float32)  # biases not all zero
    x = rng.normal(0, 1, (batch, E.PRUNER_FEATURES)).astype(np.float32)
    return p, x


@pytest.mark.parametrize("batch", [1, 37, 300])
def test_forward_matches_oracle(batch):
    p, x = case(batch)
    tr = N.Trainer(batch, params=p)
    got = tr.logits(dev(x)).cpu().numpy()
    want, _ = R.forward(p, x, bf=True)
    assert np.allclose(got, want, rtol=1e-3, atol=1e-3), np.abs(got - want).max()


@pytest.mark.parametrize("batch", [5, 64, 129])
def test_backward_matches_oracle(batch):
    p, x = case(batch, seed=batch)
    rng = np.random.default_rng(batch + 1)
    dl = rng.normal(0, 1, (batch, E.PRUNER_OUTPUTS)).astype(np.float32)
    tr = N.Trainer(batch, params=p)
    xt = dev(x)
    tr.logits(xt)
    lib = E.library()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert lib.celv2_pruner_backward(ptr(tr.p), batch, ptr(tr.acts), ptr(dev(dl)), ptr(tr.work), ptr(tr.g), st) == 0
    got = tr.g.cpu().numpy()
    _, cache = R.forward(p, x, bf=True)
    want = R.backward(p, cache, dl, bf=True)
    o = 0
    for name, shape in R.SHAPES:
        n = int(np.prod(shape))
        g, w = got[o:o + n], want[o:o + n]
        err = np.linalg.norm(g - w) / max(np.linalg.norm(w), 1e-12)
        assert err < 2e-3, (name, err)
        o += n


def test_loss_and_adam_match_oracle():
    rng = np.random.default_rng(7)
    z = rng.normal(0, 2, (50, E.PRUNER_OUTPUTS)).astype(np.float32)
    y = (rng.random((50, E.PRUNER_OUTPUTS)) < 0.4).astype(np.float32)
    w = rng.choice([0.0, 1.0, 2.0], (50, E.PRUNER_OUTPUTS)).astype(np.float32)
    lib = E.library()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    dz, loss = torch.zeros(50 * E.PRUNER_OUTPUTS, device="cuda"), torch.zeros(1, device="cuda")
    assert lib.celv2_pruner_bce(ptr(dev(z)), ptr(dev(y)), ptr(dev(w)), 50, ptr(dz), ptr(loss), st) == 0
    want_loss, want_dz = R.bce(z, y, w)
    assert abs(loss.item() - want_loss) < 1e-4 * max(1.0, abs(want_loss))
    assert np.allclose(dz.cpu().numpy().reshape(50, E.PRUNER_OUTPUTS), want_dz, atol=1e-6)
    p = rng.normal(0, 1, 1000).astype(np.float32)
    g = rng.normal(0, 1, 1000).astype(np.float32)
    pt, gt, m, v = dev(p), dev(g), torch.zeros(1000, device="cuda"), torch.zeros(1000, device="cuda")
    for step in (1, 2):
        assert lib.celv2_pruner_adam(ptr(pt), ptr(gt), ptr(m), ptr(v), 1000, 1e-2, 0.9, 0.999, 1e-8, 1e-4, step,
                                     st) == 0
    mm, vv, q = np.zeros(1000), np.zeros(1000), p.astype(np.float64)
    for step in (1, 2):
        mm = 0.9 * mm + 0.1 * g
        vv = 0.999 * vv + 0.001 * g * g
        q -= 1e-2 * ((mm / (1 - 0.9 ** step)) / (np.sqrt(vv / (1 - 0.999 ** step)) + 1e-8) + 1e-4 * q)
    assert np.allclose(pt.cpu().numpy(), q, atol=1e-5)


def levels(pyr, pw, ph):
    out, o, w, h = [], 0, pw, ph
    for _ in range(5):
        out.append(pyr[o:o + w * h].reshape(h, w))
        o += w * h
        w, h = w // 2, h // 2
    return out


def test_features_match_oracle(oracle):
    w, h = 202, 122
    src = F.textured(w, h, 5, -3)
    refs = [F.textured(w, h, i, -(i // 2)) for i in range(3)]
    pw, ph = (w + 7) & ~7, (h + 7) & ~7
    with E.CudaEngine(w, h) as e:
        e.set_config(E.CFG_FEATURES, 1)
        e.decide_inter(src, refs, 120)
        got = e.features(0)
    cur = levels(oracle.pyramid(src, False), pw, ph)
    cols, rows = field_dims(pw, ph)
    sbc, sbr = (w + 63) // 64, (h + 63) // 64
    want = np.zeros((sbc * sbr, E.PRUNER_FEATURES), np.float32)

    def clamp_read(pl, y, x):
        return pl[np.clip(y, 0, pl.shape[0] - 1), np.clip(x, 0, pl.shape[1] - 1)].astype(np.int64)

    fields = [oracle.me_fields(src, r) for r in refs]
    ref1 = [levels(oracle.pyramid(r, False), pw, ph)[1] for r in refs]
    for sb in range(sbc * sbr):
        sy, sx = divmod(sb, sbc)
        yy, xx = np.mgrid[0:16, 0:16]
        v = clamp_read(cur[2], sy * 16 + yy, sx * 16 + xx).astype(np.float32)
        want[sb, :256] = ((v - np.float32(v.sum() / 256.0)) / np.float32(64)).reshape(-1)
        for r in range(3):
            fx, fy = fields[r][1]
            for cell in range(16):
                cx, cy = min(sx * 4 + cell % 4, cols[1] - 1), min(sy * 4 + cell // 4, rows[1] - 1)
                mx, my = int(fx[cy, cx]), int(fy[cy, cx])
                iy, ix = np.mgrid[0:8, 0:8]
                a = clamp_read(cur[1], cy * 8 + iy, cx * 8 + ix)
                b = clamp_read(ref1[r], cy * 8 + my + iy, cx * 8 + mx + ix)
                want[sb, 256 + r * 16 + cell] = np.log2(1.0 + np.abs(a - b).sum()) / 14.0
        want[sb, 368:371] = 1.0
        want[sb, 375] = np.log2(float(lam.lambda_q8(120))) / 20.0
    assert np.allclose(got, want, atol=2e-6), np.abs(got - want).max()


def mask_word(prob, nrefs, tr, ti, tl, tm, band=0.0):
    """The keep word the engine's rule gives for one superblock's output probabilities
    (include/celv2_pruner.h, celv2_set_pruner)."""
    pr = prob[:nrefs]
    k = sum(1 << r for r in range(nrefs) if pr[r] >= tr) | (1 << int(np.argmax(pr)))
    k |= 0x80 if prob[7] >= ti else 0
    pl = prob[8:12]
    k |= sum(0x100 << l for l in range(4) if pl[l] >= tl) | (0x100 << int(np.argmax(pl)))
    if k & 0x80:
        k |= 0x7 << 16
        k |= sum(0x10000 << m for m in range(3, 13) if prob[12 + m - 3] >= tm)
    unsure = (np.abs(pr - tr) < band).any() or abs(prob[7] - ti) < band or (np.abs(pl - tl) < band).any()
    return 0xFFFFFFFF if unsure else k


def test_engine_applies_the_networks_masks(oracle):
    """With the pruner on, the records are the oracle's for the keep words the network chose, and
    the words are what the network's outputs and thresholds give."""
    w, h = 640, 360
    src = F.textured(w, h, 5, -3)
    refs = [F.textured(w, h, i, -(i // 2)) for i in range(4)]
    p, _ = case(1, seed=3)
    th = (0.4, 0.5, 0.45, 0.5)
    with E.CudaEngine(w, h) as e:
        e.set_config(E.CFG_FEATURES, 1)
        e.decide_inter(src, refs, 120)
        x = e.features(0)
        e.set_pruner(p, *th, 0.0)
        got = e.decide_inter(src, refs, 120)
        masks = e.pruner_masks(0)
        costs = e.sb_costs(0)
    z, _ = R.forward(p, x, bf=True)
    prob = 1 / (1 + np.exp(-z.astype(np.float64)))
    for sb in range(x.shape[0]):
        want = mask_word(prob[sb], 4, *th)
        near = mask_word(prob[sb], 4, *th, band=1e-3) == 0xFFFFFFFF  # rounding-order ties
        near |= (np.abs(prob[sb, 12:22] - th[3]) < 1e-3).any()
        assert near or masks[sb] == want, (sb, hex(masks[sb]), hex(want))
    want_rec, want_cost = oracle.decide_masked(w, h, src, refs, lam.lambda_q8(120), masks)
    assert records_equal(got.records, want_rec), first_difference(got.records, want_rec)
    assert (costs == want_cost).all()


def test_group_runs_one_network_pass(oracle):
    """In a group every inter job gets the network's masks, with or without graph replay; each job's
    records are the oracle's for those masks."""
    from celv2_b200 import synth

    w, h = 416, 240
    clip = synth.small_clip(seed=17, frames=6)
    p, _ = case(1, seed=5)
    jobs = [(5, [4, 3, 2, 1]), (4, [3, 2]), (3, []), (2, [1, 0])]
    with E.CudaEngine(w, h) as e:
        for i, f in enumerate(clip):
            e.upload(f.hy, i)
        e.set_pruner(p, 0.5, 0.5, 0.4, 0.5, 0.0)
        for graphs in (0, 1):
            e.set_config(E.CFG_GRAPHS, graphs)
            e.launch_group([s for s, _ in jobs], [r for _, r in jobs], 130, to_host=True)
            for j, (s, refs) in enumerate(jobs):
                keep = e.pruner_masks(j) if refs else None
                want, want_cost = oracle.decide_masked(w, h, clip[s].y, [clip[r].y for r in refs],
                                                       lam.lambda_q8(130), keep)
                got = e.group_records(j)
                assert records_equal(got, want), f"job {j}: {first_difference(got, want)}"
                assert (e.sb_costs(j) == want_cost).all()


def test_network_beats_the_rules_without_it():
    """On a held-out 1080p clip (a seed no training clip used; 33 frames, two mini-GOPs) at the
    benchmark's qindex, the committed network at its committed thresholds stays within the 1 %
    budget of the summed chosen-partition cost, and no rule without the network (the k nearest
    references, intra or not, every block level or only the small ones) is both at least as fast
    and at most as costly."""
    from celv2_b200 import pruner, synth
    from celv2_b200.pruner import evaluate as V

    clip = [f.hy for f in synth.hd_clip(3001, 33)]
    wts = pruner.load()
    plan = V.default_plan(33)
    with E.CudaEngine(1920, 1080) as e:
        e.reserve_group(10)
        V.upload(e, clip)
        full, _, _ = V.run(e, plan, 130)
        pruner.set_on(e, wts)
        net, ms_net, _ = V.run(e, plan, 130, reps=3)
        e.set_pruner(None)
        rules = []
        for k in (2, 3, 4):
            for intra in (True, False):
                for small in (False, True):
                    costs, ms, _ = V.run(e, plan, 130, masks=V.nearest(k, intra, small), reps=3)
                    rules.append(((k, intra, small), V.cost_increase(costs, full), ms))
    loss_net = V.cost_increase(net, full)
    assert 0.0 <= loss_net <= 0.01, loss_net
    dominating = [r for r in rules if r[1] <= loss_net and r[2] <= ms_net]
    assert not dominating, (loss_net, ms_net, dominating)


def test_network_keeps_the_budget_on_animation_content():
    """On a held-out animation-like 1080p clip (flat colours and hard edges, piecewise motion; a seed
    no training clip used; 33 frames) at the benchmark's qindex, the committed network stays within
    the 1 % budget of the summed chosen-partition cost and still saves time. Flat content is where
    pruning the large block levels costs most: a network that had seen only natural-like clips
    dropped the 64-sample level there and doubled the cost."""
    from celv2_b200 import pruner
    from celv2_b200.pruner import evaluate as V
    from celv2_b200.pruner import train as T

    clip = T._clip((T.ANIME_TEST_SEED0, 33, T.ANIME))
    wts = pruner.load()
    plan = V.default_plan(33)
    with E.CudaEngine(1920, 1080) as e:
        e.reserve_group(10)
        V.upload(e, clip)
        full, ms_full, _ = V.run(e, plan, 130, reps=3)
        pruner.set_on(e, wts)
        net, ms_net, _ = V.run(e, plan, 130, reps=3)
        e.set_pruner(None)
    loss_net = V.cost_increase(net, full)
    assert loss_net <= 0.01, loss_net
    assert ms_net < ms_full, (ms_net, ms_full)
