"""celv2_decide_key_noalloc: the KEY-frame decision for callers that cannot allocate device memory
while they run (their host provisions all GPU memory up front, or they cannot take the device
synchronisation of cudaMalloc / cudaFree). Its scratch lives in a fixed static device array, so
the test gives it caller-owned device buffers (made here with torch) and checks two calls in a
row against the existing entry point (celv2_launch with no references) and against the oracle's
KEY decision: the records must be equal byte for byte, the tolerance of every decision test here.
Sizes: 416x240 (pitch = padded width), 202x122 (a padded frame read through a pitch wider than
its padded width, so the plane's right and bottom clamps run) and 1920x1080 (510 superblocks, near
the 768-superblock limit). Collected last on purpose."""
import numpy as np
import pytest

import frames as F
from celv2_b200 import lam, synth
from celv2_b200.engine import CudaEngine, E_INVAL, library
from celv2_b200.records import SB_OUT_DTYPE, first_difference, records_equal

pytestmark = pytest.mark.gpu


def noalloc(plane: np.ndarray, w: int, h: int, q: int, pitch: int | None = None) -> np.ndarray:
    import torch

    ph, pw = plane.shape
    pitch = pitch or pw
    host = np.full((ph, pitch), 77, np.uint8)  # the columns past pw are never read
    host[:, :pw] = plane
    dev_plane = torch.from_numpy(host).cuda()
    nsb = ((w + 63) // 64) * ((h + 63) // 64)
    out = torch.empty(nsb * SB_OUT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    rc = library().celv2_decide_key_noalloc(dev_plane.data_ptr(), w, h, pitch, lam.lambda_q8(q),
                                            out.data_ptr(), stream.cuda_stream)
    assert rc == 0, library().celv2_last_error()
    stream.synchronize()
    return out.cpu().numpy().view(SB_OUT_DTYPE)


CASES = [
    ("416x240", 416, 240, None, lambda: [F.test_frame(416, 240), F.scene_frame(416, 240, 3, -2)]),
    ("202x122-pitch256", 202, 122, 256, lambda: [F.test_frame(202, 122), F.scene_frame(202, 122, 6, -3)]),
    ("1920x1080", 1920, 1080, None, lambda: [f.y for f in synth.hd_clip(seed=3, frames=2)]),
]


@pytest.mark.parametrize("name,w,h,pitch,make", CASES, ids=[c[0] for c in CASES])
def test_no_alloc_matches_launch_and_oracle_two_calls_in_a_row(oracle, name, w, h, pitch, make):
    frames = make()
    qs = (120, 40)
    with CudaEngine(w, h) as e:
        want = [e.decide_intra(f, q).records for f, q in zip(frames, qs)]
    got = [noalloc(f, w, h, q, pitch) for f, q in zip(frames, qs)]
    for f, q, g, x in zip(frames, qs, got, want):
        assert g.tobytes() == x.tobytes(), f"{name} vs celv2_launch: {first_difference(g, x)}"
        o = oracle.decide(w, h, f, [], lam.lambda_q8(q))
        assert records_equal(g, o), f"{name} vs oracle: {first_difference(g, o)}"


def test_no_alloc_rejects_frames_above_its_scratch():
    import torch

    dummy = torch.zeros(64, dtype=torch.uint8, device="cuda")
    rc = library().celv2_decide_key_noalloc(dummy.data_ptr(), 3840, 2160, 3840, 100, dummy.data_ptr(), None)
    assert rc == E_INVAL
    assert b"exceed" in library().celv2_last_error()
    # sizes whose superblock count would overflow int arithmetic are rejected before it
    for w, h in ((1 << 30, 64), (64, 1 << 30), (2**31 - 1, 2**31 - 1)):
        rc = library().celv2_decide_key_noalloc(dummy.data_ptr(), w, h, w, 100, dummy.data_ptr(), None)
        assert rc == E_INVAL, (w, h)
        assert b"at most" in library().celv2_last_error()
