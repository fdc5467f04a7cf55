"""celv2_decide_key_noalloc: the KEY-frame decision for callers that cannot allocate device memory
while they run (their host provisions all GPU memory up front, or they cannot take the device
synchronisation of cudaMalloc / cudaFree). Its scratch lives in a fixed static device array, so
the test gives it caller-owned device buffers (made here with torch) and checks two calls in a
row against the existing entry point (celv2_launch with no references): the records must be equal
byte for byte, the tolerance of every decision test here. Collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

import frames as F
from celv2_b200 import lam
from celv2_b200.engine import CudaEngine, E_INVAL, library
from celv2_b200.records import SB_OUT_DTYPE, first_difference

pytestmark = pytest.mark.gpu


def noalloc(plane: np.ndarray, w: int, h: int, q: int) -> np.ndarray:
    import torch

    dev_plane = torch.from_numpy(np.ascontiguousarray(plane)).cuda()
    nsb = ((w + 63) // 64) * ((h + 63) // 64)
    out = torch.empty(nsb * SB_OUT_DTYPE.itemsize, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    rc = library().celv2_decide_key_noalloc(dev_plane.data_ptr(), w, h, plane.shape[1], lam.lambda_q8(q),
                                            out.data_ptr(), stream.cuda_stream)
    assert rc == 0, library().celv2_last_error()
    stream.synchronize()
    return out.cpu().numpy().view(SB_OUT_DTYPE)


def test_no_alloc_matches_launch_two_calls_in_a_row():
    w, h = 416, 240
    frames = [F.test_frame(w, h), F.scene_frame(w, h, 3, -2)]
    with CudaEngine(w, h) as e:
        want = [e.decide_intra(f, q).records for f, q in zip(frames, (120, 40))]
    got = [noalloc(f, w, h, q) for f, q in zip(frames, (120, 40))]
    for g, x in zip(got, want):
        assert g.tobytes() == x.tobytes(), first_difference(g, x)


def test_no_alloc_rejects_frames_above_its_scratch():
    import torch

    dummy = torch.zeros(64, dtype=torch.uint8, device="cuda")
    rc = library().celv2_decide_key_noalloc(dummy.data_ptr(), 3840, 2160, 3840, 100, dummy.data_ptr(), None)
    assert rc == E_INVAL
    assert b"exceed" in library().celv2_last_error()
