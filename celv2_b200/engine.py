"""Python mirror of the reference's DecisionEngine interface over the CUDA engine's C ABI.

``CudaEngine`` has the reference's methods and meaning (src/gpu/decision_engine.h:9-51):
``launch(src, refs, qindex, dm, ref_keys, src_key)``, ``prepare(next, key)``,
``collect(dm, gate)``, ``set_row_streams(n)``, ``decide_inter`` / ``decide_intra``. ``RowGate``
mirrors src/gpu/decision_map.h:87-108 (decision_map.cpp:19-61). Errors are raised as the
reference raises them: ``RuntimeError`` for size mismatches and more than 7 references,
``ValueError`` (std::invalid_argument) for a key count that does not match the references.

The decisions come from the CUDA kernels in libcelv2_cuda.so; there is no CPU path. Loading the
library fails loudly when it is missing.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

from . import lam as _lam
from .records import SB_OUT_DTYPE, DecisionMap

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcelv2_cuda.so")

E_OK, E_INVAL, E_CUDA, E_STATE = 0, -1, -2, -3


class CelvFrame(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("pitch", C.c_int32),
                ("y", C.POINTER(C.c_uint8)), ("hy", C.POINTER(C.c_uint16)), ("bit_depth", C.c_int32)]


_lib = None
_lib_lock = threading.Lock()

# Every C entry point of include/celv2_cuda.h with its ctypes signature.
SIGNATURES = {
    "celv2_last_error": (C.c_char_p, []),
    "celv2_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "celv2_destroy": (None, [C.c_void_p]),
    "celv2_launch": (C.c_int, [C.c_void_p, C.POINTER(CelvFrame), C.POINTER(CelvFrame), C.c_int, C.c_int64,
                               C.POINTER(C.c_longlong), C.c_longlong]),
    "celv2_prepare": (C.c_int, [C.c_void_p, C.POINTER(CelvFrame), C.c_longlong]),
    "celv2_set_row_streams": (C.c_int, [C.c_void_p, C.c_int]),
    "celv2_geometry": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "celv2_row_order": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "celv2_wait_row": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "celv2_finish": (C.c_int, [C.c_void_p]),
    "celv2_upload": (C.c_int, [C.c_void_p, C.POINTER(CelvFrame), C.c_longlong]),
    "celv2_launch_group": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                                     C.POINTER(C.POINTER(C.c_longlong)), C.POINTER(C.c_int64), C.c_int]),
    "celv2_reserve_group": (C.c_int, [C.c_void_p, C.c_int]),
    "celv2_group_records": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "celv2_clear_store": (C.c_int, [C.c_void_p]),
    "celv2_debug_field": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_int),
                                    C.POINTER(C.c_int)]),
    "celv2_debug_intra": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "celv2_debug_inter": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "celv2_kernel_launches": (C.c_longlong, [C.c_void_p]),
    "celv2_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "celv2_stage_timing": (C.c_int, [C.c_void_p, C.c_int]),
    "celv2_stage_times": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_longlong), C.c_int]),
    "celv2_int_peak": (C.c_int, [C.c_int, C.POINTER(C.c_double)]),
    "celv2_work_counters": (C.c_int, [C.c_void_p, C.POINTER(C.c_ulonglong), C.c_int]),
    "celv2_decide_key_noalloc": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int64, C.c_void_p,
                                           C.c_void_p]),
    "celv2_launch_multi": (C.c_int, [C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                                     C.POINTER(C.POINTER(C.c_longlong)), C.POINTER(C.c_int64), C.c_int]),
    "celv2_set_config": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "celv2_get_config": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
}

CFG_PERSISTENT, CFG_GRAPHS, CFG_PERSISTENT_OFF, CFG_INTER_CHUNK, CFG_ME_CELLS_L0 = 1, 2, 3, 4, 10

STAGE_NAMES = ["upload+pyramid", "phases", "me_l4", "me_l3", "me_l2", "me_l1", "me_l0", "intra", "inter",
               "finalize"]


def library():
    """The loaded libcelv2_cuda.so (built on first use when nvcc is present)."""
    global _lib
    with _lib_lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                from . import build

                build.build()
            lib = C.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def _check(rc: int) -> None:
    if rc == E_OK:
        return
    msg = library().celv2_last_error().decode()
    if rc == E_INVAL:
        raise RuntimeError(msg)
    raise RuntimeError(f"CUDA engine error {rc}: {msg}")


def _plane_of(f):
    """(8-bit plane or None, 16-bit plane or None, bit depth) of a frame-like input."""
    if isinstance(f, np.ndarray):
        return (np.ascontiguousarray(f, dtype=np.uint8), None, 8) if f.dtype == np.uint8 else (
            None, np.ascontiguousarray(f, dtype=np.uint16), 10)
    hy = getattr(f, "hy", None)
    y = getattr(f, "y", None)
    if y is not None:
        return np.ascontiguousarray(y, dtype=np.uint8), None, 8
    return None, np.ascontiguousarray(hy, dtype=np.uint16), int(getattr(f, "bit_depth", 10))


def make_frame(f, width: int, height: int, keep: list) -> CelvFrame:
    """A celv2_frame view of a numpy plane (8-bit, or uint16 10-bit) or a synth.Frame."""
    y, hy, depth = _plane_of(f)
    cf = CelvFrame()
    cf.width, cf.height = width, height
    plane = y if y is not None else hy
    cf.pitch = plane.shape[1]
    if y is not None:
        cf.y = y.ctypes.data_as(C.POINTER(C.c_uint8))
        keep.append(y)
    else:
        cf.hy = hy.ctypes.data_as(C.POINTER(C.c_uint16))
        cf.bit_depth = depth
        keep.append(hy)
    return cf


class RowGate:
    """The reference's RowGate (src/gpu/decision_map.cpp:19-61): rows published by the collector,
    awaited by consumers; a failure is recorded once and raised to every waiter."""

    def __init__(self):
        self._cv = threading.Condition()
        self._ready = 0
        self._one: list[bool] = []
        self._error: BaseException | None = None

    def publish(self, row: int) -> None:
        with self._cv:
            if row + 1 > self._ready:
                self._ready = row + 1
            self._cv.notify_all()

    def publish_one(self, row: int) -> None:
        with self._cv:
            if len(self._one) <= row:
                self._one.extend([False] * (row + 1 - len(self._one)))
            self._one[row] = True
            while self._ready < len(self._one) and self._one[self._ready]:
                self._ready += 1
            self._cv.notify_all()

    def wait_row(self, row: int, timeout: float | None = None) -> None:
        with self._cv:
            ok = self._cv.wait_for(
                lambda: self._error is not None or self._ready > row or (row < len(self._one) and self._one[row]),
                timeout)
            if self._error is not None:
                raise self._error
            if not ok:
                raise TimeoutError(f"row {row} not published")

    def fail(self, e: BaseException) -> None:
        with self._cv:
            if self._error is None:
                self._error = e
            self._cv.notify_all()

    def ready_rows(self) -> int:
        with self._cv:
            return self._ready


class CudaEngine:
    """DecisionEngine on the B200 (src/gpu/decision_engine.h:9-51)."""

    def __init__(self, width: int, height: int, sb_size: int = 64, device: int = 0):
        self.width, self.height, self.sb_size = width, height, sb_size
        lib = library()
        h = C.c_void_p()
        _check(lib.celv2_create(width, height, sb_size, device, C.byref(h)))
        self._h = h
        sc, sr = C.c_int(), C.c_int()
        _check(lib.celv2_geometry(h, C.byref(sc), C.byref(sr)))
        self.sb_cols, self.sb_rows = sc.value, sr.value
        self.row_hook = None  # called by collect before it publishes a row (tests only)

    def close(self) -> None:
        if getattr(self, "_h", None):
            library().celv2_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- the DecisionEngine interface ----
    def launch(self, src, refs, qindex: int, dm: DecisionMap, ref_keys=None, src_key: int = -1,
               lambda_q8: int | None = None) -> None:
        refs = list(refs or [])
        if ref_keys is not None and len(ref_keys) and len(ref_keys) != len(refs):
            raise ValueError("CudaEngine: one key per reference")
        keep: list = []
        s = make_frame(src, self.width, self.height, keep)
        rarr = (CelvFrame * max(1, len(refs)))(*[make_frame(r, self.width, self.height, keep) for r in refs])
        karr = (C.c_longlong * len(refs))(*ref_keys) if ref_keys else None
        lam = _lam.lambda_q8(qindex) if lambda_q8 is None else lambda_q8
        _check(library().celv2_launch(self._h, C.byref(s), rarr, len(refs), lam, karr, src_key))
        dm.sb_size, dm.sb_cols, dm.sb_rows = self.sb_size, self.sb_cols, self.sb_rows
        dm.records = np.zeros(self.sb_cols * self.sb_rows, dtype=SB_OUT_DTYPE)

    def prepare(self, nxt, key: int) -> None:
        keep: list = []
        f = make_frame(nxt, self.width, self.height, keep)
        _check(library().celv2_prepare(self._h, C.byref(f), key))

    def set_row_streams(self, n: int) -> None:
        _check(library().celv2_set_row_streams(self._h, n))

    def row_order(self) -> list[int]:
        arr = (C.c_int * self.sb_rows)()
        _check(library().celv2_row_order(self._h, arr))
        return list(arr)

    def collect(self, dm: DecisionMap, gate: RowGate) -> None:
        """Copies every row into dm as it arrives and publishes it on gate; on failure fails the
        gate and raises. Returns with no work pending."""
        lib = library()
        try:
            for r in self.row_order():
                if self.row_hook:
                    self.row_hook(r)
                ptr = C.c_void_p()
                _check(lib.celv2_wait_row(self._h, r, C.byref(ptr)))
                n = self.sb_cols
                src = np.ctypeslib.as_array((C.c_uint8 * (n * SB_OUT_DTYPE.itemsize)).from_address(ptr.value))
                dm.records[r * n:(r + 1) * n] = src.view(SB_OUT_DTYPE)
                gate.publish_one(r)
            _check(lib.celv2_finish(self._h))
        except BaseException as e:
            gate.fail(e)
            lib.celv2_finish(self._h)
            raise

    def decide_inter(self, src, refs, qindex: int, ref_keys=None) -> DecisionMap:
        dm, gate = DecisionMap(), RowGate()
        self.launch(src, refs, qindex, dm, ref_keys)
        self.collect(dm, gate)
        return dm

    def decide_intra(self, src, qindex: int) -> DecisionMap:
        return self.decide_inter(src, [], qindex)

    # ---- device-resident path ----
    def upload(self, frame, key: int) -> None:
        keep: list = []
        f = make_frame(frame, self.width, self.height, keep)
        _check(library().celv2_upload(self._h, C.byref(f), key))

    def reserve_group(self, frames: int) -> None:
        _check(library().celv2_reserve_group(self._h, frames))

    def launch_group(self, src_keys, ref_keys, qindex, to_host: bool = False) -> None:
        n = len(src_keys)
        qs = qindex if isinstance(qindex, (list, tuple)) else [qindex] * n
        sk = (C.c_longlong * n)(*src_keys)
        nr = (C.c_int * n)(*[len(r) for r in ref_keys])
        rows = [(C.c_longlong * max(1, len(r)))(*r) for r in ref_keys]
        rk = (C.POINTER(C.c_longlong) * n)(*[C.cast(r, C.POINTER(C.c_longlong)) for r in rows])
        lams = (C.c_int64 * n)(*[_lam.lambda_q8(q) for q in qs])
        _check(library().celv2_launch_group(self._h, n, sk, nr, rk, lams, 1 if to_host else 0))

    def group_records(self, job: int) -> np.ndarray:
        ptr = C.c_void_p()
        _check(library().celv2_group_records(self._h, job, C.byref(ptr)))
        n = self.sb_cols * self.sb_rows
        raw = np.ctypeslib.as_array((C.c_uint8 * (n * SB_OUT_DTYPE.itemsize)).from_address(ptr.value))
        return raw.view(SB_OUT_DTYPE).copy()

    def finish(self) -> None:
        _check(library().celv2_finish(self._h))

    def clear_store(self) -> None:
        _check(library().celv2_clear_store(self._h))

    def set_config(self, key: int, value: int) -> None:
        _check(library().celv2_set_config(self._h, key, int(value)))

    def get_config(self, key: int) -> int:
        v = C.c_int()
        _check(library().celv2_get_config(self._h, key, C.byref(v)))
        return v.value

    def kernel_launches(self) -> int:
        return int(library().celv2_kernel_launches(self._h))

    def stream(self) -> int:
        p = C.c_void_p()
        _check(library().celv2_stream(self._h, C.byref(p)))
        return p.value or 0

    def stage_timing(self, enable: bool) -> None:
        _check(library().celv2_stage_timing(self._h, 1 if enable else 0))

    def work_counters(self) -> list[int]:
        """[searched centres at levels 0..4, distinct inter MVs, compound tiles, 0] since the last call."""
        arr = (C.c_ulonglong * 8)()
        _check(library().celv2_work_counters(self._h, arr, 8))
        return list(arr)

    def stage_times(self) -> dict:
        """{stage: (milliseconds, launches)} since the last call (stage timing must be on)."""
        n = len(STAGE_NAMES)
        ms, cnt = (C.c_double * n)(), (C.c_longlong * n)()
        _check(library().celv2_stage_times(self._h, ms, cnt, n))
        return {STAGE_NAMES[i]: (ms[i], cnt[i]) for i in range(n)}

    # ---- inspection ----
    def debug_field(self, r: int, level: int) -> np.ndarray:
        pw, ph = (self.width + 7) & ~7, (self.height + 7) & ~7
        w, h = pw, ph
        for _ in range(level):
            w, h = w // 2, h // 2
        cols, rows = (w + 7) // 8, (h + 7) // 8
        out = np.zeros((rows, cols), np.int32)
        c, rr = C.c_int(), C.c_int()
        _check(library().celv2_debug_field(self._h, r, level, out.ctypes.data_as(C.POINTER(C.c_int32)),
                                           C.byref(c), C.byref(rr)))
        return out

    def debug_intra(self) -> np.ndarray:
        out = np.zeros((self.sb_cols * self.sb_rows, 425, 13), np.int32)
        _check(library().celv2_debug_intra(self._h, out.ctypes.data_as(C.POINTER(C.c_int32))))
        return out

    def debug_inter(self) -> np.ndarray:
        out = np.zeros((self.sb_cols * self.sb_rows, 7, 425, 2), np.int32)
        _check(library().celv2_debug_inter(self._h, out.ctypes.data_as(C.POINTER(C.c_int32))))
        return out


def launch_multi(jobs, qindex, to_host: bool = False) -> None:
    """One batch over engines of different frame sizes: jobs = [(engine, src_key, [ref keys])].
    Each engine's records come back with engine.group_records(k) for its k-th job here."""
    n = len(jobs)
    qs = qindex if isinstance(qindex, (list, tuple)) else [qindex] * n
    engs = (C.c_void_p * n)(*[e._h.value if isinstance(e._h, C.c_void_p) else e._h for e, _, _ in jobs])
    sk = (C.c_longlong * n)(*[s for _, s, _ in jobs])
    nr = (C.c_int * n)(*[len(r) for _, _, r in jobs])
    rows = [(C.c_longlong * max(1, len(r)))(*r) for _, _, r in jobs]
    rk = (C.POINTER(C.c_longlong) * n)(*[C.cast(r, C.POINTER(C.c_longlong)) for r in rows])
    lams = (C.c_int64 * n)(*[_lam.lambda_q8(q) for q in qs])
    _check(library().celv2_launch_multi(n, engs, sk, nr, rk, lams, 1 if to_host else 0))


def int_peak(device: int = 0) -> float:
    """Measured INT32 ops/s of the GPU (the roofline denominator of the integer kernels)."""
    v = C.c_double()
    _check(library().celv2_int_peak(device, C.byref(v)))
    return v.value


def unpack_field(packed: np.ndarray):
    """(mvx, mvy) of a packed field ((mvy << 16) | (mvx & 0xffff))."""
    p = packed.astype(np.int64)
    mvx = ((p & 0xFFFF) ^ 0x8000) - 0x8000
    mvy = p >> 16
    return mvx.astype(np.int32), mvy.astype(np.int32)
