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
import weakref

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
    "celv2_upload_pinned": (C.c_int, [C.c_void_p, C.POINTER(CelvFrame), C.c_longlong]),
    "celv2_launch_group": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_longlong), C.POINTER(C.c_int),
                                     C.POINTER(C.POINTER(C.c_longlong)), C.POINTER(C.c_int64), C.c_int]),
    "celv2_reserve_group": (C.c_int, [C.c_void_p, C.c_int]),
    "celv2_group_records": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_void_p)]),
    "celv2_clear_store": (C.c_int, [C.c_void_p]),
    "celv2_drop_frame": (C.c_int, [C.c_void_p, C.c_longlong]),
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
    "celv2_set_output": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "celv2_host_alloc": (C.c_int, [C.c_longlong, C.POINTER(C.c_void_p)]),
    "celv2_host_free": (C.c_int, [C.c_void_p]),
    "celv2_set_keep": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    # include/celv2_pruner.h
    "celv2_pruner_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "celv2_pruner_backward": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p]),
    "celv2_pruner_bce": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                   C.c_void_p]),
    "celv2_pruner_adam": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_float,
                                    C.c_float, C.c_float, C.c_float, C.c_float, C.c_int, C.c_void_p]),
    "celv2_set_pruner": (C.c_int, [C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float]),
    "celv2_set_keep_words": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "celv2_features": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "celv2_pruner_masks": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "celv2_sb_costs": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int64)]),
}

CFG_PERSISTENT, CFG_GRAPHS, CFG_PERSISTENT_OFF, CFG_INTER_CHUNK, CFG_FEATURES, CFG_ME_CELLS_L0 = 1, 2, 3, 4, 5, 10

PRUNER_FEATURES, PRUNER_OUTPUTS, PRUNER_PARAMS, PRUNER_ACTS, PRUNER_WORK = 376, 24, 56120, 23504, 20544
# keep words (include/celv2_decision.h)
KEEP_INTRA, KEEP_LEVELS, KEEP_MODES = 0x80, 0xF00, 0x1FFF0000


def keep_level(l: int) -> int:
    return 0x100 << l


def keep_mode(m: int) -> int:
    return 0x10000 << m

STAGE_NAMES = ["upload+pyramid", "phases", "me_l4", "me_l3", "me_l2", "me_l1", "me_l0", "intra", "inter",
               "finalize", "me_refine", "pruner"]


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


class _RecordPool:
    """Page-locked record arrays (celv2_host_alloc) for the records the engine copies straight into
    the caller's DecisionMap (celv2_set_output): no copy on the host, and the device-to-host copies
    run as DMA. A buffer goes back to the pool when the last array viewing it is gone."""

    def __init__(self):
        self._free: dict[int, list[int]] = {}
        self._lock = threading.Lock()
        # free bytes kept for reuse: allocating and freeing page-locked memory is slow (and
        # cudaFreeHost waits for the device), so a pipeline's maps should cycle through the pool
        self.keep_bytes = int(os.environ.get("CELV2_RECORD_POOL_BYTES", 2 << 30))
        self._kept = 0

    def take(self, count: int):
        """(records array of `count` celv2_sb_out, its address)."""
        nbytes = count * SB_OUT_DTYPE.itemsize
        with self._lock:
            lst = self._free.get(nbytes)
            ptr = lst.pop() if lst else None
            if ptr is not None:
                self._kept -= nbytes
        if ptr is None:
            p = C.c_void_p()
            _check(library().celv2_host_alloc(nbytes, C.byref(p)))
            ptr = p.value
        buf = (C.c_uint8 * nbytes).from_address(ptr)
        fin = weakref.finalize(buf, self._give, nbytes, ptr)
        fin.atexit = False  # the process's exit releases page-locked memory anyway
        return np.ctypeslib.as_array(buf).view(SB_OUT_DTYPE), ptr

    def _give(self, nbytes: int, ptr: int) -> None:
        with self._lock:
            if self._kept + nbytes <= self.keep_bytes:
                self._free.setdefault(nbytes, []).append(ptr)
                self._kept += nbytes
                return
        library().celv2_host_free(ptr)


_records = _RecordPool()


def host_array(shape, dtype) -> np.ndarray:
    """A numpy array in page-locked host memory (celv2_host_alloc), freed with its last view: what
    celv2_upload_pinned and celv2_set_output take."""
    dt = np.dtype(dtype)
    nbytes = int(np.prod(shape)) * dt.itemsize
    p = C.c_void_p()
    _check(library().celv2_host_alloc(max(1, nbytes), C.byref(p)))
    buf = (C.c_uint8 * max(1, nbytes)).from_address(p.value)
    fin = weakref.finalize(buf, library().celv2_host_free, p.value)
    fin.atexit = False
    return np.ctypeslib.as_array(buf)[:nbytes].view(dt).reshape(shape)


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
        # record arrays queued copies still write into: held until the engine is idle, so their
        # page-locked memory cannot go back to the pool while a copy targets it
        self._inflight: list = []

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
        # the rows land in dm's own page-locked records (its contents are defined once collected)
        records, ptr = _records.take(self.sb_cols * self.sb_rows)
        lib = library()
        _check(lib.celv2_set_output(self._h, 0, ptr))
        self._inflight.append(records)
        _check(lib.celv2_launch(self._h, C.byref(s), rarr, len(refs), lam, karr, src_key))
        dm.sb_size, dm.sb_cols, dm.sb_rows = self.sb_size, self.sb_cols, self.sb_rows
        dm.records = records

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
        """Publishes every row on gate as its records arrive in dm (the launch copies them straight
        into dm.records); on failure fails the gate and raises. Returns with no work pending."""
        lib = library()
        try:
            for r in self.row_order():
                if self.row_hook:
                    self.row_hook(r)
                ptr = C.c_void_p()
                _check(lib.celv2_wait_row(self._h, r, C.byref(ptr)))
                gate.publish_one(r)
            self.finish()
        except BaseException as e:
            gate.fail(e)
            if lib.celv2_finish(self._h) == E_OK:
                self._inflight.clear()
            raise

    def decide_inter(self, src, refs, qindex: int, ref_keys=None) -> DecisionMap:
        dm, gate = DecisionMap(), RowGate()
        self.launch(src, refs, qindex, dm, ref_keys)
        self.collect(dm, gate)
        return dm

    def decide_intra(self, src, qindex: int) -> DecisionMap:
        return self.decide_inter(src, [], qindex)

    # ---- device-resident path ----
    def upload(self, frame, key: int, pinned: bool = False) -> None:
        """celv2_upload; pinned=True: celv2_upload_pinned (the plane from host_array, DMA after
        return: keep it unchanged until finish())."""
        keep: list = []
        f = make_frame(frame, self.width, self.height, keep)
        if pinned:
            _check(library().celv2_upload_pinned(self._h, C.byref(f), key))
            self._inflight.extend(keep)
        else:
            _check(library().celv2_upload(self._h, C.byref(f), key))

    def reserve_group(self, frames: int) -> None:
        _check(library().celv2_reserve_group(self._h, frames))

    def launch_group(self, src_keys, ref_keys, qindex, to_host: bool = False, dms=None) -> None:
        """One batch from the frame store (celv2_launch_group). With dms (one DecisionMap per job),
        each job's records come straight into its map's page-locked records; they are defined once
        the batch is finished (finish(), group_records())."""
        n = len(src_keys)
        if dms is not None:
            if len(dms) != n:
                raise ValueError("launch_group: one DecisionMap per job")
            to_host = True
            lib = library()
            for j, dm in enumerate(dms):
                records, ptr = _records.take(self.sb_cols * self.sb_rows)
                _check(lib.celv2_set_output(self._h, j, ptr))
                self._inflight.append(records)
                dm.sb_size, dm.sb_cols, dm.sb_rows = self.sb_size, self.sb_cols, self.sb_rows
                dm.records = records
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
        self._inflight.clear()

    def clear_store(self) -> None:
        _check(library().celv2_clear_store(self._h))
        self._group_keys = set()

    def set_output(self, job: int, ptr: int) -> None:
        """celv2_set_output: the next launch copies job's records to `ptr` (page-locked memory)."""
        _check(library().celv2_set_output(self._h, job, ptr))

    def set_keep(self, job: int, keep) -> None:
        """Pruning masks for job of the next launch, one per superblock: uint8 bytes (references and
        intra, celv2_set_keep) or uint32 keep words (references, intra, block levels, intra modes,
        celv2_set_keep_words); None: the exhaustive search."""
        if keep is None:
            _check(library().celv2_set_keep_words(self._h, job, None))
            return
        words = np.asarray(keep).dtype != np.uint8
        k = np.ascontiguousarray(keep, dtype=np.uint32 if words else np.uint8)
        if k.size != self.sb_cols * self.sb_rows:
            raise ValueError("set_keep: one mask per superblock")
        fn = library().celv2_set_keep_words if words else library().celv2_set_keep
        _check(fn(self._h, job, k.ctypes.data))

    def set_pruner(self, params, ref_threshold: float = 0.5, intra_threshold: float = 0.5,
                   level_threshold: float = 0.5, mode_threshold: float = 0.5, band: float = 0.0) -> None:
        """celv2_set_pruner: the learned pruner (FP32 parameters, CELV2_PRUNER_PARAMS) scores every
        later inter frame on its own keep words; None turns it off."""
        if params is None:
            _check(library().celv2_set_pruner(self._h, None, 0.0, 0.0, 0.0, 0.0, 0.0))
            return
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != PRUNER_PARAMS:
            raise ValueError(f"set_pruner: {PRUNER_PARAMS} parameters")
        _check(library().celv2_set_pruner(self._h, p.ctypes.data, ref_threshold, intra_threshold, level_threshold,
                                          mode_threshold, band))

    def features(self, job: int = 0) -> np.ndarray:
        """The last launch's learned-pruner features of job (nsb x CELV2_PRUNER_FEATURES)."""
        out = np.empty((self.sb_cols * self.sb_rows, PRUNER_FEATURES), dtype=np.float32)
        _check(library().celv2_features(self._h, job, out.ctypes.data))
        return out

    def pruner_masks(self, job: int = 0) -> np.ndarray:
        """The keep words the pruner chose for the last launch's job (one uint32 per superblock)."""
        out = np.empty(self.sb_cols * self.sb_rows, dtype=np.uint32)
        _check(library().celv2_pruner_masks(self._h, job, out.ctypes.data))
        return out

    def sb_costs(self, job: int = 0) -> np.ndarray:
        """The last launch's per-superblock cost of the chosen partition (int64), job's."""
        out = np.empty(self.sb_cols * self.sb_rows, dtype=np.int64)
        _check(library().celv2_sb_costs(self._h, job, out.ctypes.data_as(C.POINTER(C.c_int64))))
        return out

    def drop_frame(self, key: int) -> None:
        _check(library().celv2_drop_frame(self._h, key))

    _SRC_KEYS, _TMP_KEYS = 1 << 62, 1 << 61  # store keys of decide_group's sources / unkeyed references

    def decide_group(self, srcs, refs, qindex, ref_keys=None, wait: bool = True,
                     pinned: bool = False) -> list[DecisionMap]:
        """Frames decided together, one launch per stage: the leaves of a mini-GOP as the
        reference's Pipeline::code_group (src/pipeline.cpp:328-384) holds them. Job i decides
        srcs[i] against refs[i] (nearest first); ref_keys[i] (optional) are launch's ref_keys, so a
        reference seen before under its key is not uploaded again. The maps equal separate launch /
        collect calls' maps. Inputs are copied before it returns (pinned=True: planes from host_array,
        copied by DMA afterwards -- keep them until finish()); with wait=False the records are
        defined after finish()."""
        n = len(srcs)
        if len(refs) != n or (ref_keys is not None and len(ref_keys) != n):
            raise ValueError("decide_group: one reference list (and key list) per source")
        keyed = getattr(self, "_group_keys", set())
        counter = getattr(self, "_group_counter", 0)
        need, jobs_src, jobs_refs, tmp = set(), [], [], []
        for i in range(n):
            ks = []
            for r, f in enumerate(refs[i]):
                k = None if ref_keys is None or ref_keys[i] is None else int(ref_keys[i][r])
                if k is None:
                    counter += 1
                    k = self._TMP_KEYS | counter
                    self.upload(f, k, pinned)
                    tmp.append(k)
                elif k not in keyed:
                    if k >= self._TMP_KEYS:
                        raise ValueError("decide_group: reference keys must be below 2**61")
                    self.upload(f, k, pinned)
                    keyed.add(k)
                need.add(k)
                ks.append(k)
            counter += 1
            sk = self._SRC_KEYS | counter
            self.upload(srcs[i], sk, pinned)
            jobs_src.append(sk)
            jobs_refs.append(ks)
        for k in [k for k in keyed if k not in need]:  # keyed references this group does not use
            self.drop_frame(k)
            keyed.discard(k)
        self._group_keys, self._group_counter = keyed, counter
        dms = [DecisionMap() for _ in range(n)]
        qs = qindex if isinstance(qindex, (list, tuple)) else [qindex] * n
        self.launch_group(jobs_src, jobs_refs, qs, dms=dms)
        for k in jobs_src + tmp:  # queued work still reads them; later uploads reuse the memory
            self.drop_frame(k)
        if wait:
            self.finish()
        return dms

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


def launch_multi(jobs, qindex, to_host: bool = False, dms=None) -> None:
    """One batch over engines of different frame sizes: jobs = [(engine, src_key, [ref keys])].
    Each engine's records come back with engine.group_records(k) for its k-th job here, or, with
    dms (one DecisionMap per job), straight into the maps' records (defined once finished)."""
    n = len(jobs)
    if dms is not None:
        if len(dms) != n:
            raise ValueError("launch_multi: one DecisionMap per job")
        to_host = True
        seen: dict = {}
        for (e, _, _), dm in zip(jobs, dms):
            k = seen.get(id(e), 0)
            seen[id(e)] = k + 1
            records, ptr = _records.take(e.sb_cols * e.sb_rows)
            _check(library().celv2_set_output(e._h, k, ptr))
            e._inflight.append(records)
            dm.sb_size, dm.sb_cols, dm.sb_rows = e.sb_size, e.sb_cols, e.sb_rows
            dm.records = records
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
