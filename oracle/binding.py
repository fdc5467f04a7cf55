"""ctypes bindings of the oracle libraries (TEST INFRASTRUCTURE ONLY)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from celv2_b200.records import SB_OUT_BYTES, SB_OUT_DTYPE, first_difference, records_equal  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libcelv2ref.so")

LEVELS = 5


def build(reference: bool = True) -> None:
    """make -C oracle (the reference part only where its sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE, "all" if reference else "restatement"], check=True)


def reference_available() -> bool:
    return os.path.exists(REF_LIB)


def field_dims(pw: int, ph: int):
    cols, rows = [], []
    w, h = pw, ph
    for _ in range(LEVELS):
        cols.append((w + 7) // 8)
        rows.append((h + 7) // 8)
        w //= 2
        h //= 2
    return cols, rows


def pyramid_size(pw: int, ph: int, phases: bool) -> int:
    n, w, h = 0, pw, ph
    for l in range(LEVELS):
        n += w * h * (16 if (l == 0 and phases) else 1)
        w //= 2
        h //= 2
    return n


def _u8p(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_uint8))


def _plist(planes):
    arr = (C.POINTER(C.c_uint8) * max(1, len(planes)))()
    for i, p in enumerate(planes):
        arr[i] = _u8p(p)
    return arr


class Oracle:
    """The C restatement (oracle/celv2_oracle.c)."""

    def __init__(self):
        if not os.path.exists(LIB):
            build(reference=False)
        L = self.lib = C.CDLL(LIB)
        L.oro_decide.restype = C.c_int
        L.oro_decide.argtypes = [C.POINTER(C.c_uint8), C.c_int, C.c_int, C.POINTER(C.POINTER(C.c_uint8)), C.c_int,
                                 C.c_int64, C.c_int, C.c_void_p]
        L.oro_decide_masked.restype = C.c_int
        L.oro_decide_masked.argtypes = [C.POINTER(C.c_uint8), C.c_int, C.c_int, C.POINTER(C.POINTER(C.c_uint8)),
                                        C.c_int, C.c_int64, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.oro_build_pyramid.argtypes = [C.POINTER(C.c_uint8), C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint8)]
        L.oro_me_fields.argtypes = [C.POINTER(C.c_uint8), C.POINTER(C.c_uint8), C.c_int, C.c_int,
                                    C.POINTER(C.POINTER(C.c_int32)), C.POINTER(C.POINTER(C.c_int32))]
        L.oro_intra_satd_sb.argtypes = [C.POINTER(C.c_uint8), C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.POINTER(C.c_int32)]
        L.oro_hadamard4x4.argtypes = [C.POINTER(C.c_int)]
        L.oro_subpel_px.argtypes = [C.POINTER(C.c_uint8)] + [C.c_int] * 7
        L.oro_intra_pred.argtypes = [C.POINTER(C.c_uint8)] + [C.c_int] * 10
        L.oro_dc_value.argtypes = [C.POINTER(C.c_uint8)] + [C.c_int] * 7
        L.oro_sb_block_geom.argtypes = [C.c_int] + [C.POINTER(C.c_int)] * 4
        L.oro_round_to_8bit.argtypes = [C.POINTER(C.c_uint16), C.POINTER(C.c_uint8), C.c_size_t, C.c_int]
        L.oro_me_cell.argtypes = [C.POINTER(C.c_uint8), C.POINTER(C.c_uint8), C.c_int, C.c_int, C.c_int, C.c_int,
                                  C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_int, C.c_int, C.c_int,
                                  C.POINTER(C.c_int32), C.POINTER(C.c_int32)]

    def decide(self, width: int, height: int, src_y: np.ndarray, refs_y, lam: int, threads: int = 0) -> np.ndarray:
        src_y = np.ascontiguousarray(src_y, dtype=np.uint8)
        refs_y = [np.ascontiguousarray(r, dtype=np.uint8) for r in refs_y]
        nsb = ((width + 63) // 64) * ((height + 63) // 64)
        out = np.zeros(nsb, dtype=SB_OUT_DTYPE)
        rc = self.lib.oro_decide(_u8p(src_y), width, height, _plist(refs_y), len(refs_y), int(lam), threads,
                                 out.ctypes.data_as(C.c_void_p))
        if rc != 0:
            raise ValueError("oracle rejected the arguments")
        return out

    def decide_masked(self, width: int, height: int, src_y: np.ndarray, refs_y, lam: int, keep=None,
                      threads: int = 0):
        """(records, per-superblock costs) with pruning masks (oro_decide_masked)."""
        src_y = np.ascontiguousarray(src_y, dtype=np.uint8)
        refs_y = [np.ascontiguousarray(r, dtype=np.uint8) for r in refs_y]
        nsb = ((width + 63) // 64) * ((height + 63) // 64)
        out = np.zeros(nsb, dtype=SB_OUT_DTYPE)
        cost = np.zeros(nsb, dtype=np.int64)
        k = None if keep is None else np.ascontiguousarray(keep, dtype=np.uint32)  # bytes: references + intra
        rc = self.lib.oro_decide_masked(_u8p(src_y), width, height, _plist(refs_y), len(refs_y), int(lam), threads,
                                        None if k is None else k.ctypes.data_as(C.c_void_p),
                                        out.ctypes.data_as(C.c_void_p), cost.ctypes.data_as(C.c_void_p))
        if rc != 0:
            raise ValueError("oracle rejected the arguments")
        return out, cost

    def pyramid(self, y: np.ndarray, phases: bool) -> np.ndarray:
        ph, pw = y.shape
        out = np.zeros(pyramid_size(pw, ph, phases), np.uint8)
        self.lib.oro_build_pyramid(_u8p(np.ascontiguousarray(y)), pw, ph, int(phases), _u8p(out))
        return out

    def me_fields(self, cur_y: np.ndarray, ref_y: np.ndarray):
        """[(mvx, mvy)] per level 0..4, each rows x cols int32."""
        ph, pw = cur_y.shape
        cur = self.pyramid(cur_y, False)
        ref = self.pyramid(ref_y, True)
        cols, rows = field_dims(pw, ph)
        fx = [np.zeros((rows[l], cols[l]), np.int32) for l in range(LEVELS)]
        fy = [np.zeros((rows[l], cols[l]), np.int32) for l in range(LEVELS)]
        PX = (C.POINTER(C.c_int32) * LEVELS)(*[a.ctypes.data_as(C.POINTER(C.c_int32)) for a in fx])
        PY = (C.POINTER(C.c_int32) * LEVELS)(*[a.ctypes.data_as(C.POINTER(C.c_int32)) for a in fy])
        self.lib.oro_me_fields(_u8p(cur), _u8p(ref), pw, ph, PX, PY)
        return list(zip(fx, fy))

    def intra_satd_sb(self, y: np.ndarray, sb_col: int, sb_row: int) -> np.ndarray:
        ph, pw = y.shape
        out = np.zeros((425, 13), np.int32)
        self.lib.oro_intra_satd_sb(_u8p(np.ascontiguousarray(y)), pw, ph, sb_col, sb_row,
                                   out.ctypes.data_as(C.POINTER(C.c_int32)))
        return out

    def hadamard4x4(self, d) -> int:
        arr = (C.c_int * 16)(*[int(v) for v in d])
        return self.lib.oro_hadamard4x4(arr)

    def block_geom(self, b: int):
        v = [C.c_int() for _ in range(4)]
        self.lib.oro_sb_block_geom(b, *[C.byref(x) for x in v])
        return tuple(x.value for x in v)

    def round_to_8bit(self, hy: np.ndarray, bit_depth: int = 10) -> np.ndarray:
        hy = np.ascontiguousarray(hy, dtype=np.uint16)
        out = np.zeros(hy.shape, np.uint8)
        self.lib.oro_round_to_8bit(hy.ctypes.data_as(C.POINTER(C.c_uint16)), _u8p(out), hy.size, bit_depth)
        return out


class Reference:
    """The reference's own CpuEngine and rules, compiled from its sources (oracle/_ref)."""

    def __init__(self, lambda_table):
        if not reference_available():
            raise FileNotFoundError("oracle/_ref/libcelv2ref.so was not built (reference sources absent)")
        L = self.lib = C.CDLL(REF_LIB)
        L.refx_last_error.restype = C.c_char_p
        L.refx_set_lambda.argtypes = [C.POINTER(C.c_int64)]
        L.refx_decide_ref.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_uint8), C.POINTER(C.POINTER(C.c_uint8)),
                                      C.c_int, C.c_int, C.c_void_p]
        L.refx_build_pyramid.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_uint8), C.c_int, C.POINTER(C.c_uint8)]
        L.refx_me_fields.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_uint8), C.POINTER(C.c_uint8),
                                     C.POINTER(C.c_int32)]
        L.refx_engine_new.restype = C.c_void_p
        L.refx_engine_new.argtypes = [C.c_int, C.c_int, C.c_int]
        L.refx_engine_free.argtypes = [C.c_void_p]
        L.refx_engine_decide.argtypes = [C.c_void_p, C.POINTER(C.c_uint8), C.POINTER(C.POINTER(C.c_uint8)), C.c_int,
                                         C.c_int, C.c_void_p]
        L.refx_frames_new.restype = C.c_void_p
        L.refx_frames_new.argtypes = [C.c_int, C.c_int, C.c_int, C.POINTER(C.POINTER(C.c_uint8))]
        L.refx_frames_free.argtypes = [C.c_void_p]
        L.refx_engine_decide_idx.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int), C.c_int, C.c_int]
        L.refx_round_to_8bit.argtypes = [C.c_int, C.c_int, C.POINTER(C.c_uint16), C.POINTER(C.c_uint8)]
        self.set_lambda(lambda_table)

    def set_lambda(self, table) -> None:
        arr = (C.c_int64 * 256)(*[int(v) for v in table])
        self.lib.refx_set_lambda(arr)

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise RuntimeError(self.lib.refx_last_error().decode())

    def decide_ref(self, width, height, src_y, refs_y, qindex) -> np.ndarray:
        src_y = np.ascontiguousarray(src_y, dtype=np.uint8)
        refs_y = [np.ascontiguousarray(r, dtype=np.uint8) for r in refs_y]
        nsb = ((width + 63) // 64) * ((height + 63) // 64)
        out = np.zeros(nsb, dtype=SB_OUT_DTYPE)
        self._check(self.lib.refx_decide_ref(width, height, _u8p(src_y), _plist(refs_y), len(refs_y), qindex,
                                             out.ctypes.data_as(C.c_void_p)))
        return out

    def pyramid(self, width, height, y, phases) -> np.ndarray:
        pw, ph = (width + 7) & ~7, (height + 7) & ~7
        out = np.zeros(pyramid_size(pw, ph, phases), np.uint8)
        self._check(self.lib.refx_build_pyramid(width, height, _u8p(np.ascontiguousarray(y)), int(phases), _u8p(out)))
        return out

    def me_fields(self, width, height, cur_y, ref_y):
        pw, ph = (width + 7) & ~7, (height + 7) & ~7
        cols, rows = field_dims(pw, ph)
        total = sum(2 * c * r for c, r in zip(cols, rows))
        out = np.zeros(total, np.int32)
        self._check(self.lib.refx_me_fields(width, height, _u8p(np.ascontiguousarray(cur_y)),
                                            _u8p(np.ascontiguousarray(ref_y)),
                                            out.ctypes.data_as(C.POINTER(C.c_int32))))
        res, off = [], 0
        for l in range(LEVELS):
            n = cols[l] * rows[l]
            fx = out[off : off + n].reshape(rows[l], cols[l])
            fy = out[off + n : off + 2 * n].reshape(rows[l], cols[l])
            res.append((fx, fy))
            off += 2 * n
        return res

    def engine(self, width, height, threads):
        return RefEngine(self, width, height, threads)


class RefEngine:
    """The reference CpuEngine: launch + collect of one frame per call."""

    def __init__(self, ref: Reference, width: int, height: int, threads: int):
        self.ref, self.width, self.height = ref, width, height
        self.h = ref.lib.refx_engine_new(width, height, threads)
        if not self.h:
            raise RuntimeError(ref.lib.refx_last_error().decode())
        self.frames = None

    def decide(self, src_y, refs_y, qindex, want_records=True):
        src_y = np.ascontiguousarray(src_y, dtype=np.uint8)
        refs_y = [np.ascontiguousarray(r, dtype=np.uint8) for r in refs_y]
        out = None
        if want_records:
            nsb = ((self.width + 63) // 64) * ((self.height + 63) // 64)
            out = np.zeros(nsb, dtype=SB_OUT_DTYPE)
        self.ref._check(self.ref.lib.refx_engine_decide(self.h, _u8p(src_y), _plist(refs_y), len(refs_y), qindex,
                                                        out.ctypes.data_as(C.c_void_p) if out is not None else None))
        return out

    def hold_frames(self, ys) -> None:
        """Keep these 8-bit planes inside the reference process (no copies when deciding them)."""
        ys = [np.ascontiguousarray(y, dtype=np.uint8) for y in ys]
        if self.frames:
            self.ref.lib.refx_frames_free(self.frames)
        self.frames = self.ref.lib.refx_frames_new(self.width, self.height, len(ys), _plist(ys))

    def decide_held(self, src: int, refs, qindex: int) -> None:
        arr = (C.c_int * max(1, len(refs)))(*refs)
        self.ref._check(self.ref.lib.refx_engine_decide_idx(self.h, self.frames, src, arr, len(refs), qindex))

    def close(self):
        if self.frames:
            self.ref.lib.refx_frames_free(self.frames)
            self.frames = None
        if self.h:
            self.ref.lib.refx_engine_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
