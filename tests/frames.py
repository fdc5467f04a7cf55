"""Deterministic test pictures, restated from the reference's test fixtures.

Each generator follows the reference test file cited in its docstring so the parity and
known-answer tests run on the same kinds of content as the reference's own engine tests. Planes
are returned as padded (ph x pw) uint8 arrays, as ``Frame420::y`` holds them.
"""
from __future__ import annotations

import numpy as np


def _pad(luma: np.ndarray, w: int, h: int) -> np.ndarray:
    pw, ph = (w + 7) & ~7, (h + 7) & ~7
    out = np.zeros((ph, pw), np.uint8)
    out[:h, :w] = luma
    out[:h, w:] = out[:h, w - 1 : w]
    out[h:, :] = out[h - 1 : h, :]
    return out


def scene_frame(w: int, h: int, dx: int = 0, dy: int = 0, seed: int = 1) -> np.ndarray:
    """Shading, tiles, stripes and hashed texture shifted by (dx, dy) (tests/test_frames.h:11-37)."""
    r, c = np.mgrid[0:h, 0:w].astype(np.int64)
    x, y = c - dx, r - dy
    v = 90 + (x * 3 + y * 2) // 16 % 80
    v = np.where(((x + 1000) // 48 + (y + 1000) // 40) % 4 == 0, 200 - (y & 31), v)
    v = np.where(((x + 1000) // 23) % 7 == 0, np.where((y // 3) % 2 == 1, 30, 230), v)
    hv = ((x.astype(np.uint32) * np.uint32(73856093)) ^ (y.astype(np.uint32) * np.uint32(19349663)) ^ np.uint32(seed))
    hv = hv ^ (hv >> np.uint32(13))
    hv = (hv * np.uint32(0x5BD1E995)).astype(np.uint32)
    hv = ((hv ^ (hv >> np.uint32(15))) & np.uint32(0xFF)).astype(np.int64)
    v = np.where(((x + 1000) // 64 + (y + 1000) // 64) % 5 == 2, v + hv % 31 - 15, v)
    return _pad(np.clip(v, 0, 255).astype(np.uint8), w, h)


def textured(w: int, h: int, sx: int, sy: int) -> np.ndarray:
    """Hash texture with no flat areas, cur(x, y) = prev(x + sx, y + sy) (tests/test_gpu_me.cpp:24-39)."""
    r, c = np.mgrid[0:h, 0:w].astype(np.int64)
    x, y = c + sx, r + sy
    v = ((x + 4096).astype(np.uint32) * np.uint32(2654435761)) ^ ((y + 4096).astype(np.uint32) * np.uint32(40503))
    v = v ^ (v >> np.uint32(15))
    v = (v * np.uint32(0x2C1B3C6D)).astype(np.uint32)
    v = v ^ (v >> np.uint32(12))
    out = 64 + (x + y) // 6 % 64 + (v & np.uint32(63)).astype(np.int64)
    return _pad(out.astype(np.uint8), w, h)


def smooth(w: int, h: int, sx: float, sy: float) -> np.ndarray:
    """Value noise on a 6-pixel grid, smoothstep-blended, sampled at (x + sx, y + sy)
    (tests/test_gpu_me.cpp:116-137)."""

    def level(gx, gy):
        v = ((gx + 1000).astype(np.uint32) * np.uint32(2654435761)) ^ ((gy + 1000).astype(np.uint32) * np.uint32(40503))
        v = v ^ (v >> np.uint32(15))
        v = (v * np.uint32(0x2C1B3C6D)).astype(np.uint32)
        v = v ^ (v >> np.uint32(12))
        return 40.0 + (v % np.uint32(176)).astype(np.float64)

    r, c = np.mgrid[0:h, 0:w].astype(np.float64)
    x, y = (c + sx) / 6, (r + sy) / 6
    gx, gy = np.floor(x).astype(np.int64), np.floor(y).astype(np.int64)
    ease = lambda t: t * t * (3 - 2 * t)  # noqa: E731
    tx, ty = ease(x - gx), ease(y - gy)
    v = (level(gx, gy) * (1 - tx) + level(gx + 1, gy) * tx) * (1 - ty) + (
        level(gx, gy + 1) * (1 - tx) + level(gx + 1, gy + 1) * tx
    ) * ty
    # std::lround: halves away from zero (values are positive here)
    return _pad(np.floor(v + 0.5).astype(np.uint8), w, h)


class _Lcg:
    """The LCG of tests/test_gpu_intra.cpp:24-28."""

    def __init__(self, seed: int = 12345):
        self.s = seed

    def rnd(self, n: int) -> int:
        self.s = (self.s * 1664525 + 1013904223) & 0xFFFFFFFF
        return (self.s >> 8) % n


def test_frame(w: int, h: int, lcg: _Lcg | None = None) -> np.ndarray:
    """Smooth regions, edges and LCG texture (tests/test_gpu_intra.cpp:30-41)."""
    lcg = lcg or _Lcg()
    out = np.zeros((h, w), np.int64)
    for r in range(h):
        for c in range(w):
            v = 60 + r // 3 if (c // 37) % 2 else 180 - c // 5
            if (r // 50 + c // 70) % 3 == 0:
                v += lcg.rnd(41) - 20
            out[r, c] = v
    return _pad(np.clip(out, 0, 255).astype(np.uint8), w, h)


def glyph_frame(w: int, h: int, dx: int = 0) -> np.ndarray:
    """4-colour screen-like glyphs on a flat ground (tests/test_frames.h:52-69)."""
    ink = np.array([40, 120, 200, 240], np.uint8)
    r, c = np.mgrid[0:h, 0:w].astype(np.int64)
    x = c - dx
    cx, cy = ((x % 24) + 24) % 24, r % 20
    cell = ((x + 2400) // 24 * 7 + r // 20 * 3) % 5
    v = np.zeros((h, w), np.int64)
    v = np.where((cell == 1) & ((cx == 3) | (cx == 4) | (cy == 3)), 2, v)
    box = (cell == 2) & (cx >= 4) & (cx < 16) & (cy >= 4) & (cy < 14)
    v = np.where(box, np.where((cx < 6) | (cy > 11), 3, 1), v)
    v = np.where((cell == 3) & ((cx + cy) % 6 == 0) & (cy < 16), 3, v)
    v = np.where((cell == 4) & (cx % 4 < 2) & (cy % 4 < 2), 1, v)
    return _pad(ink[v], w, h)


def noise(w: int, h: int, seed: int) -> np.ndarray:
    """Uniform random bytes (a stand-in for the mt19937 noise of tests/test_vk_kernels.cpp:27-32)."""
    rng = np.random.default_rng(seed)
    return _pad(rng.integers(0, 256, (h, w), dtype=np.uint8), w, h)
