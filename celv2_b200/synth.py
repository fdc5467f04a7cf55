"""Seeded synthetic 4:2:0 10-bit clips for the decision engine's workloads.

The reference's benchmark clips (Xiph and private anime sources) are not available, so these
generators stand in for them with the shapes, sizes and value distributions of the workloads:

* ``sinusoid_clip`` -- luma is a sum of 2-D sinusoids (periods 8-64 px, random phases and
  amplitudes, total range within 64-960) plus axis-aligned rectangles of uniform random level.
  Motion is either one global integer+quarter-pel translation per frame with each rectangle
  moving on its own, or per-region affine motion (a grid of regions, each with its own
  translation, rotation and zoom). Gaussian noise is added per frame.
* ``animation_clip`` -- flat regions of a few uniform colours with 1-px hard edges, sparse noisy
  pixels, piecewise-translational motion and an optional scene cut.

Chroma is the 2x-downsampled luma scaled by 0.5 around 512. The engine reads only the luma plane
rounded to 8 bits (``round_to_8bit``), exactly as the reference's y4m reader hands it over.
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np

__all__ = [
    "Frame",
    "round_to_8bit",
    "pad_plane",
    "sinusoid_clip",
    "animation_clip",
    "small_clip",
    "hd_clip",
    "anime_clip",
    "write_y4m",
]


@dataclass
class Frame:
    """One 4:2:0 frame: visible ``width`` x ``height``, planes padded to multiples of 8.

    ``hy`` holds the 10-bit luma (``ph`` x ``pw`` uint16), ``y`` its 8-bit rounding (the samples
    the decision engine scores), ``hu``/``hv`` the 10-bit chroma planes (may be ``None``).
    """

    width: int
    height: int
    hy: np.ndarray
    y: np.ndarray
    hu: np.ndarray | None = None
    hv: np.ndarray | None = None
    bit_depth: int = 10

    @property
    def pw(self) -> int:
        return self.y.shape[1]

    @property
    def ph(self) -> int:
        return self.y.shape[0]


def pad_plane(p: np.ndarray, w: int, h: int, pw: int, ph: int) -> np.ndarray:
    """Edge replication of the visible ``w`` x ``h`` area to ``pw`` x ``ph``
    (reference src/io/y4m.cpp:36-42)."""
    out = np.empty((ph, pw), dtype=p.dtype)
    out[:h, :w] = p[:h, :w]
    out[:h, w:] = p[:h, w - 1 : w]
    out[h:, :] = out[h - 1 : h, :]
    return out


def round_to_8bit(hy: np.ndarray, bit_depth: int = 10) -> np.ndarray:
    """``min(255, (v + (1 << (s - 1))) >> s)`` with ``s = bit_depth - 8``
    (reference src/io/y4m.cpp:28-34)."""
    if bit_depth == 8:
        return hy.astype(np.uint8)
    s = bit_depth - 8
    return np.minimum(255, (hy.astype(np.int32) + (1 << (s - 1))) >> s).astype(np.uint8)


def _make_frame(luma: np.ndarray, width: int, height: int, with_chroma: bool) -> Frame:
    pw, ph = (width + 7) & ~7, (height + 7) & ~7
    hy = pad_plane(np.clip(np.rint(luma), 0, 1023).astype(np.uint16), width, height, pw, ph)
    hu = hv = None
    if with_chroma:
        c = hy.astype(np.float32).reshape(ph // 2, 2, pw // 2, 2).mean(axis=(1, 3))
        hu = np.clip(np.rint(512 + 0.5 * (c - 512)), 0, 1023).astype(np.uint16)
        hv = hu.copy()
    return Frame(width, height, hy, round_to_8bit(hy), hu, hv)


def sinusoid_clip(
    width: int,
    height: int,
    frames: int,
    seed: int,
    *,
    sinusoids: int = 4,
    rects: int = 3,
    global_motion: float = 6.0,
    rect_motion: float = 10.0,
    affine_regions: tuple[int, int] | None = None,
    affine_motion: float = 24.0,
    noise_sigma: float = 3.0,
    with_chroma: bool = False,
) -> list[Frame]:
    """Sinusoids + rectangles with global (or per-region affine) motion; see the module doc."""
    rng = np.random.default_rng(seed)
    periods = rng.uniform(8.0, 64.0, sinusoids)
    angles = rng.uniform(0.0, np.pi, sinusoids)
    phases = rng.uniform(0.0, 2 * np.pi, sinusoids)
    amps = rng.uniform(0.3, 1.0, sinusoids)
    amps *= 380.0 / amps.sum()  # 512 +- 380 stays inside 64..960 with the rectangles clipped below
    kx = np.cos(angles) * 2 * np.pi / periods
    ky = np.sin(angles) * 2 * np.pi / periods
    rw = rng.integers(max(8, width // 16), max(9, width // 4), rects)
    rh = rng.integers(max(8, height // 16), max(9, height // 4), rects)
    rx0 = rng.uniform(0, width, rects)
    ry0 = rng.uniform(0, height, rects)
    rlevel = rng.uniform(96.0, 928.0, rects)
    if affine_regions:
        gx, gy = affine_regions
        nreg = gx * gy
        trans = rng.uniform(-affine_motion, affine_motion, (nreg, 2))
        rot = rng.uniform(-0.01, 0.01, nreg)  # radians per frame
        zoom = rng.uniform(-0.01, 0.01, nreg)  # relative scale per frame
    def render(r0: int, r1: int, t: int, gpos: np.ndarray, rpos: np.ndarray) -> np.ndarray:
        """Rows r0 .. r1 of frame t before the noise (every sample depends on its position only)."""
        yy, xx = np.mgrid[r0:r1, 0:width].astype(np.float64)
        if affine_regions:
            # each pixel's region; its content comes from the region's affine map at frame t
            reg = (np.minimum(yy * gy // height, gy - 1) * gx + np.minimum(xx * gx // width, gx - 1)).astype(int)
            cx = (np.minimum(xx * gx // width, gx - 1) + 0.5) * width / gx
            cy = (np.minimum(yy * gy // height, gy - 1) + 0.5) * height / gy
            a = rot[reg] * t
            s = 1.0 + zoom[reg] * t
            dx, dy = xx - cx, yy - cy
            sx = (np.cos(a) * dx - np.sin(a) * dy) * s + cx - trans[reg, 0] * t
            sy = (np.sin(a) * dx + np.cos(a) * dy) * s + cy - trans[reg, 1] * t
        else:
            sx, sy = xx - gpos[0], yy - gpos[1]
        v = np.full((r1 - r0, width), 512.0)
        for k in range(sinusoids):
            v += amps[k] * np.sin(kx[k] * sx + ky[k] * sy + phases[k])
        for k in range(rects):
            x0 = rx0[k] + rpos[k, 0]
            y0 = ry0[k] + rpos[k, 1]
            m = (sx >= x0) & (sx < x0 + rw[k]) & (sy >= y0) & (sy < y0 + rh[k])
            v[m] = rlevel[k]
        return v

    # row bands on threads (numpy releases the GIL inside the array arithmetic); the noise is drawn
    # for the whole frame in order, so the clip does not depend on the band count
    bands = max(1, min(16, os.cpu_count() or 1, height // 64))
    edges = [height * i // bands for i in range(bands + 1)]
    gpos = np.zeros(2)
    rpos = np.zeros((rects, 2))
    out = []
    with ThreadPoolExecutor(bands) as pool:
        for t in range(frames):
            if t > 0:
                gpos += np.round(rng.uniform(-global_motion, global_motion, 2) * 4) / 4
                rpos += np.round(rng.uniform(-rect_motion, rect_motion, (rects, 2)) * 4) / 4
            parts = pool.map(lambda i: render(edges[i], edges[i + 1], t, gpos.copy(), rpos.copy()), range(bands))
            v = np.concatenate(list(parts), axis=0)
            v += rng.normal(0.0, noise_sigma, v.shape)
            out.append(_make_frame(np.clip(v, 64, 960), width, height, with_chroma))
    return out


def animation_clip(
    width: int,
    height: int,
    frames: int,
    seed: int,
    *,
    colours: int | tuple[int, int] = (8, 24),
    pieces: tuple[int, int] = (4, 3),
    motion: float = 48.0,
    noisy_fraction: float = 0.005,
    noise_sigma: float = 1.0,
    scene_cut: int | None = None,
    with_chroma: bool = False,
) -> list[Frame]:
    """Flat colour regions with 1-px hard edges (40 rectangles and ellipses drawn over a background,
    each of one palette colour), sparse noisy pixels, piecewise-translational motion (a grid of
    `pieces` regions, each moving by its own whole-pel velocity, up to `motion` px per frame) and an
    optional scene cut (a new palette, new shapes and new velocities from frame `scene_cut` on).
    `colours`: the palette size, or a (low, high) range it is drawn from per scene."""
    rng = np.random.default_rng(seed)
    px, py = pieces

    def scene(r: np.random.Generator):
        n = colours if isinstance(colours, int) else int(r.integers(colours[0], colours[1] + 1))
        pal = r.uniform(64.0, 960.0, n)
        nshapes = 40
        shapes = np.stack(
            [
                r.uniform(-width * 0.2, width * 1.2, nshapes),
                r.uniform(-height * 0.2, height * 1.2, nshapes),
                r.uniform(width * 0.03, width * 0.3, nshapes),
                r.uniform(height * 0.03, height * 0.3, nshapes),
                r.integers(0, n, nshapes).astype(float),
                r.integers(0, 2, nshapes).astype(float),
            ],
            axis=1,
        )
        vel = r.uniform(-motion, motion, (px * py, 2)).round()
        return pal, shapes, vel

    # piece k covers columns xs[k % px] .. xs[k % px + 1] and rows ys[k // px] .. ys[k // px + 1]
    xs = [-(-i * width // px) for i in range(px + 1)]
    ys = [-(-j * height // py) for j in range(py + 1)]
    pal, shapes, vel = scene(rng)
    out = []
    t0 = 0
    for t in range(frames):
        if scene_cut is not None and t == scene_cut:
            pal, shapes, vel = scene(rng)
            t0 = t
        dt = t - t0
        v = np.full((height, width), pal[0])
        for k in range(px * py):
            ax0, ax1, ay0, ay1 = xs[k % px], xs[k % px + 1], ys[k // px], ys[k // px + 1]
            ox, oy = vel[k, 0] * dt, vel[k, 1] * dt  # the piece shows the scene at (x - ox, y - oy)
            for x0, y0, w, h, c, ell in shapes:
                # the shape's extent in frame coordinates, one pixel of slack, clipped to the piece
                lo_x, hi_x = (x0 - w, x0 + w) if ell else (x0, x0 + w)
                lo_y, hi_y = (y0 - h, y0 + h) if ell else (y0, y0 + h)
                bx0, bx1 = max(ax0, int(np.floor(lo_x + ox)) - 1), min(ax1, int(np.ceil(hi_x + ox)) + 1)
                by0, by1 = max(ay0, int(np.floor(lo_y + oy)) - 1), min(ay1, int(np.ceil(hi_y + oy)) + 1)
                if bx0 >= bx1 or by0 >= by1:
                    continue
                sx = np.arange(bx0, bx1, dtype=np.float64)[None, :] - ox
                sy = np.arange(by0, by1, dtype=np.float64)[:, None] - oy
                if ell:
                    m = ((sx - x0) / w) ** 2 + ((sy - y0) / h) ** 2 < 1.0
                else:
                    m = (sx >= x0) & (sx < x0 + w) & (sy >= y0) & (sy < y0 + h)
                v[by0:by1, bx0:bx1][m] = pal[int(c)]
        noisy = rng.random(v.shape) < noisy_fraction
        v[noisy] += rng.normal(0.0, noise_sigma, int(noisy.sum()))
        out.append(_make_frame(v, width, height, with_chroma))
    return out


def small_clip(seed: int = 1, frames: int = 8) -> list[Frame]:
    """416x240, 8 frames: 4 sinusoids, 3 rectangles, global motion +-6 px, sigma 3."""
    return sinusoid_clip(416, 240, frames, seed, sinusoids=4, rects=3, global_motion=6.0, rect_motion=10.0,
                         noise_sigma=3.0)


def anime_clip(seed: int = 1, frames: int = 65, width: int = 3840, height: int = 2160,
               scene_cut: int | None = 33) -> list[Frame]:
    """3840x2160 animation-like content: 8-24 flat colours per scene, 1-px hard edges, 0.5% of
    pixels with noise sigma 1, piecewise-translational motion up to +-48 px, a scene cut at
    frame 33."""
    return animation_clip(width, height, frames, seed, colours=(8, 24), motion=48.0, noisy_fraction=0.005,
                          noise_sigma=1.0, scene_cut=scene_cut)


def hd_clip(seed: int = 1, frames: int = 17, width: int = 1920, height: int = 1080) -> list[Frame]:
    """1920x1080, 17 frames: 8 sinusoids, 12 rectangles, per-region affine motion up to +-24 px,
    sigma 4."""
    return sinusoid_clip(width, height, frames, seed, sinusoids=8, rects=12, affine_regions=(4, 3),
                         affine_motion=24.0, rect_motion=24.0, noise_sigma=4.0)


def write_y4m(path: str, frames: list[Frame], fps: int = 30) -> None:
    """A C420p10 y4m of the visible area (16-bit little-endian samples)."""
    f0 = frames[0]
    with open(path, "wb") as fh:
        fh.write(f"YUV4MPEG2 W{f0.width} H{f0.height} F{fps}:1 Ip A1:1 C420p10 XYSCSS=420P10\n".encode())
        cw, ch = (f0.width + 1) // 2, (f0.height + 1) // 2
        for f in frames:
            fh.write(b"FRAME\n")
            fh.write(np.ascontiguousarray(f.hy[: f.height, : f.width]).astype("<u2").tobytes())
            for c in (f.hu, f.hv):
                plane = c[:ch, :cw] if c is not None else np.full((ch, cw), 512, np.uint16)
                fh.write(np.ascontiguousarray(plane).astype("<u2").tobytes())
