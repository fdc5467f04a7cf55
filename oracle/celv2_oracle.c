/* celv2_oracle.c: CPU restatement of the reference decision engine (see celv2_oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine, never part of the product path.
 *
 * Reference files restated (paths inside the Stou-1/celv2 tree):
 *   src/gpu/intra_common.h  - clamped sample access, intra predictors, Hadamard SATD, mode bits
 *   src/gpu/inter_common.h  - quarter-pel filter, pyramid downsample, SAD, motion search and
 *                             refinement, MV candidates, compound
 *   src/gpu/sb_blocks.h     - the 425 candidate blocks of a 64x64 superblock
 *   src/gpu/kernels_ref.cpp - pyramid build, per-level motion search, per-block best choice,
 *                             bottom-up partition choice
 *   src/gpu/cpu_engine.cpp  - field sizes and the level-by-level order of the search
 *   src/io/y4m.cpp          - 8-bit rounding and edge padding of the input
 * The per-block choices are evaluated block by block and the partition choice runs bottom-up over
 * a table of square costs; the reference reaches the same blocks through a recursion
 * (kernels_ref.cpp:125-198) that evaluates each of them exactly once, so the results are equal. */
#include "celv2_oracle.h"

#include <limits.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ---- Constants (src/gpu/inter_common.h:11-55,140; src/gpu/intra_common.h:32-42) ---- */
enum {
  kPhases = 16,
  kMeRange = 8, /* every level, level 0 included (kMeRange0) */
  kMeLevels = CELV2_ME_LEVELS,
  kInterBits = 3,
  kIntraInInterBits = 32,
  kMePenalty = 4,
  kSubpelPenalty = 16,
  kPartBits = 2,
  kMaxBlockSize = 32,
  kMaxInterBlockSize = 64,
  kNumModes = CELV2_NUM_MODES,
  kBlocks = CELV2_SB_BLOCKS,
};

/* ---- Planes (src/gpu/intra_common.h:11-26) ---- */
typedef struct {
  const uint8_t* p;
  int stride, w, h;
  size_t phase; /* distance between quarter-pel phase planes; 0: whole pels only */
} plane_t;

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : v > hi ? hi : v; }

/* Plane::at: the sample at (y, x), coordinates clamped into the plane. */
static inline int at(const plane_t* s, int y, int x) {
  return s->p[(size_t)clampi(y, 0, s->h - 1) * s->stride + clampi(x, 0, s->w - 1)];
}

/* Plane::at_q: (y + qy / 4, x + qx / 4) in quarter pels, read from phase (qy & 3) * 4 + (qx & 3) at
 * the clamped whole-pel position (the phase planes hold the value at the clamped position). */
static inline int at_q(const plane_t* s, int y, int x, int qy, int qx) {
  const uint8_t* base = s->p + (size_t)((qy & 3) * 4 + (qx & 3)) * s->phase;
  const int yy = clampi(y + (qy >> 2), 0, s->h - 1), xx = clampi(x + (qx >> 2), 0, s->w - 1);
  return base[(size_t)yy * s->stride + xx];
}

/* ---- Input conditioning (src/io/y4m.cpp:28-42) ---- */
void oro_round_to_8bit(const uint16_t* hi, uint8_t* lo, size_t n, int bit_depth) {
  if (bit_depth <= 8) {
    for (size_t i = 0; i < n; i++) lo[i] = (uint8_t)hi[i];
    return;
  }
  const int shift = bit_depth - 8, half = 1 << (shift - 1);
  for (size_t i = 0; i < n; i++) {
    const int v = (hi[i] + half) >> shift;
    lo[i] = (uint8_t)(v > 255 ? 255 : v);
  }
}

void oro_pad_plane(uint8_t* p, int stride, int w, int h, int pw, int ph) {
  for (int r = 0; r < h; r++)
    for (int c = w; c < pw; c++) p[(size_t)r * stride + c] = p[(size_t)r * stride + w - 1];
  for (int r = h; r < ph; r++) memcpy(p + (size_t)r * stride, p + (size_t)(h - 1) * stride, (size_t)pw);
}

/* ---- Hadamard SATD (src/gpu/intra_common.h:131-146) ---- */
int oro_hadamard4x4(const int* d) {
  int t[16];
  for (int r = 0; r < 4; r++) {
    const int* q = d + 4 * r;
    const int s01 = q[0] + q[1], d01 = q[0] - q[1], s23 = q[2] + q[3], d23 = q[2] - q[3];
    t[4 * r + 0] = s01 + s23;
    t[4 * r + 1] = d01 + d23;
    t[4 * r + 2] = s01 - s23;
    t[4 * r + 3] = d01 - d23;
  }
  int sum = 0;
  for (int c = 0; c < 4; c++) {
    const int s01 = t[c] + t[4 + c], d01 = t[c] - t[4 + c];
    const int s23 = t[8 + c] + t[12 + c], d23 = t[8 + c] - t[12 + c];
    const int v0 = s01 + s23, v1 = d01 + d23, v2 = s01 - s23, v3 = d01 - d23;
    sum += abs(v0) + abs(v1) + abs(v2) + abs(v3);
  }
  return sum;
}

/* ---- Quarter-pel filter (src/gpu/inter_common.h:13-33) ----
 * AV2's EIGHTTAP_REGULAR rows at the quarter phases, horizontal sums unrounded, one rounding. */
static const int kTaps[4][8] = {{0, 0, 0, 128, 0, 0, 0, 0},
                                {0, 2, -14, 110, 38, -10, 2, 0},
                                {0, 2, -14, 76, 76, -14, 2, 0},
                                {0, 2, -10, 38, 110, -14, 2, 0}};

static int subpel(const plane_t* s, int y, int x, int qy, int qx) {
  int v = 0;
  for (int i = 0; i < 8; i++) {
    if (!kTaps[qy][i]) continue;
    int row = 0;
    for (int j = 0; j < 8; j++) row += kTaps[qx][j] * at(s, y + i - 3, x + j - 3);
    v += kTaps[qy][i] * row;
  }
  v = (v + (1 << 13)) >> 14;
  return v < 0 ? 0 : v > 255 ? 255 : v;
}

int oro_subpel_px(const uint8_t* p, int stride, int w, int h, int y, int x, int qy, int qx) {
  const plane_t s = {p, stride, w, h, 0};
  return subpel(&s, y, x, qy, qx);
}

/* ---- Pyramid (src/gpu/kernels_ref.cpp:213-238, src/gpu/inter_common.h:91-94) ---- */
void oro_pyr_layout(int pw, int ph, int phases, oro_pyr* L) {
  size_t off = 0;
  L->w[0] = pw, L->h[0] = ph;
  for (int l = 1; l < kMeLevels; l++) L->w[l] = L->w[l - 1] / 2, L->h[l] = L->h[l - 1] / 2;
  L->phase = phases ? (size_t)pw * ph : 0;
  for (int l = 0; l < kMeLevels; l++) {
    L->off[l] = off;
    off += (size_t)L->w[l] * L->h[l] * (l == 0 && phases ? kPhases : 1);
  }
  L->total = off;
}

void oro_build_pyramid(const uint8_t* y, int pw, int ph, int phases, uint8_t* buf) {
  oro_pyr L;
  oro_pyr_layout(pw, ph, phases, &L);
  const size_t n = (size_t)pw * ph;
  memcpy(buf, y, n);
  if (phases) {
    const plane_t s = {y, pw, pw, ph, 0};
    for (int k = 1; k < kPhases; k++) {
      uint8_t* dst = buf + (size_t)k * n;
#pragma omp parallel for schedule(static)
      for (int r = 0; r < ph; r++)
        for (int c = 0; c < pw; c++) dst[(size_t)r * pw + c] = (uint8_t)subpel(&s, r, c, k / 4, k % 4);
    }
  }
  for (int l = 1; l < kMeLevels; l++) {
    const plane_t up = {buf + L.off[l - 1], L.w[l - 1], L.w[l - 1], L.h[l - 1], 0};
    uint8_t* dst = buf + L.off[l];
    for (int r = 0; r < L.h[l]; r++)
      for (int c = 0; c < L.w[l]; c++)
        dst[(size_t)r * L.w[l] + c] = (uint8_t)((at(&up, 2 * r, 2 * c) + at(&up, 2 * r, 2 * c + 1) +
                                                 at(&up, 2 * r + 1, 2 * c) + at(&up, 2 * r + 1, 2 * c + 1) + 2) >> 2);
  }
}

/* ---- Motion search (src/gpu/inter_common.h:96-193) ---- */
static int sad8(const plane_t* cur, int x, int y, const plane_t* ref, int mvx, int mvy) {
  int sad = 0;
  for (int i = 0; i < 8; i++)
    for (int j = 0; j < 8; j++) sad += abs(at(cur, y + i, x + j) - at(ref, y + i + mvy, x + j + mvx));
  return sad;
}

/* me_search: the +-range window around (px, py) in dy-major raster order, SAD plus kMePenalty per
 * pel of distance, first strict minimum. */
static int me_search(const plane_t* cur, const plane_t* ref, int bx, int by, int px, int py, int range, int* mvx,
                     int* mvy) {
  int best = INT_MAX;
  *mvx = px, *mvy = py;
  for (int dy = -range; dy <= range; dy++)
    for (int dx = -range; dx <= range; dx++) {
      const int s = sad8(cur, bx * 8, by * 8, ref, px + dx, py + dy) + kMePenalty * (abs(dx) + abs(dy));
      if (s < best) best = s, *mvx = px + dx, *mvy = py + dy;
    }
  return best;
}

/* satd8_q: 8x8 SATD against the quarter-pel prediction at (qmx, qmy). */
static int satd8_q(const plane_t* cur, int x, int y, const plane_t* ref, int qmx, int qmy) {
  int total = 0;
  for (int ty = 0; ty < 8; ty += 4)
    for (int tx = 0; tx < 8; tx += 4) {
      int d[16];
      for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
          d[4 * i + j] = at(cur, y + ty + i, x + tx + j) - at_q(ref, y + ty + i, x + tx + j, qmy, qmx);
      total += oro_hadamard4x4(d);
    }
  return total;
}

/* me_refine (src/gpu/inter_common.h:141-154): half-pel then quarter-pel, centre first, a move
 * pays kSubpelPenalty, first strict minimum over the 8 neighbours in dy-major order. */
static void me_refine(const plane_t* cur, const plane_t* ref, int bx, int by, int* mvx, int* mvy) {
  int cx = *mvx * 4, cy = *mvy * 4;
  for (int step = 2; step >= 1; step--) {
    int best = satd8_q(cur, bx * 8, by * 8, ref, cx, cy), nx = cx, ny = cy;
    for (int dy = -1; dy <= 1; dy++)
      for (int dx = -1; dx <= 1; dx++) {
        if (!dx && !dy) continue;
        const int s = satd8_q(cur, bx * 8, by * 8, ref, cx + dx * step, cy + dy * step) + kSubpelPenalty;
        if (s < best) best = s, nx = cx + dx * step, ny = cy + dy * step;
      }
    cx = nx, cy = ny;
  }
  *mvx = cx, *mvy = cy;
}

/* me_cell (src/gpu/inter_common.h:162-193): the two best distinct centres (by SAD) among the
 * coarser MV under the cell, its left / right / above / below neighbours and zero, each scaled
 * by 2; the search around the second replaces the first's result only if strictly cheaper. */
static void me_cell(const plane_t* cur, const plane_t* ref, int bx, int by, const int32_t* pmx, const int32_t* pmy,
                    int pcols, int prows, int* mvx, int* mvy) {
  int px = 0, py = 0, px2 = 0, py2 = 0, two = 0;
  if (pmx) {
    static const int ox[5] = {0, -1, 1, 0, 0}, oy[5] = {0, 0, 0, -1, 1};
    int best = INT_MAX, second = INT_MAX;
    for (int k = 0; k < 6; k++) {
      int cx = 0, cy = 0; /* k == 5: zero */
      if (k < 5) {
        const int qx = clampi(bx / 2 + ox[k], 0, pcols - 1), qy = clampi(by / 2 + oy[k], 0, prows - 1);
        cx = 2 * pmx[qy * pcols + qx], cy = 2 * pmy[qy * pcols + qx];
      }
      if ((k > 0 && cx == px && cy == py) || (two && cx == px2 && cy == py2)) continue;
      const int s = sad8(cur, bx * 8, by * 8, ref, cx, cy);
      if (s < best) {
        if (k > 0) second = best, px2 = px, py2 = py, two = 1;
        best = s, px = cx, py = cy;
      } else if (s < second) {
        second = s, px2 = cx, py2 = cy, two = 1;
      }
    }
  }
  const int cost = me_search(cur, ref, bx, by, px, py, kMeRange, mvx, mvy);
  if (two) {
    int mx2, my2;
    if (me_search(cur, ref, bx, by, px2, py2, kMeRange, &mx2, &my2) < cost) *mvx = mx2, *mvy = my2;
  }
}

int oro_me_cell(const uint8_t* cur, const uint8_t* ref, int stride, int w, int h, int bx, int by, const int32_t* pmx,
                const int32_t* pmy, int pcols, int prows, int level0, int32_t* mvx, int32_t* mvy) {
  const plane_t c = {cur, stride, w, h, 0}, r = {ref, stride, w, h, 0};
  int mx, my;
  me_cell(&c, &r, bx, by, pmx, pmy, pcols, prows, &mx, &my);
  (void)level0;
  *mvx = mx, *mvy = my;
  return 0;
}

void oro_field_dims(int pw, int ph, int cols[CELV2_ME_LEVELS], int rows[CELV2_ME_LEVELS]) {
  int w = pw, h = ph;
  for (int l = 0; l < kMeLevels; l++) {
    cols[l] = (w + 7) / 8, rows[l] = (h + 7) / 8;
    w /= 2, h /= 2;
  }
}

/* The search of one reference, coarsest level first (src/gpu/kernels_ref.cpp:240-251 per row,
 * src/gpu/cpu_engine.cpp:68-83 level by level: a level reads all of the coarser one). */
void oro_me_fields(const uint8_t* cur_pyr, const uint8_t* ref_pyr, int pw, int ph, int32_t* mvx[CELV2_ME_LEVELS],
                   int32_t* mvy[CELV2_ME_LEVELS]) {
  oro_pyr Lc, Lr;
  oro_pyr_layout(pw, ph, 0, &Lc);
  oro_pyr_layout(pw, ph, 1, &Lr);
  int cols[kMeLevels], rows[kMeLevels];
  oro_field_dims(pw, ph, cols, rows);
  for (int l = kMeLevels - 1; l >= 0; l--) {
    const plane_t cur = {cur_pyr + Lc.off[l], Lc.w[l], Lc.w[l], Lc.h[l], 0};
    const plane_t ref = {ref_pyr + Lr.off[l], Lr.w[l], Lr.w[l], Lr.h[l], l == 0 ? Lr.phase : 0};
    const int top = l == kMeLevels - 1;
#pragma omp parallel for schedule(dynamic, 1)
    for (int by = 0; by < rows[l]; by++)
      for (int bx = 0; bx < cols[l]; bx++) {
        int mx, my;
        me_cell(&cur, &ref, bx, by, top ? NULL : mvx[l + 1], top ? NULL : mvy[l + 1], top ? 0 : cols[l + 1],
                top ? 0 : rows[l + 1], &mx, &my);
        if (l == 0) me_refine(&cur, &ref, bx, by, &mx, &my);
        mvx[l][by * cols[l] + bx] = mx, mvy[l][by * cols[l] + bx] = my;
      }
  }
}

/* ---- Superblock geometry (src/gpu/sb_blocks.h:12-37) ---- */
static int level_offset(int level) { return ((1 << (2 * level)) - 1) / 3; }

void oro_sb_block_geom(int b, int* x, int* y, int* w, int* h) {
  const int sq = b / 5, kind = b % 5;
  int level = 0;
  while (level < 3 && sq >= level_offset(level + 1)) level++;
  const int idx = sq - level_offset(level), n = 1 << level, size = 64 >> level, half = size / 2;
  const int sx = (idx % n) * size, sy = (idx / n) * size;
  *x = sx, *y = sy, *w = size, *h = size;
  if (kind == 1 || kind == 2) *h = half, *y = sy + (kind == 2 ? half : 0);
  if (kind == 3 || kind == 4) *w = half, *x = sx + (kind == 4 ? half : 0);
}

/* ---- Intra prediction from source neighbours (src/gpu/intra_common.h:32-128) ---- */
static int mode_bits(int mode) { return mode == 0 ? 1 : mode < 4 ? 3 : 9; }

static int edge_above(const plane_t* s, int x, int y, int k) {
  if (y == 0) return 128;
  if (k < 0 && x == 0) return at(s, y - 1, x);
  return at(s, y - 1, x + k);
}
static int edge_left(const plane_t* s, int x, int y, int k) {
  if (x == 0) return 128;
  if (k < 0 && y == 0) return at(s, y, x - 1);
  return at(s, y + k, x - 1);
}

static int dr_derivative(int a) { return a == 23 ? 151 : a == 45 ? 64 : 27; }

/* dr_prediction z1 / z2 / z3 without edge filter or upsampling (intra_common.h:61-85). */
static int dir_pred(const plane_t* s, int x, int y, int w, int h, int angle, int i, int j) {
  const int last = w + h - 1;
  if (angle < 90) {
    const int pos = (i + 1) * dr_derivative(angle), base = (pos >> 6) + j, shift = (pos & 63) >> 1;
    const int a0 = edge_above(s, x, y, base < last ? base : last);
    const int a1 = edge_above(s, x, y, base + 1 < last ? base + 1 : last);
    return (a0 * (32 - shift) + a1 * shift + 16) >> 5;
  }
  if (angle > 180) {
    const int pos = (j + 1) * dr_derivative(270 - angle), base = (pos >> 6) + i, shift = (pos & 63) >> 1;
    const int l0 = edge_left(s, x, y, base < last ? base : last);
    const int l1 = edge_left(s, x, y, base + 1 < last ? base + 1 : last);
    return (l0 * (32 - shift) + l1 * shift + 16) >> 5;
  }
  const int px = (j << 6) - (i + 1) * dr_derivative(180 - angle);
  const int bx = px >= 0 ? px >> 6 : -((-px + 63) >> 6);
  if (bx >= -1) {
    const int shift = (px - bx * 64) >> 1;
    return (edge_above(s, x, y, bx) * (32 - shift) + edge_above(s, x, y, bx + 1) * shift + 16) >> 5;
  }
  const int py = (i << 6) - (j + 1) * dr_derivative(angle - 90);
  const int by = py >= 0 ? py >> 6 : -((-py + 63) >> 6);
  const int shift = (py - by * 64) >> 1;
  const int b0 = by < -1 ? -1 : by, b1 = by + 1 < -1 ? -1 : by + 1;
  return (edge_left(s, x, y, b0) * (32 - shift) + edge_left(s, x, y, b1) * shift + 16) >> 5;
}

/* intra_pred (intra_common.h:89-118): modes 1..12; DC is handled by the caller. */
static int intra_pred(const plane_t* s, int x, int y, int w, int h, int mode, int i, int j) {
  const int has_a = y > 0, has_l = x > 0;
  switch (mode) {
    case 1: return has_a ? at(s, y - 1, x + j) : 128;
    case 2: return has_l ? at(s, y + i, x - 1) : 128;
    case 3: {
      const int a = has_a ? at(s, y - 1, x + j) : 128, l = has_l ? at(s, y + i, x - 1) : 128;
      const int tr = has_a ? at(s, y - 1, x + w - 1) : 128, bl = has_l ? at(s, y + h - 1, x - 1) : 128;
      const int den = w + h + 2, num = (h - i) * a + (i + 1) * bl + (w - j) * l + (j + 1) * tr;
      return (num + den / 2) / den;
    }
    case 4: return ((h - 1 - i) * edge_above(s, x, y, j) + (i + 1) * edge_left(s, x, y, h - 1) + h / 2) / h;
    case 5: return ((w - 1 - j) * edge_left(s, x, y, i) + (j + 1) * edge_above(s, x, y, w - 1) + w / 2) / w;
    case 6: {
      const int a = edge_above(s, x, y, j), l = edge_left(s, x, y, i), tl = edge_above(s, x, y, -1);
      const int base = a + l - tl, pa = abs(base - a), pl = abs(base - l), ptl = abs(base - tl);
      return pl <= pa && pl <= ptl ? l : pa <= ptl ? a : tl;
    }
    default: {
      static const int angles[6] = {45, 67, 113, 135, 157, 203};
      if (mode >= 7 && mode <= 12) return dir_pred(s, x, y, w, h, angles[mode - 7], i, j);
      return -1;
    }
  }
}

static int dc_value(const plane_t* s, int x, int y, int w, int h) {
  int sum = 0, n = 0;
  if (y > 0)
    for (int j = 0; j < w; j++) sum += at(s, y - 1, x + j), n++;
  if (x > 0)
    for (int i = 0; i < h; i++) sum += at(s, y + i, x - 1), n++;
  return n ? (sum + n / 2) / n : 128;
}

int oro_intra_pred(const uint8_t* p, int stride, int w, int h, int x, int y, int bw, int bh, int mode, int i, int j) {
  const plane_t s = {p, stride, w, h, 0};
  return intra_pred(&s, x, y, bw, bh, mode, i, j);
}
int oro_dc_value(const uint8_t* p, int stride, int w, int h, int x, int y, int bw, int bh) {
  const plane_t s = {p, stride, w, h, 0};
  return dc_value(&s, x, y, bw, bh);
}

/* block_mode_satd (intra_common.h:149-163). */
static int64_t block_mode_satd(const plane_t* s, int x, int y, int w, int h, int mode) {
  const int dc = mode == 0 ? dc_value(s, x, y, w, h) : 0;
  int64_t total = 0;
  for (int ty = 0; ty < h; ty += 4)
    for (int tx = 0; tx < w; tx += 4) {
      int d[16];
      for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
          const int p = mode == 0 ? dc : intra_pred(s, x, y, w, h, mode, ty + i, tx + j);
          d[4 * i + j] = at(s, y + ty + i, x + tx + j) - p;
        }
      total += oro_hadamard4x4(d);
    }
  return total;
}

void oro_intra_satd_sb(const uint8_t* src_y, int pw, int ph, int sb_col, int sb_row, int32_t* satd) {
  const plane_t s = {src_y, pw, pw, ph, 0};
  for (int b = 0; b < kBlocks; b++)
    for (int m = 0; m < kNumModes; m++) {
      int x, y, w, h;
      oro_sb_block_geom(b, &x, &y, &w, &h);
      satd[b * kNumModes + m] = b < 5 ? 0 : (int32_t)block_mode_satd(&s, sb_col * 64 + x, sb_row * 64 + y, w, h, m);
    }
}

/* ---- Inter candidates (src/gpu/inter_common.h:57-89,199-235) ---- */
static int mv_cells(int x, int y, int w, int h) { return ((x + w - 1) / 8 - x / 8 + 1) * ((y + h - 1) / 8 - y / 8 + 1); }

/* Field index of candidate k of block (x, y, w, h): the covered cells in raster order, then the
 * left, above, right, below, above-left, above-right, below-left and below-right neighbours,
 * clamped into the field. */
static int candidate_index(int x, int y, int w, int h, int k, int cols, int rows) {
  const int cells = mv_cells(x, y, w, h), cw = (x + w - 1) / 8 - x / 8 + 1;
  int cx = x / 8 + k % cw, cy = y / 8 + k / cw;
  if (k >= cells) {
    const int n = k - cells;
    const int l = x / 8 - 1, r = (x + w) / 8, t = y / 8 - 1, b = (y + h) / 8;
    cx = (n == 0 || n == 4 || n == 6) ? l : (n == 2 || n == 5 || n == 7) ? r : x / 8;
    cy = (n == 1 || n == 4 || n == 5) ? t : (n == 3 || n == 6 || n == 7) ? b : y / 8;
  }
  return clampi(cy, 0, rows - 1) * cols + clampi(cx, 0, cols - 1);
}

static int repeated(const int32_t* fx, const int32_t* fy, int cols, int rows, int x, int y, int w, int h, int k) {
  const int i = candidate_index(x, y, w, h, k, cols, rows);
  for (int j = 0; j < k; j++) {
    const int ij = candidate_index(x, y, w, h, j, cols, rows);
    if (fx[ij] == fx[i] && fy[ij] == fy[i]) return 1;
  }
  return 0;
}

static int64_t block_inter_satd(const plane_t* cur, const plane_t* ref, int x, int y, int w, int h, int mvx, int mvy) {
  int64_t total = 0;
  for (int ty = 0; ty < h; ty += 4)
    for (int tx = 0; tx < w; tx += 4) {
      int d[16];
      for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
          d[4 * i + j] = at(cur, y + ty + i, x + tx + j) - at_q(ref, y + ty + i, x + tx + j, mvy, mvx);
      total += oro_hadamard4x4(d);
    }
  return total;
}

static int compound_pair_ok(int a, int b, int nrefs) {
  const int lo = a < b ? a : b, limit = nrefs - 2 < 2 ? nrefs - 2 : 2;
  return a != b && lo <= limit;
}

static int64_t block_compound_satd(const plane_t* cur, const plane_t* r0, int mx0, int my0, const plane_t* r1, int mx1,
                                   int my1, int x, int y, int w, int h) {
  int64_t total = 0;
  for (int ty = 0; ty < h; ty += 4)
    for (int tx = 0; tx < w; tx += 4) {
      int d[16];
      for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
          const int yy = y + ty + i, xx = x + tx + j;
          const int p = (at_q(r0, yy, xx, my0, mx0) + at_q(r1, yy, xx, my1, mx1) + 1) >> 1;
          d[4 * i + j] = at(cur, yy, xx) - p;
        }
      total += oro_hadamard4x4(d);
    }
  return total;
}

/* ---- Per-block best choice (src/gpu/kernels_ref.cpp:28-104) ---- */
typedef struct {
  int64_t cost;
  int mode; /* 0..12 intra, kNumModes inter */
  int mvx, mvy, ref;
  int ref2, mvx2, mvy2;
} best_t;

typedef struct {
  const plane_t* plane[CELV2_MAX_REFS]; /* level 0 with phases */
  const int32_t* fx[CELV2_MAX_REFS];
  const int32_t* fy[CELV2_MAX_REFS];
  int cols, rows, n;
} refset_t;

static best_t make_best(int64_t cost, int mode, int mvx, int mvy, int ref) {
  best_t b = {cost, mode, mvx, mvy, ref, CELV2_SINGLE_REF, 0, 0};
  return b;
}

/* best_both + best_mode (kernels_ref.cpp:43-104): the intra modes in order, each reference's
 * candidates in order (repeats skipped), the best of the references, the compound of the two best,
 * all first strict minimum; records the block's candidates into o[b]; returns the block's best
 * (inter only where strictly cheaper than intra). */
static best_t block_best(const plane_t* s, const refset_t* rs, int ox, int oy, int b, int64_t lam, int intra,
                         unsigned keep_refs, unsigned keep_modes, celv2_sb_out* o) {
  int bx, by, w, h;
  oro_sb_block_geom(b, &bx, &by, &w, &h);
  const int x = ox + bx, y = oy + by;
  best_t bi = make_best(INT64_MAX, 0, 0, 0, 0), be = make_best(INT64_MAX, kNumModes, 0, 0, 0);
  for (int m = 0; m < kNumModes && intra; m++) {
    if (!(keep_modes >> m & 1u)) continue; /* a pruned mode is no candidate */
    const int64_t c = block_mode_satd(s, x, y, w, h, m) * 256 + lam * (mode_bits(m) + (rs->n > 0 ? kIntraInInterBits : 0));
    if (c < bi.cost) bi = make_best(c, m, 0, 0, 0);
  }
  best_t per[CELV2_MAX_REFS];
  int a = -1, second = -1;
  const int ncand = mv_cells(x, y, w, h) + 8;
  for (int r = 0; r < rs->n; r++) {
    per[r] = make_best(INT64_MAX, kNumModes, 0, 0, r);
    if (!(keep_refs >> r & 1u)) continue; /* a pruned reference is no candidate */
    for (int k = 0; k < ncand; k++) {
      if (repeated(rs->fx[r], rs->fy[r], rs->cols, rs->rows, x, y, w, h, k)) continue;
      const int i = candidate_index(x, y, w, h, k, rs->cols, rs->rows);
      const int64_t c = block_inter_satd(s, rs->plane[r], x, y, w, h, rs->fx[r][i], rs->fy[r][i]) * 256 +
                        lam * (kInterBits + r);
      if (c < per[r].cost) per[r] = make_best(c, kNumModes, rs->fx[r][i], rs->fy[r][i], r);
    }
    if (a < 0 || per[r].cost < per[a].cost) a = r;
  }
  for (int r = 0; r < rs->n; r++)
    if (r != a && (keep_refs >> r & 1u) && (second < 0 || per[r].cost < per[second].cost)) second = r;
  if (a >= 0) be = per[a];
  if (second >= 0 && compound_pair_ok(a, second, rs->n)) {
    const best_t p = per[a], q = per[second];
    const int64_t c = block_compound_satd(s, rs->plane[a], p.mvx, p.mvy, rs->plane[second], q.mvx, q.mvy, x, y, w, h) *
                          256 +
                      lam * (20 + a + second);
    if (c < be.cost) {
      be = p;
      be.cost = c, be.ref2 = second, be.mvx2 = q.mvx, be.mvy2 = q.mvy;
    }
  }
  /* The record (kernels_ref.cpp:93-103; MVs stay in quarter pels here). */
  o->c_inter_cost[b] = be.cost;
  o->c_intra_cost[b] = bi.cost;
  o->c_intra[b] = (uint8_t)bi.mode;
  o->c_mvx[b] = (int16_t)be.mvx, o->c_mvy[b] = (int16_t)be.mvy;
  o->c_ref[b] = (uint8_t)be.ref, o->c_ref2[b] = (uint8_t)be.ref2;
  o->c_mv2x[b] = (int16_t)be.mvx2, o->c_mv2y[b] = (int16_t)be.mvy2;
  for (int r = 0; r < rs->n; r++)
    if (per[r].cost != INT64_MAX) {
      const int64_t c8 = per[r].cost >> 8;
      o->c_rcost[r][b] = (uint32_t)(c8 < (int64_t)0xfffffffe ? c8 : (int64_t)0xfffffffe);
      o->c_rmvx[r][b] = (int16_t)per[r].mvx, o->c_rmvy[r][b] = (int16_t)per[r].mvy;
    }
  return be.cost < bi.cost ? be : bi;
}

/* A candidate record with nothing decided (the defaults of BlockCandidates, decision_map.h:93-102). */
static void blank_record(celv2_sb_out* o) {
  memset(o, 0, sizeof(*o));
  for (int b = 0; b < kBlocks; b++) {
    o->c_inter_cost[b] = INT64_MAX, o->c_intra_cost[b] = INT64_MAX;
    o->c_ref2[b] = CELV2_SINGLE_REF;
    for (int r = 0; r < CELV2_MAX_REFS; r++) o->c_rcost[r][b] = CELV2_NO_REF_COST;
  }
}

static void emit_leaf(celv2_sb_out* o, int b, const best_t* best) {
  int x, y, w, h;
  oro_sb_block_geom(b, &x, &y, &w, &h);
  const int inter = best->mode == kNumModes, k = o->nblocks++;
  o->tree[o->ntree++] = 0;
  o->w4[k] = (uint8_t)(w / 4), o->h4[k] = (uint8_t)(h / 4);
  o->mode[k] = (uint8_t)best->mode;
  o->mvx[k] = (int16_t)(inter ? best->mvx : 0), o->mvy[k] = (int16_t)(inter ? best->mvy : 0);
  o->ref[k] = (uint8_t)(inter ? best->ref : 0);
  const int two = inter && best->ref2 != CELV2_SINGLE_REF;
  o->ref2[k] = (uint8_t)(two ? best->ref2 : CELV2_SINGLE_REF);
  o->mv2x[k] = (int16_t)(two ? best->mvx2 : 0), o->mv2y[k] = (int16_t)(two ? best->mvy2 : 0);
}

/* The square at (level, qx, qy) in preorder (kernels_ref.cpp:150-160,180-197). */
static void emit_square(celv2_sb_out* o, const int* choice, const best_t* best, int level, int qx, int qy) {
  const int sq = level_offset(level) + qy * (1 << level) + qx, b = sq * 5;
  switch (choice[sq]) {
    case 0: emit_leaf(o, b, &best[b]); break;
    case 1: o->tree[o->ntree++] = 1, emit_leaf(o, b + 1, &best[b + 1]), emit_leaf(o, b + 2, &best[b + 2]); break;
    case 2: o->tree[o->ntree++] = 2, emit_leaf(o, b + 3, &best[b + 3]), emit_leaf(o, b + 4, &best[b + 4]); break;
    default: /* SPLIT; 8x8 squares (level 3) never split */
      o->tree[o->ntree++] = 3;
      for (int q = 0; q < 4 && level < 3; q++) emit_square(o, choice, best, level + 1, 2 * qx + (q & 1), 2 * qy + (q >> 1));
  }
}

/* decide_sb_ref + decide_square (kernels_ref.cpp:125-198,253-270): every block's best, then per
 * square NONE / HORZ / VERT / SPLIT bottom-up (first strict minimum; the 64x64 square takes NONE,
 * HORZ or VERT only in inter frames, 8x8 squares never split), then the preorder tree. */
static void decide_sb(const plane_t* s, const refset_t* rs, int sb_col, int sb_row, int64_t lam, unsigned keep,
                      celv2_sb_out* o, int64_t* sb_cost) {
  blank_record(o);
  const int ox = sb_col * 64, oy = sb_row * 64;
  best_t best[kBlocks];
  for (int b = 0; b < kBlocks; b++) {
    if (b < 5 && rs->n == 0) {
      best[b] = make_best(INT64_MAX, 0, 0, 0, 0);
      continue;
    }
    const int sq = b / 5, level = sq >= 21 ? 3 : sq >= 5 ? 2 : sq >= 1 ? 1 : 0;
    if (!(keep & CELV2_KEEP_LEVEL(level))) { /* a pruned level: no candidate, its record blank */
      best[b] = make_best(CELV2_PRUNED_COST, 0, 0, 0, 0);
      continue;
    }
    best[b] = block_best(s, rs, ox, oy, b, lam, b >= 5 && (keep & CELV2_KEEP_INTRA), keep & CELV2_KEEP_REFS,
                         keep >> 16, o);
  }
  int64_t sq_cost[CELV2_SB_SQUARES];
  int choice[CELV2_SB_SQUARES];
  const int64_t part = lam * kPartBits;
  for (int level = 3; level >= 0; level--) {
    const int n = 1 << level, size = 64 >> level;
    for (int i = 0; i < n * n; i++) {
      const int sq = level_offset(level) + i, b = sq * 5;
      int64_t c = INT64_MAX;
      int ch = 3;
      if (size <= kMaxBlockSize || (rs->n > 0 && size <= kMaxInterBlockSize)) {
        const int64_t horz = part + best[b + 1].cost + best[b + 2].cost;
        const int64_t vert = part + best[b + 3].cost + best[b + 4].cost;
        c = best[b].cost, ch = 0;
        if (horz < c) c = horz, ch = 1;
        if (vert < c) c = vert, ch = 2;
      }
      if (level < 3) {
        const int qx = i % n, qy = i / n;
        int64_t split = part;
        for (int q = 0; q < 4; q++)
          split += sq_cost[level_offset(level + 1) + (2 * qy + (q >> 1)) * (2 * n) + 2 * qx + (q & 1)];
        if (split < c) c = split, ch = 3;
      }
      sq_cost[sq] = c, choice[sq] = ch;
    }
  }
  if (sb_cost) *sb_cost = sq_cost[0];
  emit_square(o, choice, best, 0, 0, 0);
}

/* Pruning (an extension for testing the engine's pruned search, not a reference rule): the
 * effective keep word of a superblock (celv2_decision.h) -- all options without masks or in a KEY
 * frame; else the given references (all if none is given), intra if its bit is set, the given
 * levels and intra modes (all if none is given). */
static unsigned keep_of(const uint32_t* keep, int sb, int nrefs) {
  const unsigned all = (1u << nrefs) - 1u;
  if (!keep || nrefs == 0) return all | CELV2_KEEP_INTRA | CELV2_KEEP_LEVELS | CELV2_KEEP_MODES;
  const unsigned k = keep[sb];
  const unsigned levels = k & CELV2_KEEP_LEVELS, modes = k & CELV2_KEEP_MODES;
  return ((k & all) ? (k & all) : all) | (k & CELV2_KEEP_INTRA) | (levels ? levels : CELV2_KEEP_LEVELS) |
         (modes ? modes : CELV2_KEEP_MODES);
}

static int decide_frame(const uint8_t* src_y, int width, int height, const plane_t* ref_planes, int32_t* const* fx,
                        int32_t* const* fy, int nrefs, int64_t lam, int threads, const uint32_t* keep,
                        celv2_sb_out* out, int64_t* sb_cost) {
  const int pw = (width + 7) & ~7, ph = (height + 7) & ~7;
  const int sb_cols = (width + 63) / 64, sb_rows = (height + 63) / 64;
  const plane_t s = {src_y, pw, pw, ph, 0};
  refset_t rs;
  memset(&rs, 0, sizeof(rs));
  rs.n = nrefs, rs.cols = (pw + 7) / 8, rs.rows = (ph + 7) / 8;
  for (int r = 0; r < nrefs; r++) rs.plane[r] = &ref_planes[r], rs.fx[r] = fx[r], rs.fy[r] = fy[r];
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < sb_cols * sb_rows; i++)
    decide_sb(&s, &rs, i % sb_cols, i / sb_cols, lam, keep_of(keep, i, nrefs), &out[i], sb_cost ? &sb_cost[i] : NULL);
  return 0;
}

int oro_decide_from_fields(const uint8_t* src_y, int width, int height, const uint8_t* const* ref_pyr,
                           const int32_t* const* mvx0, const int32_t* const* mvy0, int nrefs, int64_t lambda_q8,
                           int threads, celv2_sb_out* out) {
  if (width <= 0 || height <= 0 || nrefs < 0 || nrefs > CELV2_MAX_REFS) return -1;
  const int pw = (width + 7) & ~7, ph = (height + 7) & ~7;
  plane_t planes[CELV2_MAX_REFS];
  int32_t* fx[CELV2_MAX_REFS];
  int32_t* fy[CELV2_MAX_REFS];
  for (int r = 0; r < nrefs; r++) {
    planes[r].p = ref_pyr[r], planes[r].stride = pw, planes[r].w = pw, planes[r].h = ph;
    planes[r].phase = (size_t)pw * ph;
    fx[r] = (int32_t*)mvx0[r], fy[r] = (int32_t*)mvy0[r];
  }
  return decide_frame(src_y, width, height, planes, fx, fy, nrefs, lambda_q8, threads, NULL, out, NULL);
}

int oro_decide(const uint8_t* src_y, int width, int height, const uint8_t* const* ref_y, int nrefs, int64_t lambda_q8,
               int threads, celv2_sb_out* out) {
  return oro_decide_masked(src_y, width, height, ref_y, nrefs, lambda_q8, threads, NULL, out, NULL);
}

int oro_decide_masked(const uint8_t* src_y, int width, int height, const uint8_t* const* ref_y, int nrefs,
                      int64_t lambda_q8, int threads, const uint32_t* keep, celv2_sb_out* out, int64_t* sb_cost) {
  if (width <= 0 || height <= 0 || nrefs < 0 || nrefs > CELV2_MAX_REFS) return -1;
  const int pw = (width + 7) & ~7, ph = (height + 7) & ~7;
  if (nrefs == 0)
    return decide_frame(src_y, width, height, NULL, NULL, NULL, 0, lambda_q8, threads, keep, out, sb_cost);
  if (pw < 16 || ph < 16) return -1; /* the 5-level pyramid needs a 1x1 top level */
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
  oro_pyr Lc, Lr;
  oro_pyr_layout(pw, ph, 0, &Lc);
  oro_pyr_layout(pw, ph, 1, &Lr);
  int cols[kMeLevels], rows[kMeLevels];
  oro_field_dims(pw, ph, cols, rows);
  uint8_t* cur = (uint8_t*)malloc(Lc.total);
  uint8_t* refs = (uint8_t*)malloc(Lr.total * nrefs);
  int32_t* fields = NULL;
  size_t per_ref = 0;
  for (int l = 0; l < kMeLevels; l++) per_ref += (size_t)cols[l] * rows[l] * 2;
  fields = (int32_t*)malloc(per_ref * nrefs * sizeof(int32_t));
  if (!cur || !refs || !fields) {
    free(cur), free(refs), free(fields);
    return -1;
  }
  oro_build_pyramid(src_y, pw, ph, 0, cur);
  plane_t planes[CELV2_MAX_REFS];
  int32_t* fx0[CELV2_MAX_REFS];
  int32_t* fy0[CELV2_MAX_REFS];
  for (int r = 0; r < nrefs; r++) {
    uint8_t* rp = refs + Lr.total * r;
    oro_build_pyramid(ref_y[r], pw, ph, 1, rp);
    int32_t* mvx[kMeLevels];
    int32_t* mvy[kMeLevels];
    int32_t* f = fields + per_ref * r;
    for (int l = 0; l < kMeLevels; l++) {
      mvx[l] = f, f += (size_t)cols[l] * rows[l];
      mvy[l] = f, f += (size_t)cols[l] * rows[l];
    }
    oro_me_fields(cur, rp, pw, ph, mvx, mvy);
    planes[r].p = rp, planes[r].stride = pw, planes[r].w = pw, planes[r].h = ph, planes[r].phase = Lr.phase;
    fx0[r] = mvx[0], fy0[r] = mvy[0];
  }
  const int rc = decide_frame(src_y, width, height, planes, fx0, fy0, nrefs, lambda_q8, threads, keep, out, sb_cost);
  free(cur), free(refs), free(fields);
  return rc;
}
