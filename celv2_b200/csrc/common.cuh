// common.cuh: device-side layout and integer primitives shared by the decision kernels.
//
// Planes live in HBM with a replicated margin of M samples on every side: a plane of w x h
// samples is stored in (w + 2M) x (h + 2M) bytes, and the margin repeats the nearest edge sample.
// The reference reads every plane through a clamped accessor (src/gpu/intra_common.h:17-25); with
// the margin, clamping a coordinate into [-M, size + M) gives the same sample as clamping it into
// [0, size), so kernels read directly wherever a footprint lies inside the margin and clamp to the
// allocated extent otherwise (which is still exact, and never leaves the allocation).
#pragma once
#include <cstdint>

#include "celv2_decision.h"

namespace celv2cu {

constexpr int kLevels = CELV2_ME_LEVELS;
constexpr int kMaxRefs = CELV2_MAX_REFS;
constexpr int kBlocks = CELV2_SB_BLOCKS;
constexpr int kModes = CELV2_NUM_MODES;
constexpr int kPhases = 16;
// Decision constants (reference src/gpu/inter_common.h:35-55,140, src/gpu/intra_common.h:32-42).
constexpr int kMeRange = 8;
constexpr int kMePenalty = 4;
constexpr int kSubpelPenalty = 16;
constexpr int kInterBits = 3;
constexpr int kIntraInInterBits = 32;
constexpr int kPartBits = 2;

// Margin per pyramid level. The motion search reaches at most 8 * (2^(5-l) - 1) pels from a cell
// at level l (248 at level 0, plus 3/4 pel of refinement), the superblock grid overhangs the padded
// frame by at most 56 samples and intra edges reach 95 samples past a block: 320 >> l (at least
// 32) covers all of it, so the clamping fallback never runs for in-range inputs.
__host__ __device__ constexpr int level_margin(int l) { return (320 >> l) < 32 ? 32 : (320 >> l); }

struct DevPlane {
  const uint8_t* p;   // the sample (0, 0); rows of `stride` bytes; valid rows/cols [-margin, size + margin)
  int stride, w, h, margin;
  long long phase;    // bytes between quarter-pel phase planes (level 0 of a reference), 0: none
};

struct DevPyramid {
  DevPlane lv[kLevels];
};

// One frame's decision work as the kernels see it (written by the host per launch).
struct FrameJob {
  DevPyramid cur;
  DevPyramid ref[kMaxRefs];
  int nrefs;
  int pw, ph;              // padded luma size (multiple of 8)
  int sb_cols, sb_rows;
  int fcols[kLevels], frows[kLevels];
  int* field[kMaxRefs][kLevels];  // packed MVs: (mvy << 16) | (mvx & 0xffff)
  const int* intra;        // [sb][kBlocks][kModes] SATDs (blocks < 5 unused)
  int2* inter;             // [sb][kMaxRefs][kBlocks]: (best SATD, packed MV)
  celv2_sb_out* out;       // [sb]
  long long lam;           // lambda_q8
  // Work counters for the roofline (null unless stage timing is on): [l] searched centres at
  // level l, [5] inter tile SATDs (tiles x distinct MVs per region), [6] compound 4x4 tiles.
  unsigned long long* stats;
  // Pruning (null: the exhaustive search): per superblock a keep word (include/celv2_decision.h:
  // references, intra, block levels, intra modes; see keep_mask). The kept options are scored
  // exactly as without pruning.
  const uint32_t* keep;
  long long* sb_cost;      // [sb]: the chosen partition's cost (null: not written)
};

enum { kStatInterMvs = 5, kStatCompoundTiles = 6, kStats = 8 };

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// The effective keep word of superblock sb: all options without pruning or in a KEY frame;
// otherwise the given references (all of them if none is given), intra if its bit is set, the
// given block levels and intra modes (all of them if none is given).
__device__ __forceinline__ unsigned keep_mask(const FrameJob& job, int sb) {
  const unsigned all = (1u << job.nrefs) - 1u;
  if (!job.keep || job.nrefs == 0) return all | CELV2_KEEP_INTRA | CELV2_KEEP_LEVELS | CELV2_KEEP_MODES;
  const unsigned k = job.keep[sb];
  const unsigned levels = k & CELV2_KEEP_LEVELS, modes = k & CELV2_KEEP_MODES;
  return ((k & all) ? (k & all) : all) | (k & CELV2_KEEP_INTRA) | (levels ? levels : CELV2_KEEP_LEVELS) |
         (modes ? modes : CELV2_KEEP_MODES);
}

// The square level of candidate block b: 0 for 64x64 (and its halves), 1 for 32x32, 2 for 16x16,
// 3 for 8x8.
__host__ __device__ __forceinline__ int block_level(int b) {
  const int sq = b / 5;
  return sq >= 21 ? 3 : sq >= 5 ? 2 : sq >= 1 ? 1 : 0;
}

// Whether level-0 cell (cx, cy) of reference r is read by the inter stage of a superblock that
// keeps r: superblock (sx, sy) reads the cells sx * 8 - 1 .. sx * 8 + 8 (clamped), likewise in y.
__device__ __forceinline__ bool cell_needed(const FrameJob& job, int r, int cx, int cy) {
  if (!job.keep) return true;
  const int x0 = cx >= 8 ? (cx - 1) >> 3 : 0, x1 = min(job.sb_cols - 1, (cx + 1) >> 3);
  const int y0 = cy >= 8 ? (cy - 1) >> 3 : 0, y1 = min(job.sb_rows - 1, (cy + 1) >> 3);
  for (int sy = y0; sy <= y1; sy++)
    for (int sx = x0; sx <= x1; sx++)
      if (keep_mask(job, sy * job.sb_cols + sx) >> r & 1u) return true;
  return false;
}

// The clamped sample (Plane::at, src/gpu/intra_common.h:17-21).
__device__ __forceinline__ int at(const DevPlane& s, int y, int x) {
  y = clampi(y, -s.margin, s.h + s.margin - 1);
  x = clampi(x, -s.margin, s.w + s.margin - 1);
  return s.p[(long long)y * s.stride + x];
}

// Quarter-pel sample (Plane::at_q, src/gpu/intra_common.h:23-25): phase (qy & 3) * 4 + (qx & 3) at
// the whole-pel position (y + (qy >> 2), x + (qx >> 2)).
__device__ __forceinline__ int at_q(const DevPlane& s, int y, int x, int qy, int qx) {
  const uint8_t* base = s.p + (long long)((qy & 3) * 4 + (qx & 3)) * s.phase;
  const int yy = clampi(y + (qy >> 2), -s.margin, s.h + s.margin - 1);
  const int xx = clampi(x + (qx >> 2), -s.margin, s.w + s.margin - 1);
  return base[(long long)yy * s.stride + xx];
}

// Whether the rectangle [x, x + w) x [y, y + h) lies inside the stored plane (margin included).
__device__ __forceinline__ bool inside(const DevPlane& s, int x, int y, int w, int h) {
  return x >= -s.margin && y >= -s.margin && x + w <= s.w + s.margin && y + h <= s.h + s.margin;
}

// Four bytes starting at an arbitrary byte address, from two aligned 32-bit loads.
__device__ __forceinline__ uint32_t load4(const uint8_t* p) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  const uint32_t* w = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
  const uint32_t sh = (uint32_t)(a & 3) * 8;
  const uint32_t lo = __ldg(w);
  if (sh == 0) return lo;
  return __funnelshift_r(lo, __ldg(w + 1), sh);
}

// Sum of absolute 4x4 Hadamard coefficients (src/gpu/intra_common.h:131-146): rows, then columns,
// the last column butterfly folded with the absolute values: |x + y| + |x - y| = 2 max(|x|, |y|).
__device__ __forceinline__ int hadamard4x4(int d[16]) {
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int s01 = d[4 * r] + d[4 * r + 1], d01 = d[4 * r] - d[4 * r + 1];
    const int s23 = d[4 * r + 2] + d[4 * r + 3], d23 = d[4 * r + 2] - d[4 * r + 3];
    d[4 * r] = s01 + s23, d[4 * r + 1] = d01 + d23, d[4 * r + 2] = s01 - s23, d[4 * r + 3] = d01 - d23;
  }
  int sum = 0;
#pragma unroll
  for (int c = 0; c < 4; c++) {
    const int s01 = d[c] + d[4 + c], d01 = d[c] - d[4 + c];
    const int s23 = d[8 + c] + d[12 + c], d23 = d[8 + c] - d[12 + c];
    sum += max(abs(s01), abs(s23)) + max(abs(d01), abs(d23));
  }
  return 2 * sum;
}

// Columns 0 and 2 (even) or 1 and 3 (odd) of a 4-byte row as two 16-bit lanes.
__device__ __forceinline__ uint32_t bytes_even(uint32_t w) { return __byte_perm(w, 0, 0x4240); }
__device__ __forceinline__ uint32_t bytes_odd(uint32_t w) { return __byte_perm(w, 0, 0x4341); }

// hadamard4x4 of the byte residuals cur - pred of a 4x4 tile, rows as packed bytes: cur rows given
// as their even / odd lanes (ce, co), prediction rows p. Each row's columns 0/2 and 1/3 ride as two
// 16-bit lanes of one 32-bit integer, held as lo + hi * 65536 with |lo|, |hi| <= 2040 so plain
// 32-bit adds are exact; three of the four butterfly stages run on both lanes at once, and the
// last one with the absolute values folds into |x + y| + |x - y| = 2 max(|x|, |y|). The same sum
// of 16 absolute Walsh-Hadamard coefficients as hadamard4x4.
__device__ __forceinline__ int satd4_bytes(const uint32_t* ce, const uint32_t* co, const uint32_t* p) {
  int A[4], B[4];
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int e = (int)(ce[i] - bytes_even(p[i])), o = (int)(co[i] - bytes_odd(p[i]));
    A[i] = e + o, B[i] = e - o;
  }
  int sum = 0;
#pragma unroll
  for (int h = 0; h < 2; h++) {
    const int* X = h ? B : A;
    const int s01 = X[0] + X[1], d01 = X[0] - X[1], s23 = X[2] + X[3], d23 = X[2] - X[3];
    const int v[4] = {s01 + s23, d01 + d23, s01 - s23, d01 - d23};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int lo = (int)(short)(v[k] & 0xffff), hi = (v[k] - lo) >> 16;
      sum += max(abs(lo), abs(hi));
    }
  }
  return 2 * sum;
}

// dp4a with unsigned bytes a and signed bytes b: c + sum_k a_k * b_k.
__device__ __forceinline__ int dp4a_us(uint32_t a, uint32_t b, int c) {
  int d;
  asm("dp4a.u32.s32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}

// The four 1-D Walsh-Hadamard basis rows of length 4 as signed bytes (column 0 in the low byte):
// (1,1,1,1), (1,-1,1,-1), (1,1,-1,-1), (1,-1,-1,1) -- the rows hadamard4x4's row butterflies form.
__device__ __forceinline__ uint32_t wh_row(int k) {
  return k == 0 ? 0x01010101u : k == 1 ? 0xFF01FF01u : k == 2 ? 0xFFFF0101u : 0x01FFFF01u;
}

// The same rows negated.
__device__ __forceinline__ uint32_t wh_row_neg(int k) {
  return k == 0 ? 0xFFFFFFFFu : k == 1 ? 0x01FF01FFu : k == 2 ? 0x0101FFFFu : 0xFF0101FFu;
}

// Row-transformed cur tile for satd4_rows: C[4k + i] = <row i of the tile, basis row k>.
__device__ __forceinline__ void wh_rows_cur(const uint32_t* c, int* C) {
#pragma unroll
  for (int k = 0; k < 4; k++)
#pragma unroll
    for (int i = 0; i < 4; i++) C[4 * k + i] = dp4a_us(c[i], wh_row(k), 0);
}

// hadamard4x4 of the residual cur - pred of a 4x4 tile from the row-transformed cur tile C and the
// prediction rows p (packed bytes): each residual row coefficient is one dp4a of the prediction
// row with the negated basis row, accumulated onto cur's; the column butterflies follow, the last
// one folded with the absolute values into |x + y| + |x - y| = 2 max(|x|, |y|). The same sum of
// 16 absolute coefficients.
__device__ __forceinline__ int satd4_rows(const int* C, const uint32_t* p) {
  int sum = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const uint32_t neg = wh_row_neg(k);
    const int r0 = dp4a_us(p[0], neg, C[4 * k]), r1 = dp4a_us(p[1], neg, C[4 * k + 1]);
    const int r2 = dp4a_us(p[2], neg, C[4 * k + 2]), r3 = dp4a_us(p[3], neg, C[4 * k + 3]);
    const int s01 = r0 + r1, d01 = r0 - r1, s23 = r2 + r3, d23 = r2 - r3;
    sum += max(abs(s01), abs(s23)) + max(abs(d01), abs(d23));
  }
  return 2 * sum;
}

// Residual of one 4x4 row: four cur bytes minus four prediction bytes.
__device__ __forceinline__ void residual_row(int* d, uint32_t c, uint32_t p) {
  d[0] = (int)(c & 255) - (int)(p & 255);
  d[1] = (int)((c >> 8) & 255) - (int)((p >> 8) & 255);
  d[2] = (int)((c >> 16) & 255) - (int)((p >> 16) & 255);
  d[3] = (int)(c >> 24) - (int)(p >> 24);
}

__device__ __forceinline__ int mv_x(int packed) { return (int)(short)(packed & 0xffff); }
__device__ __forceinline__ int mv_y(int packed) { return packed >> 16; }
__host__ __device__ __forceinline__ int pack_mv(int x, int y) { return (int)(((unsigned)y << 16) | ((unsigned)x & 0xffffu)); }

// ---- Superblock block geometry (src/gpu/sb_blocks.h:12-37) ----
__host__ __device__ __forceinline__ int sb_level_offset(int level) { return ((1 << (2 * level)) - 1) / 3; }

__host__ __device__ __forceinline__ void sb_block_geom(int b, int& x, int& y, int& w, int& h) {
  const int sq = b / 5, kind = b % 5;
  const int level = sq >= 21 ? 3 : sq >= 5 ? 2 : sq >= 1 ? 1 : 0;
  const int idx = sq - sb_level_offset(level), n = 1 << level, size = 64 >> level, half = size / 2;
  const int sx = (idx % n) * size, sy = (idx / n) * size;
  x = sx, y = sy, w = size, h = size;
  if (kind == 1 || kind == 2) h = half, y = sy + (kind == 2 ? half : 0);
  if (kind == 3 || kind == 4) w = half, x = sx + (kind == 4 ? half : 0);
}

__host__ __device__ __forceinline__ int mode_bits(int mode) { return mode == 0 ? 1 : mode < 4 ? 3 : 9; }

__host__ __device__ __forceinline__ bool compound_pair_ok(int a, int b, int nrefs) {
  const int lo = a < b ? a : b, limit = nrefs - 2 < 2 ? nrefs - 2 : 2;
  return a != b && lo <= limit;
}

}  // namespace celv2cu
