// intra.cu: the SATD of every candidate block under each of the 13 intra modes.
//
// Reference rules (src/gpu/intra_common.h): edge_above / edge_left (:47-56), dir_pred (:60-85),
// intra_pred (:89-118), dc_value (:120-128), block_mode_satd (:149-163). Blocks of the 64x64
// square are never intra (kMaxBlockSize 32, :39), so 420 blocks x 13 modes per superblock.
//
// One CTA per superblock:
//  1. the source samples around the superblock -- rows and columns -1 .. 95 from its origin
//     (above-right and below-left edges reach w + h - 1 past a block) -- are staged in shared
//     memory from the margin plane, which already holds the clamped values;
//  2. every block's above and left edge arrays, k = -1 .. w + h - 1, are built once with the
//     frame-edge rules applied (128 outside the frame, the corner rule at k = -1), and its DC;
//  3. the 2304 (block, 4x4 tile) items are spread over the threads; each predicts its tile under
//     the 13 modes from the edge arrays alone (no per-sample rule branches) and takes the
//     Hadamards; a segmented shuffle reduction sums a block's tiles per mode.
// The Hadamard of a residual is the cur tile's transform minus the prediction's (linearity), so
// the cur tile is transformed once per item: its rows by dp4a against the Walsh-Hadamard basis.
// DC, V and H predictions change only 1, 4 and 4 of the 16 coefficients (a constant tile only the
// DC; equal rows only the first coefficient of each column transform; constant rows only the
// first row transform), so those three modes cost a few operations on the cur transform; the ten
// others pack their prediction rows into bytes and run the dp4a row transform (satd4_rows).
// Word-wide predictions: a block's edges are one byte run per block -- the left column reversed,
// then the corner and the row above (then the left column's corner) -- so that D135's rows are
// 4-byte runs of it, D45's rows 4-byte runs of the row above, D67 / D113 (rows) and D203 / D157
// (columns) blends of two 4-byte runs with one weight per row or column (four samples at once in
// two 16-bit lanes), SmoothV / SmoothH two lanes at a time. A 4x4 SATD does not change under
// transposition (the 2-D Hadamard of the transposed residual is the transposed Hadamard), so the
// column-wise modes come last, after the cur tile's transform is redone on its columns.
// The output is raw SATDs; the finalize stage adds lambda * bits (which depend on whether the
// frame has references, unknown when prepare() runs this ahead of its launch).
#include "kernels.h"
#include "tables.h"

namespace celv2cu {

constexpr int kIntraThreads = 256;
constexpr int kRegion = 97;   // local rows / columns -1 .. 95
constexpr int kRegionStride = 100;
constexpr int kEdges = 7588;  // edge entries of the blocks of levels 1-3 (see edge_offset)

struct IntraSmem {
  uint8_t px[kRegion * kRegionStride];
  alignas(16) uint8_t edge[2 * kEdges + 16];  // per block: L reversed, A[-1], A[0..], L[-1] (+ read slack)
  int dc[kBlocks];
  int acc[kBlocks][kModes];
};

// Where block b's edge run starts (b >= 5): the run of a block with n = w + h edge samples per
// side is 2n + 2 bytes, L[n - 1] .. L[0] at 0 .. n - 1, A[-1] .. A[n - 1] at n .. 2n, L[-1] at
// 2n + 1. A square of side s holds its whole block (4s + 2 bytes) then its four halves (3s + 2
// each); levels 1, 2, 3 follow each other.
__device__ __forceinline__ int edge_offset(int b) {
  const int sq = b / 5, kind = b - sq * 5;
  const int level = sq >= 21 ? 3 : sq >= 5 ? 2 : 1;
  const int s = 64 >> level, per_sq = 8 * s + 5;
  const int base = level == 1 ? 0 : level == 2 ? 4 * 261 : 4 * 261 + 16 * 133;
  const int idx = sq - sb_level_offset(level);
  return 2 * (base + idx * per_sq + (kind == 0 ? 0 : (2 * s + 1) + (kind - 1) * (s + s / 2 + 1)));
}

// Four bytes at byte index i (any alignment) of a 16-byte-aligned shared array: two words and a
// funnel shift.
__device__ __forceinline__ uint32_t lds4(const uint8_t* base, int i) {
  const uint32_t* w = reinterpret_cast<const uint32_t*>(base) + (i >> 2);
  return __funnelshift_r(w[0], w[1], (unsigned)(i & 3) * 8);
}

// Byte order reversed (the left column is stored bottom-up).
__device__ __forceinline__ uint32_t rev4(uint32_t v) { return __byte_perm(v, 0, 0x0123); }

// Per byte (p0 * (32 - sh) + p1 * sh + 16) >> 5 -- the directional modes' blend of four samples at
// once: bytes 0 / 2 and 1 / 3 as two 16-bit lanes (at most 255 * 32 + 16 per lane, so no lane
// carries into the next).
__device__ __forceinline__ uint32_t blend4(uint32_t p0, uint32_t p1, int sh) {
  const uint32_t a = (uint32_t)(32 - sh), b = (uint32_t)sh;
  const uint32_t e = ((p0 & 0x00ff00ffu) * a + (p1 & 0x00ff00ffu) * b + 0x00100010u) >> 5;
  const uint32_t o = (((p0 >> 8) & 0x00ff00ffu) * a + ((p1 >> 8) & 0x00ff00ffu) * b + 0x00100010u) >> 5;
  return (e & 0x00ff00ffu) | ((o & 0x00ff00ffu) << 8);
}

// Rounded blend of p0, p1 with weight sh / 32 (the directional modes' interpolation).
__device__ __forceinline__ int blend32(int p0, int p1, int sh) { return (p0 * (32 - sh) + p1 * sh + 16) >> 5; }

// Four predicted samples (0..255) as the bytes of one word, sample 0 in the low byte.
__device__ __forceinline__ uint32_t pack_row(int a, int b, int c, int d) {
  return (uint32_t)a | (uint32_t)b << 8 | (uint32_t)c << 16 | (uint32_t)d << 24;
}

// One z2 sample (D113, D157): the row above while the projection stays on it, else the left
// column (intra_common.h dir_pred, the z2 branch). A points at A[0] of the block's edge run (A[-1]
// at A[-1]); L(k) of the left column.
__device__ __forceinline__ int z2_sample(int dxa, int dya, const uint8_t* E, int a0, int lr0, int lm1, int ii,
                                         int jj) {
  const int px = (jj << 6) - (ii + 1) * dxa, bx = px >> 6;
  if (bx >= -1) return blend32(E[a0 + bx], E[a0 + bx + 1], (px & 63) >> 1);
  const int py = (ii << 6) - (jj + 1) * dya, by = py >> 6;
  const int b0 = max(by, -1), b1 = max(by + 1, -1);
  return blend32(b0 < 0 ? lm1 : E[lr0 - b0], b1 < 0 ? lm1 : E[lr0 - b1], (py & 63) >> 1);
}

__global__ void __launch_bounds__(kIntraThreads, 4) k_intra(const FrameJob* __restrict__ jobs, WorkList w) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  IntraSmem& S = *reinterpret_cast<IntraSmem*>(smem_raw);
  __shared__ int unit_slot;
  const int tid = threadIdx.x;
  int unit, iter = 0;
  while (take_unit(w, unit, iter, &unit_slot)) {
  const int jb = job_of(w, unit);
  const FrameJob& job = jobs[jb];
  const int sb = unit - w.prefix[jb], sby = sb / job.sb_cols, sbx = sb - sby * job.sb_cols;
  const unsigned keep = keep_mask(job, sb);
  if (!(keep & CELV2_KEEP_INTRA)) continue;  // intra pruned for this superblock
  const int ox = sbx * 64, oy = sby * 64;
  const DevPlane src = job.cur.lv[0];

  // 1. staged samples (the margin holds the clamped values)
  for (int e = tid; e < kRegion * kRegion; e += kIntraThreads) {
    const int ly = e / kRegion - 1, lx = e % kRegion - 1;
    S.px[(ly + 1) * kRegionStride + lx + 1] = (uint8_t)at(src, oy + ly, ox + lx);
  }
  for (int e = tid; e < kBlocks * kModes; e += kIntraThreads) (&S.acc[0][0])[e] = 0;
  __syncthreads();
  // 2. edge runs (edge_above / edge_left) and DC values (dc_value) per block
  for (int b = 5 + tid; b < kBlocks; b += kIntraThreads) {
    int x, y, bw, bh;
    sb_block_geom(b, x, y, bw, bh);
    const bool top = oy + y == 0, lft = ox + x == 0;
    const int n = bw + bh;
    uint8_t* E = S.edge + edge_offset(b);
    auto s = [&](int ly, int lx) { return (int)S.px[(ly + 1) * kRegionStride + lx + 1]; };
    for (int k = -1; k < n; k++) {
      E[n + 1 + k] = (uint8_t)(top ? 128 : (k < 0 && lft) ? s(y - 1, x) : s(y - 1, x + k));  // A[k]
      E[k < 0 ? 2 * n + 1 : n - 1 - k] = (uint8_t)(lft ? 128 : (k < 0 && top) ? s(y, x - 1) : s(y + k, x - 1));  // L[k]
    }
    int sum = 0, cnt = 0;
    if (!top)
      for (int j = 0; j < bw; j++) sum += s(y - 1, x + j), cnt++;
    if (!lft)
      for (int i = 0; i < bh; i++) sum += s(y + i, x - 1), cnt++;
    S.dc[b] = cnt ? (sum + cnt / 2) / cnt : 128;
  }
  __syncthreads();

  // 3. (block, tile) items: 13 predictions + Hadamards per tile, segment sums per block
  const uint8_t* E = S.edge;
  for (int base = kIntraFirst; base < kItems; base += kIntraThreads) {
    // the items of one CTA-wide step belong to one block level (its boundaries are multiples of 256)
    if (!(keep & CELV2_KEEP_LEVEL(base < 1536 ? 1 : base < 2304 ? 2 : 3))) continue;
    const int item = base + tid;  // the intra items are a multiple of the CTA size
    int b, tx, ty;
    item_decode(item, b, tx, ty);
    const int width = item_width(item);
    int x, y, bw, bh;
    sb_block_geom(b, x, y, bw, bh);
    const int n = bw + bh, seg = edge_offset(b);
    const int a0 = seg + n + 1;  // A[k] at E[a0 + k], k >= -1
    const int lr0 = seg + n - 1; // L[k] at E[lr0 - k], k >= 0
    const int lm1 = E[seg + 2 * n + 1];  // L[-1]
    const int r0 = ty * 4 - y, c0 = tx * 4 - x;  // the tile's origin inside the block
    // the cur tile: rows as packed bytes, row-transformed (C)
    const int cur0 = (ty * 4 + 1) * kRegionStride + tx * 4 + 1;
    int C[16];
    {
      uint32_t cw[4];
#pragma unroll
      for (int i = 0; i < 4; i++) cw[i] = lds4(S.px, cur0 + i * kRegionStride);
      wh_rows_cur(cw, C);
    }
    const int seg_lead = (tid & ((width < 32 ? width : 32) - 1)) == 0;
    {
      // DC, V, H: per basis row k the column transform's outputs; T the sum of all 16 absolute
      // coefficients (the cur tile's SATD), Hk0 the first outputs and V0 their absolute sum, U0 the
      // absolute sum of row k = 0's
      int Hk0[4], T = 0, V0 = 0, U0 = 0;
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int s01 = C[4 * k] + C[4 * k + 1], d01 = C[4 * k] - C[4 * k + 1];
        const int s23 = C[4 * k + 2] + C[4 * k + 3], d23 = C[4 * k + 2] - C[4 * k + 3];
        const int a = abs(s01 + s23) + abs(s01 - s23) + abs(d01 + d23) + abs(d01 - d23);
        T += a, Hk0[k] = s01 + s23, V0 += abs(s01 + s23);
        if (k == 0) U0 = a;
      }
      // DC: only coefficient (0, 0) moves, by 16 v
      const int dc = T - abs(Hk0[0]) + abs(Hk0[0] - 16 * S.dc[b]);
      // V: every row is the above row a; the first output of each column transform moves by 4 a_k
      const uint32_t a = lds4(E, a0 + c0);
      int v = T - V0;
#pragma unroll
      for (int k = 0; k < 4; k++) v += abs(Hk0[k] - 4 * dp4a_us(a, wh_row(k), 0));
      // H: row i is the constant l_i; row transform k = 0 moves by 4 l_i
      const uint32_t l4 = rev4(lds4(E, lr0 - r0 - 3));  // L[r0 .. r0 + 3]
      const int r0v = C[0] - 4 * (int)(l4 & 255), r1v = C[1] - 4 * (int)((l4 >> 8) & 255);
      const int r2v = C[2] - 4 * (int)((l4 >> 16) & 255), r3v = C[3] - 4 * (int)(l4 >> 24);
      const int s01 = r0v + r1v, d01 = r0v - r1v, s23 = r2v + r3v, d23 = r2v - r3v;
      const int h = T - U0 + abs(s01 + s23) + abs(s01 - s23) + abs(d01 + d23) + abs(d01 - d23);
      const int s0 = segment_sum(dc, width), s1 = segment_sum(v, width), s2 = segment_sum(h, width);
      if (seg_lead) atomicAdd(&S.acc[b][0], s0), atomicAdd(&S.acc[b][1], s1), atomicAdd(&S.acc[b][2], s2);
    }
    const int lgw = 31 - __clz(bw), lgh = 31 - __clz(bh);
    const int den = bw + bh + 2;
    // n / den for n < 2^15 as a multiply-high by ceil(2^32 / den): exact while n * (den * ceil(2^32 /
    // den) - 2^32) < 2^32 (division by invariant integers using multiplication, Granlund and
    // Montgomery 1994); here n < 256 den and den <= 66
    const unsigned magic = 0xffffffffu / (unsigned)den + 1u;
#pragma unroll 1
    for (int m = 3; m < kModes; m++) {  // the ten modes with their own prediction rows
      uint32_t pw[4];
      if (m == 11 && (keep & (CELV2_KEEP_MODE(11) | CELV2_KEEP_MODE(12)))) {
        // D157 and D203 predict columns: from here on C is the transform of the cur tile's columns
        uint32_t cw[4], col[4];
#pragma unroll
        for (int i = 0; i < 4; i++) cw[i] = lds4(S.px, cur0 + i * kRegionStride);
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const unsigned sel = (unsigned)j | (unsigned)(4 + j) << 4;
          col[j] = __byte_perm(__byte_perm(cw[0], cw[1], sel), __byte_perm(cw[2], cw[3], sel), 0x5410);
        }
        wh_rows_cur(col, C);
      }
      if (!(keep & CELV2_KEEP_MODE(m))) continue;  // a pruned mode (uniform over the CTA)
      switch (m) {
        case 3: {  // Smooth: bilinear blend of above, left, top-right and bottom-left
          const int tr = E[a0 + bw - 1], bl = E[lr0 - (bh - 1)];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            int v[4];
            const int ii = r0 + i, li = E[lr0 - ii];
#pragma unroll
            for (int j = 0; j < 4; j++) {
              const int jj = c0 + j;
              const int num = (bh - ii) * E[a0 + jj] + (ii + 1) * bl + (bw - jj) * li + (jj + 1) * tr;
              v[j] = (int)__umulhi((unsigned)(num + den / 2), magic);
            }
            pw[i] = pack_row(v[0], v[1], v[2], v[3]);
          }
          break;
        }
        case 4: {  // SmoothV (h a power of two, the numerator non-negative): two 16-bit lanes at once
          const uint32_t a4 = lds4(E, a0 + c0), ae = a4 & 0x00ff00ffu, ao = (a4 >> 8) & 0x00ff00ffu;
          const int bl = E[lr0 - (bh - 1)];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const int ii = r0 + i;
            const uint32_t wa = (uint32_t)(bh - 1 - ii), add = (uint32_t)((ii + 1) * bl + bh / 2) * 0x00010001u;
            const uint32_t e = ((ae * wa + add) >> lgh) & 0x00ff00ffu, o = ((ao * wa + add) >> lgh) & 0x00ff00ffu;
            pw[i] = e | o << 8;
          }
          break;
        }
        case 5: {  // SmoothH: per row the left sample l, per column weights (bw - 1 - jj, jj + 1)
          const int tr = E[a0 + bw - 1];
          const uint32_t we = (uint32_t)(bw - 1 - c0) | (uint32_t)(bw - 3 - c0) << 16;
          const uint32_t wo = (uint32_t)(bw - 2 - c0) | (uint32_t)(bw - 4 - c0) << 16;
          const uint32_t te = ((uint32_t)(c0 + 1) | (uint32_t)(c0 + 3) << 16) * (uint32_t)tr + (uint32_t)(bw / 2) * 0x00010001u;
          const uint32_t to = ((uint32_t)(c0 + 2) | (uint32_t)(c0 + 4) << 16) * (uint32_t)tr + (uint32_t)(bw / 2) * 0x00010001u;
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const uint32_t l = E[lr0 - (r0 + i)];
            const uint32_t e = ((l * we + te) >> lgw) & 0x00ff00ffu, o = ((l * wo + to) >> lgw) & 0x00ff00ffu;
            pw[i] = e | o << 8;
          }
          break;
        }
        case 6: {  // Paeth
          const int tl = E[a0 - 1];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            int v[4];
            const int l = E[lr0 - (r0 + i)];
#pragma unroll
            for (int j = 0; j < 4; j++) {
              const int a = E[a0 + c0 + j], bse = a + l - tl;
              const int pa = abs(bse - a), pl = abs(bse - l), ptl = abs(bse - tl);
              v[j] = pl <= pa && pl <= ptl ? l : pa <= ptl ? a : tl;
            }
            pw[i] = pack_row(v[0], v[1], v[2], v[3]);
          }
          break;
        }
        case 7: {  // D45: derivative 64, no blend: row i is A[r0 + i + 1 + c0 ..] (never past A[w + h - 1])
#pragma unroll
          for (int i = 0; i < 4; i++) pw[i] = lds4(E, a0 + r0 + i + 1 + c0);
          break;
        }
        case 8: {  // D67: derivative 27, one weight per row
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const int pos = (r0 + i + 1) * 27, b0 = a0 + (pos >> 6) + c0;
            pw[i] = blend4(lds4(E, b0), lds4(E, b0 + 1), (pos & 63) >> 1);
          }
          break;
        }
        case 9: {  // D113: a row whose first sample projects onto the row above stays on it
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const int ii = r0 + i, px = (c0 << 6) - (ii + 1) * 27, bx = px >> 6;
            if (bx >= -1) {
              pw[i] = blend4(lds4(E, a0 + bx), lds4(E, a0 + bx + 1), (px & 63) >> 1);
            } else {
              uint32_t row = 0;
#pragma unroll 1
              for (int j = 3; j >= 0; j--) row = row << 8 | (uint32_t)z2_sample(27, 151, E, a0, lr0, lm1, ii, c0 + j);
              pw[i] = row;
            }
          }
          break;
        }
        case 10: {  // D135: derivatives 64 / 64, no blend: row i is a 4-byte run of L reversed, A[-1], A
#pragma unroll
          for (int i = 0; i < 4; i++) pw[i] = lds4(E, a0 - 1 + c0 - r0 - i);
          break;
        }
        case 11: {  // D157, by columns: a column whose top sample projects onto the left column
                    // (row above not reached, no clamp at L[-1]) stays on it
#pragma unroll
          for (int j = 0; j < 4; j++) {
            const int jj = c0 + j, py = (r0 << 6) - (jj + 1) * 27, by = py >> 6;
            if ((jj << 6) - (r0 + 1) * 151 < -64 && by >= 0) {
              const uint32_t l0 = rev4(lds4(E, lr0 - by - 3)), l1 = rev4(lds4(E, lr0 - by - 4));
              pw[j] = blend4(l0, l1, (py & 63) >> 1);
            } else {
              uint32_t col = 0;
#pragma unroll 1
              for (int i = 3; i >= 0; i--) col = col << 8 | (uint32_t)z2_sample(151, 27, E, a0, lr0, lm1, r0 + i, jj);
              pw[j] = col;
            }
          }
          break;
        }
        default: {  // z3: D203 (derivative 27), by columns from the column left
#pragma unroll
          for (int j = 0; j < 4; j++) {
            const int pos = (c0 + j + 1) * 27, b0 = (pos >> 6) + r0;
            const uint32_t l0 = rev4(lds4(E, lr0 - b0 - 3)), l1 = rev4(lds4(E, lr0 - b0 - 4));
            pw[j] = blend4(l0, l1, (pos & 63) >> 1);
          }
          break;
        }
      }
      const int s = segment_sum(satd4_rows(C, pw), width);
      if (seg_lead) atomicAdd(&S.acc[b][m], s);
    }
  }
  __syncthreads();
  int* out = const_cast<int*>(job.intra) + (long long)sb * kBlocks * kModes;
  for (int e = tid; e < kBlocks * kModes; e += kIntraThreads) out[e] = (&S.acc[0][0])[e];
  }  // units
}

void launch_intra(const FrameJob* jobs, const WorkList& w, cudaStream_t st) {
  const int units = w.prefix[w.njobs];
  if (units <= 0) return;
  const int grid = w.queue ? persistent_grid((const void*)k_intra, kIntraThreads, sizeof(IntraSmem), units) : units;
  k_intra<<<grid, kIntraThreads, sizeof(IntraSmem), st>>>(jobs, w);
}

cudaError_t intra_attributes() {
  const cudaError_t e = cudaFuncSetAttribute(k_intra, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(IntraSmem));
  if (e == cudaSuccess) persistent_grid((const void*)k_intra, kIntraThreads, sizeof(IntraSmem), 1);  // fills the grid cache
  return e;
}

}  // namespace celv2cu
