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
  uint8_t above[kEdges], left[kEdges];
  int dc[kBlocks];
  int acc[kBlocks][kModes];
};

// Where block b's edge arrays start (b >= 5): a square of side s holds its whole block
// (2s + 1 entries) then its four halves (1.5s + 1 each); levels 1, 2, 3 follow each other.
__device__ __forceinline__ int edge_offset(int b) {
  const int sq = b / 5, kind = b - sq * 5;
  const int level = sq >= 21 ? 3 : sq >= 5 ? 2 : 1;
  const int s = 64 >> level, per_sq = 8 * s + 5;
  const int base = level == 1 ? 0 : level == 2 ? 4 * 261 : 4 * 261 + 16 * 133;
  const int idx = sq - sb_level_offset(level);
  return base + idx * per_sq + (kind == 0 ? 0 : (2 * s + 1) + (kind - 1) * (s + s / 2 + 1));
}

// Rounded blend of p0, p1 with weight sh / 32 (the directional modes' interpolation).
__device__ __forceinline__ int blend32(int p0, int p1, int sh) { return (p0 * (32 - sh) + p1 * sh + 16) >> 5; }

// Four predicted samples (0..255) as the bytes of one word, sample 0 in the low byte.
__device__ __forceinline__ uint32_t pack_row(int a, int b, int c, int d) {
  return (uint32_t)a | (uint32_t)b << 8 | (uint32_t)c << 16 | (uint32_t)d << 24;
}

// z1 (D45, D67): from the row above, derivative dxa (intra_common.h dir_pred, the z1 branch).
__device__ __forceinline__ void pred_z1(int dxa, const uint8_t* A, int r0, int c0, int last, uint32_t* pw) {
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int pos = (r0 + i + 1) * dxa, b0 = (pos >> 6) + c0, sh = (pos & 63) >> 1;
    int v[4];
#pragma unroll
    for (int j = 0; j < 4; j++) v[j] = blend32(A[min(b0 + j, last)], A[min(b0 + j + 1, last)], sh);
    pw[i] = pack_row(v[0], v[1], v[2], v[3]);
  }
}

// z2 (D113, D135, D157): the row above while the projection stays on it, else the left column.
// (The derivatives stay run-time values: per-mode constants let the compiler spread the three
// modes' code and spill.)
__device__ __forceinline__ void pred_z2(int dxa, int dya, const uint8_t* A, const uint8_t* L, int r0, int c0, uint32_t* pw) {
#pragma unroll
  for (int i = 0; i < 4; i++) {
    int v[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int ii = r0 + i, jj = c0 + j;
      const int px = (jj << 6) - (ii + 1) * dxa, bx = px >> 6;
      if (bx >= -1) {
        v[j] = blend32(A[bx], A[bx + 1], (px & 63) >> 1);
      } else {
        const int py = (ii << 6) - (jj + 1) * dya, by = py >> 6;
        v[j] = blend32(L[max(by, -1)], L[max(by + 1, -1)], (py & 63) >> 1);
      }
    }
    pw[i] = pack_row(v[0], v[1], v[2], v[3]);
  }
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
  if (!(keep_mask(job, sb) & 0x80u)) continue;  // intra pruned for this superblock
  const int ox = sbx * 64, oy = sby * 64;
  const DevPlane src = job.cur.lv[0];

  // 1. staged samples (the margin holds the clamped values)
  for (int e = tid; e < kRegion * kRegion; e += kIntraThreads) {
    const int ly = e / kRegion - 1, lx = e % kRegion - 1;
    S.px[(ly + 1) * kRegionStride + lx + 1] = (uint8_t)at(src, oy + ly, ox + lx);
  }
  for (int e = tid; e < kBlocks * kModes; e += kIntraThreads) (&S.acc[0][0])[e] = 0;
  __syncthreads();
  // 2. edge arrays (edge_above / edge_left) and DC values (dc_value) per block
  for (int b = 5 + tid; b < kBlocks; b += kIntraThreads) {
    int x, y, bw, bh;
    sb_block_geom(b, x, y, bw, bh);
    const bool top = oy + y == 0, lft = ox + x == 0;
    const int off = edge_offset(b), n = bw + bh;
    auto s = [&](int ly, int lx) { return (int)S.px[(ly + 1) * kRegionStride + lx + 1]; };
    for (int k = -1; k < n; k++) {
      S.above[off + k + 1] = (uint8_t)(top ? 128 : (k < 0 && lft) ? s(y - 1, x) : s(y - 1, x + k));
      S.left[off + k + 1] = (uint8_t)(lft ? 128 : (k < 0 && top) ? s(y, x - 1) : s(y + k, x - 1));
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
  for (int base = kIntraFirst; base < kItems; base += kIntraThreads) {
    const int item = base + tid;  // the intra items are a multiple of the CTA size
    int b, tx, ty;
    item_decode(item, b, tx, ty);
    const int width = item_width(item);
    int x, y, bw, bh;
    sb_block_geom(b, x, y, bw, bh);
    const uint8_t* A = S.above + edge_offset(b) + 1;  // A[k], k >= -1
    const uint8_t* L = S.left + edge_offset(b) + 1;
    const int last = bw + bh - 1;
    const int r0 = ty * 4 - y, c0 = tx * 4 - x;  // the tile's origin inside the block
    // the cur tile: rows as packed bytes, row-transformed (C), and per basis row k the column
    // transform's outputs, their absolute sum T, the first outputs Hk0 and their sum V0, and U0
    // the absolute sum of row k = 0's outputs
    int C[16];
    {
      uint32_t cw[4];
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const uint8_t* q = S.px + (ty * 4 + i + 1) * kRegionStride + tx * 4 + 1;
        cw[i] = pack_row(q[0], q[1], q[2], q[3]);
      }
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
      const uint32_t a = pack_row(A[c0], A[c0 + 1], A[c0 + 2], A[c0 + 3]);
      int v = T - V0;
#pragma unroll
      for (int k = 0; k < 4; k++) v += abs(Hk0[k] - 4 * dp4a_us(a, wh_row(k), 0));
      // H: row i is the constant l_i; row transform k = 0 moves by 4 l_i
      const int r0v = C[0] - 4 * L[r0], r1v = C[1] - 4 * L[r0 + 1];
      const int r2v = C[2] - 4 * L[r0 + 2], r3v = C[3] - 4 * L[r0 + 3];
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
      switch (m) {
        case 3: {  // Smooth: bilinear blend of above, left, top-right and bottom-left
          const int tr = A[bw - 1], bl = L[bh - 1];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            int v[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
              const int ii = r0 + i, jj = c0 + j;
              const int num = (bh - ii) * A[jj] + (ii + 1) * bl + (bw - jj) * L[ii] + (jj + 1) * tr;
              v[j] = (int)__umulhi((unsigned)(num + den / 2), magic);
            }
            pw[i] = pack_row(v[0], v[1], v[2], v[3]);
          }
          break;
        }
        case 4: {  // SmoothV (h is a power of two, the numerator non-negative)
          const int bl = L[bh - 1];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const int ii = r0 + i;
            int v[4];
#pragma unroll
            for (int j = 0; j < 4; j++) v[j] = ((bh - 1 - ii) * A[c0 + j] + (ii + 1) * bl + bh / 2) >> lgh;
            pw[i] = pack_row(v[0], v[1], v[2], v[3]);
          }
          break;
        }
        case 5: {  // SmoothH
          const int tr = A[bw - 1];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            int v[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
              const int jj = c0 + j;
              v[j] = ((bw - 1 - jj) * L[r0 + i] + (jj + 1) * tr + bw / 2) >> lgw;
            }
            pw[i] = pack_row(v[0], v[1], v[2], v[3]);
          }
          break;
        }
        case 6: {  // Paeth
          const int tl = A[-1];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            int v[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
              const int a = A[c0 + j], l = L[r0 + i], bse = a + l - tl;
              const int pa = abs(bse - a), pl = abs(bse - l), ptl = abs(bse - tl);
              v[j] = pl <= pa && pl <= ptl ? l : pa <= ptl ? a : tl;
            }
            pw[i] = pack_row(v[0], v[1], v[2], v[3]);
          }
          break;
        }
        case 7:
        case 8: pred_z1(m == 7 ? 64 : 27, A, r0, c0, last, pw); break;  // D45, D67
        case 9:
        case 10:
        case 11:  // D113, D135, D157
          pred_z2(m == 9 ? 27 : m == 10 ? 64 : 151, m == 9 ? 151 : m == 10 ? 64 : 27, A, L, r0, c0, pw);
          break;
        default: {  // z3: D203 (derivative 27), from the column left
          int v[16];
#pragma unroll
          for (int j = 0; j < 4; j++) {
            const int pos = (c0 + j + 1) * 27, b0 = (pos >> 6) + r0, sh = (pos & 63) >> 1;
#pragma unroll
            for (int i = 0; i < 4; i++) v[4 * i + j] = blend32(L[min(b0 + i, last)], L[min(b0 + i + 1, last)], sh);
          }
#pragma unroll
          for (int i = 0; i < 4; i++) pw[i] = pack_row(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
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
