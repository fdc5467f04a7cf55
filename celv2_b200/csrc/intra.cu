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

// n / d for 0 <= n < 2^20, from a float estimate corrected to the exact quotient.
__device__ __forceinline__ int exact_div(int n, int d, float rcp) {
  int q = __float2int_rz((float)n * rcp);
  if ((q + 1) * d <= n) q++;
  if (q * d > n) q--;
  return q;
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
    int cur[16];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) cur[4 * i + j] = S.px[(ty * 4 + i + 1) * kRegionStride + tx * 4 + j + 1];
    const int lgw = 31 - __clz(bw), lgh = 31 - __clz(bh);
    const int den = bw + bh + 2;
    const float rcp = 1.0f / (float)den;
#pragma unroll 1
    for (int m = 0; m < kModes; m++) {
      int d[16];
      switch (m) {
        case 0: {
          const int v = S.dc[b];
#pragma unroll
          for (int k = 0; k < 16; k++) d[k] = cur[k] - v;
          break;
        }
        case 1:
#pragma unroll
          for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) d[4 * i + j] = cur[4 * i + j] - A[c0 + j];
          break;
        case 2:
#pragma unroll
          for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) d[4 * i + j] = cur[4 * i + j] - L[r0 + i];
          break;
        case 3: {  // Smooth: bilinear blend of above, left, top-right and bottom-left
          const int tr = A[bw - 1], bl = L[bh - 1];
#pragma unroll
          for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) {
              const int ii = r0 + i, jj = c0 + j;
              const int num = (bh - ii) * A[jj] + (ii + 1) * bl + (bw - jj) * L[ii] + (jj + 1) * tr;
              d[4 * i + j] = cur[4 * i + j] - exact_div(num + den / 2, den, rcp);
            }
          break;
        }
        case 4: {  // SmoothV (h is a power of two, the numerator non-negative)
          const int bl = L[bh - 1];
#pragma unroll
          for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) {
              const int ii = r0 + i;
              d[4 * i + j] = cur[4 * i + j] - (((bh - 1 - ii) * A[c0 + j] + (ii + 1) * bl + bh / 2) >> lgh);
            }
          break;
        }
        case 5: {  // SmoothH
          const int tr = A[bw - 1];
#pragma unroll
          for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) {
              const int jj = c0 + j;
              d[4 * i + j] = cur[4 * i + j] - (((bw - 1 - jj) * L[r0 + i] + (jj + 1) * tr + bw / 2) >> lgw);
            }
          break;
        }
        case 6: {  // Paeth
          const int tl = A[-1];
#pragma unroll
          for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) {
              const int a = A[c0 + j], l = L[r0 + i], bse = a + l - tl;
              const int pa = abs(bse - a), pl = abs(bse - l), ptl = abs(bse - tl);
              d[4 * i + j] = cur[4 * i + j] - (pl <= pa && pl <= ptl ? l : pa <= ptl ? a : tl);
            }
          break;
        }
        case 7:
        case 8: {  // z1: D45 (derivative 64), D67 (27), from the row above
          const int dxa = m == 7 ? 64 : 27;
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const int pos = (r0 + i + 1) * dxa, b0 = (pos >> 6) + c0, sh = (pos & 63) >> 1;
#pragma unroll
            for (int j = 0; j < 4; j++) {
              const int p0 = A[min(b0 + j, last)], p1 = A[min(b0 + j + 1, last)];
              d[4 * i + j] = cur[4 * i + j] - ((p0 * (32 - sh) + p1 * sh + 16) >> 5);
            }
          }
          break;
        }
        case 12: {  // z3: D203 (derivative 27), from the column left
#pragma unroll
          for (int j = 0; j < 4; j++) {
            const int pos = (c0 + j + 1) * 27, b0 = (pos >> 6) + r0, sh = (pos & 63) >> 1;
#pragma unroll
            for (int i = 0; i < 4; i++) {
              const int p0 = L[min(b0 + i, last)], p1 = L[min(b0 + i + 1, last)];
              d[4 * i + j] = cur[4 * i + j] - ((p0 * (32 - sh) + p1 * sh + 16) >> 5);
            }
          }
          break;
        }
        default: {  // z2: D113, D135, D157 -- the row above while the projection stays on it
          const int dxa = m == 9 ? 27 : m == 10 ? 64 : 151, dya = m == 9 ? 151 : m == 10 ? 64 : 27;
#pragma unroll
          for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) {
              const int ii = r0 + i, jj = c0 + j;
              const int px = (jj << 6) - (ii + 1) * dxa, bx = px >> 6;
              int p;
              if (bx >= -1) {
                const int sh = (px & 63) >> 1;
                p = (A[bx] * (32 - sh) + A[bx + 1] * sh + 16) >> 5;
              } else {
                const int py = (ii << 6) - (jj + 1) * dya, by = py >> 6, sh = (py & 63) >> 1;
                p = (L[max(by, -1)] * (32 - sh) + L[max(by + 1, -1)] * sh + 16) >> 5;
              }
              d[4 * i + j] = cur[4 * i + j] - p;
            }
          break;
        }
      }
      const int s = segment_sum(hadamard4x4(d), width);
      if ((tid & ((width < 32 ? width : 32) - 1)) == 0) atomicAdd(&S.acc[b][m], s);
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
