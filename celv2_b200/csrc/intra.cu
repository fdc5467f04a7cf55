// intra.cu: the SATD of every candidate block under each of the 13 intra modes.
//
// Reference rules (src/gpu/intra_common.h): edge_above / edge_left (:47-56), dir_pred (:60-85),
// intra_pred (:89-118), dc_value (:120-128), block_mode_satd (:149-163). Blocks of the 64x64
// square are never intra (kMaxBlockSize 32, :39), so 420 blocks x 13 modes per superblock.
//
// One CTA per superblock:
//  1. the source samples the predictions and residuals read -- rows and columns -1 .. 95 around
//     the superblock origin (above-right / below-left edges reach w + h - 1 past a block) -- are
//     staged in shared memory from the margin plane (which already holds the clamped values);
//  2. every block's DC value is computed once;
//  3. the 2304 (block, 4x4 tile) items are spread over the threads; each computes its tile's
//     13 predictions and Hadamards, and a segmented shuffle reduction sums a block's tiles.
// The output is raw SATDs; the finalize stage adds lambda * bits (which depend on whether the
// frame has references, unknown when prepare() runs this ahead of its launch).
#include "kernels.h"
#include "tables.h"

namespace celv2cu {

constexpr int kIntraThreads = 256;
constexpr int kRegion = 97;   // local rows / columns -1 .. 95
constexpr int kRegionStride = 100;

struct IntraSmem {
  uint8_t px[kRegion * kRegionStride];
  int dc[kBlocks];
  int acc[kBlocks][kModes];
};

// A block's view of the staged samples: local coordinates relative to the superblock origin.
struct IntraBlock {
  const uint8_t* px;
  int x, y, w, h;     // local block position and size
  bool top, left;     // the block touches the frame's top / left edge
  __device__ __forceinline__ int s(int ly, int lx) const { return px[(ly + 1) * kRegionStride + lx + 1]; }
  // edge_above / edge_left (intra_common.h:47-56)
  __device__ __forceinline__ int above(int k) const {
    if (top) return 128;
    if (k < 0 && left) return s(y - 1, x);
    return s(y - 1, x + k);
  }
  __device__ __forceinline__ int leftc(int k) const {
    if (left) return 128;
    if (k < 0 && top) return s(y, x - 1);
    return s(y + k, x - 1);
  }
};

__device__ __forceinline__ int dr_derivative(int a) { return a == 23 ? 151 : a == 45 ? 64 : 27; }

// dr_prediction z1 / z2 / z3 without edge filter (intra_common.h:61-85). Not inlined: the six
// directional modes share one copy, which keeps the per-tile loop within the register budget.
__device__ __noinline__ int dir_pred(const IntraBlock& B, int angle, int i, int j) {
  const int last = B.w + B.h - 1;
  if (angle < 90) {
    const int pos = (i + 1) * dr_derivative(angle), base = (pos >> 6) + j, shift = (pos & 63) >> 1;
    const int a0 = B.above(base < last ? base : last), a1 = B.above(base + 1 < last ? base + 1 : last);
    return (a0 * (32 - shift) + a1 * shift + 16) >> 5;
  }
  if (angle > 180) {
    const int pos = (j + 1) * dr_derivative(270 - angle), base = (pos >> 6) + i, shift = (pos & 63) >> 1;
    const int l0 = B.leftc(base < last ? base : last), l1 = B.leftc(base + 1 < last ? base + 1 : last);
    return (l0 * (32 - shift) + l1 * shift + 16) >> 5;
  }
  const int px = (j << 6) - (i + 1) * dr_derivative(180 - angle);
  const int bx = px >= 0 ? px >> 6 : -((-px + 63) >> 6);
  if (bx >= -1) {
    const int shift = (px - bx * 64) >> 1;
    return (B.above(bx) * (32 - shift) + B.above(bx + 1) * shift + 16) >> 5;
  }
  const int py = (i << 6) - (j + 1) * dr_derivative(angle - 90);
  const int by = py >= 0 ? py >> 6 : -((-py + 63) >> 6);
  const int shift = (py - by * 64) >> 1;
  const int b0 = by < -1 ? -1 : by, b1 = by + 1 < -1 ? -1 : by + 1;
  return (B.leftc(b0) * (32 - shift) + B.leftc(b1) * shift + 16) >> 5;
}

// intra_pred (intra_common.h:89-118) for modes 1..12 at block sample (i, j).
__device__ __forceinline__ int intra_pred(const IntraBlock& B, int mode, int i, int j) {
  switch (mode) {
    case 1: return B.top ? 128 : B.s(B.y - 1, B.x + j);
    case 2: return B.left ? 128 : B.s(B.y + i, B.x - 1);
    case 3: {
      const int a = B.top ? 128 : B.s(B.y - 1, B.x + j), l = B.left ? 128 : B.s(B.y + i, B.x - 1);
      const int tr = B.top ? 128 : B.s(B.y - 1, B.x + B.w - 1), bl = B.left ? 128 : B.s(B.y + B.h - 1, B.x - 1);
      const int den = B.w + B.h + 2, num = (B.h - i) * a + (i + 1) * bl + (B.w - j) * l + (j + 1) * tr;
      return (num + den / 2) / den;
    }
    case 4: return ((B.h - 1 - i) * B.above(j) + (i + 1) * B.leftc(B.h - 1) + B.h / 2) / B.h;
    case 5: return ((B.w - 1 - j) * B.leftc(i) + (j + 1) * B.above(B.w - 1) + B.w / 2) / B.w;
    case 6: {
      const int a = B.above(j), l = B.leftc(i), tl = B.above(-1);
      const int base = a + l - tl, pa = abs(base - a), pl = abs(base - l), ptl = abs(base - tl);
      return pl <= pa && pl <= ptl ? l : pa <= ptl ? a : tl;
    }
    default: {
      constexpr int kAngle[6] = {45, 67, 113, 135, 157, 203};
      return dir_pred(B, kAngle[mode - 7], i, j);
    }
  }
}

__global__ void __launch_bounds__(kIntraThreads) k_intra(const FrameJob* __restrict__ jobs, WorkList w) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  IntraSmem& S = *reinterpret_cast<IntraSmem*>(smem_raw);
  const int tid = threadIdx.x;
  const int unit = blockIdx.x;
  const int jb = job_of(w, unit);
  const FrameJob& job = jobs[jb];
  const int sb = unit - w.prefix[jb], sby = sb / job.sb_cols, sbx = sb - sby * job.sb_cols;
  const int ox = sbx * 64, oy = sby * 64;
  const DevPlane src = job.cur.lv[0];

  // 1. staged samples (clamped positions are what the margin holds)
  for (int e = tid; e < kRegion * kRegion; e += kIntraThreads) {
    const int ly = e / kRegion - 1, lx = e % kRegion - 1;
    S.px[(ly + 1) * kRegionStride + lx + 1] = (uint8_t)at(src, oy + ly, ox + lx);
  }
  for (int e = tid; e < kBlocks * kModes; e += kIntraThreads) (&S.acc[0][0])[e] = 0;
  __syncthreads();
  // 2. DC values (dc_value, intra_common.h:120-128)
  for (int b = tid; b < kBlocks; b += kIntraThreads) {
    int x, y, bw, bh;
    sb_block_geom(b, x, y, bw, bh);
    const bool has_a = oy + y > 0, has_l = ox + x > 0;
    int sum = 0, n = 0;
    if (has_a)
      for (int j = 0; j < bw; j++) sum += S.px[y * kRegionStride + x + j + 1], n++;
    if (has_l)
      for (int i = 0; i < bh; i++) sum += S.px[(y + i + 1) * kRegionStride + x], n++;
    S.dc[b] = n ? (sum + n / 2) / n : 128;
  }
  __syncthreads();
  // 3. (block, tile) items: 13 predictions + Hadamards per tile, segment sums per block
  for (int base = kIntraFirst; base < kItems; base += kIntraThreads) {
    const int item = base + tid;  // kIntraItems is a multiple of the CTA size: always valid
    const uint32_t it = job.items[item];
    const int b = item_block(it), width = item_width(item);
    IntraBlock B;
    B.px = S.px;
    sb_block_geom(b, B.x, B.y, B.w, B.h);
    B.top = oy + B.y == 0, B.left = ox + B.x == 0;
    const int tx = item_tx(it) * 4, ty = item_ty(it) * 4;  // superblock-local tile origin
    int cur[16];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) cur[4 * i + j] = B.s(ty + i, tx + j);
    const int bi = ty - B.y, bj = tx - B.x;  // tile origin inside the block
#pragma unroll 1
    for (int m = 0; m < kModes; m++) {
      int d[16];
      if (m == 0) {
#pragma unroll
        for (int k = 0; k < 16; k++) d[k] = cur[k] - S.dc[b];
      } else {
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int j = 0; j < 4; j++) d[4 * i + j] = cur[4 * i + j] - intra_pred(B, m, bi + i, bj + j);
      }
      const int s = segment_sum(hadamard4x4(d), width);
      if ((tid & ((width < 32 ? width : 32) - 1)) == 0) atomicAdd(&S.acc[b][m], s);
    }
  }
  __syncthreads();
  int* out = const_cast<int*>(job.intra) + (long long)sb * kBlocks * kModes;
  for (int e = tid; e < kBlocks * kModes; e += kIntraThreads) out[e] = (&S.acc[0][0])[e];
}

void launch_intra(const FrameJob* jobs, const WorkList& w, cudaStream_t st) {
  const int units = w.prefix[w.njobs];
  if (units <= 0) return;
  k_intra<<<units, kIntraThreads, sizeof(IntraSmem), st>>>(jobs, w);
}

cudaError_t intra_attributes() {
  return cudaFuncSetAttribute(k_intra, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(IntraSmem));
}

}  // namespace celv2cu
