// planes.cu: the engine's input planes in HBM -- 8-bit luma with replicated margins, its 2x2
// pyramid and a reference's quarter-pel phase planes.
//
// Reference rules: round_to_8bit (src/io/y4m.cpp:28-34), build_pyramid_ref
// (src/gpu/kernels_ref.cpp:213-238), downsample_px and subpel_px (src/gpu/inter_common.h:13-33,
// 91-94). Every kernel writes the whole stored extent of its plane, margin included: the value at
// a margin position is the plane's value at the clamped position, which is what the reference's
// clamped reads return (for phase planes: the phase value at the clamped whole-pel position).
// All of these are HBM-bound byte kernels: one thread per output sample, row-major, so each warp
// writes 32 consecutive bytes of a row and reads a small neighbourhood that L1 serves.
#include "kernels.h"

namespace celv2cu {

// 8-bit luma (pw x ph, row pitch `pitch`) into level 0 with its margin: four stored samples per
// thread, one 32-bit store (rows and margins are multiples of 8 bytes).
__global__ void k_expand_u8(const uint8_t* __restrict__ raw, int pitch, DevPlane dst) {
  const int W = dst.w + 2 * dst.margin, H = dst.h + 2 * dst.margin;
  const int x = 4 * (blockIdx.x * blockDim.x + threadIdx.x) - dst.margin;
  const int y = blockIdx.y * blockDim.y + threadIdx.y - dst.margin;
  if (x + dst.margin >= W || y + dst.margin >= H) return;
  const uint8_t* row = raw + (long long)clampi(y, 0, dst.h - 1) * pitch;
  uint32_t v = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) v |= (uint32_t)row[clampi(x + k, 0, dst.w - 1)] << (8 * k);
  *reinterpret_cast<uint32_t*>(const_cast<uint8_t*>(dst.p) + (long long)y * dst.stride + x) = v;
}

// High-depth luma rounded to 8 bits on the way in: min(255, (v + half) >> shift); four stored
// samples per thread as for k_expand_u8.
__global__ void k_expand_u16(const uint16_t* __restrict__ raw, int pitch, int bit_depth, DevPlane dst) {
  const int W = dst.w + 2 * dst.margin, H = dst.h + 2 * dst.margin;
  const int x = 4 * (blockIdx.x * blockDim.x + threadIdx.x) - dst.margin;
  const int y = blockIdx.y * blockDim.y + threadIdx.y - dst.margin;
  if (x + dst.margin >= W || y + dst.margin >= H) return;
  const uint16_t* row = raw + (long long)clampi(y, 0, dst.h - 1) * pitch;
  const int shift = bit_depth - 8;
  uint32_t v = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int s = row[clampi(x + k, 0, dst.w - 1)];
    const int r = shift > 0 ? (s + (1 << (shift - 1))) >> shift : s;
    v |= (uint32_t)(r > 255 ? 255 : r) << (8 * k);
  }
  *reinterpret_cast<uint32_t*>(const_cast<uint8_t*>(dst.p) + (long long)y * dst.stride + x) = v;
}

// Level l + 1 from level l: (a + b + c + d + 2) >> 2 of the 2x2 block at the clamped position.
__global__ void k_downsample(DevPlane src, DevPlane dst) {
  const int W = dst.w + 2 * dst.margin, H = dst.h + 2 * dst.margin;
  const int x = blockIdx.x * blockDim.x + threadIdx.x - dst.margin;
  const int y = blockIdx.y * blockDim.y + threadIdx.y - dst.margin;
  if (x + dst.margin >= W || y + dst.margin >= H) return;
  const int sx = clampi(x, 0, dst.w - 1) * 2, sy = clampi(y, 0, dst.h - 1) * 2;
  const int v = at(src, sy, sx) + at(src, sy, sx + 1) + at(src, sy + 1, sx) + at(src, sy + 1, sx + 1);
  const_cast<uint8_t*>(dst.p)[(long long)y * dst.stride + x] = (uint8_t)((v + 2) >> 2);
}

// AV2 EIGHTTAP_REGULAR at the quarter phases (src/gpu/inter_common.h:13-19); taps 0 and 7 are zero
// at every phase.
__constant__ int c_taps[4][8] = {{0, 0, 0, 128, 0, 0, 0, 0},
                                 {0, 2, -14, 110, 38, -10, 2, 0},
                                 {0, 2, -14, 76, 76, -14, 2, 0},
                                 {0, 2, -10, 38, 110, -14, 2, 0}};
constexpr int kPhTW = 64, kPhTH = 16, kPhRows = kPhTH + 7;

// The 15 quarter-pel phase planes of level 0 (phase k at lv0.p + k * lv0.phase), separably: one
// CTA per 64 x 16 tile of stored positions. A position's value is the phase value at its clamped
// whole-pel position, and clamping is monotonic, so the tile's clamped centres span at most 64 x 16
// consecutive columns and rows from (cx0, cy0): their 8 x 8 source neighbourhoods are staged once,
// the horizontal sums at phases 1-3 formed once per (row, column) in shared memory, and each thread
// combines a column of them vertically into the 15 phases of 4 positions.
__global__ void __launch_bounds__(256) k_subpel_phases(DevPlane lv0) {
  __shared__ uint8_t src[kPhRows][kPhTW + 8];  // rows cy0 - 3 .., columns cx0 - 3 ..
  __shared__ int hs[3][kPhRows][kPhTW];         // horizontal sums at phases qx = 1, 2, 3 (unrounded)
  const int W = lv0.w + 2 * lv0.margin, H = lv0.h + 2 * lv0.margin;
  const int x0 = blockIdx.x * kPhTW - lv0.margin, y0 = blockIdx.y * kPhTH - lv0.margin;
  const int cx0 = clampi(x0, 0, lv0.w - 1), cy0 = clampi(y0, 0, lv0.h - 1);
  const int tid = threadIdx.x;
  for (int e = tid; e < kPhRows * (kPhTW + 7); e += 256) {
    const int r = e / (kPhTW + 7), c = e - r * (kPhTW + 7);
    src[r][c] = (uint8_t)at(lv0, cy0 + r - 3, cx0 + c - 3);
  }
  __syncthreads();
  for (int e = tid; e < kPhRows * kPhTW; e += 256) {
    const int r = e / kPhTW, c = e - r * kPhTW;
    int px[8];
#pragma unroll
    for (int j = 1; j < 7; j++) px[j] = src[r][c + j];
#pragma unroll
    for (int q = 1; q < 4; q++) {
      int v = 0;
#pragma unroll
      for (int j = 1; j < 7; j++) v += c_taps[q][j] * px[j];
      hs[q - 1][r][c] = v;
    }
  }
  __syncthreads();
  const int tx = tid & 63, ty = tid >> 6;  // column; rows 4 ty .. 4 ty + 3
  const int x = x0 + tx;
  if (x + lv0.margin >= W) return;
  const int c = clampi(x, 0, lv0.w - 1) - cx0;
#pragma unroll
  for (int k4 = 0; k4 < 4; k4++) {
    const int y = y0 + ty * 4 + k4;
    if (y + lv0.margin >= H) return;
    const int r = clampi(y, 0, lv0.h - 1) - cy0;  // the centre row; taps reach rows r .. r + 7
    uint8_t* base = const_cast<uint8_t*>(lv0.p) + (long long)y * lv0.stride + x;
    int col[4][8];  // col[qx][i]: horizontal sum at phase qx of row r + i
#pragma unroll
    for (int i = 1; i < 7; i++) {
      col[0][i] = 128 * src[r + i][c + 3];
#pragma unroll
      for (int q = 1; q < 4; q++) col[q][i] = hs[q - 1][r + i][c];
    }
#pragma unroll
    for (int k = 1; k < kPhases; k++) {
      const int qy = k >> 2, qx = k & 3;
      int v = 0;
#pragma unroll
      for (int i = 1; i < 7; i++) v += c_taps[qy][i] * col[qx][i];
      v = (v + (1 << 13)) >> 14;
      base[(long long)k * lv0.phase] = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
    }
  }
}

static dim3 plane_grid(const DevPlane& p, dim3 block) {
  const int W = p.w + 2 * p.margin, H = p.h + 2 * p.margin;
  return dim3((W + block.x - 1) / block.x, (H + block.y - 1) / block.y);
}

// Four stored samples per thread: the grid covers the stored width in words (it is a multiple of
// 8 bytes, as are the margin and the stride, so every word store is aligned).
static dim3 expand_grid(const DevPlane& p, dim3 block) {
  const int W = p.w + 2 * p.margin, H = p.h + 2 * p.margin;
  return dim3((W / 4 + block.x - 1) / block.x, (H + block.y - 1) / block.y);
}

void launch_expand_u8(const uint8_t* raw, int pitch, const DevPlane& lv0, cudaStream_t st) {
  const dim3 b(64, 4);
  k_expand_u8<<<expand_grid(lv0, b), b, 0, st>>>(raw, pitch, lv0);
}

void launch_expand_u16(const uint16_t* raw, int pitch, int bit_depth, const DevPlane& lv0, cudaStream_t st) {
  const dim3 b(64, 4);
  k_expand_u16<<<expand_grid(lv0, b), b, 0, st>>>(raw, pitch, bit_depth, lv0);
}

void launch_pyramid(const DevPyramid& pyr, cudaStream_t st) {
  const dim3 b(128, 2);
  for (int l = 1; l < kLevels; l++) k_downsample<<<plane_grid(pyr.lv[l], b), b, 0, st>>>(pyr.lv[l - 1], pyr.lv[l]);
}

void launch_phases(const DevPlane& lv0, cudaStream_t st) {
  const dim3 grid((lv0.w + 2 * lv0.margin + kPhTW - 1) / kPhTW, (lv0.h + 2 * lv0.margin + kPhTH - 1) / kPhTH);
  k_subpel_phases<<<grid, 256, 0, st>>>(lv0);
}

}  // namespace celv2cu
