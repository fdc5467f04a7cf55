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

// 8-bit luma (pw x ph, row pitch `pitch`) into level 0 with its margin.
__global__ void k_expand_u8(const uint8_t* __restrict__ raw, int pitch, DevPlane dst) {
  const int W = dst.w + 2 * dst.margin, H = dst.h + 2 * dst.margin;
  const int x = blockIdx.x * blockDim.x + threadIdx.x - dst.margin;
  const int y = blockIdx.y * blockDim.y + threadIdx.y - dst.margin;
  if (x + dst.margin >= W || y + dst.margin >= H) return;
  const int sx = clampi(x, 0, dst.w - 1), sy = clampi(y, 0, dst.h - 1);
  const_cast<uint8_t*>(dst.p)[(long long)y * dst.stride + x] = raw[(long long)sy * pitch + sx];
}

// High-depth luma rounded to 8 bits on the way in: min(255, (v + half) >> shift).
__global__ void k_expand_u16(const uint16_t* __restrict__ raw, int pitch, int bit_depth, DevPlane dst) {
  const int W = dst.w + 2 * dst.margin, H = dst.h + 2 * dst.margin;
  const int x = blockIdx.x * blockDim.x + threadIdx.x - dst.margin;
  const int y = blockIdx.y * blockDim.y + threadIdx.y - dst.margin;
  if (x + dst.margin >= W || y + dst.margin >= H) return;
  const int sx = clampi(x, 0, dst.w - 1), sy = clampi(y, 0, dst.h - 1);
  const int v = raw[(long long)sy * pitch + sx];
  const int shift = bit_depth - 8;
  const int r = shift > 0 ? (v + (1 << (shift - 1))) >> shift : v;
  const_cast<uint8_t*>(dst.p)[(long long)y * dst.stride + x] = (uint8_t)(r > 255 ? 255 : r);
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

// AV2 EIGHTTAP_REGULAR at the quarter phases (src/gpu/inter_common.h:13-19).
__constant__ int c_taps[4][8] = {{0, 0, 0, 128, 0, 0, 0, 0},
                                 {0, 2, -14, 110, 38, -10, 2, 0},
                                 {0, 2, -14, 76, 76, -14, 2, 0},
                                 {0, 2, -10, 38, 110, -14, 2, 0}};

// The 15 quarter-pel phase planes of level 0 (phase k at lv0.p + k * lv0.phase): one thread per
// stored position computes the four horizontal sums of each of the 8 rows once and combines them
// into all 15 phases, so the 8x8 source neighbourhood is read once per position.
__global__ void k_subpel_phases(DevPlane lv0) {
  const int W = lv0.w + 2 * lv0.margin, H = lv0.h + 2 * lv0.margin;
  const int x = blockIdx.x * blockDim.x + threadIdx.x - lv0.margin;
  const int y = blockIdx.y * blockDim.y + threadIdx.y - lv0.margin;
  if (x + lv0.margin >= W || y + lv0.margin >= H) return;
  const int cx = clampi(x, 0, lv0.w - 1), cy = clampi(y, 0, lv0.h - 1);
  int hs[4][8];  // hs[qx][i]: horizontal sum of row cy + i - 3 at phase qx (unrounded)
#pragma unroll
  for (int i = 0; i < 8; i++) {
    int px[8];
#pragma unroll
    for (int j = 0; j < 8; j++) px[j] = at(lv0, cy + i - 3, cx + j - 3);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      int s = 0;
#pragma unroll
      for (int j = 0; j < 8; j++) s += c_taps[q][j] * px[j];
      hs[q][i] = s;
    }
  }
  uint8_t* base = const_cast<uint8_t*>(lv0.p) + (long long)y * lv0.stride + x;
#pragma unroll
  for (int k = 1; k < kPhases; k++) {
    const int qy = k >> 2, qx = k & 3;
    int v = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) v += c_taps[qy][i] * hs[qx][i];
    v = (v + (1 << 13)) >> 14;
    base[(long long)k * lv0.phase] = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
  }
}

static dim3 plane_grid(const DevPlane& p, dim3 block) {
  const int W = p.w + 2 * p.margin, H = p.h + 2 * p.margin;
  return dim3((W + block.x - 1) / block.x, (H + block.y - 1) / block.y);
}

void launch_expand_u8(const uint8_t* raw, int pitch, const DevPlane& lv0, cudaStream_t st) {
  const dim3 b(128, 2);
  k_expand_u8<<<plane_grid(lv0, b), b, 0, st>>>(raw, pitch, lv0);
}

void launch_expand_u16(const uint16_t* raw, int pitch, int bit_depth, const DevPlane& lv0, cudaStream_t st) {
  const dim3 b(128, 2);
  k_expand_u16<<<plane_grid(lv0, b), b, 0, st>>>(raw, pitch, bit_depth, lv0);
}

void launch_pyramid(const DevPyramid& pyr, cudaStream_t st) {
  const dim3 b(128, 2);
  for (int l = 1; l < kLevels; l++) k_downsample<<<plane_grid(pyr.lv[l], b), b, 0, st>>>(pyr.lv[l - 1], pyr.lv[l]);
}

void launch_phases(const DevPlane& lv0, cudaStream_t st) {
  const dim3 b(64, 4);
  k_subpel_phases<<<plane_grid(lv0, b), b, 0, st>>>(lv0);
}

}  // namespace celv2cu
