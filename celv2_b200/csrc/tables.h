// tables.h: the superblock's (block, 4x4 tile) work items (see tables.cu for their order).
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace celv2cu {

constexpr int kItems = 3072;       // every block's tiles
constexpr int kIntraFirst = 768;   // first item of a block below 64x64
constexpr int kIntraItems = kItems - kIntraFirst;

// item: block (9 bits) | tile column in the superblock (4 bits) << 9 | tile row (4 bits) << 13
__host__ __device__ __forceinline__ uint32_t pack_item(int b, int tx, int ty) {
  return (uint32_t)b | ((uint32_t)tx << 9) | ((uint32_t)ty << 13);
}
__device__ __forceinline__ int item_block(uint32_t it) { return (int)(it & 511); }
__device__ __forceinline__ int item_tx(uint32_t it) { return (int)((it >> 9) & 15); }
__device__ __forceinline__ int item_ty(uint32_t it) { return (int)((it >> 13) & 15); }

// Tiles per block of the class item i belongs to (the reduction segment width).
__device__ __forceinline__ int item_width(int i) {
  return i < 256 ? 256 : i < 768 ? 128 : i < 1024 ? 64 : i < 1536 ? 32 : i < 1792 ? 16 : i < 2304 ? 8 : i < 2560 ? 4 : 2;
}

// The item table in device memory (one per device, made once; FrameJob::items points at it).
cudaError_t make_items(uint32_t** dev);

// Sum of v over the lanes of this lane's segment of `width` lanes (power of two); every lane of
// the segment ends with the sum. For width >= 32 the whole warp is one segment.
__device__ __forceinline__ int segment_sum(int v, int width) {
  const int span = width < 32 ? width : 32;
  for (int off = span >> 1; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

}  // namespace celv2cu
