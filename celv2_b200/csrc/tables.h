// tables.h: the superblock's (block, 4x4 tile) work items.
//
// Item order: blocks grouped by size class, largest first -- 64x64 (1 block x 256 tiles),
// 64x32 / 32x64 (4 x 128), 32x32 (4 x 64), 32x16 / 16x32 (16 x 32), 16x16 (16 x 16), 16x8 / 8x16
// (64 x 8), 8x8 (64 x 4), 8x4 / 4x8 (256 x 2): 3072 items, every class boundary a multiple of 32,
// so a warp's 32 consecutive items hold whole blocks (or 32 tiles of one) and a block's tile sums
// reduce with shuffles over a power-of-two segment. Intra items are the last 2304 (blocks below
// 64x64 size, kMaxBlockSize, src/gpu/intra_common.h:39). Within a block, tiles are in raster order.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace celv2cu {

constexpr int kItems = 3072;       // every block's tiles
constexpr int kIntraFirst = 768;   // first item of a block below 64x64
constexpr int kIntraItems = kItems - kIntraFirst;

// Tiles per block of the class item i belongs to (the reduction segment width).
__device__ __forceinline__ int item_width(int i) {
  return i < 256 ? 256 : i < 768 ? 128 : i < 1024 ? 64 : i < 1536 ? 32 : i < 1792 ? 16 : i < 2304 ? 8 : i < 2560 ? 4 : 2;
}

// Item i's block and tile position in the superblock (tile units of 4 samples), from the class
// structure: class c covers squares of level c / 2, whole (even c) or as halves (odd c).
__device__ __forceinline__ void item_decode(int i, int& b, int& tx, int& ty) {
  const int c = i < 256 ? 0 : i < 768 ? 1 : i < 1024 ? 2 : i < 1536 ? 3 : i < 1792 ? 4 : i < 2304 ? 5 : i < 2560 ? 6 : 7;
  const int start = c == 0 ? 0 : c == 1 ? 256 : c == 2 ? 768 : c == 3 ? 1024 : c == 4 ? 1536 : c == 5 ? 1792 : c == 6 ? 2304 : 2560;
  const int level = c >> 1;
  const int lwt = (c & 1) ? (2 * (4 - level) - 1) : (2 * (4 - level));  // log2(tiles per block)
  const int k = i - start, blk = k >> lwt, t = k & ((1 << lwt) - 1);
  const int sq = sb_level_offset(level) + ((c & 1) ? (blk >> 2) : blk);
  const int kind = (c & 1) ? 1 + (blk & 3) : 0;
  b = sq * 5 + kind;
  int x, y, w, h;
  sb_block_geom(b, x, y, w, h);
  const int tw = w >> 2;
  tx = (x >> 2) + (t % tw), ty = (y >> 2) + (t / tw);
}

// Sum of v over the lanes of this lane's segment of `width` lanes (power of two); every lane of
// the segment ends with the sum. For width >= 32 the whole warp is one segment.
__device__ __forceinline__ int segment_sum(int v, int width) {
  const int span = width < 32 ? width : 32;
  for (int off = span >> 1; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

}  // namespace celv2cu
