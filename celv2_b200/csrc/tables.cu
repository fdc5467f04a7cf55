// tables.cu: the (block, 4x4 tile) work items of a superblock, shared by the intra and compound
// stages.
//
// Item order: blocks grouped by size class, largest first -- 64x64 (1 block x 256 tiles),
// 64x32 / 32x64 (4 x 128), 32x32 (4 x 64), 32x16 / 16x32 (16 x 32), 16x16 (16 x 16), 16x8 / 8x16
// (64 x 8), 8x8 (64 x 4), 8x4 / 4x8 (256 x 2): 3072 items, every class boundary a multiple of 32,
// so a warp's 32 consecutive items hold whole blocks (or 32 tiles of one) and a block's tile sums
// reduce with shuffles over a power-of-two segment. Intra items are the last 2304 (blocks below
// 64x64 size, kMaxBlockSize, src/gpu/intra_common.h:39).
#include <vector>

#include "tables.h"

namespace celv2cu {

static void build_items(std::vector<uint32_t>& items) {
  items.clear();
  // size classes in order: (level, kinds)
  struct Cls { int level; bool halves; };
  const Cls classes[8] = {{0, false}, {0, true}, {1, false}, {1, true}, {2, false}, {2, true}, {3, false}, {3, true}};
  for (const Cls& c : classes) {
    const int n = 1 << c.level;
    for (int i = 0; i < n * n; i++) {
      const int sq = sb_level_offset(c.level) + i;
      for (int kind = c.halves ? 1 : 0; kind < (c.halves ? 5 : 1); kind++) {
        const int b = sq * 5 + kind;
        int x, y, w, h;
        sb_block_geom(b, x, y, w, h);
        for (int ty = 0; ty < h / 4; ty++)
          for (int tx = 0; tx < w / 4; tx++) items.push_back(pack_item(b, x / 4 + tx, y / 4 + ty));
      }
    }
  }
}

cudaError_t make_items(uint32_t** dev) {
  std::vector<uint32_t> items;
  build_items(items);
  if ((int)items.size() != kItems) return cudaErrorInvalidValue;
  cudaError_t e = cudaMalloc(dev, kItems * sizeof(uint32_t));
  if (e != cudaSuccess) return e;
  return cudaMemcpy(*dev, items.data(), kItems * sizeof(uint32_t), cudaMemcpyHostToDevice);
}

}  // namespace celv2cu
