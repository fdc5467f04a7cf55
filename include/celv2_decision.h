/* celv2_decision.h: the per-superblock decision record the CUDA decision engine emits.
 *
 * The layout is, field for field and byte for byte, the reference encoder's device decision record
 * `celv2::SbOut` (src/gpu/sb_out.h:13-31), so the reference host code converts it into a
 * DecisionMap with its own `celv2::sb_out_to_decision` (src/gpu/decision_map.cpp:65-105) unchanged.
 * Plain C, no CUDA or torch types: this is the boundary format.
 *
 * Conventions (reference src/gpu/sb_blocks.h:1-37, src/gpu/decision_map.h:17-102):
 *  - a 64x64 superblock has 425 candidate blocks: 85 squares (64x64, then 4 of 32x32, 16 of 16x16,
 *    64 of 8x8, raster order per level), each whole (kind 0) and as its top, bottom, left and right
 *    half (kinds 1-4); block b = square * 5 + kind;
 *  - motion vectors are in quarter pels here (the DecisionMap holds them doubled, in 1/8 pel);
 *  - mode 13 (CELV2_NUM_MODES) marks an inter block, 0..12 are the intra modes DC, V, H, Smooth,
 *    SmoothV, SmoothH, Paeth, D45, D67, D113, D135, D157, D203;
 *  - tree[] is the partition tree in preorder (0 NONE, 1 HORZ, 2 VERT, 3 SPLIT), the leaves are in
 *    coding order;
 *  - entries past ntree / nblocks are zero in every record this project writes. */
#ifndef CELV2_DECISION_H
#define CELV2_DECISION_H

#include <stdint.h>

#define CELV2_SB_SIZE 64
#define CELV2_SB_OUT_CAP 256
#define CELV2_SB_SQUARES 85
#define CELV2_SB_BLOCKS 425
#define CELV2_MAX_REFS 7
#define CELV2_NUM_MODES 13
#define CELV2_ME_LEVELS 5
#define CELV2_SINGLE_REF 255
#define CELV2_NO_REF_COST 0xffffffffu

typedef struct celv2_sb_out {
  int32_t ntree, nblocks;
  uint8_t tree[CELV2_SB_OUT_CAP];
  uint8_t w4[CELV2_SB_OUT_CAP], h4[CELV2_SB_OUT_CAP], mode[CELV2_SB_OUT_CAP];
  int16_t mvx[CELV2_SB_OUT_CAP], mvy[CELV2_SB_OUT_CAP];
  uint8_t ref[CELV2_SB_OUT_CAP];
  uint8_t ref2[CELV2_SB_OUT_CAP];
  int16_t mv2x[CELV2_SB_OUT_CAP], mv2y[CELV2_SB_OUT_CAP];
  /* every candidate block: best inter choice and best intra mode, costs SATD*256 + lambda*bits
   * (INT64_MAX where there is none) */
  int64_t c_inter_cost[CELV2_SB_BLOCKS], c_intra_cost[CELV2_SB_BLOCKS];
  int16_t c_mvx[CELV2_SB_BLOCKS], c_mvy[CELV2_SB_BLOCKS], c_mv2x[CELV2_SB_BLOCKS], c_mv2y[CELV2_SB_BLOCKS];
  uint8_t c_ref[CELV2_SB_BLOCKS], c_ref2[CELV2_SB_BLOCKS], c_intra[CELV2_SB_BLOCKS];
  /* each reference's best single-reference MV with its cost >> 8, saturated at 0xfffffffe;
   * 0xffffffff where the reference has none */
  uint32_t c_rcost[CELV2_MAX_REFS][CELV2_SB_BLOCKS];
  int16_t c_rmvx[CELV2_MAX_REFS][CELV2_SB_BLOCKS], c_rmvy[CELV2_MAX_REFS][CELV2_SB_BLOCKS];
} celv2_sb_out;

/* Keep words of the pruned search (no counterpart in the reference, which always searches
 * exhaustively): per superblock of an inter frame, which options the exact scorer evaluates.
 *  bits 0-6   reference r (none set: all of them);
 *  bit 7      the intra modes;
 *  bits 8-11  the candidate blocks of square level l (0: 64x64, 64x32, 32x64; 1: 32x32, 32x16,
 *             16x32; 2: 16x16, 16x8, 8x16; 3: 8x8, 8x4, 4x8) (none set: all levels);
 *  bits 16-28 intra mode m (none set: all modes).
 * A kept option is scored exactly as the exhaustive search scores it; a block of a pruned level is
 * no candidate (its record reads as one with no choice: costs INT64_MAX, reference costs
 * CELV2_NO_REF_COST) and the partition choice takes it at cost CELV2_PRUNED_COST, so that any
 * non-empty set of levels leaves a complete partition. A KEY frame always scores everything. */
#define CELV2_KEEP_REFS 0x7Fu
#define CELV2_KEEP_INTRA 0x80u
#define CELV2_KEEP_LEVEL(l) (0x100u << (l))
#define CELV2_KEEP_LEVELS 0xF00u
#define CELV2_KEEP_MODE(m) (0x10000u << (m))
#define CELV2_KEEP_MODES 0x1FFF0000u
#define CELV2_PRUNED_COST (1LL << 56)

#ifdef __cplusplus
static_assert(sizeof(celv2_sb_out) == 38872, "celv2_sb_out must keep the reference SbOut layout");
#else
_Static_assert(sizeof(celv2_sb_out) == 38872, "celv2_sb_out must keep the reference SbOut layout");
#endif

#endif /* CELV2_DECISION_H */
