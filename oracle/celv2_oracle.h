/* celv2_oracle.h: CPU restatement of the reference decision engine's integer rules, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the CUDA engine is compared against: only the
 * tests, the smoke check and the benchmark's CPU-baseline leg load it. The product path never
 * calls it and has no CPU fallback.
 *
 * Every function cites the reference file:line it restates (paths inside the Stou-1/celv2 tree).
 * The restatement is pinned against the reference itself: oracle/Makefile compiles the
 * reference's own CpuEngine sources into oracle/_ref/, and tests/golden/ holds decision digests
 * the reference produced (tests/golden/make_golden.py). */
#ifndef CELV2_ORACLE_H
#define CELV2_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#include "celv2_decision.h"

#ifdef __cplusplus
extern "C" {
#endif

/* 10-bit (or 12-bit) samples to the 8-bit ones the engine scores: min(255, (v + half) >> shift)
 * (src/io/y4m.cpp:28-34). */
void oro_round_to_8bit(const uint16_t* hi, uint8_t* lo, size_t n, int bit_depth);

/* Edge replication of the visible w x h area into a pw x ph plane (src/io/y4m.cpp:36-42). */
void oro_pad_plane(uint8_t* p, int stride, int w, int h, int pw, int ph);

/* Pyramid geometry (src/gpu/kernels_ref.cpp:213-238): level 0 is pw x ph, level l+1 halves
 * level l (floor); a reference's level 0 is followed by its 15 quarter-pel phase planes. */
typedef struct oro_pyr {
  int w[CELV2_ME_LEVELS], h[CELV2_ME_LEVELS];
  size_t off[CELV2_ME_LEVELS]; /* byte offset of each level in the buffer */
  size_t phase;                /* distance between phase planes of level 0 (0: none) */
  size_t total;                /* buffer size in bytes */
} oro_pyr;
void oro_pyr_layout(int pw, int ph, int phases, oro_pyr* L);
void oro_build_pyramid(const uint8_t* y, int pw, int ph, int phases, uint8_t* buf);

/* Motion fields (integer pels, level 0 quarter pels) of every level, coarsest first
 * (src/gpu/kernels_ref.cpp:240-251, src/gpu/cpu_engine.cpp:40-46,68-83). Field l has
 * cols = (w_l + 7) / 8 by rows = (h_l + 7) / 8 cells, row-major. */
void oro_field_dims(int pw, int ph, int cols[CELV2_ME_LEVELS], int rows[CELV2_ME_LEVELS]);
void oro_me_fields(const uint8_t* cur_pyr, const uint8_t* ref_pyr, int pw, int ph, int32_t* mvx[CELV2_ME_LEVELS],
                   int32_t* mvy[CELV2_ME_LEVELS]);

/* One frame's decisions, every superblock's record in raster order (sb_cols x sb_rows records):
 * the source and up to 7 references (nearest first) as padded pw x ph 8-bit luma planes; nrefs 0
 * is a KEY frame. Returns 0, or -1 on bad arguments. threads <= 0: all OpenMP threads. */
int oro_decide(const uint8_t* src_y, int width, int height, const uint8_t* const* ref_y, int nrefs,
               int64_t lambda_q8, int threads, celv2_sb_out* out);

/* oro_decide with pruning masks (an extension for testing the engine's pruned search; no
 * reference rule): keep (NULL: none) holds one keep word per superblock (celv2_decision.h: the
 * references, intra, the block levels and the intra modes kept); a KEY frame always scores
 * everything. A superblock scores what it keeps exactly as oro_decide does and picks among it; a
 * block of a pruned level is no candidate and enters the partition choice at CELV2_PRUNED_COST.
 * sb_cost (NULL: not written) receives each superblock's chosen partition cost. */
int oro_decide_masked(const uint8_t* src_y, int width, int height, const uint8_t* const* ref_y, int nrefs,
                      int64_t lambda_q8, int threads, const uint32_t* keep, celv2_sb_out* out, int64_t* sb_cost);

/* The same from prebuilt pyramids and level-0 fields (for the stage-by-stage tests). */
int oro_decide_from_fields(const uint8_t* src_y, int width, int height, const uint8_t* const* ref_pyr,
                           const int32_t* const* mvx0, const int32_t* const* mvy0, int nrefs, int64_t lambda_q8,
                           int threads, celv2_sb_out* out);

/* Per-candidate-block intra SATDs of one superblock: satd[b * 13 + mode] for blocks b >= 5 (the
 * 64x64 square's blocks are never intra, kMaxBlockSize), 0 for b < 5. */
void oro_intra_satd_sb(const uint8_t* src_y, int pw, int ph, int sb_col, int sb_row, int32_t* satd);

/* Primitives, exposed for unit tests. */
int oro_hadamard4x4(const int* d);
int oro_subpel_px(const uint8_t* p, int stride, int w, int h, int y, int x, int qy, int qx);
int oro_intra_pred(const uint8_t* p, int stride, int w, int h, int x, int y, int bw, int bh, int mode, int i,
                   int j);
int oro_dc_value(const uint8_t* p, int stride, int w, int h, int x, int y, int bw, int bh);
void oro_sb_block_geom(int b, int* x, int* y, int* w, int* h);
int oro_me_cell(const uint8_t* cur, const uint8_t* ref, int stride, int w, int h, int bx, int by, const int32_t* pmx,
                const int32_t* pmy, int pcols, int prows, int level0, int32_t* mvx, int32_t* mvy);

#ifdef __cplusplus
}
#endif

#endif /* CELV2_ORACLE_H */
