// finalize.cu: per superblock, every block's best choice and the partition tree, written as the
// decision record (include/celv2_decision.h).
//
// Reference rules (src/gpu/kernels_ref.cpp): best_both / best_mode (:43-104) -- intra modes in
// order with mode bits (+32 in inter frames), each reference's best (from the inter stage), the
// best of the references and the second best (first strict minimum), the compound of the two
// (src/gpu/inter_common.h:199-220) when the pair is allowed, inter only where strictly cheaper than
// intra; the per-block records (:93-103); decide_square (:125-198) -- bottom-up NONE / HORZ /
// VERT / SPLIT, first strict minimum, the 64x64 square NONE / HORZ / VERT only in inter frames,
// 8x8 squares never split; the preorder tree with its leaves.
//
// One CTA per superblock: a thread per block for the choices, the compound SATDs as (block, tile)
// items reduced per block like the intra stage's, the DP level by level, one thread for the
// preorder walk, then all threads write the record with coalesced stores.
#include <cstddef>

#include "kernels.h"
#include "tables.h"

namespace celv2cu {

constexpr int kFinThreads = 256;
constexpr long long kMax = 0x7fffffffffffffffLL;

struct FinSmem {
  long long inter_cost[kBlocks];  // best single-reference cost (kMax: none)
  int inter_mv[kBlocks], inter_ref[kBlocks];
  int comp_a[kBlocks], comp_b[kBlocks];  // compound pair (comp_a -1: none)
  int comp_mv0[kBlocks], comp_mv1[kBlocks];
  int comp_sum[kBlocks];
  long long best_cost[kBlocks];
  int best_mode[kBlocks], best_mv[kBlocks], best_ref[kBlocks], best_ref2[kBlocks], best_mv2[kBlocks];
  long long sq_cost[CELV2_SB_SQUARES];
  int sq_choice[CELV2_SB_SQUARES];
  unsigned char tree[CELV2_SB_OUT_CAP];
  short leaf[CELV2_SB_OUT_CAP];
  int ntree, nblocks;
};

__global__ void __launch_bounds__(kFinThreads, 4) k_finalize(const FrameJob* __restrict__ jobs, WorkList w) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  FinSmem& S = *reinterpret_cast<FinSmem*>(smem_raw);
  __shared__ int unit_slot;
  const int tid = threadIdx.x;
  int unit, iter = 0;
  while (take_unit(w, unit, iter, &unit_slot)) {
  const int jb = job_of(w, unit);
  const FrameJob& job = jobs[jb];
  const int sb = unit - w.prefix[jb], sby = sb / job.sb_cols, sbx = sb - sby * job.sb_cols;
  const int ox = sbx * 64, oy = sby * 64;
  const int nrefs = job.nrefs;
  const long long lam = job.lam;
  celv2_sb_out* o = job.out + sb;
  const int2* inter = job.inter + (long long)sb * kMaxRefs * kBlocks;
  // pruned references, intra, block levels and intra modes are not candidates
  const unsigned keep = keep_mask(job, sb);

  // 1. each reference's best, the best two references, the records per reference
  unsigned comp_tiles = 0;  // work counter: compound 4x4 tiles
  for (int b = tid; b < kBlocks; b += kFinThreads) {
    long long rc[kMaxRefs];
    int rmv[kMaxRefs];
    int a = -1, second = -1;
    const bool live = keep & CELV2_KEEP_LEVEL(block_level(b));  // a block of a pruned level: no choice
    for (int r = 0; r < nrefs; r++) {
      if (!live || !(keep >> r & 1u)) {
        rc[r] = kMax, rmv[r] = 0;
        continue;
      }
      const int2 v = inter[r * kBlocks + b];
      rc[r] = (long long)v.x * 256 + lam * (kInterBits + r);
      rmv[r] = v.y;
      if (a < 0 || rc[r] < rc[a]) a = r;
    }
    for (int r = 0; r < nrefs; r++)
      if (r != a && live && (keep >> r & 1u) && (second < 0 || rc[r] < rc[second])) second = r;
#pragma unroll
    for (int r = 0; r < kMaxRefs; r++) {
      const bool has = r < nrefs && live && (keep >> r & 1u);
      const long long c8 = has ? rc[r] >> 8 : 0;
      o->c_rcost[r][b] = has ? (unsigned)(c8 < 0xfffffffeLL ? c8 : 0xfffffffeLL) : CELV2_NO_REF_COST;
      o->c_rmvx[r][b] = (short)(has ? mv_x(rmv[r]) : 0);
      o->c_rmvy[r][b] = (short)(has ? mv_y(rmv[r]) : 0);
    }
    S.inter_cost[b] = a >= 0 ? rc[a] : kMax;
    S.inter_mv[b] = a >= 0 ? rmv[a] : 0;
    S.inter_ref[b] = a >= 0 ? a : 0;
    const bool comp = second >= 0 && compound_pair_ok(a, second, nrefs);
    if (comp) {
      int bx, by, bw, bh;
      sb_block_geom(b, bx, by, bw, bh);
      comp_tiles += (unsigned)(bw / 4) * (bh / 4);
    }
    S.comp_a[b] = comp ? a : -1;
    S.comp_b[b] = comp ? second : 0;
    S.comp_mv0[b] = comp ? rmv[a] : 0;
    S.comp_mv1[b] = comp ? rmv[second] : 0;
    S.comp_sum[b] = 0;
  }
  if (job.stats) {  // one atomic per warp
    comp_tiles = __reduce_add_sync(0xffffffffu, comp_tiles);
    if ((tid & 31) == 0 && comp_tiles) atomicAdd(job.stats + kStatCompoundTiles, (unsigned long long)comp_tiles);
  }
  __syncthreads();

  // 2. compound SATDs (block_compound_satd): (cur - ((p0 + p1 + 1) >> 1)) per 4x4 tile
  if (nrefs >= 2) {
    const DevPlane cur = job.cur.lv[0];
    for (int item = tid; item < kItems; item += kFinThreads) {
      int b, tx, ty;
      item_decode(item, b, tx, ty);
      const int width = item_width(item);
      int s = 0;
      if (S.comp_a[b] >= 0) {  // uniform over the block's segment
        const int m0 = S.comp_mv0[b], m1 = S.comp_mv1[b];
        const int mx0 = mv_x(m0), my0 = mv_y(m0), mx1 = mv_x(m1), my1 = mv_y(m1);
        DevPlane p0 = job.ref[S.comp_a[b]].lv[0], p1 = job.ref[S.comp_b[b]].lv[0];
        p0.p += (long long)((my0 & 3) * 4 + (mx0 & 3)) * p0.phase;
        p1.p += (long long)((my1 & 3) * 4 + (mx1 & 3)) * p1.phase;
        const int x = ox + tx * 4, y = oy + ty * 4;
        const int x0 = x + (mx0 >> 2), y0 = y + (my0 >> 2), x1 = x + (mx1 >> 2), y1 = y + (my1 >> 2);
        if (inside(p0, x0, y0, 4, 4) && inside(p1, x1, y1, 4, 4)) {
          uint32_t ce[4], co[4], pr[4];
#pragma unroll
          for (int i = 0; i < 4; i++) {
            const uint32_t c = load4(cur.p + (long long)(y + i) * cur.stride + x);
            const uint32_t a = load4(p0.p + (long long)(y0 + i) * p0.stride + x0);
            const uint32_t q = load4(p1.p + (long long)(y1 + i) * p1.stride + x1);
            ce[i] = bytes_even(c), co[i] = bytes_odd(c);
            pr[i] = __vavgu4(a, q);  // per byte (a + q + 1) >> 1
          }
          s = satd4_bytes(ce, co, pr);
        } else {
          const DevPlane r0 = job.ref[S.comp_a[b]].lv[0], r1 = job.ref[S.comp_b[b]].lv[0];
          int d[16];
#pragma unroll
          for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) {
              const int pr = (at_q(r0, y + i, x + j, my0, mx0) + at_q(r1, y + i, x + j, my1, mx1) + 1) >> 1;
              d[4 * i + j] = at(cur, y + i, x + j) - pr;
            }
          s = hadamard4x4(d);
        }
      }
      s = segment_sum(s, width);
      if ((tid & ((width < 32 ? width : 32) - 1)) == 0 && S.comp_a[b] >= 0) atomicAdd(&S.comp_sum[b], s);
    }
  }
  __syncthreads();

  // 3. the block's inter choice (compound where strictly cheaper), intra choice, records, best
  const int* intra = job.intra + (long long)sb * kBlocks * kModes;
  for (int b = tid; b < kBlocks; b += kFinThreads) {
    long long ci = S.inter_cost[b];
    int mv = S.inter_mv[b], ref = S.inter_ref[b], ref2 = CELV2_SINGLE_REF, mv2 = 0;
    if (S.comp_a[b] >= 0) {
      const long long cc = (long long)S.comp_sum[b] * 256 + lam * (20 + S.comp_a[b] + S.comp_b[b]);
      if (cc < ci) ci = cc, ref2 = S.comp_b[b], mv2 = S.comp_mv1[b];
    }
    long long c = kMax;
    int m = 0;
    const bool live = keep & CELV2_KEEP_LEVEL(block_level(b));
    if (b >= 5 && live && (keep & CELV2_KEEP_INTRA))
      for (int k = 0; k < kModes; k++) {
        if (!(keep & CELV2_KEEP_MODE(k))) continue;
        const long long ck = (long long)intra[b * kModes + k] * 256 + lam * (mode_bits(k) + (nrefs > 0 ? kIntraInInterBits : 0));
        if (ck < c) c = ck, m = k;
      }
    o->c_inter_cost[b] = ci;
    o->c_intra_cost[b] = c;
    o->c_intra[b] = (unsigned char)m;
    o->c_mvx[b] = (short)mv_x(mv), o->c_mvy[b] = (short)mv_y(mv);
    o->c_ref[b] = (unsigned char)ref, o->c_ref2[b] = (unsigned char)ref2;
    o->c_mv2x[b] = (short)mv_x(mv2), o->c_mv2y[b] = (short)mv_y(mv2);
    const bool take_inter = ci < c;
    S.best_cost[b] = live ? (take_inter ? ci : c) : CELV2_PRUNED_COST;
    S.best_mode[b] = take_inter ? kModes : m;
    S.best_mv[b] = take_inter ? mv : 0;
    S.best_ref[b] = take_inter ? ref : 0;
    S.best_ref2[b] = take_inter ? ref2 : CELV2_SINGLE_REF;
    S.best_mv2[b] = take_inter ? mv2 : 0;
  }
  __syncthreads();

  // 4. partition choice bottom-up (decide_square)
  const long long part = lam * kPartBits;
  for (int level = 3; level >= 0; level--) {
    const int n = 1 << level, size = 64 >> level;
    if (tid < n * n) {
      const int sq = sb_level_offset(level) + tid, b = sq * 5;
      long long c = kMax;
      int ch = 3;
      if (size <= 32 || nrefs > 0) {
        const long long horz = part + S.best_cost[b + 1] + S.best_cost[b + 2];
        const long long vert = part + S.best_cost[b + 3] + S.best_cost[b + 4];
        c = S.best_cost[b], ch = 0;
        if (horz < c) c = horz, ch = 1;
        if (vert < c) c = vert, ch = 2;
      }
      if (level < 3) {
        const int qx = tid % n, qy = tid / n, c0 = sb_level_offset(level + 1);
        long long split = part;
        for (int q = 0; q < 4; q++) split += S.sq_cost[c0 + (2 * qy + (q >> 1)) * (2 * n) + 2 * qx + (q & 1)];
        if (split < c) c = split, ch = 3;
      }
      S.sq_cost[sq] = c, S.sq_choice[sq] = ch;
    }
    __syncthreads();
  }
  if (tid == 0 && job.sb_cost) job.sb_cost[sb] = S.sq_cost[0];

  // 5. the preorder tree and its leaves
  if (tid == 0) {
    int ntree = 0, nleaf = 0;
    int stack[16], sp = 0;
    stack[sp++] = 0;  // (level << 8) | (qy << 4) | qx
    while (sp > 0) {
      const int e = stack[--sp], level = e >> 8, qy = (e >> 4) & 15, qx = e & 15;
      const int sq = sb_level_offset(level) + qy * (1 << level) + qx, b = sq * 5, ch = S.sq_choice[sq];
      if (ch == 0) {
        S.tree[ntree++] = 0, S.leaf[nleaf++] = (short)b;
      } else if (ch == 1 || ch == 2) {
        const int k = ch == 1 ? 1 : 3;
        S.tree[ntree++] = (unsigned char)ch;
        S.tree[ntree++] = 0, S.leaf[nleaf++] = (short)(b + k);
        S.tree[ntree++] = 0, S.leaf[nleaf++] = (short)(b + k + 1);
      } else {
        S.tree[ntree++] = 3;
        for (int q = 3; q >= 0 && level < 3; q--)  // reversed so quadrant 0 comes out first
          stack[sp++] = ((level + 1) << 8) | ((2 * qy + (q >> 1)) << 4) | (2 * qx + (q & 1));
      }
    }
    S.ntree = ntree, S.nblocks = nleaf;
    o->ntree = ntree, o->nblocks = nleaf;
    // the record's padding bytes
    reinterpret_cast<unsigned char*>(o)[offsetof(celv2_sb_out, c_rcost) - 1] = 0;
    *reinterpret_cast<unsigned*>(reinterpret_cast<unsigned char*>(o) + sizeof(celv2_sb_out) - 4) = 0;
  }
  __syncthreads();
  // 6. tree and leaf fields, zero past the end
  for (int k = tid; k < CELV2_SB_OUT_CAP; k += kFinThreads) {
    o->tree[k] = k < S.ntree ? S.tree[k] : 0;
    if (k < S.nblocks) {
      const int b = S.leaf[k];
      int x, y, bw, bh;
      sb_block_geom(b, x, y, bw, bh);
      const bool in = S.best_mode[b] == kModes;
      const bool two = in && S.best_ref2[b] != CELV2_SINGLE_REF;
      o->w4[k] = (unsigned char)(bw / 4), o->h4[k] = (unsigned char)(bh / 4);
      o->mode[k] = (unsigned char)S.best_mode[b];
      o->mvx[k] = (short)(in ? mv_x(S.best_mv[b]) : 0), o->mvy[k] = (short)(in ? mv_y(S.best_mv[b]) : 0);
      o->ref[k] = (unsigned char)(in ? S.best_ref[b] : 0);
      o->ref2[k] = (unsigned char)(two ? S.best_ref2[b] : CELV2_SINGLE_REF);
      o->mv2x[k] = (short)(two ? mv_x(S.best_mv2[b]) : 0), o->mv2y[k] = (short)(two ? mv_y(S.best_mv2[b]) : 0);
    } else {
      o->w4[k] = o->h4[k] = o->mode[k] = 0;
      o->mvx[k] = o->mvy[k] = 0;
      o->ref[k] = o->ref2[k] = 0;
      o->mv2x[k] = o->mv2y[k] = 0;
    }
  }
  }  // units
}

void launch_finalize(const FrameJob* jobs, const WorkList& w, cudaStream_t st) {
  const int units = w.prefix[w.njobs];
  if (units <= 0) return;
  const int grid = w.queue ? persistent_grid((const void*)k_finalize, kFinThreads, sizeof(FinSmem), units) : units;
  k_finalize<<<grid, kFinThreads, sizeof(FinSmem), st>>>(jobs, w);
}

cudaError_t finalize_attributes() {
  const cudaError_t e = cudaFuncSetAttribute(k_finalize, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(FinSmem));
  if (e == cudaSuccess) persistent_grid((const void*)k_finalize, kFinThreads, sizeof(FinSmem), 1);  // fills the grid cache
  return e;
}

}  // namespace celv2cu
