// inter.cu: each reference's best single-reference candidate for every candidate block.
//
// Reference rules: mv_cells / candidate_mv_index / repeated_candidate
// (src/gpu/inter_common.h:60-89), block_inter_satd (:223-235) and the per-reference loop of
// best_both (src/gpu/kernels_ref.cpp:54-66): candidates in order, repeats skipped, first strict
// minimum of SATD * 256 + lambda * (3 + r) -- i.e. of the SATD, the bits being constant per
// reference.
//
// Work reuse: a block's SATD at an MV is the sum of its 4x4 tiles' SATDs at that MV (the blocks'
// tiles all sit on the superblock's 4x4 grid), and every candidate MV of a superblock's blocks is
// the level-0 MV of one of the 10 x 10 cells around it. So one CTA per (superblock, reference):
//  1. gathers those 100 MVs (clamped into the field) and their distinct set D, and gives every
//     (block, candidate) slot its MV's index in D (the slot's cell is a constant of the block
//     geometry, tabulated once), and per MV of D the offset of the superblock's prediction in its
//     phase plane;
//  2. for chunks of D: one thread per 4x4 tile (its cur samples in registers) computes the tile's
//     SATD at every MV of the chunk -- a warp reads two contiguous image rows per load -- and the
//     four tiles of an 8x8 cell, which sit in one warp, sum by shuffles; then the 16x16 sums;
//  3. every candidate slot whose MV is in the chunk takes its SATD from those sums, and a shared
//     atomicMin of (SATD << 7 | candidate index) keeps each block's least. That is the reference's
//     first strict minimum over the candidates in order: a repeated MV (which the reference skips)
//     has the same SATD as its first occurrence and a larger index, so it never wins.
// 256 |D| Hadamards per (superblock, reference) instead of up to 68,352 for the blocks one by one.
// Pruned search: where the superblock keeps no 64-level blocks (no 64x64, 64x32, 32x64), a second
// kernel (k_inter_regions) scores each of its 32x32 regions (16x16 with no 32-level blocks either)
// on its own: a kept block and all its candidates' cells lie inside its region and the ring of
// cells around it, so the region's tiles are scored at the distinct MVs of its 6 x 6 (4 x 4) cells
// only -- exactly the SATDs the whole-superblock pass gives them. The whole-superblock kernel
// (k_inter) keeps its own code and registers: the units of the two kinds go to the two kernels.
// The result per (block, reference) is the winning SATD and MV; the lambda terms are added by the
// finalize stage, which alone needs the costs.
#include <algorithm>

#include "kernels.h"

namespace celv2cu {

constexpr int kInterThreads = 256;  // one per 4x4 tile of the superblock
constexpr int kNb = 100;            // 10 x 10 cells around the superblock
constexpr int kChunk = 64;          // distinct MVs per pass at most
constexpr int kSlots = 4296;        // candidates of the 425 blocks (cells covered + 8 neighbours)

// Every (block, candidate) slot as b | k << 9 | cell << 16 (its neighbourhood cell), ordered by
// block size, block kind, candidate index, block: a warp's slots then take one path through
// block_satd and name 32 different blocks (no divergence, no colliding shared atomics).
__device__ unsigned g_slot[kSlots];
// Block b's candidate k sits in neighbourhood cell g_cand_cell[c_cand_off[b] + k].
__constant__ short c_cand_off[kBlocks];
__device__ unsigned char g_cand_cell[kSlots];

constexpr int kMaxRegions = 16;  // 16x16 regions of a superblock
constexpr int kRegCells = 256;   // regions x neighbourhood cells at most (16 x 16, 4 x 36, 1 x 100)

// Per candidate slot (in g_slot's order) and per block: level | 32x32 region << 2 | 16x16 region
// << 4. The slots of one level are contiguous in g_slot's order: level l's from c_level_slot[l].
__device__ unsigned char g_slot_aux[kSlots];
__device__ unsigned char g_block_aux[kBlocks];
__constant__ int c_level_slot[5];

// The region pass's shared state.
struct RegionSmem {
  int rnb[kInterThreads];      // per thread (region, local cell): the cell's packed MV
  int D[kRegCells];            // per region r: its distinct MVs at D[r * ncell ..], first occurrence order
  int moff[kRegCells];         // per (region, MV): the superblock's prediction, bytes from the reference's level 0
  unsigned char mfast[kRegCells];  // per (region, MV): the region's prediction lies inside the margin
  unsigned char dmap[kMaxRegions][kNb];  // per region: neighbourhood cell -> its MV's index in the region's D
  unsigned bal[kInterThreads / 32];      // per warp: which lanes hold a first occurrence
  int nd[kMaxRegions];
  int nd_max;
  unsigned key[kBlocks];              // per block: least (SATD << 7 | candidate index) so far
};

// The per-chunk sums follow RegionSmem in shared memory, sized by the launch's chunk (a smaller
// chunk leaves more of the SM's memory to the L1 cache the prediction rows go through).
struct ChunkSums {
  unsigned short (*tile)[256];   // [chunk][256] 4x4 SATDs (at most 16 x 4 x 255 = 16,320)
  unsigned short (*whole8)[64];  // [chunk][64] 8x8 sums (at most 65,280)
  int (*sum16)[16];              // [chunk][16] 16x16 sums
};

__host__ __device__ constexpr size_t inter_smem_bytes(int chunk) {
  return (sizeof(RegionSmem) + 15) / 16 * 16 + (size_t)chunk * (256 * 2 + 64 * 2 + 16 * 4);
}

__device__ __forceinline__ ChunkSums chunk_sums(unsigned char* base, int chunk) {
  unsigned char* p = base + (sizeof(RegionSmem) + 15) / 16 * 16;
  ChunkSums c;
  c.tile = reinterpret_cast<unsigned short (*)[256]>(p);
  c.whole8 = reinterpret_cast<unsigned short (*)[64]>(p + (size_t)chunk * 512);
  c.sum16 = reinterpret_cast<int (*)[16]>(p + (size_t)chunk * 640);
  return c;
}

// The whole-superblock pass's shared state (every kept level, the 64-level blocks among them).
struct WholeSmem {
  int nb[kNb];  // packed MV of each neighbourhood cell
  int D[kNb];   // distinct MVs, first occurrence order
  int first_idx[kNb];
  unsigned char dmap[kNb];
  int moff[kNb];  // per MV of D: the superblock's prediction, bytes from the reference's level 0
  unsigned char mfast[kNb];           // per MV of D: its 64 x 64 prediction lies inside the margin
  unsigned char list[kSlots];         // per candidate slot: its MV index in D
  unsigned key[kBlocks];              // per block: least (SATD << 7 | candidate index) so far
  unsigned short tile[kChunk][256];   // 4x4 SATDs (at most 16 x 4 x 255 = 16,320)
  unsigned short whole8[kChunk][64];  // 8x8 sums (at most 65,280)
  int sum16[kChunk][16];
  int nd;
};

// SATD of block b at chunk-local MV dd from the shared sums (WholeSmem or ChunkSums).
template <typename Sums>
__device__ __forceinline__ int block_satd(const Sums& S, int b, int dd) {
  const int sq = b / 5, kind = b - sq * 5;
  if (sq >= 21) {  // 8x8 cell c: its tiles t, t + 1, t + 16, t + 17
    const int c = sq - 21, t = (c >> 3) * 32 + (c & 7) * 2;
    const unsigned short* T = S.tile[dd];
    switch (kind) {
      case 0: return S.whole8[dd][c];
      case 1: return T[t] + T[t + 1];
      case 2: return T[t + 16] + T[t + 17];
      case 3: return T[t] + T[t + 16];
      default: return T[t + 1] + T[t + 17];
    }
  }
  if (sq >= 5) {  // 16x16: children are 8x8 cells
    const int i = sq - 5, c = (i >> 2) * 16 + (i & 3) * 2;
    const unsigned short* W = S.whole8[dd];
    switch (kind) {
      case 0: return S.sum16[dd][i];
      case 1: return W[c] + W[c + 1];
      case 2: return W[c + 8] + W[c + 9];
      case 3: return W[c] + W[c + 8];
      default: return W[c + 1] + W[c + 9];
    }
  }
  const int* s = S.sum16[dd];
  if (sq >= 1) {  // 32x32: children are 16x16 squares
    const int i = sq - 1, c0 = (i >> 1) * 8 + (i & 1) * 2;
    const int tl = s[c0], tr = s[c0 + 1], bl = s[c0 + 4], br = s[c0 + 5];
    switch (kind) {
      case 0: return tl + tr + bl + br;
      case 1: return tl + tr;
      case 2: return bl + br;
      case 3: return tl + bl;
      default: return tr + br;
    }
  }
  int q[4];  // the 32x32 quadrants
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int c0 = (i >> 1) * 8 + (i & 1) * 2;
    q[i] = s[c0] + s[c0 + 1] + s[c0 + 4] + s[c0 + 5];
  }
  switch (kind) {
    case 0: return q[0] + q[1] + q[2] + q[3];
    case 1: return q[0] + q[1];
    case 2: return q[2] + q[3];
    case 3: return q[0] + q[2];
    default: return q[1] + q[3];
  }
}

// Neighbourhood index (10 x 10, origin one cell above-left of the superblock) of candidate k of
// the block at superblock-local (bx, by), size bw x bh (candidate_mv_index, inter_common.h:65-78).
__host__ __device__ __forceinline__ int candidate_cell(int bx, int by, int bw, int bh, int k) {
  const int lx = bx >> 3, ly = by >> 3;
  const int cw = ((bx + bw - 1) >> 3) - lx + 1, ch = ((by + bh - 1) >> 3) - ly + 1, cells = cw * ch;
  int cx, cy;
  if (k < cells) {
    const int kr = k / cw;
    cx = lx + (k - kr * cw), cy = ly + kr;
  } else {
    const int n = k - cells;
    const int nl = lx - 1, nr = (bx + bw) >> 3, nt = ly - 1, nbm = (by + bh) >> 3;
    cx = (n == 0 || n == 4 || n == 6) ? nl : (n == 2 || n == 5 || n == 7) ? nr : lx;
    cy = (n == 1 || n == 4 || n == 5) ? nt : (n == 3 || n == 6 || n == 7) ? nbm : ly;
  }
  return (cy + 1) * 10 + cx + 1;
}

__global__ void __launch_bounds__(kInterThreads, 4) k_inter(const FrameJob* __restrict__ jobs, WorkList w, int chunk) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WholeSmem& S = *reinterpret_cast<WholeSmem*>(smem_raw);
  __shared__ int warp_cnt[kInterThreads / 32];
  __shared__ int unit_slot;
  const int tid = threadIdx.x, lane = tid & 31;
  int unit, iter = 0;
  while (take_unit(w, unit, iter, &unit_slot)) {
  const int jb = job_of(w, unit);
  const FrameJob& job = jobs[jb];
  const int nsb = job.sb_cols * job.sb_rows;
  const int u = unit - w.prefix[jb];
  const int r = u / nsb, sb = u - r * nsb, sby = sb / job.sb_cols, sbx = sb - sby * job.sb_cols;
  const unsigned keep = keep_mask(job, sb);
  // a pruned (superblock, reference) is not scored; without 64-level blocks k_inter_regions scores it
  if (!(keep >> r & 1u) || !(keep & CELV2_KEEP_LEVEL(0))) continue;
  const int ox = sbx * 64, oy = sby * 64;
  const int cols = job.fcols[0], rows = job.frows[0];
  const int* field = job.field[r][0];

  // 1. neighbourhood MVs, their distinct set (first occurrence order), the blocks' lists
  if (tid < kNb) {
    const int ny = tid / 10, nx = tid - ny * 10;
    const int cx = clampi(sbx * 8 - 1 + nx, 0, cols - 1), cy = clampi(sby * 8 - 1 + ny, 0, rows - 1);
    S.nb[tid] = field[cy * cols + cx];
  }
  for (int b = tid; b < kBlocks; b += kInterThreads) S.key[b] = 0xffffffffu;
  __syncthreads();
  bool is_first = false;
  int firstj = 0;
  if (tid < kNb) {
    const int v = S.nb[tid];
    while (S.nb[firstj] != v) firstj++;
    is_first = firstj == tid;
  }
  const unsigned bal = __ballot_sync(0xffffffffu, is_first);
  if (lane == 0) warp_cnt[tid >> 5] = __popc(bal);
  __syncthreads();
  if (tid < kNb) {
    int pos = __popc(bal & ((1u << lane) - 1u));
    for (int k = 0; k < (tid >> 5); k++) pos += warp_cnt[k];
    if (is_first) S.D[pos] = S.nb[tid], S.first_idx[tid] = pos;
  }
  if (tid == 0) S.nd = warp_cnt[0] + warp_cnt[1] + warp_cnt[2] + warp_cnt[3];
  __syncthreads();
  if (tid < kNb) S.dmap[tid] = (unsigned char)S.first_idx[firstj];
  const int nd = S.nd;
  if (tid == 0 && job.stats) atomicAdd(job.stats + kStatInterMvs, (unsigned long long)nd * 256);
  const DevPlane cur = job.cur.lv[0], ref = job.ref[r].lv[0];
  if (tid < nd) {
    const int m = S.D[tid], mx = mv_x(m), my = mv_y(m), x = ox + (mx >> 2), y = oy + (my >> 2);
    const long long o = (long long)((my & 3) * 4 + (mx & 3)) * ref.phase + (long long)y * ref.stride + x;
    S.moff[tid] = (int)o;
    S.mfast[tid] = inside(ref, x, y, 64, 64) && o == (long long)(int)o;
  }
  __syncthreads();
  for (int e = tid; e < kSlots; e += kInterThreads) S.list[e] = S.dmap[g_slot[e] >> 16];

  // this thread's tile: its cur rows, row-transformed, in registers (the grid lies inside the margin)
  const int tx = tid & 15, ty = tid >> 4;
  int C[16];
  {
    uint32_t c[4];
#pragma unroll
    for (int i = 0; i < 4; i++) c[i] = load4(cur.p + (long long)(oy + ty * 4 + i) * cur.stride + ox + tx * 4);
    wh_rows_cur(c, C);
  }
  // the tile's prediction rows at MV d start at tile_base + moff[d]; words a row apart are ws apart
  const uintptr_t tile_base = reinterpret_cast<uintptr_t>(ref.p) + (uintptr_t)(ty * 4 * ref.stride + tx * 4);
  const int ws = ref.stride >> 2;  // strides are multiples of 64
  // chunks of equal size, at most `chunk` MVs each
  const int nchunks = (nd + chunk - 1) / chunk, csize = (nd + nchunks - 1) / nchunks;
  __syncthreads();  // lists complete

  for (int c0 = 0; c0 < nd; c0 += csize) {
    const int nc = min(csize, nd - c0);
    // 2. tile SATDs at every MV of the chunk (two MVs per step for load parallelism); an 8x8
    //    cell's tiles are lanes l, l + 1, l + 16, l + 17 of one warp
    for (int dd = 0; dd < nc; dd += 2) {
      int sat[2];
      const int dA = c0 + dd, dB = c0 + min(dd + 1, nc - 1);
      if (S.mfast[dA] & S.mfast[dB]) {
        // both MVs' rows from aligned word pairs, all 16 loads issued before either SATD
        uint32_t wv[2][4][2];
        uint32_t shv[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const uintptr_t a = tile_base + (uintptr_t)(intptr_t)S.moff[h ? dB : dA];
          const uint32_t* wp = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
          shv[h] = (uint32_t)(a & 3) * 8;
#pragma unroll
          for (int i = 0; i < 4; i++) wv[h][i][0] = __ldg(wp + i * ws), wv[h][i][1] = __ldg(wp + i * ws + 1);
        }
#pragma unroll
        for (int h = 0; h < 2; h++) {
          uint32_t pr[4];
#pragma unroll
          for (int i = 0; i < 4; i++) pr[i] = __funnelshift_r(wv[h][i][0], wv[h][i][1], shv[h]);
          sat[h] = satd4_rows(C, pr);
        }
      } else {
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int d = h ? dB : dA;
        uint32_t pr[4];
        if (S.mfast[d]) {
          const uintptr_t a = tile_base + (uintptr_t)(intptr_t)S.moff[d];
          const uint32_t* wp = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
          const uint32_t sh = (uint32_t)(a & 3) * 8;
#pragma unroll
          for (int i = 0; i < 4; i++) pr[i] = __funnelshift_r(__ldg(wp + i * ws), __ldg(wp + i * ws + 1), sh);
        } else {
          const int m = S.D[d], mx = mv_x(m), my = mv_y(m);
          DevPlane ph = ref;
          ph.p = ref.p + (long long)((my & 3) * 4 + (mx & 3)) * ref.phase;
          const int x = ox + tx * 4 + (mx >> 2), y = oy + ty * 4 + (my >> 2);
#pragma unroll
          for (int i = 0; i < 4; i++) {
            pr[i] = 0;
#pragma unroll
            for (int k = 0; k < 4; k++) pr[i] |= (uint32_t)at(ph, y + i, x + k) << (8 * k);
          }
        }
        sat[h] = satd4_rows(C, pr);
      }
      }
#pragma unroll
      for (int h = 0; h < 2; h++) {
        int v = sat[h] + __shfl_xor_sync(0xffffffffu, sat[h], 1);
        v += __shfl_xor_sync(0xffffffffu, v, 16);
        if (dd + h < nc) {
          S.tile[dd + h][tid] = (unsigned short)sat[h];
          if (lane < 16 && !(lane & 1)) S.whole8[dd + h][(tid >> 5) * 8 + (lane >> 1)] = (unsigned short)v;
        }
      }
    }
    __syncthreads();
    for (int e = tid; e < nc * 16; e += kInterThreads) {
      const int dd = e >> 4, i = e & 15, c = (i >> 2) * 16 + (i & 3) * 2;
      const unsigned short* W = S.whole8[dd];
      S.sum16[dd][i] = W[c] + W[c + 1] + W[c + 8] + W[c + 9];
    }
    __syncthreads();
    // 3. every candidate slot whose MV is in this chunk
    for (int e = tid; e < kSlots; e += kInterThreads) {
      const int d = (int)S.list[e] - c0;
      if (d < 0 || d >= nc) continue;
      const unsigned bp = g_slot[e];
      const int b = bp & 511, k = (bp >> 9) & 127;
      atomicMin(&S.key[b], ((unsigned)block_satd(S, b, d) << 7) | (unsigned)k);
    }
    __syncthreads();  // the next chunk overwrites the sums
  }
  int2* out = job.inter + ((long long)sb * kMaxRefs + r) * kBlocks;
  for (int b = tid; b < kBlocks; b += kInterThreads) {
    const unsigned k = S.key[b];
    out[b] = make_int2((int)(k >> 7), S.D[S.dmap[g_cand_cell[c_cand_off[b] + (k & 127)]]]);
  }
  }  // units
}

// One (superblock, reference) unit of the region pass, regions of R x R samples (32 or 16).
template <int R>
__device__ __forceinline__ void region_unit(RegionSmem& S, const ChunkSums& Q, const FrameJob& job, int r, int sb,
                                            int sbx, int sby, unsigned keep, int chunk) {
  constexpr int nr = 64 / R, nreg = nr * nr, rcells = R / 8, rc = rcells + 2, ncell = rc * rc;
  constexpr int per = kInterThreads / nreg;  // threads per region: 64 (R = 32) or 16 (R = 16)
  static_assert(per >= ncell && (per & (per - 1)) == 0 && nreg * ncell <= kRegCells, "region layout");
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ox = sbx * 64, oy = sby * 64;
  const int cols = job.fcols[0], rows = job.frows[0];
  const int* field = job.field[r][0];

  // 1. thread (region reg, local cell lc) reads its neighbourhood cell's MV (clamped into the field)
  const int reg = tid / per, lc = tid % per;
  const bool live = lc < ncell;
  const int c10 = ((reg / nr) * rcells + lc / rc) * 10 + (reg % nr) * rcells + lc % rc;
  int v = 0;
  if (live) {
    const int cx = clampi(sbx * 8 - 1 + c10 % 10, 0, cols - 1), cy = clampi(sby * 8 - 1 + c10 / 10, 0, rows - 1);
    v = __ldg(field + cy * cols + cx);
  }
  S.rnb[tid] = v;
  for (int b = tid; b < kBlocks; b += kInterThreads) S.key[b] = 0xffffffffu;
  if (tid == 0) S.nd_max = 0;
  __syncthreads();
  // the region's first local cell holding this MV; the first occurrences, in local cell order, are
  // the region's distinct MVs: an MV's index is the number of first occurrences before its own
  int firstlc = lc;
  if (live) {
    const int* rn = S.rnb + reg * per;
    for (int k = 0; k < lc; k++)
      if (rn[k] == v) {
        firstlc = k;
        break;
      }
  }
  const bool is_first = live && firstlc == lc;
  const unsigned bal = __ballot_sync(0xffffffffu, is_first);
  if (lane == 0) S.bal[warp] = bal;
  const int nd_sum = __syncthreads_count(is_first);
  int pos, nd;
  if constexpr (per == 16) {  // two regions per warp, a half each
    const unsigned rb = (bal >> ((reg & 1) * 16)) & 0xffffu;
    pos = __popc(rb & ((1u << firstlc) - 1u)), nd = __popc(rb);
  } else {  // a region over two warps: local cells 0-31 and 32-35
    const unsigned ba = S.bal[2 * reg], bb = S.bal[2 * reg + 1];
    pos = firstlc < 32 ? __popc(ba & ((1u << firstlc) - 1u)) : __popc(ba) + __popc(bb & ((1u << (firstlc - 32)) - 1u));
    nd = __popc(ba) + __popc(bb);
  }
  if (live) S.dmap[reg][c10] = (unsigned char)pos;
  const DevPlane cur = job.cur.lv[0], ref = job.ref[r].lv[0];
  if (is_first) {  // per (region, MV): the prediction's offset, inside the margin or not
    const int e = reg * ncell + pos, mx = mv_x(v), my = mv_y(v);
    const int x = ox + (mx >> 2), y = oy + (my >> 2);
    const long long o = (long long)((my & 3) * 4 + (mx & 3)) * ref.phase + (long long)y * ref.stride + x;
    S.D[e] = v;
    S.moff[e] = (int)o;
    S.mfast[e] = inside(ref, x + (reg % nr) * R, y + (reg / nr) * R, R, R) && o == (long long)(int)o;
  }
  if (lc == 0) S.nd[reg] = nd, atomicMax(&S.nd_max, nd);
  if (tid == 0 && job.stats) atomicAdd(job.stats + kStatInterMvs, (unsigned long long)nd_sum * (R / 4) * (R / 4));

  // this thread's tile: its cur rows, row-transformed, in registers (the grid lies inside the margin)
  const int tx = tid & 15, ty = tid >> 4;
  const int treg = (ty / (R / 4)) * nr + tx / (R / 4);  // the tile's region
  int C[16];
  {
    uint32_t c[4];
#pragma unroll
    for (int i = 0; i < 4; i++) c[i] = load4(cur.p + (long long)(oy + ty * 4 + i) * cur.stride + ox + tx * 4);
    wh_rows_cur(c, C);
  }
  // the tile's prediction rows at MV d start at tile_base + moff[d]; words a row apart are ws apart
  const uintptr_t tile_base = reinterpret_cast<uintptr_t>(ref.p) + (uintptr_t)(ty * 4 * ref.stride + tx * 4);
  const int ws = ref.stride >> 2;  // strides are multiples of 64
  __syncthreads();  // MVs, maps, offsets complete
  const int tnd = S.nd[treg], tbase = treg * ncell, nd_max = S.nd_max;
  const int wnd = __reduce_max_sync(0xffffffffu, tnd);  // the most MVs of this warp's regions
  // the candidate slots of the kept levels (contiguous by level in g_slot's order; levels 1-3 here)
  const unsigned lv = (keep & CELV2_KEEP_LEVELS) >> 8;
  const int slot_lo = c_level_slot[__ffs(lv) - 1], slot_hi = c_level_slot[32 - __clz(lv)];
  // chunks of equal size, at most `chunk` MVs each
  const int nchunks = (nd_max + chunk - 1) / chunk, csize = (nd_max + nchunks - 1) / nchunks;

  for (int c0 = 0; c0 < nd_max; c0 += csize) {
    const int nc = min(csize, nd_max - c0);
    const int tnc = min(nc, tnd - c0);  // this tile's region's MVs in the chunk
    const int wnc = min(nc, wnd - c0);  // this warp's
    // 2. tile SATDs at the region's MVs of the chunk (two MVs per step for load parallelism); an
    //    8x8 cell's tiles are lanes l, l + 1, l + 16, l + 17 of one warp (and of one region)
    for (int dd = 0; dd < wnc; dd += 2) {
      int sat[2];
#pragma unroll
      for (int h = 0; h < 2; h++) {
        // a tile whose region has no MV left scores its region's first MV (always there); those
        // sums are never read: a region's slots name only its own MVs
        const int d = tbase + (tnc > 0 ? c0 + min(dd + h, tnc - 1) : 0);
        uint32_t pr[4];
        if (S.mfast[d]) {  // the usual case: rows from aligned words
          const uintptr_t a = tile_base + (uintptr_t)(intptr_t)S.moff[d];
          const uint32_t* wp = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
          const uint32_t sh = (uint32_t)(a & 3) * 8;
          if (sh == 0) {
#pragma unroll
            for (int i = 0; i < 4; i++) pr[i] = __ldg(wp + i * ws);
          } else {
#pragma unroll
            for (int i = 0; i < 4; i++) pr[i] = __funnelshift_r(__ldg(wp + i * ws), __ldg(wp + i * ws + 1), sh);
          }
        } else {
          const int m = S.D[d], mx = mv_x(m), my = mv_y(m);
          DevPlane ph = ref;
          ph.p = ref.p + (long long)((my & 3) * 4 + (mx & 3)) * ref.phase;
          const int x = ox + tx * 4 + (mx >> 2), y = oy + ty * 4 + (my >> 2);
#pragma unroll
          for (int i = 0; i < 4; i++) {
            pr[i] = 0;
#pragma unroll
            for (int k = 0; k < 4; k++) pr[i] |= (uint32_t)at(ph, y + i, x + k) << (8 * k);
          }
        }
        sat[h] = satd4_rows(C, pr);
      }
#pragma unroll
      for (int h = 0; h < 2; h++) {
        int v8 = sat[h] + __shfl_xor_sync(0xffffffffu, sat[h], 1);
        v8 += __shfl_xor_sync(0xffffffffu, v8, 16);
        if (dd + h < wnc) {
          Q.tile[dd + h][tid] = (unsigned short)sat[h];
          if (lane < 16 && !(lane & 1)) Q.whole8[dd + h][(tid >> 5) * 8 + (lane >> 1)] = (unsigned short)v8;
        }
      }
    }
    __syncthreads();
    // 16x16 sums (a 16x16 square lies in one region, so its four 8x8 sums exist wherever it is read)
    for (int k = tid; k < nc * 16; k += kInterThreads) {
      const int dd = k >> 4, i = k & 15, c = (i >> 2) * 16 + (i & 3) * 2;
      const unsigned short* W = Q.whole8[dd];
      Q.sum16[dd][i] = W[c] + W[c + 1] + W[c + 8] + W[c + 9];
    }
    __syncthreads();
    // 3. every candidate slot of a kept level whose MV (in its block's region) is in this chunk
    for (int k = slot_lo + tid; k < slot_hi; k += kInterThreads) {
      const unsigned aux = __ldg(g_slot_aux + k);
      if (!(keep & CELV2_KEEP_LEVEL(aux & 3u))) continue;
      const unsigned bp = __ldg(g_slot + k);
      const int d = (int)S.dmap[R == 32 ? (aux >> 2) & 3u : aux >> 4][bp >> 16] - c0;
      if (d < 0 || d >= nc) continue;
      const int b = bp & 511;
      atomicMin(&S.key[b], ((unsigned)block_satd(Q, b, d) << 7) | ((bp >> 9) & 127u));
    }
    __syncthreads();  // the next chunk overwrites the sums
  }
  int2* out = job.inter + ((long long)sb * kMaxRefs + r) * kBlocks;
  for (int b = tid; b < kBlocks; b += kInterThreads) {
    const unsigned aux = __ldg(g_block_aux + b);
    if (!(keep & CELV2_KEEP_LEVEL(aux & 3u))) continue;  // a pruned block: never read
    const int breg = R == 32 ? (aux >> 2) & 3u : aux >> 4;
    const unsigned k = S.key[b];
    out[b] = make_int2((int)(k >> 7), S.D[breg * ncell + S.dmap[breg][g_cand_cell[c_cand_off[b] + (k & 127)]]]);
  }
}

__global__ void __launch_bounds__(kInterThreads, 4) k_inter_regions(const FrameJob* __restrict__ jobs, WorkList w, int chunk) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  RegionSmem& S = *reinterpret_cast<RegionSmem*>(smem_raw);
  const ChunkSums Q = chunk_sums(smem_raw, chunk);
  __shared__ int unit_slot;
  int unit, iter = 0;
  while (take_unit(w, unit, iter, &unit_slot)) {
    const int jb = job_of(w, unit);
    const FrameJob& job = jobs[jb];
    const int nsb = job.sb_cols * job.sb_rows;
    const int u = unit - w.prefix[jb];
    const int r = u / nsb, sb = u - r * nsb, sby = sb / job.sb_cols, sbx = sb - sby * job.sb_cols;
    const unsigned keep = keep_mask(job, sb);
    // a pruned (superblock, reference) is not scored; with 64-level blocks k_inter scores it
    if (!(keep >> r & 1u) || (keep & CELV2_KEEP_LEVEL(0))) continue;
    // regions: its 32x32 squares, or 16x16 ones where the 32-level blocks are pruned too
    if (keep & CELV2_KEEP_LEVEL(1))
      region_unit<32>(S, Q, job, r, sb, sbx, sby, keep, chunk);
    else
      region_unit<16>(S, Q, job, r, sb, sbx, sby, keep, chunk);
  }
}

void launch_inter(const FrameJob* jobs, const WorkList& w, int chunk, bool regions, unsigned* region_queue,
                  cudaStream_t st) {
  const int units = w.prefix[w.njobs];
  if (units <= 0) return;
  chunk = chunk < 8 ? 8 : chunk > kChunk ? kChunk : chunk;
  const int grid = w.queue ? persistent_grid((const void*)k_inter, kInterThreads, sizeof(WholeSmem), units) : units;
  k_inter<<<grid, kInterThreads, sizeof(WholeSmem), st>>>(jobs, w, chunk);
  if (!regions) return;  // no job has keep words: every unit keeps its 64-level blocks
  WorkList wr = w;
  wr.queue = w.queue ? region_queue : nullptr;
  const size_t smem = inter_smem_bytes(chunk);
  const int rgrid = wr.queue ? persistent_grid((const void*)k_inter_regions, kInterThreads, smem, units) : units;
  k_inter_regions<<<rgrid, kInterThreads, smem, st>>>(jobs, wr, chunk);
}

cudaError_t inter_attributes() {
  short off[kBlocks];
  static unsigned slot[kSlots];
  static unsigned char cell[kSlots];
  static unsigned long long order[kSlots];  // sort key << 32 | slot
  int o = 0;
  for (int b = 0; b < kBlocks; b++) {
    int x, y, w, h;
    sb_block_geom(b, x, y, w, h);
    const int n = ((x + w - 1) / 8 - x / 8 + 1) * ((y + h - 1) / 8 - y / 8 + 1) + 8;
    const int sq = b / 5, size = sq >= 21 ? 3 : sq >= 5 ? 2 : sq >= 1 ? 1 : 0, kind = b - sq * 5;
    off[b] = (short)o;
    for (int k = 0; k < n && o + k < kSlots; k++) {
      const int c = candidate_cell(x, y, w, h, k);
      cell[o + k] = (unsigned char)c;
      const unsigned desc = (unsigned)b | (unsigned)k << 9 | (unsigned)c << 16;
      order[o + k] = (unsigned long long)(size << 19 | kind << 16 | k << 9 | b) << 32 | desc;
    }
    o += n;
  }
  if (o != kSlots) return cudaErrorInvalidValue;
  std::sort(order, order + kSlots);
  // level | 32x32 region << 2 | 16x16 region << 4 of a block (its region: where its top-left lies)
  auto aux_of = [](int b) {
    int x, y, w, h;
    sb_block_geom(b, x, y, w, h);
    return (unsigned char)(block_level(b) | ((y / 32) * 2 + x / 32) << 2 | ((y / 16) * 4 + x / 16) << 4);
  };
  static unsigned char slot_aux[kSlots];
  unsigned char block_aux[kBlocks];
  int level_slot[5] = {0, 0, 0, 0, kSlots};
  for (int b = 0; b < kBlocks; b++) block_aux[b] = aux_of(b);
  for (int e = 0; e < kSlots; e++) {
    slot[e] = (unsigned)order[e];
    slot_aux[e] = block_aux[slot[e] & 511];
  }
  for (int l = 1; l < 4; l++) {  // the first slot of level l (the slots are ordered by level)
    int e = 0;
    while (e < kSlots && (slot_aux[e] & 3) < l) e++;
    level_slot[l] = e;
  }
  cudaError_t e = cudaMemcpyToSymbol(c_cand_off, off, sizeof off);
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_slot_aux, slot_aux, sizeof slot_aux);
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_block_aux, block_aux, sizeof block_aux);
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_level_slot, level_slot, sizeof level_slot);
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_cand_cell, cell, sizeof cell);
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_slot, slot, sizeof slot);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(k_inter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(WholeSmem));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_inter_regions, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)inter_smem_bytes(kChunk));
  if (e == cudaSuccess) persistent_grid((const void*)k_inter, kInterThreads, sizeof(WholeSmem), 1);  // fills the grid cache
  return e;
}

}  // namespace celv2cu
