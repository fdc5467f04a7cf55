// me.cu: hierarchical integer motion search, one pyramid level per launch, all references and
// all frames of a batch together.
//
// Reference rules (src/gpu/inter_common.h): sad8 (:96-104), me_search (:108-119), satd8_q
// (:122-133), me_refine (:141-154), me_cell (:162-193); driven level by level, coarsest first,
// as src/gpu/cpu_engine.cpp:68-83 does.
//
// One CTA per 30 (or 15) consecutive 8x8 cells of one (job, reference):
//  A. the cells' cur blocks are staged in shared memory; one thread per (cell, predictor centre)
//     computes the six centre SADs;
//  B. one thread per cell replays the reference's sequential choice of the two best distinct
//     centres, and the searches (one or two per cell) get their 24 x 32-byte reference windows
//     staged in shared memory with aligned 8-byte loads;
//  C. one thread per (search, dx) column slides down the window's 24 rows: each row's 8 bytes at
//     column dx are loaded once (two funnel shifts of three words) and feed, with vabsdiff4, every
//     one of the 17 dy accumulators whose 8x8 block covers that row -- 24 row loads instead of
//     17 x 8 per column. The column's best (cost << 9 | raster index) goes to a shared atomicMin,
//     which yields the reference's first strict minimum in dy-major order;
// Level 0's quarter-pel refinement is its own kernel (k_me_refine): a warp per position of a step,
// a lane per cell.
// Integer ALU bound: 289 x 16 byte-SIMD absolute-difference accumulates per searched centre.
#include "kernels.h"

namespace celv2cu {

constexpr int kMeThreads = 256;
constexpr int kWinRows = 24, kWinWords = 8;    // a window row: 32 bytes from an 8-byte boundary
constexpr int kWinStride = kWinRows * kWinWords + 8;  // +8 words: neighbouring windows use other banks
// A merged search: the two centres of a cell at most 2 apart in x and y searched as one union
// window of at most 19 x 19 positions (instead of two 17 x 17): 26 rows of 40 bytes, in the space
// of two windows.
constexpr int kMergeMax = 2, kUnion = 17 + kMergeMax, kMWinRows = kUnion + 7, kMWinWords = 10;
static_assert(kMWinRows * kMWinWords <= 2 * kWinStride, "a merged window fits two windows' space");

// Shared state of a CTA of CELLS cells (15 or 30: fewer cells per CTA give small pyramid levels
// more CTAs; the autotuner picks per level). Nearly every cell searches two centres, so a CTA's
// search phase has about 2 x 17 x CELLS (search, column) items: 30 and 15 cells make 1,020 and 510,
// four and two nearly full rounds of 256 threads (32 and 16 cells left a last round 25% and 12%
// full).
template <int CELLS>
struct MeSmem {
  static constexpr int kSearches = 2 * CELLS;  // at most two centres per cell
  uint32_t cur[CELLS][16];
  int csad[CELLS][6];
  int ccx[CELLS][6], ccy[CELLS][6];
  int scell[kSearches], sx[kSearches], sy[kSearches], soff[kSearches];
  unsigned skey[kSearches];
  // merged searches (entries from the back of the list): the second centre and its key
  int sx2[kSearches], sy2[kSearches];
  unsigned skey2[kSearches];
  int first_search[CELLS], two[CELLS];  // two: 0 one centre, 1 two searches, 2 one merged search
  int need[CELLS];  // the cell is searched (level 0 of a pruned job: some superblock reads it)
  int nsearch, nmerged;
  alignas(16) uint32_t win[kSearches * kWinStride];
};

// An asynchronous 8-byte global -> shared copy (cp.async; both addresses 8-byte aligned).
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gsrc) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// 4 bytes of a plane at (x .. x + 3, y), clamped like Plane::at where the row leaves the margin.
__device__ __forceinline__ uint32_t row4(const DevPlane& s, int x, int y) {
  if (y >= -s.margin && y < s.h + s.margin && x >= -s.margin && x + 4 <= s.w + s.margin)
    return load4(s.p + (long long)y * s.stride + x);
  uint32_t v = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) v |= (uint32_t)at(s, y, x + k) << (8 * k);
  return v;
}

// acc + the sum of the four byte absolute differences of a and b (PTX vabsdiff4 with its add).
__device__ __forceinline__ unsigned sad4_acc(unsigned a, unsigned b, unsigned acc) {
  unsigned d;
  asm("vabsdiff4.u32.u32.u32.add %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(acc));
  return d;
}

// sad8 of a cur block (shared memory) against the reference at (x, y).
__device__ __forceinline__ int sad8(const uint32_t* c, const DevPlane& ref, int x, int y) {
  unsigned s = 0;
  if (inside(ref, x, y, 8, 8)) {
    const uint8_t* p = ref.p + (long long)y * ref.stride + x;
#pragma unroll
    for (int i = 0; i < 8; i++) {
      s = sad4_acc(c[2 * i], load4(p + (long long)i * ref.stride), s);
      s = sad4_acc(c[2 * i + 1], load4(p + (long long)i * ref.stride + 4), s);
    }
    return (int)s;
  }
#pragma unroll
  for (int i = 0; i < 8; i++) {
    s = sad4_acc(c[2 * i], row4(ref, x, y + i), s);
    s = sad4_acc(c[2 * i + 1], row4(ref, x + 4, y + i), s);
  }
  return (int)s;
}

// The 4-byte windows at p and p + 1 (any alignment) from two aligned 32-bit loads.
__device__ __forceinline__ void load_pair(const uint8_t* p, uint32_t& lo4, uint32_t& hi4) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  const uint32_t* w = reinterpret_cast<const uint32_t*>(a & ~uintptr_t(3));
  const uint32_t sh = (uint32_t)(a & 3) * 8, w0 = __ldg(w), w1 = __ldg(w + 1);
  lo4 = __funnelshift_r(w0, w1, sh);
  hi4 = __funnelshift_rc(w0, w1, sh + 8);  // a shift of 32 gives w1
}

// The refinement step's position n (raster 0..8 with the centre, 4, visited first).
__device__ __forceinline__ int refine_pos(int t) { return t == 0 ? 4 : (t <= 4 ? t - 1 : t); }

template <int CELLS>
__global__ void __launch_bounds__(kMeThreads, 4) k_me_level(const FrameJob* __restrict__ jobs, WorkList w, int level) {
  constexpr int kMeCells = CELLS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  MeSmem<CELLS>& S = *reinterpret_cast<MeSmem<CELLS>*>(smem_raw);
  __shared__ int unit_slot;
  const int tid = threadIdx.x;
  int unit, iter = 0;
  while (take_unit(w, unit, iter, &unit_slot)) {
  const int jb = job_of(w, unit);
  const FrameJob& job = jobs[jb];
  const int cols = job.fcols[level], rows = job.frows[level], ncell = cols * rows;
  const int groups = (ncell + kMeCells - 1) / kMeCells;
  const int u = unit - w.prefix[jb];
  const int r = u / groups, cell0 = (u - r * groups) * kMeCells;
  const int ncells = min(kMeCells, ncell - cell0);
  const DevPlane cur = job.cur.lv[level], ref = job.ref[r].lv[level];

  // ---- A. cur blocks, predictor centres and their SADs (me_cell, inter_common.h:164-186) ----
  for (int e = tid; e < kMeCells * 16; e += kMeThreads) {
    const int c = e >> 4, k = e & 15;
    const int cell = cell0 + (c < ncells ? c : 0), by = cell / cols, bx = cell - by * cols;
    S.cur[c][k] = row4(cur, bx * 8 + 4 * (k & 1), by * 8 + (k >> 1));
  }
  if (tid < kMeCells) {
    const int cell = cell0 + tid, by = cell / cols, bx = cell - by * cols;
    S.need[tid] = tid < ncells && (level != 0 || cell_needed(job, r, bx, by));
  }
  if (tid == 0) S.nsearch = 0, S.nmerged = 0;
  __syncthreads();
  const bool top = level == kLevels - 1;
  if (!top && tid < kMeCells * 6) {
    const int c = tid / 6, k = tid - c * 6;
    if (c < ncells && S.need[c]) {
      const int cell = cell0 + c, by = cell / cols, bx = cell - by * cols;
      int cx = 0, cy = 0;  // k == 5: zero
      if (k < 5) {
        const int* pf = job.field[r][level + 1];
        const int pcols = job.fcols[level + 1], prows = job.frows[level + 1];
        const int ox = k == 1 ? -1 : k == 2 ? 1 : 0, oy = k == 3 ? -1 : k == 4 ? 1 : 0;
        const int m = pf[clampi(by / 2 + oy, 0, prows - 1) * pcols + clampi(bx / 2 + ox, 0, pcols - 1)];
        cx = 2 * mv_x(m), cy = 2 * mv_y(m);
      }
      S.ccx[c][k] = cx, S.ccy[c][k] = cy;
      S.csad[c][k] = sad8(S.cur[c], ref, bx * 8 + cx, by * 8 + cy);
    }
  }
  __syncthreads();

  // ---- B. the two best distinct centres per cell, the search list ----
  if (tid < ncells && !S.need[tid]) S.first_search[tid] = -1, S.two[tid] = 0;
  if (tid < ncells && S.need[tid]) {
    const int c = tid;
    int px = 0, py = 0, px2 = 0, py2 = 0;
    bool two = false;
    if (!top) {
      int best = 0x7fffffff, second = 0x7fffffff;
      for (int k = 0; k < 6; k++) {
        const int cx = S.ccx[c][k], cy = S.ccy[c][k], s = S.csad[c][k];
        if ((k > 0 && cx == px && cy == py) || (two && cx == px2 && cy == py2)) continue;
        if (s < best) {
          if (k > 0) second = best, px2 = px, py2 = py, two = true;
          best = s, px = cx, py = cy;
        } else if (s < second) {
          second = s, px2 = cx, py2 = cy, two = true;
        }
      }
    }
    const int cell = cell0 + c, by = cell / cols, bx = cell - by * cols;
    if (two && abs(px - px2) <= kMergeMax && abs(py - py2) <= kMergeMax) {
      // one union window for both centres, its entry from the back of the list
      const int s = MeSmem<CELLS>::kSearches - 1 - atomicAdd(&S.nmerged, 1);
      const int ux = min(px, px2) - kMeRange, wx0 = bx * 8 + ux;
      S.first_search[c] = s, S.two[c] = 2;
      S.scell[s] = c, S.sx[s] = px, S.sy[s] = py, S.sx2[s] = px2, S.sy2[s] = py2;
      S.soff[s] = wx0 - (wx0 & ~7);
      S.skey[s] = S.skey2[s] = 0xffffffffu;
    } else {
    const int s0 = atomicAdd(&S.nsearch, two ? 2 : 1);
    S.first_search[c] = s0, S.two[c] = two;
    for (int k = 0; k < (two ? 2 : 1); k++) {
      const int cxs = k ? px2 : px, cys = k ? py2 : py;
      const int wx0 = bx * 8 + cxs - kMeRange;
      S.scell[s0 + k] = c, S.sx[s0 + k] = cxs, S.sy[s0 + k] = cys;
      S.soff[s0 + k] = wx0 - (wx0 & ~7);  // the window starts on the 8-byte boundary below wx0
      S.skey[s0 + k] = 0xffffffffu;
    }
    }
  }
  __syncthreads();
  const int nsearch = S.nsearch, nmerged = S.nmerged;
  // windows: rows y0 + cy - 8 .. + 23, 32 bytes from the 8-byte boundary at or below x0 + cx - 8;
  // inside the margin as asynchronous 8-byte copies (all in flight at once: one memory latency for
  // the whole staging), else word by word with clamping. Plane rows start 8-byte aligned (strides
  // and margins are multiples of 8), and so do the window rows in shared memory.
  for (int e = tid; e < nsearch * kWinRows * 4; e += kMeThreads) {
    const int s = e / (kWinRows * 4), rem = e - s * (kWinRows * 4);
    const int rr = rem >> 2, qd = rem & 3;
    const int cell = cell0 + S.scell[s], by = cell / cols, bx = cell - by * cols;
    const int wx = (bx * 8 + S.sx[s] - kMeRange) & ~7, wy = by * 8 + S.sy[s] - kMeRange;
    uint32_t* dst = S.win + s * kWinStride + rr * kWinWords + 2 * qd;
    if (inside(ref, wx, wy, 4 * kWinWords, kWinRows)) {
      cp_async8(dst, ref.p + (long long)(wy + rr) * ref.stride + wx + 8 * qd);
    } else {
      dst[0] = row4(ref, wx + 8 * qd, wy + rr), dst[1] = row4(ref, wx + 8 * qd + 4, wy + rr);
    }
  }
  // merged windows: rows from min(cy) - 8, 40 bytes from the 8-byte boundary at or below min(cx) - 8;
  // merged search m (entry kSearches - 1 - m) in the window space of entries kSearches - 2 - 2m, +1
  for (int e = tid; e < nmerged * kMWinRows * 5; e += kMeThreads) {
    const int m = e / (kMWinRows * 5), rem = e - m * (kMWinRows * 5);
    const int rr = rem / 5, qd = rem - rr * 5, s = MeSmem<CELLS>::kSearches - 1 - m;
    const int cell = cell0 + S.scell[s], by = cell / cols, bx = cell - by * cols;
    const int wx = (bx * 8 + min(S.sx[s], S.sx2[s]) - kMeRange) & ~7;
    const int wy = by * 8 + min(S.sy[s], S.sy2[s]) - kMeRange;
    uint32_t* dst = S.win + (MeSmem<CELLS>::kSearches - 2 - 2 * m) * kWinStride + rr * kMWinWords + 2 * qd;
    if (inside(ref, wx, wy, 4 * kMWinWords, kMWinRows)) {
      cp_async8(dst, ref.p + (long long)(wy + rr) * ref.stride + wx + 8 * qd);
    } else {
      dst[0] = row4(ref, wx + 8 * qd, wy + rr), dst[1] = row4(ref, wx + 8 * qd + 4, wy + rr);
    }
  }
  cp_async_wait_all();
  __syncthreads();

  // ---- C. +-8 search (me_search, inter_common.h:108-119): a thread per (search, dx), then a
  //      thread per (merged search, union column), in one loop so the two kinds share rounds ----
  const int nplain = nsearch * 17, nitems = nplain + nmerged * kUnion;
  for (int item = tid; item < nitems; item += kMeThreads) {
    if (item < nplain) {
    const int s = item / 17, dx = item - s * 17;
    const uint32_t* c = S.cur[S.scell[s]];
    uint32_t cw[16];
#pragma unroll
    for (int k = 0; k < 16; k++) cw[k] = c[k];
    const int b = S.soff[s] + dx, wi = b >> 2;
    const unsigned sh = (unsigned)(b & 3) * 8;
    const uint32_t* wr = S.win + s * kWinStride + wi;
    unsigned acc[17];
#pragma unroll
    for (int k = 0; k < 17; k++) acc[k] = 0;
#pragma unroll
    for (int rr = 0; rr < kWinRows; rr++) {
      const uint32_t u0 = wr[rr * kWinWords], u1 = wr[rr * kWinWords + 1], u2 = wr[rr * kWinWords + 2];
      const uint32_t w0 = __funnelshift_r(u0, u1, sh), w1 = __funnelshift_r(u1, u2, sh);
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const int dy = rr - i;
        if (dy >= 0 && dy <= 16) acc[dy] = sad4_acc(cw[2 * i + 1], w1, sad4_acc(cw[2 * i], w0, acc[dy]));
      }
    }
    unsigned best = 0xffffffffu;
    const unsigned pen_x = kMePenalty * abs(dx - kMeRange);
#pragma unroll
    for (int dy = 0; dy < 17; dy++) {
      const unsigned cost = acc[dy] + pen_x + kMePenalty * abs(dy - kMeRange);
      const unsigned key = (cost << 9) | (unsigned)(dy * 17 + dx);
      best = key < best ? key : best;
    }
    atomicMin(&S.skey[s], best);
    } else {
    // merged searches: a thread per union column (at most 19); every union position's SAD is the
    // same for both centres, and each centre takes its own penalty and raster index -- the same
    // keys as its own 17 x 17 search, so the same first strict minimum. All 19 union rows are
    // summed (fixed trip counts; rows past the centres' union are never keyed)
    const int m = (item - nplain) / kUnion, du = item - nplain - m * kUnion, s = MeSmem<CELLS>::kSearches - 1 - m;
    const int cx1 = S.sx[s], cy1 = S.sy[s], cx2 = S.sx2[s], cy2 = S.sy2[s];
    const int ux = min(cx1, cx2), uy = min(cy1, cy2);  // union position 0 = centre offset -8
    if (du >= 17 + abs(cx1 - cx2)) continue;
    const uint32_t* c = S.cur[S.scell[s]];
    uint32_t cw[16];
#pragma unroll
    for (int k = 0; k < 16; k++) cw[k] = c[k];
    const int b = S.soff[s] + du, wi = b >> 2;
    const unsigned sh = (unsigned)(b & 3) * 8;
    const uint32_t* wr = S.win + (MeSmem<CELLS>::kSearches - 2 - 2 * m) * kWinStride + wi;
    unsigned acc[kUnion];
#pragma unroll
    for (int k = 0; k < kUnion; k++) acc[k] = 0;
#pragma unroll
    for (int rr = 0; rr < kMWinRows; rr++) {
      const uint32_t u0 = wr[rr * kMWinWords], u1 = wr[rr * kMWinWords + 1], u2 = wr[rr * kMWinWords + 2];
      const uint32_t w0 = __funnelshift_r(u0, u1, sh), w1 = __funnelshift_r(u1, u2, sh);
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const int dy = rr - i;
        if (dy >= 0 && dy < kUnion) acc[dy] = sad4_acc(cw[2 * i + 1], w1, sad4_acc(cw[2 * i], w0, acc[dy]));
      }
    }
#pragma unroll
    for (int t = 0; t < 2; t++) {
      // union column du is the offset ux - 8 + du, column ux + du - c of the window around centre c
      const int dx = ux + du - (t ? cx2 : cx1);  // column in this centre's 17 x 17 window
      const int oy = uy - (t ? cy2 : cy1);       // union row 0's row in its window
      if (dx < 0 || dx > 16) continue;
      unsigned best = 0xffffffffu;
      const unsigned pen_x = kMePenalty * abs(dx - kMeRange);
#pragma unroll
      for (int du_y = 0; du_y < kUnion; du_y++) {
        const int dy = oy + du_y;
        if (dy < 0 || dy > 16) continue;
        const unsigned cost = acc[du_y] + pen_x + kMePenalty * abs(dy - kMeRange);
        const unsigned key = (cost << 9) | (unsigned)(dy * 17 + dx);
        best = key < best ? key : best;
      }
      atomicMin(t ? &S.skey2[s] : &S.skey[s], best);
    }
    }
  }
  __syncthreads();
  if (tid < ncells && S.need[tid]) {
    const int s0 = S.first_search[tid];
    const unsigned k1 = S.skey[s0];
    int mx = S.sx[s0] + (int)(k1 & 511) % 17 - kMeRange, my = S.sy[s0] + (int)(k1 & 511) / 17 - kMeRange;
    if (S.two[tid]) {  // the second centre's result only if strictly cheaper (me_cell, :189-192)
      const bool merged = S.two[tid] == 2;
      const unsigned k2 = merged ? S.skey2[s0] : S.skey[s0 + 1];
      const int sx2 = merged ? S.sx2[s0] : S.sx[s0 + 1], sy2 = merged ? S.sy2[s0] : S.sy[s0 + 1];
      if ((k2 >> 9) < (k1 >> 9)) mx = sx2 + (int)(k2 & 511) % 17 - kMeRange, my = sy2 + (int)(k2 & 511) / 17 - kMeRange;
    }
    // level 0 in quarter pels: k_me_refine refines it in place
    job.field[r][level][cell0 + tid] = level == 0 ? pack_mv(mx * 4, my * 4) : pack_mv(mx, my);
  }
  if (job.stats && tid < 32) {  // searched centres, one atomic per unit (the cells sit in warp 0)
    const unsigned n = __reduce_add_sync(0xffffffffu, tid < ncells && S.need[tid] ? (S.two[tid] ? 2u : 1u) : 0u);
    if (tid == 0) atomicAdd(job.stats + level, (unsigned long long)n);
  }
  }  // units
}

// ---- quarter-pel refinement of level 0 (me_refine, inter_common.h:141-154) ----
// One CTA per 32 consecutive level-0 cells of one (job, reference), 4 warps: warp t holds tile t
// of the cells' four 4x4 tiles, a lane per cell, the cur tile row-transformed once into registers.
// In each step a lane scores its tile at the step's nine positions; the lanes of a load read the
// same row of the same tile for 32 neighbouring cells, which where their MVs agree -- most of a
// frame -- is one contiguous run of a phase plane's row (a lane per (cell, position, tile)
// scattered each warp's loads over nine phase planes and was bound by the L1's wavefronts; a warp
// per position re-read the cur coefficients from shared memory nine times a step). The four tiles'
// SATDs meet in shared memory and every lane replays its cell's centre-first strict choice from
// them (the same in all four warps, so one barrier per step). The second step's centre is the
// first step's winner, whose SATD the first step has already computed.
constexpr int kRefineCells = 32, kRefineTiles = 4, kRefineThreads = 32 * kRefineTiles;

__global__ void __launch_bounds__(kRefineThreads, 8) k_me_refine(const FrameJob* __restrict__ jobs, WorkList w) {
  __shared__ int sat[2][9][kRefineTiles][kRefineCells];  // [step][position][tile][cell]
  __shared__ int unit_slot;
  const int tid = threadIdx.x, c = tid & 31, t = tid >> 5;
  int unit, iter = 0;
  while (take_unit(w, unit, iter, &unit_slot)) {
  const int jb = job_of(w, unit);
  const FrameJob& job = jobs[jb];
  const int cols = job.fcols[0], ncell = cols * job.frows[0];
  const int groups = (ncell + kRefineCells - 1) / kRefineCells;
  const int u = unit - w.prefix[jb];
  const int r = u / groups, cell0 = (u - r * groups) * kRefineCells;
  const int ncells = min(kRefineCells, ncell - cell0);
  const int cell = cell0 + min(c, ncells - 1), by = cell / cols, bx = cell - by * cols;
  const bool need = c < ncells && cell_needed(job, r, bx, by);
  // a unit none of whose cells a kept reference reads (pruned search): nothing to refine
  if (!__syncthreads_or(need)) continue;
  const DevPlane cur = job.cur.lv[0], ref = job.ref[r].lv[0];
  int* field = job.field[r][0];
  // this lane's tile of its cell: origin, cur rows row-transformed
  const int ox = bx * 8 + 4 * (t & 1), oy = by * 8 + 4 * (t >> 1);
  int C[16];
  {
    uint32_t cw[4];
#pragma unroll
    for (int i = 0; i < 4; i++) cw[i] = row4(cur, ox, oy + i);
    wh_rows_cur(cw, C);
  }
  const int m = field[cell];
  int cx = mv_x(m), cy = mv_y(m);  // quarter pels
  int centre = 0;                  // the centre's SATD (the cell's four tiles), once known
#pragma unroll
  for (int s = 0; s < 2; s++) {
    const int step = 2 - s;
    // the half-pel step around a whole-pel MV reads four phase planes only (phase 2 one pel left
    // or up of phase 0 at -1/2 pel, at the same pel at +1/2): the rows of the 5 x 5 footprint are
    // loaded once per plane and the positions that share a plane take 4-byte windows of them
    const int X = ox + (cx >> 2), Y = oy + (cy >> 2);
    if (s == 0 && !((cx | cy) & 3) && inside(ref, X - 1, Y - 1, 5, 5)) {
      const long long rs = ref.stride;
      const uint8_t* p00 = ref.p + (long long)Y * rs + X;
      uint32_t pr[5], lf[5], rt[5];
#pragma unroll
      for (int i = 0; i < 4; i++) pr[i] = load4(p00 + i * rs);
      sat[0][0][t][c] = satd4_rows(C, pr);  // the centre, phase (0, 0)
      const uint8_t* p20 = p00 + 8 * ref.phase;  // phase (2, 0): rows Y - 1 .. Y + 3
#pragma unroll
      for (int i = 0; i < 5; i++) pr[i] = load4(p20 + (i - 1) * rs);
      sat[0][2][t][c] = satd4_rows(C, pr);      // (0, -1/2)
      sat[0][7][t][c] = satd4_rows(C, pr + 1);  // (0, +1/2)
      const uint8_t* p02 = p00 + 2 * ref.phase - 1;  // phase (0, 2): columns X - 1 .. X + 3
#pragma unroll
      for (int i = 0; i < 4; i++) load_pair(p02 + i * rs, lf[i], rt[i]);
      sat[0][4][t][c] = satd4_rows(C, lf);  // (-1/2, 0)
      sat[0][5][t][c] = satd4_rows(C, rt);  // (+1/2, 0)
      const uint8_t* p22 = p00 + 10 * ref.phase - 1;  // phase (2, 2): both
#pragma unroll
      for (int i = 0; i < 5; i++) load_pair(p22 + (i - 1) * rs, lf[i], rt[i]);
      sat[0][1][t][c] = satd4_rows(C, lf);      // (-1/2, -1/2)
      sat[0][3][t][c] = satd4_rows(C, rt);      // (+1/2, -1/2)
      sat[0][6][t][c] = satd4_rows(C, lf + 1);  // (-1/2, +1/2)
      sat[0][8][t][c] = satd4_rows(C, rt + 1);  // (+1/2, +1/2)
    } else {
#pragma unroll
    for (int k = s; k < 9; k++) {  // the second step's centre (k = 0) is the first step's winner
      const int n = refine_pos(k);
      const int qx = cx + (n % 3 - 1) * step, qy = cy + (n / 3 - 1) * step;
      DevPlane ph = ref;
      ph.p = ref.p + (long long)((qy & 3) * 4 + (qx & 3)) * ref.phase;
      const int x = ox + (qx >> 2), y = oy + (qy >> 2);
      uint32_t pr[4];
      if (inside(ph, x, y, 4, 4)) {
        const uint8_t* p = ph.p + (long long)y * ph.stride + x;
#pragma unroll
        for (int i = 0; i < 4; i++) pr[i] = load4(p + (long long)i * ph.stride);
      } else {
#pragma unroll
        for (int i = 0; i < 4; i++) pr[i] = row4(ph, x, y + i);
      }
      sat[s][k][t][c] = satd4_rows(C, pr);
    }
    }
    __syncthreads();
    // the cell's choice (me_refine: the centre first, a move must save kSubpelPenalty)
    int best = s == 0 ? sat[0][0][0][c] + sat[0][0][1][c] + sat[0][0][2][c] + sat[0][0][3][c] : centre;
    int raw = best, nx = cx, ny = cy;
#pragma unroll
    for (int k = 1; k < 9; k++) {
      const int v = sat[s][k][0][c] + sat[s][k][1][c] + sat[s][k][2][c] + sat[s][k][3][c];
      const int n = refine_pos(k);
      if (v + kSubpelPenalty < best) best = v + kSubpelPenalty, raw = v, nx = cx + (n % 3 - 1) * step, ny = cy + (n / 3 - 1) * step;
    }
    centre = raw, cx = nx, cy = ny;
  }
  if (t == 0 && need) field[cell] = pack_mv(cx, cy);
  }  // units
}

int refine_units(int nrefs, int cols, int rows) { return nrefs * ((cols * rows + kRefineCells - 1) / kRefineCells); }

void launch_me_refine(const FrameJob* jobs, const WorkList& w, cudaStream_t st) {
  const int units = w.prefix[w.njobs];
  if (units <= 0) return;
  const int grid = w.queue ? persistent_grid((const void*)k_me_refine, kRefineThreads, 0, units) : units;
  k_me_refine<<<grid, kRefineThreads, 0, st>>>(jobs, w);
}

int me_units(int nrefs, int cols, int rows, int cells) { return nrefs * ((cols * rows + cells - 1) / cells); }

template <int CELLS>
static void launch_cells(const FrameJob* jobs, const WorkList& w, int level, cudaStream_t st) {
  const int units = w.prefix[w.njobs];
  const size_t smem = sizeof(MeSmem<CELLS>);
  const int grid = w.queue ? persistent_grid((const void*)k_me_level<CELLS>, kMeThreads, smem, units) : units;
  k_me_level<CELLS><<<grid, kMeThreads, smem, st>>>(jobs, w, level);
}

void launch_me_level(const FrameJob* jobs, const WorkList& w, int level, int cells, cudaStream_t st) {
  if (w.prefix[w.njobs] <= 0) return;
  if (cells == 15)
    launch_cells<15>(jobs, w, level, st);
  else
    launch_cells<30>(jobs, w, level, st);
}

template <int CELLS>
static cudaError_t attributes_cells() {
  const size_t smem = sizeof(MeSmem<CELLS>);
  const cudaError_t e = cudaFuncSetAttribute(k_me_level<CELLS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) persistent_grid((const void*)k_me_level<CELLS>, kMeThreads, smem, 1);  // fills the grid cache
  return e;
}

cudaError_t me_attributes() {
  cudaError_t e = attributes_cells<15>();
  if (e == cudaSuccess) e = attributes_cells<30>();
  if (e == cudaSuccess) persistent_grid((const void*)k_me_refine, kRefineThreads, 0, 1);  // fills the grid cache
  return e;
}

}  // namespace celv2cu
