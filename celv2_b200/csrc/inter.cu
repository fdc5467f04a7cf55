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
//  1. gathers those 100 MVs (clamped into the field) and their distinct set D;
//  2. computes, for every 8x8 cell and every MV of D, the SATDs of the cell's four 4x4 tiles and
//     keeps the cell's top / bottom / left / right halves (2 tiles each) -- 256 |D| Hadamards
//     instead of up to 68,352 for the blocks one by one;
//  3. sums them into 16x16, 32x32 and 64x64 squares;
//  4. gives every block its candidates in the reference's order, skips repeats with a per-block
//     seen-set over D, and reads each candidate's SATD with one or two shared-memory loads.
// The result per (block, reference) is the winning SATD and MV; the lambda terms are added by
// the finalize stage, which alone needs the costs.
#include "kernels.h"

namespace celv2cu {

constexpr int kInterThreads = 256;
constexpr int kNb = 100;  // 10 x 10 cells around the superblock

// The SATD of the 8x8 cell at (x, y) against phase plane `ph` at whole-pel offset (mx, my):
// its top, bottom, left and right halves (two 4x4 Hadamards each).
__device__ __forceinline__ void cell_halves(const uint32_t c[16], const DevPlane& ph, int x, int y, int& top, int& bot,
                                            int& lft, int& rgt) {
  int t[4];
  const bool in = inside(ph, x, y, 8, 8);
  const uint8_t* p = ph.p + (long long)y * ph.stride + x;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const int tx = q & 1, ty = q >> 1;
    int d[16];
#pragma unroll
    for (int i = 0; i < 4; i++) {
      uint32_t pr;
      if (in) {
        pr = load4(p + (long long)(4 * ty + i) * ph.stride + 4 * tx);
      } else {
        pr = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) pr |= (uint32_t)at(ph, y + 4 * ty + i, x + 4 * tx + k) << (8 * k);
      }
      residual_row(d + 4 * i, c[2 * (4 * ty + i) + tx], pr);
    }
    t[q] = hadamard4x4(d);
  }
  top = t[0] + t[1], bot = t[2] + t[3], lft = t[0] + t[2], rgt = t[1] + t[3];
}

struct InterSmem {
  int nb[kNb];         // packed MV of each neighbourhood cell
  unsigned char dmap[kNb];
  int D[kNb];          // distinct MVs
  int nd;
  int first_idx[kNb];
  ushort4 halves[kNb][64];  // per d, per 8x8 cell: top, bottom, left, right
  int sum16[kNb][16];
  int sum32[kNb][4];
  int sum64[kNb];
  unsigned seen[kInterThreads][4];
};

// SATD of block b at distinct MV d from the shared sums.
__device__ __forceinline__ int block_satd(const InterSmem& S, int b, int d) {
  const int sq = b / 5, kind = b - sq * 5;
  auto whole8 = [&](int cx, int cy) {
    const ushort4 h = S.halves[d][cy * 8 + cx];
    return (int)h.x + (int)h.y;
  };
  if (sq >= 21) {  // 8x8
    const ushort4 h = S.halves[d][sq - 21];
    return kind == 0 ? (int)h.x + (int)h.y : kind == 1 ? (int)h.x : kind == 2 ? (int)h.y : kind == 3 ? (int)h.z : (int)h.w;
  }
  if (sq >= 5) {  // 16x16: children are 8x8 cells
    const int i = sq - 5, qx = i & 3, qy = i >> 2, cx = 2 * qx, cy = 2 * qy;
    switch (kind) {
      case 0: return S.sum16[d][i];
      case 1: return whole8(cx, cy) + whole8(cx + 1, cy);
      case 2: return whole8(cx, cy + 1) + whole8(cx + 1, cy + 1);
      case 3: return whole8(cx, cy) + whole8(cx, cy + 1);
      default: return whole8(cx + 1, cy) + whole8(cx + 1, cy + 1);
    }
  }
  if (sq >= 1) {  // 32x32: children are 16x16 squares
    const int i = sq - 1, qx = i & 1, qy = i >> 1, c0 = (2 * qy) * 4 + 2 * qx;
    const int* s = S.sum16[d];
    switch (kind) {
      case 0: return S.sum32[d][i];
      case 1: return s[c0] + s[c0 + 1];
      case 2: return s[c0 + 4] + s[c0 + 5];
      case 3: return s[c0] + s[c0 + 4];
      default: return s[c0 + 1] + s[c0 + 5];
    }
  }
  const int* s = S.sum32[d];
  switch (kind) {
    case 0: return S.sum64[d];
    case 1: return s[0] + s[1];
    case 2: return s[2] + s[3];
    case 3: return s[0] + s[2];
    default: return s[1] + s[3];
  }
}

__global__ void __launch_bounds__(kInterThreads, 2) k_inter(const FrameJob* __restrict__ jobs, WorkList w) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  InterSmem& S = *reinterpret_cast<InterSmem*>(smem_raw);
  const int tid = threadIdx.x;
  const int unit = blockIdx.x;
  const int jb = job_of(w, unit);
  const FrameJob& job = jobs[jb];
  const int nsb = job.sb_cols * job.sb_rows;
  const int u = unit - w.prefix[jb];
  const int r = u / nsb, sb = u - r * nsb, sby = sb / job.sb_cols, sbx = sb - sby * job.sb_cols;
  const int ox = sbx * 64, oy = sby * 64;
  const int cols = job.fcols[0], rows = job.frows[0];
  const int* field = job.field[r][0];

  // 1. neighbourhood MVs and their distinct set (first occurrence order)
  if (tid < kNb) {
    const int ny = tid / 10, nx = tid - ny * 10;
    const int cx = clampi(sbx * 8 - 1 + nx, 0, cols - 1), cy = clampi(sby * 8 - 1 + ny, 0, rows - 1);
    S.nb[tid] = field[cy * cols + cx];
  }
  __syncthreads();
  bool is_first = false;
  int firstj = 0;
  if (tid < kNb) {
    const int v = S.nb[tid];
    while (S.nb[firstj] != v) firstj++;
    is_first = firstj == tid;
  }
  // prefix count of first occurrences (4 warps cover the 100 entries)
  const unsigned bal = __ballot_sync(0xffffffffu, is_first);
  __shared__ int warp_cnt[kInterThreads / 32];
  if ((tid & 31) == 0) warp_cnt[tid >> 5] = __popc(bal);
  __syncthreads();
  if (tid < kNb) {
    int pos = __popc(bal & ((1u << (tid & 31)) - 1u));
    for (int k = 0; k < (tid >> 5); k++) pos += warp_cnt[k];
    if (is_first) S.D[pos] = S.nb[tid], S.first_idx[tid] = pos;
  }
  if (tid == 0) {
    int n = 0;
    for (int k = 0; k < (kNb + 31) / 32; k++) n += warp_cnt[k];
    S.nd = n;
  }
  __syncthreads();
  if (tid < kNb) S.dmap[tid] = (unsigned char)S.first_idx[firstj];
  const int nd = S.nd;
  if (tid == 0 && job.stats) atomicAdd(job.stats + kStatInterMvs, (unsigned long long)nd);

  // 2. per 8x8 cell and distinct MV: the tile SATD halves
  {
    const int cell = tid & 63, cx = cell & 7, cy = cell >> 3;
    const DevPlane cur = job.cur.lv[0];
    const DevPlane ref = job.ref[r].lv[0];
    const int x = ox + cx * 8, y = oy + cy * 8;
    uint32_t c[16];
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const uint8_t* p = cur.p + (long long)(y + i) * cur.stride + x;
      c[2 * i] = load4(p), c[2 * i + 1] = load4(p + 4);  // the SB grid lies inside the cur margin
    }
    for (int d = tid >> 6; d < nd; d += kInterThreads / 64) {
      const int m = S.D[d], mx = mv_x(m), my = mv_y(m);
      DevPlane ph = ref;
      ph.p = ref.p + (long long)((my & 3) * 4 + (mx & 3)) * ref.phase;
      int t, b, l, rr;
      cell_halves(c, ph, x + (mx >> 2), y + (my >> 2), t, b, l, rr);
      S.halves[d][cell] = make_ushort4((unsigned short)t, (unsigned short)b, (unsigned short)l, (unsigned short)rr);
    }
  }
  __syncthreads();
  // 3. 16x16, 32x32, 64x64 sums
  for (int e = tid; e < nd * 16; e += kInterThreads) {
    const int d = e >> 4, i = e & 15, cx = 2 * (i & 3), cy = 2 * (i >> 2);
    int s = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const ushort4 h = S.halves[d][(cy + (q >> 1)) * 8 + cx + (q & 1)];
      s += (int)h.x + (int)h.y;
    }
    S.sum16[d][i] = s;
  }
  __syncthreads();
  for (int e = tid; e < nd * 4; e += kInterThreads) {
    const int d = e >> 2, i = e & 3, c0 = (2 * (i >> 1)) * 4 + 2 * (i & 1);
    S.sum32[d][i] = S.sum16[d][c0] + S.sum16[d][c0 + 1] + S.sum16[d][c0 + 4] + S.sum16[d][c0 + 5];
  }
  __syncthreads();
  for (int d = tid; d < nd; d += kInterThreads) S.sum64[d] = S.sum32[d][0] + S.sum32[d][1] + S.sum32[d][2] + S.sum32[d][3];
  __syncthreads();

  // 4. every block's candidates in order (repeats skipped), first strict minimum
  int2* out = job.inter + ((long long)sb * kMaxRefs + r) * kBlocks;
  unsigned* seen = S.seen[tid];
  for (int b = tid; b < kBlocks; b += kInterThreads) {
    int bx, by, bw, bh;
    sb_block_geom(b, bx, by, bw, bh);
    seen[0] = seen[1] = seen[2] = seen[3] = 0;
    const int lx = bx >> 3, ly = by >> 3;
    const int cw = ((bx + bw - 1) >> 3) - lx + 1, ch = ((by + bh - 1) >> 3) - ly + 1, cells = cw * ch;
    const int nl = lx - 1, nr = (bx + bw) >> 3, nt = ly - 1, nbm = (by + bh) >> 3;
    int best = 0x7fffffff, bestd = 0;
    for (int k = 0; k < cells + 8; k++) {
      int cx, cy;
      if (k < cells) {
        const int kr = k / cw;
        cx = lx + (k - kr * cw), cy = ly + kr;
      } else {
        const int n = k - cells;
        cx = (n == 0 || n == 4 || n == 6) ? nl : (n == 2 || n == 5 || n == 7) ? nr : lx;
        cy = (n == 1 || n == 4 || n == 5) ? nt : (n == 3 || n == 6 || n == 7) ? nbm : ly;
      }
      const int d = S.dmap[(cy + 1) * 10 + cx + 1];
      const unsigned bit = 1u << (d & 31);
      if (seen[d >> 5] & bit) continue;  // repeated_candidate: an earlier candidate had this MV
      seen[d >> 5] |= bit;
      const int s = block_satd(S, b, d);
      if (s < best) best = s, bestd = d;
    }
    out[b] = make_int2(best, S.D[bestd]);
  }
}

void launch_inter(const FrameJob* jobs, const WorkList& w, cudaStream_t st) {
  const int units = w.prefix[w.njobs];
  if (units <= 0) return;
  k_inter<<<units, kInterThreads, sizeof(InterSmem), st>>>(jobs, w);
}

cudaError_t inter_attributes() {
  return cudaFuncSetAttribute(k_inter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(InterSmem));
}

}  // namespace celv2cu
