// me.cu: hierarchical integer motion search, one pyramid level per launch, all references and
// all frames of a batch together.
//
// Reference rules (src/gpu/inter_common.h): sad8 (:96-104), me_search (:108-119), satd8_q
// (:122-133), me_refine (:141-154), me_cell (:162-193); driven level by level, coarsest first,
// as src/gpu/cpu_engine.cpp:68-83 does.
//
// One warp per (job, reference, 8x8 cell):
//  1. the cur block is held in registers (8 rows x 2 words of packed bytes);
//  2. lanes 0-5 compute the SADs of the six predictor centres at once; every lane then replays
//     the reference's sequential choice of the two best distinct centres (uniform in the warp);
//  3. per searched centre the 24 x 27-byte reference window is staged in shared memory as four
//     byte-shifted copies, so an 8-byte row at any offset is two aligned 32-bit words; each lane
//     takes positions lane, lane + 32, ... of the 289, sums the 8 rows with __vsadu4, and the
//     warp reduces (cost << 9 | raster index) with a min -- which is the reference's first strict
//     minimum in dy-major order;
//  4. at level 0 lanes 0-8 compute the nine 8x8 quarter-pel SATDs of each refinement step and
//     every lane replays the centre-first strict choice.
// Integer ALU bound: per cell and centre 289 x 16 __vsadu4 on shared-memory words.
#include "kernels.h"

namespace celv2cu {

constexpr int kMeWarps = 8;
constexpr int kWinRows = 24, kWinWords = 6;

// 4 bytes of a plane at (x .. x + 3, y), clamped like Plane::at where the row leaves the margin.
__device__ __forceinline__ uint32_t row4(const DevPlane& s, int x, int y) {
  if (y >= -s.margin && y < s.h + s.margin && x >= -s.margin && x + 4 <= s.w + s.margin)
    return load4(s.p + (long long)y * s.stride + x);
  uint32_t v = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) v |= (uint32_t)at(s, y, x + k) << (8 * k);
  return v;
}

// sad8 of the cur block (registers) against the reference at (x, y).
__device__ __forceinline__ int sad8(const uint32_t c[16], const DevPlane& ref, int x, int y) {
  unsigned s = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    s = __vsadu4(c[2 * i], row4(ref, x, y + i)) + s;
    s = __vsadu4(c[2 * i + 1], row4(ref, x + 4, y + i)) + s;
  }
  return (int)s;
}

// satd8_q: the 8x8 SATD of the cur block against the quarter-pel prediction at (qx, qy).
__device__ __forceinline__ int satd8_q(const uint32_t c[16], const DevPlane& ref, int x0, int y0, int qx, int qy) {
  DevPlane ph = ref;
  ph.p = ref.p + (long long)((qy & 3) * 4 + (qx & 3)) * ref.phase;
  const int x = x0 + (qx >> 2), y = y0 + (qy >> 2);
  int total = 0;
#pragma unroll
  for (int ty = 0; ty < 2; ty++)
#pragma unroll
    for (int tx = 0; tx < 2; tx++) {
      int d[16];
#pragma unroll
      for (int i = 0; i < 4; i++) residual_row(d + 4 * i, c[2 * (4 * ty + i) + tx], row4(ph, x + 4 * tx, y + 4 * ty + i));
      total += hadamard4x4(d);
    }
  return total;
}

__global__ void __launch_bounds__(kMeWarps * 32) k_me_level(const FrameJob* __restrict__ jobs, WorkList w, int level) {
  __shared__ uint32_t win[kMeWarps][4][kWinRows][kWinWords];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int unit = blockIdx.x * kMeWarps + warp;
  if (unit >= w.prefix[w.njobs]) return;  // whole warps only; no block-wide barrier below
  const int jb = job_of(w, unit);
  const FrameJob& job = jobs[jb];
  const int cols = job.fcols[level], rows = job.frows[level], ncell = cols * rows;
  const int u = unit - w.prefix[jb];
  const int r = u / ncell, cell = u - r * ncell, by = cell / cols, bx = cell - by * cols;
  const DevPlane cur = job.cur.lv[level], ref = job.ref[r].lv[level];
  const int x0 = bx * 8, y0 = by * 8;

  uint32_t c[16];
#pragma unroll
  for (int i = 0; i < 8; i++) c[2 * i] = row4(cur, x0, y0 + i), c[2 * i + 1] = row4(cur, x0 + 4, y0 + i);

  // ---- 2. predictor centres (me_cell, inter_common.h:164-186) ----
  int px = 0, py = 0, px2 = 0, py2 = 0;
  bool two = false;
  if (level < kLevels - 1) {
    const int* pf = job.field[r][level + 1];
    const int pcols = job.fcols[level + 1], prows = job.frows[level + 1];
    int cx[6], cy[6];
#pragma unroll
    for (int k = 0; k < 6; k++) {
      cx[k] = 0, cy[k] = 0;
      if (k < 5) {
        const int ox = k == 1 ? -1 : k == 2 ? 1 : 0, oy = k == 3 ? -1 : k == 4 ? 1 : 0;
        const int qx = clampi(bx / 2 + ox, 0, pcols - 1), qy = clampi(by / 2 + oy, 0, prows - 1);
        const int m = pf[qy * pcols + qx];
        cx[k] = 2 * mv_x(m), cy[k] = 2 * mv_y(m);
      }
    }
    int mine = 0;
#pragma unroll
    for (int k = 0; k < 6; k++)
      if (lane == k) mine = sad8(c, ref, x0 + cx[k], y0 + cy[k]);
    int best = 0x7fffffff, second = 0x7fffffff;
#pragma unroll
    for (int k = 0; k < 6; k++) {
      const int s = __shfl_sync(0xffffffffu, mine, k);
      if ((k > 0 && cx[k] == px && cy[k] == py) || (two && cx[k] == px2 && cy[k] == py2)) continue;
      if (s < best) {
        if (k > 0) second = best, px2 = px, py2 = py, two = true;
        best = s, px = cx[k], py = cy[k];
      } else if (s < second) {
        second = s, px2 = cx[k], py2 = cy[k], two = true;
      }
    }
  }

  // ---- 3. +-8 search around each centre (me_search, inter_common.h:108-119) ----
  uint32_t(*W)[kWinRows][kWinWords] = win[warp];
  auto search = [&](int cxs, int cys) -> unsigned {
    const int wx0 = x0 + cxs - kMeRange, wy0 = y0 + cys - kMeRange;
    __syncwarp();
    for (int e = lane; e < 4 * kWinRows * kWinWords; e += 32) {
      const int s = e / (kWinRows * kWinWords), rem = e - s * (kWinRows * kWinWords);
      const int rr = rem / kWinWords, ww = rem - rr * kWinWords;
      W[s][rr][ww] = row4(ref, wx0 + 4 * ww + s, wy0 + rr);
    }
    __syncwarp();
    unsigned best = 0xffffffffu;
    for (int idx = lane; idx < 289; idx += 32) {
      const int dyi = idx / 17, dxi = idx - dyi * 17;
      const int s = dxi & 3, wo = dxi >> 2;
      unsigned sad = 0;
#pragma unroll
      for (int i = 0; i < 8; i++) {
        sad = __vsadu4(c[2 * i], W[s][dyi + i][wo]) + sad;
        sad = __vsadu4(c[2 * i + 1], W[s][dyi + i][wo + 1]) + sad;
      }
      const unsigned cost = sad + kMePenalty * (abs(dxi - kMeRange) + abs(dyi - kMeRange));
      const unsigned key = (cost << 9) | (unsigned)idx;
      best = key < best ? key : best;
    }
    return __reduce_min_sync(0xffffffffu, best);
  };
  unsigned k1 = search(px, py);
  int mx = px + (int)(k1 & 511) % 17 - kMeRange, my = py + (int)(k1 & 511) / 17 - kMeRange;
  if (two) {
    const unsigned k2 = search(px2, py2);
    if ((k2 >> 9) < (k1 >> 9)) mx = px2 + (int)(k2 & 511) % 17 - kMeRange, my = py2 + (int)(k2 & 511) / 17 - kMeRange;
  }

  // ---- 4. quarter-pel refinement at level 0 (me_refine, inter_common.h:141-154) ----
  if (level == 0) {
    int cxq = mx * 4, cyq = my * 4;
    for (int step = 2; step >= 1; step--) {
      int mine = 0;
      if (lane < 9) {
        const int n = lane == 0 ? 4 : (lane <= 4 ? lane - 1 : lane);  // raster 0..8, centre (4) first
        const int dx = n % 3 - 1, dy = n / 3 - 1;
        mine = satd8_q(c, ref, x0, y0, cxq + dx * step, cyq + dy * step);
      }
      int best = __shfl_sync(0xffffffffu, mine, 0), nx = cxq, ny = cyq;
#pragma unroll
      for (int t = 1; t < 9; t++) {
        const int s = __shfl_sync(0xffffffffu, mine, t) + kSubpelPenalty;
        const int n = t <= 4 ? t - 1 : t;
        if (s < best) best = s, nx = cxq + (n % 3 - 1) * step, ny = cyq + (n / 3 - 1) * step;
      }
      cxq = nx, cyq = ny;
    }
    mx = cxq, my = cyq;
  }
  if (lane == 0) {
    job.field[r][level][cell] = pack_mv(mx, my);
    if (job.stats) atomicAdd(job.stats + level, two ? 2ull : 1ull);
  }
}

void launch_me_level(const FrameJob* jobs, const WorkList& w, int level, cudaStream_t st) {
  const int units = w.prefix[w.njobs];
  if (units <= 0) return;
  k_me_level<<<(units + kMeWarps - 1) / kMeWarps, kMeWarps * 32, 0, st>>>(jobs, w, level);
}

}  // namespace celv2cu
