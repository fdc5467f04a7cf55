// kernels.h: host-side launchers of the decision engine's CUDA stages.
//
// Every stage takes a list of frame jobs (FrameJob, device memory) so one launch scores several
// frames -- the leaf B frames of a mini-GOP, or frames of several streams of different sizes --
// and each CTA finds its job and unit from a prefix table of the jobs' unit counts.
#pragma once
#include <cuda_runtime.h>

#include "common.cuh"

namespace celv2cu {

constexpr int kMaxJobs = 32;

// Units of one stage per job, as prefix sums: job j owns units [prefix[j], prefix[j + 1]).
// queue: the stage's work queue in device memory (zero before the launch) -- a persistent grid's
// CTAs take units from it in order until it runs dry; null: one CTA per unit (blockIdx.x).
struct WorkList {
  int njobs;
  int prefix[kMaxJobs + 1];
  unsigned* queue;
};

// The next unit of this CTA into `unit` (every thread gets it); false when the stage is done.
// Starts with a barrier, so the previous unit's shared state is free for the next one. No CTA
// ever waits for another: a drained queue simply ends the loop.
__device__ __forceinline__ bool take_unit(const WorkList& w, int& unit, int& iter, int* slot) {
  const int total = w.prefix[w.njobs];
  if (!w.queue) {
    if (iter++) return false;
    unit = blockIdx.x;
    return unit < total;
  }
  __syncthreads();
  if (threadIdx.x == 0) *slot = (int)atomicAdd(w.queue, 1u);
  __syncthreads();
  unit = *slot;
  return unit < total;
}

// CTAs of a persistent grid for a kernel: the SM count times the CTAs an SM holds, at most units.
int persistent_grid(const void* kernel, int threads, size_t smem, int units);

// Unit u's job (a linear scan: at most kMaxJobs jobs).
__device__ __forceinline__ int job_of(const WorkList& w, int u) {
  int j = 0;
  while (j + 1 < w.njobs && u >= w.prefix[j + 1]) j++;
  return j;
}

void launch_expand_u8(const uint8_t* raw, int pitch, const DevPlane& lv0, cudaStream_t st);
void launch_expand_u16(const uint16_t* raw, int pitch, int bit_depth, const DevPlane& lv0, cudaStream_t st);
void launch_pyramid(const DevPyramid& pyr, cudaStream_t st);
void launch_phases(const DevPlane& lv0, cudaStream_t st);

// Motion search of one pyramid level for every (job, reference, 8x8 cell), whole-pel (level 0's
// field in quarter pels). Units: me_units(nrefs, fcols[level], frows[level], cells) per job (groups
// of `cells` cells of one reference; cells 16 or 32).
int me_units(int nrefs, int cols, int rows, int cells);
void launch_me_level(const FrameJob* jobs, const WorkList& w, int level, int cells, cudaStream_t st);
// Level 0's quarter-pel refinement, in place. Units: refine_units(nrefs, fcols[0], frows[0]) per job.
int refine_units(int nrefs, int cols, int rows);
void launch_me_refine(const FrameJob* jobs, const WorkList& w, cudaStream_t st);

// Intra SATDs of every candidate block and mode. Units: sb_cols * sb_rows per job.
void launch_intra(const FrameJob* jobs, const WorkList& w, cudaStream_t st);

// Each reference's best candidate MV per candidate block, the distinct MVs of a superblock taken
// in chunks of at most `chunk` (<= 64). Units: nrefs * sb_cols * sb_rows per job. Units that keep
// their 64-level blocks are scored whole (k_inter); with `regions` (some job has keep words) a
// second kernel scores the others region by region, draining `region_queue` (zero beforehand).
void launch_inter(const FrameJob* jobs, const WorkList& w, int chunk, bool regions, unsigned* region_queue,
                  cudaStream_t st);

// Per-block choice, compound, partition choice and the decision records. Units: superblocks.
void launch_finalize(const FrameJob* jobs, const WorkList& w, cudaStream_t st);

// The learned pruner (pruner.cu): one job's features (nsb x CELV2_PRUNER_FEATURES), the network's
// forward pass into a cache of batch x CELV2_PRUNER_ACTS floats (logits last), and the masks.
void launch_features(const FrameJob* djob, int nsb, float* out, cudaStream_t st);
void pruner_forward(const float* params, const float* x, int batch, float* acts, cudaStream_t st);
// The pruner's decision rule: per output group the probability a kept option needs (references,
// intra, block levels, intra modes), and the band around them inside which a superblock falls back
// to the full search.
struct PrunerThresholds {
  float ref, intra, level, mode, band;
};
void launch_masks(const float* logits, int nsb, int nrefs, const PrunerThresholds& th, uint32_t* keep,
                  cudaStream_t st);
// The engine's inference: the network and the mask of every superblock of one job in one kernel,
// from bf16 weight copies (infer_weights: infer_weight_elems() bf16 elements).
size_t infer_weight_elems();
void infer_weights(const float* params, void* wb, cudaStream_t st);
void launch_infer(const float* params, const void* wb, const float* feats, int nsb, int nrefs,
                  const PrunerThresholds& th, uint32_t* keep, cudaStream_t st);

// Set-up of the constant tables (once per device).
cudaError_t init_tables();

}  // namespace celv2cu
