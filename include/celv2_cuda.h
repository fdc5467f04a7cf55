/* celv2_cuda.h: the C ABI of the B200 decision engine (libcelv2_cuda.so).
 *
 * The engine is a drop-in third implementation of the reference encoder's DecisionEngine
 * (src/gpu/decision_engine.h:9-51) next to its CpuEngine and VulkanEngine: it decides every
 * 64x64 superblock of a frame -- hierarchical motion search over up to 7 references with
 * quarter-pel refinement, intra / inter / compound SATD scoring and the bottom-up partition
 * choice -- and emits the decision records of include/celv2_decision.h, byte-identical to the
 * reference CpuEngine's decisions on the same 8-bit luma planes and lambda. Plain pointers and
 * sizes only; a C++ adapter deriving from DecisionEngine sits on top (celv2_b200/host/cuda_engine.h).
 *
 * Every function returns 0 on success and a negative CELV2_E* code on failure, with a message
 * for the calling thread in celv2_last_error(). One thread drives launch / prepare of an engine;
 * the row waits may come from another thread. Several engines may share a GPU.
 */
#ifndef CELV2_CUDA_H
#define CELV2_CUDA_H

#include <stdint.h>

#include "celv2_decision.h"

#ifdef __cplusplus
extern "C" {
#endif

enum {
  CELV2_OK = 0,
  CELV2_EINVAL = -1,   /* bad argument (the reference throws std::runtime_error / invalid_argument) */
  CELV2_ECUDA = -2,    /* CUDA runtime error (no device, out of memory, launch failure) */
  CELV2_ESTATE = -3,   /* call out of order (e.g. a row wait with no launch) */
};

typedef struct celv2_engine celv2_engine;

/* A frame's luma, as the reference's Frame420 holds it (src/io/y4m.h:11-23): visible width x
 * height, planes padded by edge replication to pw = (width + 7) & ~7 by ph = (height + 7) & ~7.
 * Give either the 8-bit plane `y` (Frame420::y, already rounded), or the high-depth plane `hy`
 * (Frame420::hy) with its bit_depth, which the engine rounds to 8 bits on the device exactly as
 * round_to_8bit does (src/io/y4m.cpp:28-34). pitch: samples per row (0: pw). */
typedef struct celv2_frame {
  int32_t width, height;
  int32_t pitch;
  const uint8_t* y;
  const uint16_t* hy;
  int32_t bit_depth;
} celv2_frame;

/* VulkanEngine(width, height, sb_size, device) (src/vk/vk_engine.h:18, vk_engine.cpp:172-180):
 * throws on a zero size and on sb_size != 64; here CELV2_EINVAL. */
int celv2_create(int width, int height, int sb_size, int device, celv2_engine** out);
void celv2_destroy(celv2_engine* e);

/* DecisionEngine::launch (decision_engine.h:12-18; vk_engine.cpp:207-312): queues the decision of
 * every superblock row and returns. refs nearest first, at most 7; nrefs 0 is a KEY frame.
 * ref_keys (NULL, or one per reference): a reference whose key was seen before is the same
 * picture, and its upload, pyramid and phases are reused. src_key: the key a prepare() used.
 * The inputs are copied before this returns. lambda_q8: the encoder's lambda_q8(qindex)
 * (src/core/quant.cpp:31-39). Errors as the reference's: a size mismatch or more than 7
 * references (std::runtime_error there) -> CELV2_EINVAL; a failure leaves no work running. */
int celv2_launch(celv2_engine* e, const celv2_frame* src, const celv2_frame* refs, int nrefs, int64_t lambda_q8,
                 const long long* ref_keys, long long src_key);

/* DecisionEngine::prepare (decision_engine.h:19-22; vk_engine.cpp:188-205): starts the next
 * frame's reference-free work (upload, pyramid, intra SATDs) behind the queued work, on a second
 * stream. A key < 0 or a size mismatch does nothing. */
int celv2_prepare(celv2_engine* e, const celv2_frame* next, long long key);

/* DecisionEngine::set_row_streams (decision_engine.h:30-33; vk_engine.cpp:288-294): rows come
 * back as the first row of each of n runs, then the second, ... (1: top to bottom). */
int celv2_set_row_streams(celv2_engine* e, int n);

/* Superblock columns and rows of the engine's frames. */
int celv2_geometry(const celv2_engine* e, int* sb_cols, int* sb_rows);

/* The order the last launch brings rows back in (sb_rows entries). */
int celv2_row_order(const celv2_engine* e, int* rows);

/* The collect side (DecisionEngine::collect, decision_engine.h:27-29): blocks until superblock
 * row `row` of the last launch is in host memory and returns its sb_cols records (valid until the
 * next launch). */
int celv2_wait_row(celv2_engine* e, int row, const celv2_sb_out** records);

/* Returns with no work of the last launch pending (collect's end). */
int celv2_finish(celv2_engine* e);

/* The calling thread's last error message ("" if none). */
const char* celv2_last_error(void);

/* ---- Device-resident path (frames already in HBM; batching) ---- */

/* Uploads a frame into the engine's keyed frame store (pyramid and quarter-pel phases), as a
 * reference would be; key >= 0. Later launches find it by key (celv2_launch's ref_keys too). It
 * stays until celv2_drop_frame / celv2_clear_store: celv2_launch's own cache of references does not
 * evict it. The upload runs behind the queued work. */
int celv2_upload(celv2_engine* e, const celv2_frame* f, long long key);
/* celv2_upload from a plane in page-locked host memory (celv2_host_alloc; else CELV2_EINVAL), by
 * DMA after the call returns, with no copy on the host: the caller keeps the plane unchanged
 * until the engine is idle (celv2_finish). No counterpart in the reference. */
int celv2_upload_pinned(celv2_engine* e, const celv2_frame* f, long long key);

/* One batch of frames decided from the frame store: job i decides the frame with key src_keys[i]
 * against the nrefs[i] frames ref_keys[i][0..]. All jobs' stages run as one launch per stage.
 * Records stay in device memory unless `to_host` is nonzero, in which case they come back to the
 * engine's host buffer (celv2_group_records). At most 32 jobs, nsb * jobs within the engine's
 * group capacity (celv2_create sizes it for 8 frames; celv2_reserve_group raises it). */
int celv2_launch_group(celv2_engine* e, int njobs, const long long* src_keys, const int* nrefs,
                       const long long* const* ref_keys, const int64_t* lambda_q8, int to_host);
int celv2_reserve_group(celv2_engine* e, int frames);
/* The same across engines of different frame sizes on one GPU (frames of several streams): job i
 * decides a frame of engines[i]'s store. One launch per stage for all of them -- each stage a
 * persistent kernel draining one work queue, the largest jobs first -- on engines[0]'s stream.
 * Engine e's jobs take its group slots in their order here (celv2_group_records(e, k) is e's k-th
 * job). No counterpart in the reference, whose engines are each made for one frame size
 * (src/vk/vk_engine.h:18). */
int celv2_launch_multi(int njobs, celv2_engine* const* engines, const long long* src_keys, const int* nrefs,
                       const long long* const* ref_keys, const int64_t* lambda_q8, int to_host);
int celv2_group_records(celv2_engine* e, int job, const celv2_sb_out** records);

/* Drops every frame of the store. */
int celv2_clear_store(celv2_engine* e);
/* Drops the stored frame with this key (none: nothing happens); a later upload reuses its device
 * memory. Queued work that reads it still sees it: uploads run behind the queued work. */
int celv2_drop_frame(celv2_engine* e, long long key);

/* ---- Records straight into the caller's memory ----
 * No counterpart in the reference, whose engines hand the records over through their own
 * buffers. celv2_set_output names where the NEXT launch (celv2_launch: job 0; celv2_launch_group
 * or celv2_launch_multi: this engine's job-th frame) copies its sb_cols * sb_rows records: page-
 * locked host memory from celv2_host_alloc (any other memory: CELV2_EINVAL), or NULL for the
 * engine's own buffer. It applies to that one launch; celv2_wait_row and celv2_group_records then
 * return pointers into it. The caller keeps the memory until the launch is collected. */
int celv2_set_output(celv2_engine* e, int job, celv2_sb_out* records);
int celv2_host_alloc(long long bytes, void** out);
int celv2_host_free(void* p);

/* ---- Pruned search ----
 * No counterpart in the reference. celv2_set_keep_words gives the NEXT launch's job (numbered as
 * for celv2_set_output) one keep word per superblock (sb_cols * sb_rows, raster order; NULL:
 * exhaustive): the references, intra, the block levels and the intra modes it keeps
 * (include/celv2_decision.h). A superblock then scores only what it keeps -- exactly as the
 * exhaustive search scores it -- and picks among that: its pruned references' records read
 * CELV2_NO_REF_COST, with intra pruned no block is intra, the blocks of a pruned level read as
 * blocks with no choice. A KEY frame always scores everything. The motion search skips the level-0
 * cells no superblock's kept references read; the inter stage scores only the tiles and motion
 * vectors the kept levels' blocks use; the intra stage skips pruned levels and modes.
 * celv2_set_keep: the same from one byte per superblock (bits 0-7 of the word: the references and
 * intra; every level and mode kept).
 * celv2_sb_costs copies the last launch's per-superblock cost of the chosen partition (the sum the
 * partition choice minimises, lambda-weighted SATD plus rate) for one job; it waits for the work. */
int celv2_set_keep(celv2_engine* e, int job, const uint8_t* keep);
int celv2_set_keep_words(celv2_engine* e, int job, const uint32_t* keep);
int celv2_sb_costs(celv2_engine* e, int job, int64_t* out);

/* ---- A KEY-frame decision that allocates nothing ----
 * No counterpart in the reference. For callers that cannot allocate device memory while they run
 * (a host application that provisions all GPU memory up front, a path that cannot take the device
 * synchronisation of cudaMalloc / cudaFree): decides an intra-only frame from the caller's padded
 * 8-bit luma plane (`luma`, device memory, pw x ph with row pitch `pitch` >= pw) into the caller's
 * sb_cols * sb_rows records (`out`, device memory), on `stream` (a cudaStream_t, NULL: the default
 * stream), with the same records as celv2_launch with no references. Its scratch is a fixed static
 * device array: frames above CELV2_NOALLOC_MAX_SUPERBLOCKS superblocks are rejected (CELV2_EINVAL);
 * the first call on a device sets it up (call it before any stream capture); calls whose GPU work
 * overlaps race on the shared scratch. */
#define CELV2_NOALLOC_MAX_SUPERBLOCKS 768
int celv2_decide_key_noalloc(const uint8_t* luma, int width, int height, int pitch, int64_t lambda_q8,
                             celv2_sb_out* out, void* stream);

/* ---- Inspection (tests) ---- */

/* The last launch's motion field of reference r at pyramid level l: cols x rows packed MVs
 * (mvy << 16 | (mvx & 0xffff)); cols / rows receive the size. Synchronises. */
int celv2_debug_field(celv2_engine* e, int r, int level, int32_t* out, int* cols, int* rows);
/* The last launch's intra SATDs: sb_cols * sb_rows * 425 * 13 int32. Synchronises. */
int celv2_debug_intra(celv2_engine* e, int32_t* out);
/* The last launch's per-reference bests: sb_cols * sb_rows * 7 * 425 (SATD, packed MV) pairs. */
int celv2_debug_inter(celv2_engine* e, int32_t* out);
/* Kernel launches the engine has issued so far (all stages). */
long long celv2_kernel_launches(const celv2_engine* e);

/* ---- Configuration ----
 * How the stages run; none of it changes a decision.
 *  CELV2_CFG_PERSISTENT: 1 (default) -- each stage is one persistent kernel whose CTAs drain a
 *    device-side queue of the batch's work units (superblocks, cell groups); 0 -- one CTA per unit.
 *  CELV2_CFG_GRAPHS: 1 -- celv2_launch_group captures a batch's whole stage sequence (descriptor
 *    copy, queue resets, stage kernels) as a CUDA graph once per batch shape (the jobs' reference
 *    counts) and replays it, the record copies following it; 0 (default) -- launches stage by
 *    stage.
 *  CELV2_CFG_PERSISTENT_OFF: a bit mask of stages that run one CTA per unit even when
 *    CELV2_CFG_PERSISTENT is on (bit l: motion-search level l, 5 intra, 6 inter, 7 finalize,
 *    8 level 0's quarter-pel refinement).
 *  CELV2_CFG_INTER_CHUNK: distinct MVs per pass of the inter stage, 8..64 (default 64).
 *  CELV2_CFG_ME_CELLS_L0 + l: 8x8 cells per motion-search CTA at pyramid level l, 15 or 30
 *    (default 30).
 *  CELV2_CFG_FEATURES: 1 -- every inter frame's learned-pruner features are kept for
 *    celv2_features (include/celv2_pruner.h); 0 (default) -- only when the pruner runs.
 * The autotuner (celv2_b200/tune.py) times these per frame size and sets the fastest. */
enum {
  CELV2_CFG_PERSISTENT = 1,
  CELV2_CFG_GRAPHS = 2,
  CELV2_CFG_PERSISTENT_OFF = 3,
  CELV2_CFG_INTER_CHUNK = 4,
  CELV2_CFG_FEATURES = 5,
  CELV2_CFG_ME_CELLS_L0 = 10,
};
int celv2_set_config(celv2_engine* e, int key, int value);
int celv2_get_config(const celv2_engine* e, int key, int* value);

/* ---- Measurement ---- */

/* The engine's main stream (a cudaStream_t), for timing events around its work. */
int celv2_stream(const celv2_engine* e, void** stream);
/* Stage timing: when enabled, every stage launch is bracketed by CUDA events on its stream.
 * celv2_stage_times returns (and resets) the summed milliseconds and launch counts per stage, in
 * the order: uploads (8-bit level 0 + pyramid), quarter-pel phases, motion search levels 4, 3, 2,
 * 1, 0, intra, inter, finalize, level 0's quarter-pel refinement, the learned pruner (CELV2_STAGES
 * entries). */
#define CELV2_STAGES 12
int celv2_stage_timing(celv2_engine* e, int enable);
int celv2_stage_times(celv2_engine* e, double* ms, long long* launches, int n);
/* Work the kernels executed while stage timing was on, then reset: [l] motion-search centres
 * searched at level l (0..4), [5] 4x4 tile SATDs of the inter stage (tiles x distinct candidate
 * MVs, summed over (superblock, reference) and its regions), [6] compound 4x4 tiles
 * (CELV2_WORK_COUNTERS entries). */
#define CELV2_WORK_COUNTERS 8
int celv2_work_counters(celv2_engine* e, unsigned long long* out, int n);
/* The GPU's measured INT32 throughput (integer ops per second): the roofline denominator of the
 * integer-bound decision kernels. */
int celv2_int_peak(int device, double* ops_per_s);

#ifdef __cplusplus
}
#endif

#endif /* CELV2_CUDA_H */
