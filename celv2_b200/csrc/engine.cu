// engine.cu: the host side of the B200 decision engine behind the C ABI of include/celv2_cuda.h.
//
// Structure (per engine, one resolution, one GPU):
//  - a frame store in HBM: keyed slots holding a frame's 5-level pyramid with replicated margins
//    and, for references, the 15 quarter-pel phase planes (the reference Vulkan engine's RefSlot,
//    src/vk/vk_engine.cpp:71-78,239-258: the slot of a key is reused, else one this launch does not
//    need, else a new one);
//  - two source slots: while one frame is decided, prepare() builds the next one's pyramid and
//    intra SATDs on a second stream (vk_engine.cpp:80-87,188-205);
//  - per launch: the stage kernels on the main stream -- motion search level by level for every
//    reference, intra (unless prepared), inter candidates, finalize -- then one device-to-host
//    copy per superblock row with an event, so rows are collected as they arrive
//    (vk_engine.cpp:288-328);
//  - uploads go through a ring of pinned staging buffers: launch() copies the caller's planes into
//    pinned memory before it returns (the reference requires that the inputs may change at once,
//    decision_engine.h:12-16).
// No CPU fallback: every decision is made by the kernels; a missing GPU is an error.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "celv2_cuda.h"
#include "celv2_pruner.h"
#include "kernels.h"
#include "tables.h"

namespace celv2cu {
void set_last_error(const std::string& msg);
cudaError_t measure_int_peak(int device, double* ops_per_s);
cudaError_t me_attributes();
cudaError_t inter_attributes();
cudaError_t intra_attributes();
cudaError_t finalize_attributes();
}  // namespace celv2cu

using namespace celv2cu;

namespace {
thread_local std::string g_error;
std::mutex g_grid_mu;
struct GridKey {
  const void* kernel;
  int device, threads;
  size_t smem;
};
std::vector<std::pair<GridKey, int>> g_grid_cache;  // CTAs per SM x SMs, per kernel and device
}  // namespace

// The calling thread's message for celv2_last_error (entry points outside this file set it too).
void celv2cu::set_last_error(const std::string& msg) { g_error = msg; }

int celv2cu::persistent_grid(const void* kernel, int threads, size_t smem, int units) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_grid_mu);
  for (const auto& e : g_grid_cache)
    if (e.first.kernel == kernel && e.first.device == dev && e.first.threads == threads && e.first.smem == smem)
      return units < e.second ? units : e.second;
  int per_sm = 1, sms = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int full = (per_sm < 1 ? 1 : per_sm) * sms;
  g_grid_cache.push_back({GridKey{kernel, dev, threads, smem}, full});
  return units < full ? units : full;
}

namespace {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error(CELV2_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}
#define CK(x) check((x), #x)

void invalid(const std::string& m) { throw Error(CELV2_EINVAL, m); }

template <typename F>
int guarded(F&& f) {
  try {
    f();
    return CELV2_OK;
  } catch (const Error& e) {
    g_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_error = e.what();
    return CELV2_ECUDA;
  }
}

std::mutex g_init_mu;
std::vector<char> g_ready;  // per device: kernel attributes set

void init_device(int dev) {
  std::lock_guard<std::mutex> lk(g_init_mu);
  if ((int)g_ready.size() <= dev) g_ready.resize(dev + 1, 0);
  if (g_ready[dev]) return;
  CK(me_attributes());
  CK(inter_attributes());
  CK(intra_attributes());
  CK(finalize_attributes());
  // the constant tables' copies (from pageable memory) land before any kernel on another stream
  CK(cudaDeviceSynchronize());
  g_ready[dev] = 1;
}

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Geometry of one frame size: padded luma, pyramid levels, fields, superblocks.
struct Geometry {
  int width = 0, height = 0, pw = 0, ph = 0;
  int w[kLevels], h[kLevels], margin[kLevels], stride[kLevels];
  size_t level_bytes[kLevels], level_off[kLevels];
  size_t pyr_bytes = 0, pyr_bytes_phases = 0;
  int fcols[kLevels], frows[kLevels];
  int sb_cols = 0, sb_rows = 0, nsb = 0;
  size_t field_ints = 0;  // all levels of one reference

  void set(int width_, int height_) {
    width = width_, height = height_;
    pw = (width + 7) & ~7, ph = (height + 7) & ~7;
    for (int l = 0; l < kLevels; l++) {
      w[l] = l ? w[l - 1] / 2 : pw;
      h[l] = l ? h[l - 1] / 2 : ph;
      margin[l] = level_margin(l);
      stride[l] = (int)align_up((size_t)w[l] + 2 * margin[l], 64);
      level_bytes[l] = align_up((size_t)stride[l] * (h[l] + 2 * margin[l]), 256);
      fcols[l] = (w[l] + 7) / 8, frows[l] = (h[l] + 7) / 8;
    }
    // level 0 first (its 15 phases follow it when present), then levels 1-4
    size_t off = 0;
    level_off[0] = 0;
    off = level_bytes[0];
    for (int l = 1; l < kLevels; l++) level_off[l] = off, off += level_bytes[l];
    pyr_bytes = off;
    pyr_bytes_phases = off + (kPhases - 1) * level_bytes[0];
    sb_cols = (width + 63) / 64, sb_rows = (height + 63) / 64, nsb = sb_cols * sb_rows;
    field_ints = 0;
    for (int l = 0; l < kLevels; l++) field_ints += (size_t)fcols[l] * frows[l];
  }
};

// A frame's pyramid in HBM.
struct Slot {
  long long key = -1;
  long long used = -1;
  bool phases = false;
  bool resident = false;  // uploaded into the store (celv2_upload): launch()'s reference cache leaves it
  // Store uploads run on the engine's upload stream: `ready` marks this slot's upload done; the
  // launches that read the slot record `last_use` on their stream, which a later upload into the
  // slot waits for.
  cudaEvent_t ready = nullptr, last_use = nullptr;
  bool ready_pending = false, use_pending = false;
  uint8_t* mem = nullptr;
  size_t bytes = 0;
  DevPyramid pyr{};
};

// One pinned staging buffer with its device copy (an upload in flight).
struct Stage {
  void* host = nullptr;
  void* dev = nullptr;
  size_t bytes = 0;
  cudaEvent_t done = nullptr;
  bool pending = false;
};

// Stages timed by CUDA events when stage timing is on (celv2_stage_timing).
enum StageId { kStUpload, kStPhases, kStMe4, kStMe3, kStMe2, kStMe1, kStMe0, kStIntra, kStInter, kStFinalize, kStRefine,
               kStPruner, kStages };

// A job's learned-pruner work, queued between motion-search levels 1 and 0: its features into
// `feats` (when non-null), and with `net` the network and the masks into `keep`.
struct NetJob {
  float* feats = nullptr;
  bool net = false;
  const float* params = nullptr;
  const void* wb = nullptr;  // bf16 weight copies of the inference kernel
  uint32_t* keep = nullptr;
  PrunerThresholds th{};
};

// Per-frame device buffers of a decision.
struct JobBuffers {
  int* fields = nullptr;     // kMaxRefs * field_ints
  int* intra = nullptr;      // nsb * kBlocks * kModes
  int2* inter = nullptr;     // nsb * kMaxRefs * kBlocks
  celv2_sb_out* out = nullptr;
  celv2_sb_out* out2 = nullptr;  // group buffers: out, out2, out3 in turn (see group_parity)
  celv2_sb_out* out3 = nullptr;
  // group record buffer set p (0: out, 1: out2, 2: out3)
  celv2_sb_out* records(int p) const { return p == 0 ? out : p == 1 ? out2 : out3; }
  uint32_t* keep = nullptr;      // pruning keep words of the job, when given (nsb)
  long long* sb_cost = nullptr;  // per superblock, the chosen partition's cost (nsb)
  float* feats = nullptr;        // the learned pruner's features (nsb x CELV2_PRUNER_FEATURES)
  bool owns_feats = false;       // group slots share one block (consecutive slots, consecutive rows)
};

}  // namespace

struct celv2_engine {
  int device = 0;
  Geometry g;
  cudaStream_t st = nullptr, prep_st = nullptr;
  cudaEvent_t prep_done = nullptr;
  std::vector<Slot*> store;      // keyed frames (references, resident frames)
  Slot srcs[2];                  // sources of launch / prepare
  int cur_src = 0;
  long long launches = 0;
  long long launches_group = -1;  // the value of `launches` after the last group launch
  std::vector<Stage> stages;
  int next_stage = 0;
  JobBuffers single;             // the launch() path
  int* intra_prep[2] = {nullptr, nullptr};  // intra SATDs per source slot
  celv2_sb_out* host_out = nullptr;          // pinned, nsb records
  // caller memory for the next launch's records (celv2_set_output), per job; where the last
  // launch's records went (launch: last_out; group: group_out[job])
  celv2_sb_out* next_out[kMaxJobs] = {};
  std::vector<uint32_t> next_keep[kMaxJobs];  // keep words for the next launch's jobs (celv2_set_keep)
  celv2_sb_out* last_out = nullptr;
  celv2_sb_out* group_out[kMaxJobs] = {};
  std::vector<cudaEvent_t> row_done;
  std::vector<int> order;
  int row_streams = 1;
  bool pending = false;
  int last_nrefs = 0;
  FrameJob* djobs = nullptr;     // 2 * kMaxJobs + 1 device descriptors (the last: prepare's)
  // Descriptors go to the device from a ring of pinned buffers: an asynchronous copy from pageable
  // memory may wait for the stream, which would serialise back-to-back launches.
  static constexpr int kRing = 8, kRingJobs = 2 * kMaxJobs + 1;
  // Store slots an upload may add rather than wait for a dropped slot's readers (a caller that
  // issues far ahead of the GPU would otherwise grow the store without bound).
  static constexpr int kStoreSlotsIdle = 48;
  FrameJob* ring = nullptr;
  cudaEvent_t ring_done[kRing] = {};
  bool ring_pending[kRing] = {};
  int ring_next = 0;
  // group path
  int group_cap = 0;
  std::vector<JobBuffers> group;
  float* group_feats = nullptr;  // the group slots' pruner features, slot after slot
  celv2_sb_out* group_host = nullptr;
  int group_jobs = 0;
  // Group records go to the host on copy_st, overlapping the next groups' stages, which write the
  // other device record buffers: three sets in turn (group_parity), so a group waits only for the
  // copies of the group three back (with two, the group after a large batch waited for that
  // batch's records to cross PCIe); copied[p] marks buffer set p's copies done.
  cudaStream_t copy_st = nullptr;
  cudaStream_t up_st = nullptr;  // celv2_upload's stream (frame-store uploads)
  static constexpr int kRecordSets = 3;
  cudaEvent_t stages_done = nullptr, copied[kRecordSets] = {};
  bool copy_pending[kRecordSets] = {};
  int group_parity = 0;
  long long kernel_launches = 0;
  // stage timing: an event pair around each stage launch, harvested when the stream is idle
  bool timing = false;
  struct Timed {
    int stage;
    cudaEvent_t a, b;
  };
  std::vector<Timed> timed;
  std::vector<cudaEvent_t> event_pool;
  double stage_ms[kStages] = {};
  long long stage_n[kStages] = {};
  unsigned long long* stats = nullptr;  // device work counters (kStats), while timing
  // stage work queues (device counters): [0..4] motion search levels, [5] intra, [6] inter,
  // [7] finalize, [8] level 0's refinement, [9] inter by regions, of the main stream; [15]
  // prepare's intra
  unsigned* queues = nullptr;
  bool persistent = true;      // the queue-draining persistent stage kernels (else one CTA per unit)
  unsigned persistent_off = 0; // stages (bit i: queue i) that run one CTA per unit anyway
  int me_cells[kLevels] = {30, 30, 30, 30, 30};
  // the learned pruner: features on request, the network when parameters are set
  bool features_on = false;
  float* pruner_params = nullptr;  // device, CELV2_PRUNER_PARAMS floats
  void* nn_wb = nullptr;           // device, bf16 weight copies for the inference kernel
  PrunerThresholds pruner_th{0.5f, 0.5f, 0.5f, 0.5f, 0.f};

  // The pruner work of a job of this engine (buffers b; keep_given: celv2_set_keep masks win).
  NetJob net_for(const FrameJob& job, const JobBuffers& b, bool keep_given) const {
    NetJob n;
    if (job.nrefs == 0) return n;
    const bool net = pruner_params && !keep_given;
    if (!features_on && !net) return n;
    n.feats = b.feats, n.net = net, n.params = pruner_params, n.wb = nn_wb, n.keep = b.keep;
    n.th = pruner_th;
    return n;
  }
  int inter_chunk = 64;

  template <typename F>
  void stage(int id, cudaStream_t stream, F&& f) {
    if (!timing) {
      f();
      return;
    }
    cudaEvent_t ev[2];
    for (cudaEvent_t& e : ev) {
      if (event_pool.empty()) {
        CK(cudaEventCreate(&e));
      } else {
        e = event_pool.back();
        event_pool.pop_back();
      }
    }
    CK(cudaEventRecord(ev[0], stream));
    f();
    CK(cudaEventRecord(ev[1], stream));
    timed.push_back({id, ev[0], ev[1]});
  }

  void harvest() {
    for (const Timed& t : timed) {
      CK(cudaEventSynchronize(t.b));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, t.a, t.b));
      stage_ms[t.stage] += ms;
      stage_n[t.stage]++;
      event_pool.push_back(t.a), event_pool.push_back(t.b);
    }
    timed.clear();
  }

  ~celv2_engine() {
    cudaSetDevice(device);
    if (st) cudaStreamSynchronize(st);
    if (prep_st) cudaStreamSynchronize(prep_st);
    if (copy_st) cudaStreamSynchronize(copy_st);
    if (up_st) cudaStreamSynchronize(up_st);
    free_graphs();
    for (Slot* s : store) free_slot(s);
    for (Slot& s : srcs) cudaFree(s.mem);
    for (Stage& s : stages) {
      cudaFreeHost(s.host), cudaFree(s.dev);
      if (s.done) cudaEventDestroy(s.done);
    }
    free_buffers(single);
    for (JobBuffers& b : group) free_buffers(b);
    for (int* p : intra_prep) cudaFree(p);
    cudaFreeHost(host_out);
    cudaFreeHost(group_host);
    for (cudaEvent_t e : row_done) cudaEventDestroy(e);
    for (const Timed& t : timed) cudaEventDestroy(t.a), cudaEventDestroy(t.b);
    cudaFree(stats);
    cudaFree(queues);
    cudaFree(pruner_params);
    cudaFree(nn_wb);
    cudaFree(group_feats);
    for (cudaEvent_t e : event_pool) cudaEventDestroy(e);
    cudaFree(djobs);
    cudaFreeHost(ring);
    for (cudaEvent_t e : ring_done)
      if (e) cudaEventDestroy(e);
    if (prep_done) cudaEventDestroy(prep_done);
    if (stages_done) cudaEventDestroy(stages_done);
    for (cudaEvent_t e : copied)
      if (e) cudaEventDestroy(e);
    if (st) cudaStreamDestroy(st);
    if (prep_st) cudaStreamDestroy(prep_st);
    if (copy_st) cudaStreamDestroy(copy_st);
    if (up_st) cudaStreamDestroy(up_st);
  }

  static void free_slot(Slot* s) {
    cudaFree(s->mem);
    if (s->ready) cudaEventDestroy(s->ready);
    if (s->last_use) cudaEventDestroy(s->last_use);
    delete s;
  }

  static void free_buffers(JobBuffers& b) {
    cudaFree(b.fields), cudaFree(b.intra), cudaFree(b.inter), cudaFree(b.out), cudaFree(b.out2), cudaFree(b.out3);
    cudaFree(b.keep), cudaFree(b.sb_cost);
    if (b.owns_feats) cudaFree(b.feats);
    b = JobBuffers{};
  }

  void alloc_buffers(JobBuffers& b, bool with_intra) {
    CK(cudaMalloc(&b.fields, kMaxRefs * g.field_ints * sizeof(int)));
    if (with_intra) CK(cudaMalloc(&b.intra, (size_t)g.nsb * kBlocks * kModes * sizeof(int)));
    CK(cudaMalloc(&b.inter, (size_t)g.nsb * kMaxRefs * kBlocks * sizeof(int2)));
    CK(cudaMalloc(&b.out, (size_t)g.nsb * sizeof(celv2_sb_out)));
    if (with_intra) {
      CK(cudaMalloc(&b.out2, (size_t)g.nsb * sizeof(celv2_sb_out)));
      CK(cudaMalloc(&b.out3, (size_t)g.nsb * sizeof(celv2_sb_out)));
    }
    CK(cudaMalloc(&b.keep, (size_t)g.nsb * sizeof(uint32_t)));
    CK(cudaMalloc(&b.sb_cost, (size_t)g.nsb * sizeof(long long)));
    if (!with_intra) {  // the group slots' features are one block (reserve_group)
      CK(cudaMalloc(&b.feats, (size_t)g.nsb * CELV2_PRUNER_FEATURES * sizeof(float)));
      b.owns_feats = true;
    }
  }

  void init(int width, int height, int dev) {
    device = dev;
    CK(cudaSetDevice(dev));
    init_device(dev);
    g.set(width, height);
    CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&prep_st, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&prep_done, cudaEventDisableTiming));
    CK(cudaStreamCreateWithFlags(&copy_st, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&up_st, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&stages_done, cudaEventDisableTiming));
    for (cudaEvent_t& e : copied) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CK(cudaMalloc(&djobs, kRingJobs * sizeof(FrameJob)));
    CK(cudaMalloc(&queues, 16 * sizeof(unsigned)));
    CK(cudaMallocHost(&ring, (size_t)kRing * kRingJobs * sizeof(FrameJob)));
    for (cudaEvent_t& e : ring_done) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    alloc_buffers(single, false);
    for (int*& p : intra_prep) CK(cudaMalloc(&p, (size_t)g.nsb * kBlocks * kModes * sizeof(int)));
    CK(cudaMallocHost(&host_out, (size_t)g.nsb * sizeof(celv2_sb_out)));
    last_out = host_out;
    row_done.resize(g.sb_rows);
    for (cudaEvent_t& e : row_done) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    stages.resize(16);
    for (Stage& s : stages) CK(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming));
    for (Slot& s : srcs) alloc_slot(s, false);
  }

  // ---- frame pyramids ----
  void alloc_slot(Slot& s, bool phases) {
    // + slack: an unaligned 4-byte read (load4) may touch up to 3 bytes past the last row
    const size_t need = (phases ? g.pyr_bytes_phases : g.pyr_bytes) + 256;
    if (s.mem && s.bytes >= need) return;
    if (s.mem) CK(cudaFree(s.mem));
    s.mem = nullptr;
    CK(cudaMalloc(&s.mem, need));
    s.bytes = need;
    for (int l = 0; l < kLevels; l++) {
      DevPlane& p = s.pyr.lv[l];
      // level 0's phases sit right after it: levels 1-4 move behind the phases
      const size_t off = l == 0 ? 0 : (phases ? g.level_off[l] + (kPhases - 1) * g.level_bytes[0] : g.level_off[l]);
      p.p = s.mem + off + (size_t)g.margin[l] * g.stride[l] + g.margin[l];
      p.stride = g.stride[l], p.w = g.w[l], p.h = g.h[l], p.margin = g.margin[l];
      p.phase = l == 0 && phases ? (long long)g.level_bytes[0] : 0;
    }
    s.phases = false;
  }

  Stage& take_stage(size_t bytes) {
    Stage& s = stages[next_stage];
    next_stage = (next_stage + 1) % (int)stages.size();
    if (s.pending) CK(cudaEventSynchronize(s.done)), s.pending = false;
    if (s.bytes < bytes) {
      if (s.host) CK(cudaFreeHost(s.host));
      if (s.dev) CK(cudaFree(s.dev));
      s.host = s.dev = nullptr;
      CK(cudaMallocHost(&s.host, bytes));
      CK(cudaMalloc(&s.dev, bytes));
      s.bytes = bytes;
    }
    return s;
  }

  void check_frame(const celv2_frame* f, const char* what) {
    if (!f) invalid(std::string(what) + ": null frame");
    if (f->width != g.width || f->height != g.height)
      invalid(std::string("CudaEngine: ") + what + " size does not match the engine");
    if (!f->y && !f->hy) invalid(std::string(what) + ": no luma plane");
    if (!f->y && (f->bit_depth < 9 || f->bit_depth > 16)) invalid(std::string(what) + ": bit depth must be 9..16");
    if (f->pitch && f->pitch < g.pw) invalid(std::string(what) + ": pitch below the padded width");
  }

  // Copies f's luma into pinned memory (synchronously: the caller may change it afterwards), then
  // queues its upload, the 8-bit level 0, the pyramid and (phases) the quarter-pel planes.
  // Uploads f into s on `stream`: 8-bit level 0 and pyramid, the phase planes too when `phases`
  // (room for them when `room`).
  // direct: the plane is page-locked and stays unchanged until the upload ran (DMA from it, no
  // staging copy on the host).
  void upload(const celv2_frame* f, Slot& s, bool phases, cudaStream_t stream, bool room = false,
              bool direct = false) {
    alloc_slot(s, phases || room || s.phases);
    const bool wide = f->y == nullptr;
    const int pitch = f->pitch ? f->pitch : g.pw;
    const size_t row = (size_t)g.pw * (wide ? 2 : 1);
    Stage& sg = take_stage(row * g.ph);
    const uint8_t* src = wide ? reinterpret_cast<const uint8_t*>(f->hy) : f->y;
    const size_t spitch = (size_t)pitch * (wide ? 2 : 1);
    if (direct) {
      CK(cudaMemcpy2DAsync(sg.dev, row, src, spitch, row, g.ph, cudaMemcpyHostToDevice, stream));
    } else {
      if (spitch == row) {
        std::memcpy(sg.host, src, row * g.ph);
      } else {
        for (int r = 0; r < g.ph; r++) std::memcpy((uint8_t*)sg.host + r * row, src + r * spitch, row);
      }
      CK(cudaMemcpyAsync(sg.dev, sg.host, row * g.ph, cudaMemcpyHostToDevice, stream));
    }
    stage(kStUpload, stream, [&] {
      if (wide)
        launch_expand_u16((const uint16_t*)sg.dev, g.pw, f->bit_depth, s.pyr.lv[0], stream);
      else
        launch_expand_u8((const uint8_t*)sg.dev, g.pw, s.pyr.lv[0], stream);
    });
    CK(cudaEventRecord(sg.done, stream));
    sg.pending = true;
    stage(kStUpload, stream, [&] { launch_pyramid(s.pyr, stream); });
    kernel_launches += 1 + (kLevels - 1);
    s.phases = false;
    if (phases) make_phases(s, stream);
  }

  void make_phases(Slot& s, cudaStream_t stream) {
    if (s.phases) return;
    stage(kStPhases, stream, [&] { launch_phases(s.pyr.lv[0], stream); });
    kernel_launches++;
    s.phases = true;
  }

  // The store's slot for `key` (keys of this launch are protected), else a free or new one.
  Slot* ref_slot(long long key, const long long* keys, int nkeys, long long now, bool& fresh) {
    fresh = false;
    if (key >= 0)
      for (Slot* s : store)
        if (s->key == key) return s;
    Slot* pick = nullptr;
    for (Slot* s : store) {
      if (s->used == now || s->resident) continue;
      bool needed = false;
      for (int i = 0; i < nkeys && keys; i++) needed |= s->key >= 0 && s->key == keys[i];
      if (needed) continue;
      if (!pick || s->used < pick->used) pick = s;
    }
    if (!pick) {
      pick = new Slot;
      store.push_back(pick);
    }
    pick->key = -1;
    fresh = true;
    return pick;
  }

  void fill_job(FrameJob& job, const DevPyramid& cur, Slot* const* refs, int nrefs, const JobBuffers& b,
                const int* intra, long long lam) {
    std::memset(&job, 0, sizeof job);
    job.cur = cur;
    for (int r = 0; r < nrefs; r++) job.ref[r] = refs[r]->pyr;
    job.nrefs = nrefs;
    job.pw = g.pw, job.ph = g.ph;
    job.sb_cols = g.sb_cols, job.sb_rows = g.sb_rows;
    for (int l = 0; l < kLevels; l++) job.fcols[l] = g.fcols[l], job.frows[l] = g.frows[l];
    for (int r = 0; r < kMaxRefs; r++) {
      size_t off = r * g.field_ints;
      for (int l = 0; l < kLevels; l++) {
        job.field[r][l] = b.fields + off;
        off += (size_t)g.fcols[l] * g.frows[l];
      }
    }
    job.intra = intra;
    job.inter = b.inter;
    job.out = b.out;
    job.lam = lam;
    job.stats = timing ? stats : nullptr;
    job.sb_cost = b.sb_cost;
  }

  // The keep words named for the next launch's jobs (celv2_set_keep); clears them.
  std::array<std::vector<uint32_t>, kMaxJobs> take_keeps() {
    std::array<std::vector<uint32_t>, kMaxJobs> k;
    for (int j = 0; j < kMaxJobs; j++) k[j].swap(next_keep[j]);
    return k;
  }

  // A job's masks copied into b.keep on `stream` through the staging ring; null when none.
  const uint32_t* put_keep(const std::vector<uint32_t>& k, const JobBuffers& b, cudaStream_t stream) {
    if (k.empty()) return nullptr;
    const size_t bytes = (size_t)g.nsb * sizeof(uint32_t);
    Stage& sg = take_stage(bytes);
    std::memcpy(sg.host, k.data(), bytes);
    CK(cudaMemcpyAsync(b.keep, sg.host, bytes, cudaMemcpyHostToDevice, stream));
    CK(cudaEventRecord(sg.done, stream));
    sg.pending = true;
    return b.keep;
  }

  // Queues the copy of n descriptors to dst (device) through the pinned ring.
  void put_jobs(const FrameJob* jobs, int n, FrameJob* dst, cudaStream_t stream) {
    const int i = ring_next;
    ring_next = (ring_next + 1) % kRing;
    if (ring_pending[i]) CK(cudaEventSynchronize(ring_done[i])), ring_pending[i] = false;
    FrameJob* h = ring + (size_t)i * kRingJobs;
    std::memcpy(h, jobs, n * sizeof(FrameJob));
    CK(cudaMemcpyAsync(dst, h, n * sizeof(FrameJob), cudaMemcpyHostToDevice, stream));
    CK(cudaEventRecord(ring_done[i], stream));
    ring_pending[i] = true;
  }

  // Queues the stage kernels of the jobs whose descriptors are in djobs (intra for all of them
  // or none); returns the kernels launched.
  int enqueue_stages(const std::vector<FrameJob>& jobs, bool with_intra, cudaStream_t stream,
                     const std::vector<NetJob>& nets) {
    const int n = (int)jobs.size();
    int launched = 0;
    if (persistent) CK(cudaMemsetAsync(queues, 0, 10 * sizeof(unsigned), stream));
    auto q = [&](int i) { return persistent && !(persistent_off >> i & 1) ? queues + i : nullptr; };
    WorkList w{};
    w.njobs = n;
    for (int l = kLevels - 1; l >= 0; l--) {
      for (int j = 0; j < n; j++)
        w.prefix[j + 1] = w.prefix[j] + me_units(jobs[j].nrefs, jobs[j].fcols[l], jobs[j].frows[l], me_cells[l]);
      if (l == 0 && !nets.empty())  // the learned pruner, from the level-1 motion search
        stage(kStPruner, stream, [&] { launched += enqueue_pruner(jobs, nets, stream); });
      w.queue = q(l);
      if (w.prefix[n] > 0) {
        stage(kStMe0 - l, stream, [&] { launch_me_level(djobs, w, l, me_cells[l], stream); });
        launched++;
      }
    }
    for (int j = 0; j < n; j++)
      w.prefix[j + 1] = w.prefix[j] + refine_units(jobs[j].nrefs, jobs[j].fcols[0], jobs[j].frows[0]);
    w.queue = q(8);
    if (w.prefix[n] > 0) {
      stage(kStRefine, stream, [&] { launch_me_refine(djobs, w, stream); });
      launched++;
    }
    if (with_intra) {
      for (int j = 0; j < n; j++) w.prefix[j + 1] = w.prefix[j] + jobs[j].sb_cols * jobs[j].sb_rows;
      w.queue = q(5);
      stage(kStIntra, stream, [&] { launch_intra(djobs, w, stream); });
      launched++;
    }
    for (int j = 0; j < n; j++) w.prefix[j + 1] = w.prefix[j] + jobs[j].nrefs * jobs[j].sb_cols * jobs[j].sb_rows;
    w.queue = q(6);
    if (w.prefix[n] > 0) {
      bool any_keep = false;
      for (const FrameJob& jb : jobs) any_keep |= jb.keep != nullptr;
      stage(kStInter, stream, [&] { launch_inter(djobs, w, inter_chunk, any_keep, q(9), stream); });
      launched++;
    }
    for (int j = 0; j < n; j++) w.prefix[j + 1] = w.prefix[j] + jobs[j].sb_cols * jobs[j].sb_rows;
    w.queue = q(7);
    stage(kStFinalize, stream, [&] { launch_finalize(djobs, w, stream); });
    launched++;
    CK(cudaGetLastError());
    return launched;
  }

  // The pruner's features per job, then per job one kernel running the network on each
  // superblock and writing its mask; returns the kernels launched.
  int enqueue_pruner(const std::vector<FrameJob>& jobs, const std::vector<NetJob>& nets, cudaStream_t stream) {
    const int n = std::min((int)jobs.size(), (int)nets.size());
    int launched = 0;
    for (int j = 0; j < n; j++) {
      const NetJob& nj = nets[j];
      if (!nj.feats) continue;
      const int nsb = jobs[j].sb_cols * jobs[j].sb_rows;
      launch_features(djobs + j, nsb, nj.feats, stream);
      launched++;
      if (nj.net) {
        launch_infer(nj.params, nj.wb, nj.feats, nsb, jobs[j].nrefs, nj.th, nj.keep, stream);
        launched++;
      }
    }
    return launched;
  }

  // The stage kernels of the jobs, their descriptors sent through the pinned ring.
  void run_stages(const std::vector<FrameJob>& jobs, bool with_intra, cudaStream_t stream,
                  const std::vector<NetJob>& nets = {}) {
    put_jobs(jobs.data(), (int)jobs.size(), djobs, stream);
    kernel_launches += enqueue_stages(jobs, with_intra, stream, nets);
  }

  void wait_idle() {
    CK(cudaStreamSynchronize(up_st));
    CK(cudaStreamSynchronize(st));
    CK(cudaStreamSynchronize(copy_st));
    pending = false;
    if (!timed.empty()) {
      CK(cudaStreamSynchronize(prep_st));
      harvest();
    }
  }

  void launch(const celv2_frame* src, const celv2_frame* refs, int nrefs, long long lam, const long long* keys,
              long long src_key) {
    celv2_sb_out* dest = take_outputs()[0];  // this launch's, even when it fails
    if (!dest) dest = host_out;
    const std::vector<uint32_t> keep0 = std::move(take_keeps()[0]);
    check_frame(src, "source");
    if (nrefs < 0 || nrefs > kMaxRefs) invalid("CudaEngine: too many references");
    for (int r = 0; r < nrefs; r++) check_frame(&refs[r], "reference");
    if (nrefs > 0 && (g.pw < 16 || g.ph < 16)) invalid("CudaEngine: inter frames need at least 9x9 pixels");
    if (pending) wait_idle();
    try {
      // the prepared source, else an upload into the other slot
      int use = -1;
      for (int i = 0; i < 2; i++)
        if (src_key >= 0 && srcs[i].key == src_key) use = i;
      const bool prepared = use >= 0;
      if (prepared) {
        CK(cudaStreamWaitEvent(st, prep_done, 0));
      } else {
        use = 1 - cur_src;
        CK(cudaStreamSynchronize(prep_st));  // a prepare() into this slot may still run
        upload(src, srcs[use], false, st);
      }
      srcs[use].key = -1;  // used: a later prepare() may overwrite it
      cur_src = use;
      const long long now = ++launches;
      Slot* used[kMaxRefs];
      for (int r = 0; r < nrefs; r++) {
        bool fresh;
        Slot* s = ref_slot(keys ? keys[r] : -1, keys, keys ? nrefs : 0, now, fresh);
        if (fresh) {
          wait_ready(*s, st);  // a dropped store frame's upload may still run
          upload(&refs[r], *s, true, st);
          s->key = keys ? keys[r] : -1;
        } else {
          wait_ready(*s, st);  // a frame of the store
          make_phases(*s, st);
        }
        s->used = now;
        used[r] = s;
      }
      std::vector<FrameJob> jobs(1);
      fill_job(jobs[0], srcs[use].pyr, used, nrefs, single, intra_prep[use], lam);
      jobs[0].keep = put_keep(keep0, single, st);
      const std::vector<NetJob> nets{net_for(jobs[0], single, !keep0.empty())};
      if (nets[0].net) jobs[0].keep = single.keep;
      run_stages(jobs, !prepared, st, nets);
      mark_used(used, nrefs, st);
      last_nrefs = nrefs;
      // rows back to the host in row-stream order
      const int streams = std::max(1, std::min(row_streams, g.sb_rows));
      const int run = (g.sb_rows + streams - 1) / streams;
      order.clear();
      for (int i = 0; i < run; i++)
        for (int s = 0; s < streams; s++)
          if (s * run + i < g.sb_rows) order.push_back(s * run + i);
      for (int r : order) {
        const size_t first = (size_t)r * g.sb_cols;
        CK(cudaMemcpyAsync(dest + first, single.out + first, g.sb_cols * sizeof(celv2_sb_out),
                           cudaMemcpyDeviceToHost, st));
        CK(cudaEventRecord(row_done[r], st));
      }
      last_out = dest;
      pending = true;
    } catch (...) {
      cudaStreamSynchronize(st);  // a failure leaves no work running
      cudaStreamSynchronize(prep_st);
      pending = false;
      throw;
    }
  }

  void prepare(const celv2_frame* next, long long key) {
    if (key < 0 || !next || next->width != g.width || next->height != g.height) return;
    check_frame(next, "next frame");
    Slot& s = srcs[1 - cur_src];
    s.key = -1;
    // the slot's previous use (two launches back) was collected; the current launch uses the other
    upload(next, s, false, prep_st);
    std::vector<FrameJob> jobs(1);
    JobBuffers none{};
    fill_job(jobs[0], s.pyr, nullptr, 0, none, intra_prep[1 - cur_src], 0);
    // the intra stage alone, from a descriptor area of its own (the main stream owns djobs[0..])
    FrameJob* dprep = djobs + kRingJobs - 1;
    put_jobs(jobs.data(), 1, dprep, prep_st);
    WorkList w{};
    w.njobs = 1;
    w.prefix[1] = g.nsb;
    if (persistent) {
      CK(cudaMemsetAsync(queues + 15, 0, sizeof(unsigned), prep_st));
      w.queue = queues + 15;
    }
    stage(kStIntra, prep_st, [&] { launch_intra(dprep, w, prep_st); });
    kernel_launches++;
    CK(cudaGetLastError());
    CK(cudaEventRecord(prep_done, prep_st));
    s.key = key;
  }

  const celv2_sb_out* wait_row(int row) {
    if (row < 0 || row >= g.sb_rows) invalid("row out of range");
    if (!pending && launches == 0) throw Error(CELV2_ESTATE, "no launch to collect");
    CK(cudaEventSynchronize(row_done[row]));
    return last_out + (size_t)row * g.sb_cols;
  }

  // The caller memory named for the next launch's jobs (null: the engine's buffer); clears it.
  std::array<celv2_sb_out*, kMaxJobs> take_outputs() {
    std::array<celv2_sb_out*, kMaxJobs> o;
    for (int j = 0; j < kMaxJobs; j++) o[j] = next_out[j], next_out[j] = nullptr;
    return o;
  }

  // The device record buffer set (JobBuffers::records) of the next group, after `stream` waits for
  // the host copies that still read it (kRecordSets groups back).
  int take_parity(cudaStream_t stream) {
    const int par = group_parity;
    group_parity = (par + 1) % kRecordSets;
    if (copy_pending[par]) {
      CK(cudaStreamWaitEvent(stream, copied[par], 0));
      copy_pending[par] = false;
    }
    return par;
  }

  // ---- group path ----
  void reserve_group(int frames) {
    if (frames <= group_cap) return;
    wait_idle();
    free_graphs();  // they hold the old buffers' addresses
    group_jobs = 0;  // the last group's records go with the old host buffer
    for (JobBuffers& b : group) free_buffers(b);
    cudaFree(group_feats);
    group_feats = nullptr;
    group.assign(frames, JobBuffers{});
    for (JobBuffers& b : group) alloc_buffers(b, true);
    const size_t per = (size_t)g.nsb * CELV2_PRUNER_FEATURES;
    CK(cudaMalloc(&group_feats, per * frames * sizeof(float)));
    for (int j = 0; j < frames; j++) group[j].feats = group_feats + per * j;
    if (group_host) CK(cudaFreeHost(group_host));
    CK(cudaMallocHost(&group_host, (size_t)frames * g.nsb * sizeof(celv2_sb_out)));
    group_cap = frames;
  }

  Slot* find(long long key) {
    for (Slot* s : store)
      if (key >= 0 && s->key == key) return s;
    return nullptr;
  }

  void upload_store(const celv2_frame* f, long long key, bool direct = false) {
    check_frame(f, "frame");
    if (key < 0) invalid("store keys must be >= 0");
    // No wait for queued work: it runs on this stream, ahead of the upload.
    Slot* s = find(key);
    if (!s) {
      // a dropped store frame's memory (it has the events): the least recently read one whose
      // readers have all finished; with none finished, a new slot while the store holds fewer
      // than kStoreSlotsIdle, else the least recently read one (the upload then waits for it)
      Slot* lru = nullptr;
      for (Slot* x : store) {
        if (x->key >= 0 || x->resident || !x->last_use) continue;
        if (!lru || x->used < lru->used) lru = x;
        if ((!s || x->used < s->used) && (!x->use_pending || cudaEventQuery(x->last_use) == cudaSuccess)) s = x;
      }
      if (!s && (int)store.size() >= kStoreSlotsIdle) s = lru;
    }
    if (!s) {
      s = new Slot;
      store.push_back(s);
    }
    if (!s->ready) {
      CK(cudaEventCreateWithFlags(&s->ready, cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&s->last_use, cudaEventDisableTiming));
    }
    s->key = -1;
    // on the upload stream, after the queued work that reads the slot's old contents; the phase
    // planes are made by the first launch that uses the frame as a reference
    if (s->use_pending) CK(cudaStreamWaitEvent(up_st, s->last_use, 0));
    s->use_pending = false;
    upload(f, *s, false, up_st, true, direct);
    CK(cudaEventRecord(s->ready, up_st));
    s->ready_pending = true;
    s->key = key;
    s->used = launches;
    s->resident = true;
  }

  // `stream` waits for s's store upload, if one is in flight.
  void wait_ready(Slot& s, cudaStream_t stream) {
    if (s.ready_pending) CK(cudaStreamWaitEvent(stream, s.ready, 0));
  }

  // The slots a launch on `stream` reads: a later upload into them waits for this point. Their
  // recency (`used`) becomes this launch's, so an upload into a dropped slot takes the one whose
  // last reader was queued longest ago -- the one least likely to make the upload stream wait for
  // work still in flight (the slots of the batch just queued are the most recent).
  void mark_used(Slot* const* slots, int n, cudaStream_t stream) {
    for (int i = 0; i < n; i++) {
      Slot* x = slots[i];
      if (!x->last_use) continue;  // not a store slot (launch()'s own cache, on this stream)
      CK(cudaEventRecord(x->last_use, stream));
      x->use_pending = true;
      x->used = launches;
    }
  }

  void launch_group(int njobs, const long long* src_keys, const int* nrefs, const long long* const* ref_keys,
                    const int64_t* lams, bool to_host) {
    const std::array<celv2_sb_out*, kMaxJobs> dests = take_outputs();
    const std::array<std::vector<uint32_t>, kMaxJobs> keeps = take_keeps();
    if (njobs <= 0 || njobs > kMaxJobs - 1) invalid("1..31 jobs per group");
    if (!to_host)
      for (int j = 0; j < njobs; j++)
        if (dests[j]) invalid("group: set_output names host memory, but to_host 0 leaves the records on the device");
    if (njobs > group_cap) reserve_group(std::max(njobs, 8));
    std::vector<FrameJob> jobs(njobs);
    std::vector<Slot*> reads;
    for (int j = 0; j < njobs; j++) {
      Slot* cur = find(src_keys[j]);
      if (!cur) invalid("group: no stored frame with the source key");
      if (nrefs[j] < 0 || nrefs[j] > kMaxRefs) invalid("group: too many references");
      if (nrefs[j] > 0 && !ref_keys) invalid("group: null reference keys");
      if (nrefs[j] > 0 && (g.pw < 16 || g.ph < 16)) invalid("group: inter frames need at least 9x9 pixels");
      Slot* refs[kMaxRefs];
      for (int r = 0; r < nrefs[j]; r++) {
        refs[r] = find(ref_keys[j][r]);
        if (!refs[r]) invalid("group: no stored frame with a reference key");
      }
      wait_ready(*cur, st);
      reads.push_back(cur);
      for (int r = 0; r < nrefs[j]; r++) {
        wait_ready(*refs[r], st);
        make_phases(*refs[r], st);
        reads.push_back(refs[r]);
      }
      fill_job(jobs[j], cur->pyr, refs, nrefs[j], group[j], group[j].intra, lams[j]);
    }
    std::vector<NetJob> nets(njobs);
    for (int j = 0; j < njobs; j++) {
      jobs[j].keep = put_keep(keeps[j], group[j], st);
      nets[j] = net_for(jobs[j], group[j], !keeps[j].empty());
      if (nets[j].net) jobs[j].keep = group[j].keep;
    }
    const int par = take_parity(st);
    for (int j = 0; j < njobs; j++) jobs[j].out = group[j].records(par);
    if (use_graphs && !timing)
      launch_graph(jobs, nets);
    else
      run_stages(jobs, true, st, nets);
    mark_used(reads.data(), (int)reads.size(), st);
    if (to_host) {
      CK(cudaEventRecord(stages_done, st));
      CK(cudaStreamWaitEvent(copy_st, stages_done, 0));
      for (int j = 0; j < njobs; j++) {
        group_out[j] = dests[j] ? dests[j] : group_host + (size_t)j * g.nsb;
        CK(cudaMemcpyAsync(group_out[j], jobs[j].out, g.nsb * sizeof(celv2_sb_out), cudaMemcpyDeviceToHost, copy_st));
      }
      CK(cudaEventRecord(copied[par], copy_st));
      copy_pending[par] = true;
    } else {
      for (int j = 0; j < njobs; j++) group_out[j] = nullptr;  // records left on the device
    }
    group_jobs = njobs;
    ++launches;
    launches_group = launches;
    pending = true;
  }

  // ---- CUDA graphs: a batch's whole stage sequence captured once per shape, then replayed ----
  // The descriptors are not part of the graph: each replay is preceded by their copy into djobs
  // through the pinned ring (stream order puts it after the previous batch's kernels), so a replay
  // never waits on the host for an earlier replay of the same graph.
  struct Graph {
    std::vector<int> key;  // each job's reference count
    cudaGraphExec_t exec = nullptr;
    int kernels = 0;
  };
  bool use_graphs = false;
  std::vector<Graph> graphs;

  void free_graphs() {
    for (Graph& gr : graphs)
      if (gr.exec) cudaGraphExecDestroy(gr.exec);
    graphs.clear();
  }

  void launch_graph(const std::vector<FrameJob>& jobs, const std::vector<NetJob>& nets) {
    // the shape: per job its reference count, whether it has keep words (which decides whether the
    // region pass of the inter stage is launched at all), features and the network
    std::vector<int> key;
    for (size_t j = 0; j < jobs.size(); j++)
      key.push_back(jobs[j].nrefs * 8 + (jobs[j].keep ? 4 : 0) + (nets[j].feats ? 2 : 0) + (nets[j].net ? 1 : 0));
    Graph* gr = nullptr;
    for (Graph& x : graphs)
      if (x.key == key) gr = &x;
    const int n = (int)jobs.size();
    if (!gr) {
      graphs.emplace_back();
      gr = &graphs.back();
      gr->key = key;
      cudaGraph_t graph = nullptr;
      CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      try {
        gr->kernels = enqueue_stages(jobs, true, st, nets);
      } catch (...) {
        cudaStreamEndCapture(st, &graph);
        if (graph) cudaGraphDestroy(graph);
        graphs.pop_back();
        throw;
      }
      CK(cudaStreamEndCapture(st, &graph));
      const cudaError_t e = cudaGraphInstantiate(&gr->exec, graph, 0);
      cudaGraphDestroy(graph);
      CK(e);
    }
    put_jobs(jobs.data(), n, djobs, st);
    CK(cudaGraphLaunch(gr->exec, st));
    kernel_launches += gr->kernels;
  }
};

namespace {

// Jobs of several engines (each its own resolution and frame store) in one launch per stage, on
// the first engine's stream. Engine e's jobs take its group slots in order of appearance.
void launch_multi(int njobs, celv2_engine* const* engines, const long long* src_keys, const int* nrefs,
                  const long long* const* ref_keys, const int64_t* lams, bool to_host) {
  celv2_engine* lead = engines[0];
  std::vector<celv2_engine*> uniq;
  for (int j = 0; j < std::min(njobs, kMaxJobs); j++)
    if (engines[j] && std::find(uniq.begin(), uniq.end(), engines[j]) == uniq.end()) uniq.push_back(engines[j]);
  // the caller memory named for this launch, which takes it even when it fails
  std::vector<std::array<celv2_sb_out*, kMaxJobs>> dests;
  std::vector<std::array<std::vector<uint32_t>, kMaxJobs>> keeps;
  for (celv2_engine* e : uniq) dests.push_back(e->take_outputs()), keeps.push_back(e->take_keeps());
  if (njobs <= 0 || njobs > kMaxJobs - 1) invalid("1..31 jobs per batch");
  for (int j = 0; j < njobs; j++) {
    if (!engines[j]) invalid("null engine");
    if (engines[j]->device != lead->device) invalid("a batch runs on one GPU");
  }
  if (!to_host)
    for (const auto& d : dests)
      for (celv2_sb_out* p : d)
        if (p) invalid("batch: set_output names host memory, but to_host 0 leaves the records on the device");
  // Every key and reference is checked before any state changes (record buffer parities, waits,
  // phase planes), so a rejected batch leaves every engine as it was.
  std::vector<Slot*> cur_of(njobs);
  std::vector<std::array<Slot*, kMaxRefs>> refs_of(njobs);
  for (int j = 0; j < njobs; j++) {
    celv2_engine* e = engines[j];
    cur_of[j] = e->find(src_keys[j]);
    if (!cur_of[j]) invalid("batch: no stored frame with the source key");
    if (nrefs[j] < 0 || nrefs[j] > kMaxRefs) invalid("batch: too many references");
    if (nrefs[j] > 0 && !ref_keys) invalid("batch: null reference keys");
    if (nrefs[j] > 0 && (e->g.pw < 16 || e->g.ph < 16)) invalid("batch: inter frames need at least 9x9 pixels");
    for (int r = 0; r < nrefs[j]; r++) {
      refs_of[j][r] = e->find(ref_keys[j][r]);
      if (!refs_of[j][r]) invalid("batch: no stored frame with a reference key");
    }
  }
  for (celv2_engine* e : uniq) {
    int count = 0;
    for (int j = 0; j < njobs; j++) count += engines[j] == e;
    if (count > e->group_cap) e->reserve_group(std::max(count, 8));
  }
  // the other engines' queued work first: the lead stream waits for each of their streams
  for (celv2_engine* e : uniq)
    if (e != lead) {
      cudaEvent_t ev;
      CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      CK(cudaEventRecord(ev, e->st));
      CK(cudaStreamWaitEvent(lead->st, ev, 0));
      cudaEventDestroy(ev);
    }
  struct Entry {
    FrameJob job;
    NetJob net;
    celv2_engine* e;
    int slot;
    long long work;
    celv2_sb_out* dest;  // the caller's memory for the records, or null
  };
  std::vector<int> par;  // each engine's device record buffer set for this batch
  for (celv2_engine* e : uniq) par.push_back(e->take_parity(lead->st));
  std::vector<Entry> entries;
  std::vector<int> next(uniq.size(), 0);
  std::vector<std::vector<Slot*>> reads(uniq.size());  // each engine's store slots this batch reads
  for (int j = 0; j < njobs; j++) {
    celv2_engine* e = engines[j];
    const int ei = (int)(std::find(uniq.begin(), uniq.end(), e) - uniq.begin());
    const int slot = next[ei]++;
    Slot* cur = cur_of[j];
    Slot* const* refs = refs_of[j].data();
    e->wait_ready(*cur, lead->st);
    reads[ei].push_back(cur);
    for (int r = 0; r < nrefs[j]; r++) {
      e->wait_ready(*refs[r], lead->st);
      e->make_phases(*refs[r], lead->st);
      reads[ei].push_back(refs[r]);
    }
    Entry en;
    e->fill_job(en.job, cur->pyr, refs, nrefs[j], e->group[slot], e->group[slot].intra, lams[j]);
    en.job.keep = e->put_keep(keeps[ei][slot], e->group[slot], lead->st);
    en.net = e->net_for(en.job, e->group[slot], !keeps[ei][slot].empty());
    if (en.net.net) en.job.keep = e->group[slot].keep;
    en.job.out = e->group[slot].records(par[ei]);
    en.e = e, en.slot = slot, en.work = (long long)(nrefs[j] + 1) * e->g.nsb, en.dest = dests[ei][slot];
    entries.push_back(en);
  }
  // the largest jobs first, so the queues' last units are small ones
  std::stable_sort(entries.begin(), entries.end(), [](const Entry& a, const Entry& b) { return a.work > b.work; });
  std::vector<FrameJob> jobs;
  std::vector<NetJob> nets;
  for (const Entry& en : entries) jobs.push_back(en.job), nets.push_back(en.net);
  lead->run_stages(jobs, true, lead->st, nets);
  for (size_t i = 0; i < uniq.size(); i++) uniq[i]->mark_used(reads[i].data(), (int)reads[i].size(), lead->st);
  if (to_host) {  // on the lead's copy stream, overlapping later work
    CK(cudaEventRecord(lead->stages_done, lead->st));
    CK(cudaStreamWaitEvent(lead->copy_st, lead->stages_done, 0));
  }
  for (const Entry& en : entries) {
    if (!to_host) {
      en.e->group_out[en.slot] = nullptr;  // records left on the device
      continue;
    }
    celv2_sb_out* d = en.dest ? en.dest : en.e->group_host + (size_t)en.slot * en.e->g.nsb;
    en.e->group_out[en.slot] = d;
    CK(cudaMemcpyAsync(d, en.job.out, en.e->g.nsb * sizeof(celv2_sb_out), cudaMemcpyDeviceToHost, lead->copy_st));
  }
  if (to_host)
    for (size_t i = 0; i < uniq.size(); i++) {
      celv2_engine* e = uniq[i];
      CK(cudaEventRecord(e->copied[par[i]], lead->copy_st));
      e->copy_pending[par[i]] = true;
      if (e != lead) CK(cudaStreamWaitEvent(e->copy_st, e->copied[par[i]], 0));  // e's waits cover them
    }
  // every engine's later work waits for this batch
  cudaEvent_t done;
  CK(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
  CK(cudaEventRecord(done, lead->st));
  for (size_t i = 0; i < uniq.size(); i++) {
    celv2_engine* e = uniq[i];
    if (e != lead) CK(cudaStreamWaitEvent(e->st, done, 0));
    e->group_jobs = next[i];
    ++e->launches;
    e->launches_group = e->launches;
    e->pending = true;
  }
  cudaEventDestroy(done);
}

}  // namespace

extern "C" {

const char* celv2_last_error(void) { return g_error.c_str(); }

int celv2_launch_multi(int njobs, celv2_engine* const* engines, const long long* src_keys, const int* nrefs,
                       const long long* const* ref_keys, const int64_t* lambda_q8, int to_host) {
  return guarded([&] {
    if (!engines || !src_keys || !nrefs || !lambda_q8 || njobs <= 0 || !engines[0]) invalid("null argument");
    CK(cudaSetDevice(engines[0]->device));
    launch_multi(njobs, engines, src_keys, nrefs, ref_keys, lambda_q8, to_host != 0);
  });
}

int celv2_create(int width, int height, int sb_size, int device, celv2_engine** out) {
  if (out) *out = nullptr;
  return guarded([&] {
    if (!out) invalid("null output pointer");
    if (width <= 0 || height <= 0) invalid("CudaEngine: frame size must be positive");
    if (sb_size != 64) invalid("CudaEngine: only 64x64 superblocks are supported");
    int n = 0;
    CK(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) invalid("CudaEngine: no such CUDA device");
    auto* e = new celv2_engine;
    try {
      e->init(width, height, device);
    } catch (...) {
      delete e;
      throw;
    }
    *out = e;
  });
}

void celv2_destroy(celv2_engine* e) { delete e; }

int celv2_launch(celv2_engine* e, const celv2_frame* src, const celv2_frame* refs, int nrefs, int64_t lambda_q8,
                 const long long* ref_keys, long long src_key) {
  return guarded([&] {
    if (!e) invalid("null engine");
    if (nrefs > 0 && !refs) {
      e->take_outputs(), e->take_keeps();
      invalid("null references");
    }
    CK(cudaSetDevice(e->device));
    e->launch(src, refs, nrefs, lambda_q8, ref_keys, src_key);
  });
}

int celv2_prepare(celv2_engine* e, const celv2_frame* next, long long key) {
  return guarded([&] {
    if (!e) invalid("null engine");
    CK(cudaSetDevice(e->device));
    e->prepare(next, key);
  });
}

int celv2_set_row_streams(celv2_engine* e, int n) {
  return guarded([&] {
    if (!e) invalid("null engine");
    e->row_streams = n < 1 ? 1 : n;
  });
}

int celv2_geometry(const celv2_engine* e, int* sb_cols, int* sb_rows) {
  return guarded([&] {
    if (!e) invalid("null engine");
    if (sb_cols) *sb_cols = e->g.sb_cols;
    if (sb_rows) *sb_rows = e->g.sb_rows;
  });
}

int celv2_row_order(const celv2_engine* e, int* rows) {
  return guarded([&] {
    if (!e || !rows) invalid("null argument");
    if (e->order.empty()) throw Error(CELV2_ESTATE, "no launch yet");
    std::copy(e->order.begin(), e->order.end(), rows);
  });
}

int celv2_wait_row(celv2_engine* e, int row, const celv2_sb_out** records) {
  return guarded([&] {
    if (!e || !records) invalid("null argument");
    CK(cudaSetDevice(e->device));
    *records = e->wait_row(row);
  });
}

int celv2_finish(celv2_engine* e) {
  return guarded([&] {
    if (!e) invalid("null engine");
    CK(cudaSetDevice(e->device));
    e->wait_idle();
    CK(cudaStreamSynchronize(e->prep_st));
  });
}

int celv2_upload(celv2_engine* e, const celv2_frame* f, long long key) {
  return guarded([&] {
    if (!e) invalid("null engine");
    CK(cudaSetDevice(e->device));
    e->upload_store(f, key);
  });
}

int celv2_upload_pinned(celv2_engine* e, const celv2_frame* f, long long key) {
  return guarded([&] {
    if (!e) invalid("null engine");
    if (!f || (!f->y && !f->hy)) invalid("upload_pinned: no luma plane");
    CK(cudaSetDevice(e->device));
    cudaPointerAttributes a{};
    const void* plane = f->y ? (const void*)f->y : (const void*)f->hy;
    if (cudaPointerGetAttributes(&a, plane) != cudaSuccess || a.type != cudaMemoryTypeHost) {
      cudaGetLastError();
      invalid("upload_pinned: the plane must be page-locked host memory (celv2_host_alloc)");
    }
    e->upload_store(f, key, true);
  });
}

int celv2_launch_group(celv2_engine* e, int njobs, const long long* src_keys, const int* nrefs,
                       const long long* const* ref_keys, const int64_t* lambda_q8, int to_host) {
  return guarded([&] {
    if (!e) invalid("null engine");
    if (!src_keys || !nrefs || !lambda_q8) {
      e->take_outputs(), e->take_keeps();  // named for this launch, which fails
      invalid("null argument");
    }
    CK(cudaSetDevice(e->device));
    e->launch_group(njobs, src_keys, nrefs, ref_keys, lambda_q8, to_host != 0);
  });
}

int celv2_reserve_group(celv2_engine* e, int frames) {
  return guarded([&] {
    if (!e) invalid("null engine");
    if (frames < 1 || frames > kMaxJobs - 1) invalid("1..31 frames per group");
    CK(cudaSetDevice(e->device));
    e->reserve_group(frames);
  });
}

int celv2_group_records(celv2_engine* e, int job, const celv2_sb_out** records) {
  return guarded([&] {
    if (!e || !records) invalid("null argument");
    if (job < 0 || job >= e->group_jobs) invalid("no such job in the last group");
    if (!e->group_out[job])
      throw Error(CELV2_ESTATE, "group_records: the last group left its records on the device (to_host 0)");
    CK(cudaSetDevice(e->device));
    e->wait_idle();
    *records = e->group_out[job];
  });
}

int celv2_set_keep(celv2_engine* e, int job, const uint8_t* keep) {
  return guarded([&] {
    if (!e) invalid("null engine");
    if (job < 0 || job >= kMaxJobs - 1) invalid("set_keep: job out of range");
    if (keep)
      e->next_keep[job].assign(keep, keep + e->g.nsb);  // references and intra; every level and mode
    else
      e->next_keep[job].clear();
  });
}

int celv2_set_keep_words(celv2_engine* e, int job, const uint32_t* keep) {
  return guarded([&] {
    if (!e) invalid("null engine");
    if (job < 0 || job >= kMaxJobs - 1) invalid("set_keep_words: job out of range");
    if (keep)
      e->next_keep[job].assign(keep, keep + e->g.nsb);
    else
      e->next_keep[job].clear();
  });
}

int celv2_sb_costs(celv2_engine* e, int job, int64_t* out) {
  return guarded([&] {
    if (!e || !out) invalid("null argument");
    const bool group = e->group_jobs > 0 && e->launches_group == e->launches;
    if (job < 0 || (group ? job >= e->group_jobs : job != 0)) invalid("sb_costs: no such job in the last launch");
    CK(cudaSetDevice(e->device));
    e->wait_idle();
    const long long* src = group ? e->group[job].sb_cost : e->single.sb_cost;
    CK(cudaMemcpy(out, src, (size_t)e->g.nsb * sizeof(long long), cudaMemcpyDeviceToHost));
  });
}

int celv2_set_output(celv2_engine* e, int job, celv2_sb_out* records) {
  return guarded([&] {
    if (!e) invalid("null engine");
    if (job < 0 || job >= kMaxJobs - 1) invalid("set_output: job out of range");
    if (records) {
      cudaPointerAttributes a{};
      if (cudaPointerGetAttributes(&a, records) != cudaSuccess || a.type != cudaMemoryTypeHost) {
        cudaGetLastError();
        invalid("set_output: records must be page-locked host memory (celv2_host_alloc)");
      }
    }
    e->next_out[job] = records;
  });
}

int celv2_host_alloc(long long bytes, void** out) {
  return guarded([&] {
    if (!out || bytes <= 0) invalid("host_alloc: a positive size and an output pointer");
    *out = nullptr;
    CK(cudaHostAlloc(out, (size_t)bytes, cudaHostAllocPortable));
  });
}

int celv2_host_free(void* p) {
  return guarded([&] {
    if (p) CK(cudaFreeHost(p));
  });
}

int celv2_clear_store(celv2_engine* e) {
  return guarded([&] {
    if (!e) invalid("null engine");
    CK(cudaSetDevice(e->device));
    e->wait_idle();
    for (Slot* s : e->store) celv2_engine::free_slot(s);
    e->store.clear();
  });
}

int celv2_drop_frame(celv2_engine* e, long long key) {
  return guarded([&] {
    if (!e) invalid("null engine");
    if (Slot* s = e->find(key)) s->key = -1, s->resident = false;  // keeps its recency (`used`)
  });
}

int celv2_debug_field(celv2_engine* e, int r, int level, int32_t* out, int* cols, int* rows) {
  return guarded([&] {
    if (!e || !out) invalid("null argument");
    if (r < 0 || r >= kMaxRefs || level < 0 || level >= kLevels) invalid("bad reference or level");
    CK(cudaSetDevice(e->device));
    e->wait_idle();
    size_t off = r * e->g.field_ints;
    for (int l = 0; l < level; l++) off += (size_t)e->g.fcols[l] * e->g.frows[l];
    const size_t n = (size_t)e->g.fcols[level] * e->g.frows[level];
    CK(cudaMemcpy(out, e->single.fields + off, n * sizeof(int), cudaMemcpyDeviceToHost));
    if (cols) *cols = e->g.fcols[level];
    if (rows) *rows = e->g.frows[level];
  });
}

int celv2_debug_intra(celv2_engine* e, int32_t* out) {
  return guarded([&] {
    if (!e || !out) invalid("null argument");
    CK(cudaSetDevice(e->device));
    e->wait_idle();
    CK(cudaMemcpy(out, e->intra_prep[e->cur_src], (size_t)e->g.nsb * kBlocks * kModes * sizeof(int),
                  cudaMemcpyDeviceToHost));
  });
}

int celv2_debug_inter(celv2_engine* e, int32_t* out) {
  return guarded([&] {
    if (!e || !out) invalid("null argument");
    CK(cudaSetDevice(e->device));
    e->wait_idle();
    CK(cudaMemcpy(out, e->single.inter, (size_t)e->g.nsb * kMaxRefs * kBlocks * sizeof(int2), cudaMemcpyDeviceToHost));
  });
}

long long celv2_kernel_launches(const celv2_engine* e) { return e ? e->kernel_launches : 0; }

int celv2_set_pruner(celv2_engine* e, const float* params, float ref_threshold, float intra_threshold,
                     float level_threshold, float mode_threshold, float band) {
  return guarded([&] {
    if (!e) invalid("null engine");
    auto unit = [](float v) { return v >= 0.f && v <= 1.f; };
    if (params && !(unit(ref_threshold) && unit(intra_threshold) && unit(level_threshold) && unit(mode_threshold) &&
                    band >= 0.f))
      invalid("set_pruner: thresholds must lie in [0, 1] and the band be >= 0");
    CK(cudaSetDevice(e->device));
    e->wait_idle();
    e->free_graphs();  // captured batches hold the old settings
    if (!params) {
      cudaFree(e->pruner_params), cudaFree(e->nn_wb);
      e->pruner_params = nullptr, e->nn_wb = nullptr;
      return;
    }
    if (!e->pruner_params) {
      CK(cudaMalloc(&e->pruner_params, CELV2_PRUNER_PARAMS * sizeof(float)));
      CK(cudaMalloc(&e->nn_wb, infer_weight_elems() * 2));
    }
    // on the engine's stream, ahead of the kernel that reads them (a synchronous copy from pageable
    // memory may return before its DMA lands, and the engine's streams do not wait for it)
    CK(cudaMemcpyAsync(e->pruner_params, params, CELV2_PRUNER_PARAMS * sizeof(float), cudaMemcpyHostToDevice, e->st));
    infer_weights(e->pruner_params, e->nn_wb, e->st);
    CK(cudaStreamSynchronize(e->st));
    e->pruner_th = PrunerThresholds{ref_threshold, intra_threshold, level_threshold, mode_threshold, band};
  });
}

namespace {
// The buffers of job `job` of the last launch (a group's, or launch()'s own).
const JobBuffers& last_buffers(const celv2_engine* e, int job) {
  const bool group = e->group_jobs > 0 && e->launches_group == e->launches;
  if (job < 0 || (group ? job >= e->group_jobs : job != 0)) invalid("no such job in the last launch");
  return group ? e->group[job] : e->single;
}
}  // namespace

int celv2_features(celv2_engine* e, int job, float* out) {
  return guarded([&] {
    if (!e || !out) invalid("null argument");
    const JobBuffers& b = last_buffers(e, job);
    CK(cudaSetDevice(e->device));
    e->wait_idle();
    CK(cudaMemcpy(out, b.feats, (size_t)e->g.nsb * CELV2_PRUNER_FEATURES * sizeof(float), cudaMemcpyDeviceToHost));
  });
}

int celv2_pruner_masks(celv2_engine* e, int job, uint32_t* out) {
  return guarded([&] {
    if (!e || !out) invalid("null argument");
    const JobBuffers& b = last_buffers(e, job);
    CK(cudaSetDevice(e->device));
    e->wait_idle();
    CK(cudaMemcpy(out, b.keep, (size_t)e->g.nsb * sizeof(uint32_t), cudaMemcpyDeviceToHost));
  });
}

int celv2_set_config(celv2_engine* e, int key, int value) {
  return guarded([&] {
    if (!e) invalid("null engine");
    CK(cudaSetDevice(e->device));
    e->wait_idle();
    switch (key) {
      case CELV2_CFG_PERSISTENT: e->persistent = value != 0, e->free_graphs(); break;
      case CELV2_CFG_GRAPHS: e->use_graphs = value != 0; break;
      case CELV2_CFG_FEATURES: e->features_on = value != 0, e->free_graphs(); break;
      case CELV2_CFG_PERSISTENT_OFF: e->persistent_off = (unsigned)value & 0x1ff, e->free_graphs(); break;
      case CELV2_CFG_INTER_CHUNK:
        if (value < 8 || value > 64) invalid("inter chunk must be 8..64");
        e->inter_chunk = value, e->free_graphs();
        break;
      case CELV2_CFG_ME_CELLS_L0:
      case CELV2_CFG_ME_CELLS_L0 + 1:
      case CELV2_CFG_ME_CELLS_L0 + 2:
      case CELV2_CFG_ME_CELLS_L0 + 3:
      case CELV2_CFG_ME_CELLS_L0 + 4:
        if (value != 15 && value != 30) invalid("motion-search cells per CTA must be 15 or 30");
        e->me_cells[key - CELV2_CFG_ME_CELLS_L0] = value, e->free_graphs();
        break;
      default: invalid("unknown configuration key");
    }
  });
}

int celv2_get_config(const celv2_engine* e, int key, int* value) {
  return guarded([&] {
    if (!e || !value) invalid("null argument");
    switch (key) {
      case CELV2_CFG_PERSISTENT: *value = e->persistent; break;
      case CELV2_CFG_FEATURES: *value = e->features_on; break;
      case CELV2_CFG_GRAPHS: *value = e->use_graphs; break;
      case CELV2_CFG_PERSISTENT_OFF: *value = (int)e->persistent_off; break;
      case CELV2_CFG_INTER_CHUNK: *value = e->inter_chunk; break;
      case CELV2_CFG_ME_CELLS_L0:
      case CELV2_CFG_ME_CELLS_L0 + 1:
      case CELV2_CFG_ME_CELLS_L0 + 2:
      case CELV2_CFG_ME_CELLS_L0 + 3:
      case CELV2_CFG_ME_CELLS_L0 + 4: *value = e->me_cells[key - CELV2_CFG_ME_CELLS_L0]; break;
      default: invalid("unknown configuration key");
    }
  });
}

int celv2_stream(const celv2_engine* e, void** stream) {
  return guarded([&] {
    if (!e || !stream) invalid("null argument");
    *stream = e->st;
  });
}

int celv2_stage_timing(celv2_engine* e, int enable) {
  return guarded([&] {
    if (!e) invalid("null engine");
    CK(cudaSetDevice(e->device));
    e->wait_idle();
    e->timing = enable != 0;
    if (e->timing && !e->stats) {
      CK(cudaMalloc(&e->stats, kStats * sizeof(unsigned long long)));
      CK(cudaMemset(e->stats, 0, kStats * sizeof(unsigned long long)));
    }
  });
}

int celv2_work_counters(celv2_engine* e, unsigned long long* out, int n) {
  return guarded([&] {
    if (!e || !out) invalid("null argument");
    CK(cudaSetDevice(e->device));
    e->wait_idle();
    CK(cudaStreamSynchronize(e->prep_st));
    unsigned long long v[kStats] = {};
    if (e->stats) {
      CK(cudaMemcpy(v, e->stats, sizeof v, cudaMemcpyDeviceToHost));
      CK(cudaMemset(e->stats, 0, sizeof v));
    }
    for (int i = 0; i < n && i < kStats; i++) out[i] = v[i];
  });
}

int celv2_stage_times(celv2_engine* e, double* ms, long long* launches, int n) {
  return guarded([&] {
    if (!e || !ms || !launches) invalid("null argument");
    CK(cudaSetDevice(e->device));
    e->wait_idle();
    CK(cudaStreamSynchronize(e->prep_st));
    e->harvest();
    for (int i = 0; i < n && i < kStages; i++) ms[i] = e->stage_ms[i], launches[i] = e->stage_n[i];
    std::fill(e->stage_ms, e->stage_ms + kStages, 0.0);
    std::fill(e->stage_n, e->stage_n + kStages, 0LL);
  });
}

int celv2_int_peak(int device, double* ops_per_s) {
  return guarded([&] {
    if (!ops_per_s) invalid("null argument");
    CK(measure_int_peak(device, ops_per_s));
  });
}

}  // extern "C"
