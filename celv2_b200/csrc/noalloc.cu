// noalloc.cu: a KEY-frame (intra-only) decision that allocates no device memory.
//
// Who needs it: callers that cannot allocate GPU memory while they run. An encoder embedded in a
// host application that provisions all device memory up front through its own allocator (and
// forbids runtime cudaMalloc), or a latency-critical path that cannot take the implicit device
// synchronisation cudaMalloc / cudaFree may bring. They pass their own device buffers for the
// input plane and the output records; everything else this call needs lives in one file-scope
// static __device__ array of fixed size.
//
// What it runs: the intra SATD kernel, whose output (the per-block, per-mode SATDs) is scratch
// that the finalize kernel reads to make the decision records -- the same kernels and records as
// celv2_launch with no references. The kernels' job descriptor sits in the same array.
//
// Limits and behaviour:
//  - frames of at most CELV2_NOALLOC_MAX_SUPERBLOCKS (768) 64x64 superblocks; larger ones are
//    rejected with CELV2_EINVAL (1920x1080 has 510);
//  - every GPU that loads the library holds the array (about 17 MB) until the process exits;
//  - the first call on a device, with that device current, looks up the array's device address
//    (cudaGetSymbolAddress) and sets the kernels' shared-memory attributes, once per device; make
//    that first call before any stream capture;
//  - every call shares the array and it keeps the last call's contents. Each call rewrites all of
//    the scratch it reads (every SATD entry of every superblock it decides, and the descriptor),
//    so nothing has to start at zero; but calls whose GPU work overlaps (on different streams, or
//    from threads that do not order their calls) race on the array;
//  - the job descriptor reaches the array as a kernel parameter (k_put_job), so no host memory is
//    read after the call returns.
#include <cuda_runtime.h>

#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "celv2_cuda.h"
#include "kernels.h"

namespace celv2cu {
cudaError_t intra_attributes();
cudaError_t finalize_attributes();
void set_last_error(const std::string& msg);
}  // namespace celv2cu

using namespace celv2cu;

namespace {

constexpr int kMaxSb = CELV2_NOALLOC_MAX_SUPERBLOCKS;
constexpr int kMaxSide = 1 << 16;  // width, height and pitch bound (samples)
// The descriptor first (rounded up to 256 bytes), then the intra SATDs of kMaxSb superblocks.
constexpr size_t kJobInts = (sizeof(FrameJob) + 255) / 256 * 64;
constexpr size_t kScratchInts = kJobInts + (size_t)kMaxSb * kBlocks * kModes;

static __device__ __align__(256) int g_noalloc_scratch[kScratchInts];

std::mutex g_mu;
std::vector<int*> g_scratch_addr;  // per device: the array's device address, once looked up

// The device address of the array on the current device `dev` (set up on the first call).
// Writes the job descriptor into the scratch array. The descriptor travels as a kernel parameter,
// which the launch copies, so nothing on the host is read once the call has returned.
__global__ void k_put_job(FrameJob job, FrameJob* dst) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *dst = job;
}

int* scratch_on(int dev) {
  std::lock_guard<std::mutex> lk(g_mu);
  if ((int)g_scratch_addr.size() <= dev) g_scratch_addr.resize(dev + 1, nullptr);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) throw std::runtime_error(std::string("scratch address: ") + cudaGetErrorString(e));
    if ((e = intra_attributes()) != cudaSuccess || (e = finalize_attributes()) != cudaSuccess)
      throw std::runtime_error(std::string("kernel attributes: ") + cudaGetErrorString(e));
    g_scratch_addr[dev] = static_cast<int*>(p);
  }
  return g_scratch_addr[dev];
}

}  // namespace

extern "C" int celv2_decide_key_noalloc(const uint8_t* luma, int width, int height, int pitch, int64_t lambda_q8,
                                        celv2_sb_out* out, void* stream) {
  if (!luma || !out) {
    set_last_error("decide_key_noalloc: null plane or output");
    return CELV2_EINVAL;
  }
  if (width <= 0 || height <= 0) {
    set_last_error("decide_key_noalloc: frame size must be positive");
    return CELV2_EINVAL;
  }
  // bounded before any arithmetic on the sizes (no int overflow); the superblock limit below is
  // far tighter for any real frame
  if (width > kMaxSide || height > kMaxSide || pitch > kMaxSide) {
    set_last_error("decide_key_noalloc: width, height and pitch must be at most " + std::to_string(kMaxSide) +
                   " (and the frame within " + std::to_string(kMaxSb) + " superblocks)");
    return CELV2_EINVAL;
  }
  const int pw = (width + 7) & ~7, ph = (height + 7) & ~7;
  const int sb_cols = (width + 63) / 64, sb_rows = (height + 63) / 64;
  if (pitch < pw) {
    set_last_error("decide_key_noalloc: pitch below the padded width");
    return CELV2_EINVAL;
  }
  if (sb_cols * sb_rows > kMaxSb) {
    set_last_error("decide_key_noalloc: " + std::to_string(sb_cols * sb_rows) +
                   " superblocks exceed this entry point's fixed scratch of " + std::to_string(kMaxSb) +
                   " (use celv2_launch)");
    return CELV2_EINVAL;
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_last_error(std::string("decide_key_noalloc: ") + cudaGetErrorString(e));
    return CELV2_ECUDA;
  }
  int* scratch;
  try {
    scratch = scratch_on(dev);
  } catch (const std::exception& ex) {
    set_last_error(std::string("decide_key_noalloc: ") + ex.what());
    return CELV2_ECUDA;
  }
  FrameJob job{};
  // The caller's padded plane as a plane without margin: reads clamp into [0, ph) x [0, pw),
  // exactly the reference's Plane::at.
  job.cur.lv[0] = DevPlane{luma, pitch, pw, ph, 0, 0};
  job.nrefs = 0;
  job.pw = pw, job.ph = ph, job.sb_cols = sb_cols, job.sb_rows = sb_rows;
  job.intra = scratch + kJobInts;
  job.inter = nullptr;
  job.out = out;
  job.lam = lambda_q8;
  job.stats = nullptr;
  FrameJob* djob = reinterpret_cast<FrameJob*>(scratch);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_put_job<<<1, 32, 0, st>>>(job, djob);
  e = cudaGetLastError();
  if (e == cudaSuccess) {
    WorkList w{};
    w.njobs = 1;
    w.prefix[1] = sb_cols * sb_rows;
    launch_intra(djob, w, st);
    launch_finalize(djob, w, st);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    set_last_error(std::string("decide_key_noalloc: ") + cudaGetErrorString(e));
    return CELV2_ECUDA;
  }
  return CELV2_OK;
}
