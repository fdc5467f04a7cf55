// cuda_engine.cpp: DecisionEngine over the CUDA engine's C ABI (see cuda_engine.h).
#include "cuda_engine.h"

#include <cstddef>
#include <stdexcept>
#include <vector>

#include "celv2_cuda.h"
#include "gpu/decision_map.h"
#include "gpu/kernels_ref.h"  // lambda_q8 (src/core/quant.cpp:31-39)
#include "gpu/sb_out.h"

// The records are the encoder's SbOut, field for field.
static_assert(sizeof(celv2_sb_out) == sizeof(celv2::SbOut), "record size");
static_assert(offsetof(celv2_sb_out, c_inter_cost) == offsetof(celv2::SbOut, c_inter_cost), "record layout");
static_assert(offsetof(celv2_sb_out, c_rcost) == offsetof(celv2::SbOut, c_rcost), "record layout");
static_assert(offsetof(celv2_sb_out, c_rmvy) == offsetof(celv2::SbOut, c_rmvy), "record layout");

namespace {

void check(int rc) {
  if (rc == CELV2_OK) return;
  throw std::runtime_error(std::string("CudaEngine: ") + celv2_last_error());
}

celv2_frame view(const Frame420& f) {
  celv2_frame v{};
  v.width = f.width, v.height = f.height, v.pitch = f.stride_y();
  v.y = f.y.data();  // the decisions score Frame420::y, the 8-bit rounding (src/io/y4m.h:14-18)
  return v;
}

}  // namespace

CudaEngine::CudaEngine(int width, int height, int sb_size, int device) : width_(width), height_(height) {
  check(celv2_create(width, height, sb_size, device, &e_));
  check(celv2_geometry(e_, &sb_cols_, &sb_rows_));
  name_ = "CUDA device " + std::to_string(device);
}

CudaEngine::~CudaEngine() { celv2_destroy(e_); }

void CudaEngine::set_row_streams(int n) { check(celv2_set_row_streams(e_, n)); }

void CudaEngine::launch(const Frame420& src, const std::vector<const Frame420*>& refs, int qindex, DecisionMap& dm,
                        const std::vector<long long>& ref_keys, long long src_key) {
  if (!ref_keys.empty() && ref_keys.size() != refs.size())
    throw std::invalid_argument("CudaEngine: one key per reference");
  const celv2_frame s = view(src);
  std::vector<celv2_frame> r;
  for (const Frame420* f : refs) r.push_back(view(*f));
  check(celv2_launch(e_, &s, r.data(), static_cast<int>(r.size()), lambda_q8(qindex),
                     ref_keys.empty() ? nullptr : ref_keys.data(), src_key));
  dm.sb_size = 64;
  dm.sb_cols = sb_cols_;
  dm.sb_rows = sb_rows_;
  dm.sbs.assign(static_cast<size_t>(sb_cols_) * sb_rows_, SbDecision{});
}

void CudaEngine::prepare(const Frame420& next, long long key) {
  const celv2_frame n = view(next);
  check(celv2_prepare(e_, &n, key));
}

void CudaEngine::collect(DecisionMap& dm, RowGate& gate) {
  try {
    std::vector<int> order(sb_rows_);
    check(celv2_row_order(e_, order.data()));
    for (int r : order) {
      const celv2_sb_out* rec = nullptr;
      check(celv2_wait_row(e_, r, &rec));
      const size_t first = static_cast<size_t>(r) * sb_cols_;
      for (int c = 0; c < sb_cols_; c++)
        celv2::sb_out_to_decision(*reinterpret_cast<const celv2::SbOut*>(rec + c), dm.sbs[first + c]);
      gate.publish_one(r);
    }
    check(celv2_finish(e_));
  } catch (...) {
    gate.fail(std::current_exception());
    celv2_finish(e_);
    throw;
  }
}
