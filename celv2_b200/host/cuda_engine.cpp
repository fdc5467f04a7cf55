// cuda_engine.cpp: DecisionEngine over the CUDA engine's C ABI (see cuda_engine.h).
#include "cuda_engine.h"

#include <algorithm>
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

void CudaEngine::launch_group(const std::vector<const Frame420*>& srcs,
                              const std::vector<std::vector<const Frame420*>>& refs,
                              const std::vector<std::vector<long long>>& keys, const std::vector<int>& qindex,
                              std::vector<DecisionMap>& dms) {
  const size_t n = srcs.size();
  if (n == 0 || n > 31 || refs.size() != n || qindex.size() != n || (!keys.empty() && keys.size() != n))
    throw std::invalid_argument("CudaEngine::launch_group: 1..31 frames, one reference list and qindex each");
  constexpr long long kOwn = 1LL << 61;  // store keys of sources and unkeyed references
  std::vector<long long> need, temp, src_keys(n);
  std::vector<std::vector<long long>> ref_keys(n);
  for (size_t i = 0; i < n; i++) {
    if (!keys.empty() && !keys[i].empty() && keys[i].size() != refs[i].size())
      throw std::invalid_argument("CudaEngine: one key per reference");
    if (refs[i].size() > 7) throw std::runtime_error("CudaEngine: too many references");
    for (size_t r = 0; r < refs[i].size(); r++) {
      const celv2_frame f = view(*refs[i][r]);
      long long k;
      if (keys.empty() || keys[i].empty()) {
        k = kOwn + next_key_++;
        check(celv2_upload(e_, &f, k));
        temp.push_back(k);
      } else {
        k = keys[i][r];
        if (k < 0 || k >= kOwn) throw std::invalid_argument("CudaEngine: reference keys must be in [0, 2^61)");
        if (std::find(keyed_.begin(), keyed_.end(), k) == keyed_.end()) {
          check(celv2_upload(e_, &f, k));
          keyed_.push_back(k);
        }
      }
      need.push_back(k);
      ref_keys[i].push_back(k);
    }
    const celv2_frame s = view(*srcs[i]);
    src_keys[i] = kOwn + next_key_++;
    check(celv2_upload(e_, &s, src_keys[i]));
    temp.push_back(src_keys[i]);
  }
  // keyed references this group does not use leave the store
  for (auto it = keyed_.begin(); it != keyed_.end();)
    if (std::find(need.begin(), need.end(), *it) == need.end()) {
      check(celv2_drop_frame(e_, *it));
      it = keyed_.erase(it);
    } else {
      ++it;
    }
  std::vector<int> nrefs(n);
  std::vector<const long long*> rk(n);
  std::vector<int64_t> lams(n);
  for (size_t i = 0; i < n; i++)
    nrefs[i] = static_cast<int>(ref_keys[i].size()), rk[i] = ref_keys[i].data(), lams[i] = lambda_q8(qindex[i]);
  check(celv2_launch_group(e_, static_cast<int>(n), src_keys.data(), nrefs.data(), rk.data(), lams.data(), 1));
  group_jobs_ = static_cast<int>(n);
  for (long long k : temp) check(celv2_drop_frame(e_, k));  // the queued work still reads them
  dms.resize(n);
  for (DecisionMap& dm : dms) {
    dm.sb_size = 64;
    dm.sb_cols = sb_cols_;
    dm.sb_rows = sb_rows_;
    dm.sbs.assign(static_cast<size_t>(sb_cols_) * sb_rows_, SbDecision{});
  }
}

void CudaEngine::collect_group(std::vector<DecisionMap>& dms, const std::vector<RowGate*>& gates) {
  try {
    if (static_cast<int>(dms.size()) != group_jobs_ || gates.size() != dms.size())
      throw std::invalid_argument("CudaEngine::collect_group: one map and gate per launched frame");
    for (int j = 0; j < group_jobs_; j++) {
      const celv2_sb_out* rec = nullptr;
      check(celv2_group_records(e_, j, &rec));
      for (size_t i = 0; i < dms[j].sbs.size(); i++)
        celv2::sb_out_to_decision(*reinterpret_cast<const celv2::SbOut*>(rec + i), dms[j].sbs[i]);
      for (int r = 0; r < sb_rows_; r++) gates[j]->publish_one(r);
    }
    group_jobs_ = 0;
  } catch (...) {
    for (RowGate* g : gates)
      if (g) g->fail(std::current_exception());
    celv2_finish(e_);
    group_jobs_ = 0;
    throw;
  }
}
