// cuda_engine.h: the B200 decision engine as a DecisionEngine of the reference encoder.
//
// A drop-in third engine next to CpuEngine and VulkanEngine (src/gpu/decision_engine.h:9-51),
// selected as Device::Cuda / --device cuda in make_engine (src/pipeline.cpp:43-72). It forwards to the C ABI of
// include/celv2_cuda.h and converts the device records with the encoder's own
// celv2::sb_out_to_decision (src/gpu/decision_map.cpp:65-105), whose SbOut layout the records
// keep byte for byte. Compiled inside the reference tree: it includes "gpu/decision_engine.h".
#pragma once
#include <string>
#include <vector>

#include "gpu/decision_engine.h"

struct celv2_engine;

class CudaEngine : public DecisionEngine {
 public:
  // As VulkanEngine(width, height, sb_size, device) (src/vk/vk_engine.h:18): throws
  // std::runtime_error on a zero size, on sb_size != 64 and when no CUDA device can be used.
  CudaEngine(int width, int height, int sb_size, int device = 0);
  ~CudaEngine() override;
  CudaEngine(const CudaEngine&) = delete;
  CudaEngine& operator=(const CudaEngine&) = delete;

  using DecisionEngine::launch;
  void launch(const Frame420& src, const std::vector<const Frame420*>& refs, int qindex, DecisionMap& dm,
              const std::vector<long long>& ref_keys = {}, long long src_key = -1) override;
  void prepare(const Frame420& next, long long key) override;
  void collect(DecisionMap& dm, RowGate& gate) override;
  void set_row_streams(int n) override;
  const std::string& device_name() const { return name_; }

  // Several frames decided together, one kernel launch per stage for all of them: the leaves of a
  // mini-GOP, which Pipeline::code_group (src/pipeline.cpp:328-384) otherwise hands to launch()
  // one at a time. Frame i is srcs[i] against refs[i] (nearest first; keys[i] empty or one key per
  // reference, as launch()'s ref_keys, so a reference seen before is not uploaded again) at
  // qindex[i]; dms[i] is sized as launch() sizes it. The decisions equal separate launches'. The
  // inputs are copied before it returns. At most 31 frames; collect_group must follow.
  void launch_group(const std::vector<const Frame420*>& srcs, const std::vector<std::vector<const Frame420*>>& refs,
                    const std::vector<std::vector<long long>>& keys, const std::vector<int>& qindex,
                    std::vector<DecisionMap>& dms);
  // Fills every dms[i] and publishes all of its rows on *gates[i], frame by frame; on failure
  // fails every gate and rethrows. Returns with no work pending.
  void collect_group(std::vector<DecisionMap>& dms, const std::vector<RowGate*>& gates);

 private:
  celv2_engine* e_ = nullptr;
  int width_, height_, sb_cols_ = 0, sb_rows_ = 0;
  std::string name_;
  // launch_group's frame store: keyed references it uploaded, and a counter for the store keys of
  // sources and unkeyed references (above the caller's key range)
  std::vector<long long> keyed_;
  long long next_key_ = 0;
  int group_jobs_ = 0;
};
