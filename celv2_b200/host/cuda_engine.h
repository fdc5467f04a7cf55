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

 private:
  celv2_engine* e_ = nullptr;
  int width_, height_, sb_cols_ = 0, sb_rows_ = 0;
  std::string name_;
};
