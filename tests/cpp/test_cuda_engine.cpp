// The CUDA engine behind the reference's own DecisionEngine interface, against the reference's
// CpuEngine and decide_*_ref rules: the engine tests of the reference (tests/test_gpu_intra.cpp,
// tests/test_gpu_me.cpp) with CudaEngine in the place of VulkanEngine. Built by oracle/Makefile
// (target adapter-test) from the reference's sources and test headers where they lie; run by
// tests/test_gpu_adapter.py on a machine with a B200. Exit status 0 when every case passes.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <exception>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "check.h"
#include "cuda_engine.h"
#include "gpu/cpu_engine.h"
#include "gpu/kernels_ref.h"
#include "io/y4m.h"
#include "test_frames.h"

// lambda_q8 for this test program: a stand-in table (AVM's quantizer is not available). Both
// engines read the same value for a qindex, which is all that parity needs.
int64_t lambda_q8(int qindex) {
  const double step = 1.0 + qindex / 8.0, pivot = 1.0 + 120 / 8.0;
  return static_cast<int64_t>(0.002 * step * step * std::pow(pivot / step, 0.8) * 256.0 + 0.5);
}

namespace {

// Every field the decision map carries: trees, leaves, and each candidate block's choices.
bool identical(const DecisionMap& a, const DecisionMap& b) {
  if (a.sb_size != b.sb_size || a.sb_cols != b.sb_cols || a.sb_rows != b.sb_rows || a.sbs.size() != b.sbs.size())
    return false;
  for (size_t i = 0; i < a.sbs.size(); i++) {
    const SbDecision &x = a.sbs[i], &y = b.sbs[i];
    if (x.tree != y.tree || x.blocks.size() != y.blocks.size() || x.cands.size() != y.cands.size()) {
      std::fprintf(stderr, "  superblock %zu: tree or sizes differ\n", i);
      return false;
    }
    for (size_t k = 0; k < x.blocks.size(); k++) {
      const BlockDecision &p = x.blocks[k], &q = y.blocks[k];
      if (p.w4 != q.w4 || p.h4 != q.h4 || p.inter != q.inter || p.intra != q.intra || p.mv_row != q.mv_row ||
          p.mv_col != q.mv_col || p.ref != q.ref || p.ref2 != q.ref2 || p.mv2_row != q.mv2_row || p.mv2_col != q.mv2_col) {
        std::fprintf(stderr, "  superblock %zu leaf %zu differs\n", i, k);
        return false;
      }
    }
    for (size_t k = 0; k < x.cands.size(); k++) {
      const BlockCandidates &p = x.cands[k], &q = y.cands[k];
      const BlockDecision &u = p.inter, &v = q.inter;
      bool same = p.inter_cost == q.inter_cost && p.intra_cost == q.intra_cost && p.intra == q.intra &&
                  u.w4 == v.w4 && u.h4 == v.h4 && u.mv_row == v.mv_row && u.mv_col == v.mv_col && u.ref == v.ref &&
                  u.ref2 == v.ref2 && u.mv2_row == v.mv2_row && u.mv2_col == v.mv2_col;
      for (int r = 0; r < BlockCandidates::kRefs; r++)
        same = same && p.ref_cost[r] == q.ref_cost[r] && p.ref_mv_col[r] == q.ref_mv_col[r] &&
               p.ref_mv_row[r] == q.ref_mv_row[r];
      if (!same) {
        std::fprintf(stderr, "  superblock %zu candidate %zu differs\n", i, k);
        return false;
      }
    }
  }
  return true;
}

DecisionMap run(DecisionEngine& e, const Frame420& src, const std::vector<const Frame420*>& refs, int q,
                const std::vector<long long>& keys = {}) {
  DecisionMap dm;
  RowGate gate;
  e.launch(src, refs, q, dm, keys);
  e.collect(dm, gate);
  if (gate.ready_rows() != dm.sb_rows) throw std::runtime_error("not every row was published");
  return dm;
}

}  // namespace

static int cpu_engine_matches_cuda() {
  for (const auto& wh : {std::pair<int, int>{202, 122}, std::pair<int, int>{640, 360}, std::pair<int, int>{32, 32}}) {
    const int w = wh.first, h = wh.second;
    const Frame420 prev = scene_frame(w, h), src = scene_frame(w, h, 3, -2);
    CpuEngine cpu(w, h, 64, 8);
    CudaEngine cuda(w, h, 64);
    for (bool key : {true, false}) {
      const std::vector<const Frame420*> refs = key ? std::vector<const Frame420*>{} : std::vector<const Frame420*>{&prev};
      for (int q : {40, 120, 220}) CHECK(identical(run(cpu, src, refs, q), run(cuda, src, refs, q)));
    }
  }
  return 0;
}

static int launch_collect_matches_decide() {
  for (const auto& wh : {std::pair<int, int>{202, 122}, std::pair<int, int>{640, 360}}) {
    const Frame420 src = scene_frame(wh.first, wh.second, 5, 1), prev = scene_frame(wh.first, wh.second);
    CudaEngine a(wh.first, wh.second, 64), b(wh.first, wh.second, 64);
    for (bool key : {false, true}) {
      const DecisionMap want = key ? a.decide_intra(src, 120) : a.decide_inter(src, prev, 120);
      Frame420 s = src, p = prev;  // launch must not read the caller's frames after it returns
      DecisionMap dm;
      b.launch(s, key ? nullptr : &p, 120, dm);
      std::fill(s.y.begin(), s.y.end(), uint8_t{0});
      std::fill(p.y.begin(), p.y.end(), uint8_t{255});
      RowGate gate;
      b.collect(dm, gate);
      CHECK(identical(dm, want));
      CHECK_EQ(gate.ready_rows(), dm.sb_rows);
    }
  }
  return 0;
}

static int multi_ref_matches_rules() {
  for (const auto& wh : {std::pair<int, int>{202, 122}, std::pair<int, int>{640, 360}}) {
    const int w = wh.first, h = wh.second;
    const Frame420 src = scene_frame(w, h, 6, -3), r0 = scene_frame(w, h, 40, 30, 5), r1 = scene_frame(w, h, 6, -3),
                   r2 = scene_frame(w, h, 3, -1);
    const std::vector<const Frame420*> refs{&r0, &r1, &r2};
    CudaEngine cuda(w, h, 64);
    const DecisionMap g = run(cuda, src, refs, 120);
    CHECK(identical(g, decide_inter_ref(src, refs, 64, 120)));
    int used[3] = {};
    for (const auto& sb : g.sbs)
      for (const auto& b : sb.blocks)
        if (b.inter) used[b.ref]++;
    CHECK(used[1] > used[0] && used[1] > used[2]);  // the matching scene, two frames back, wins
  }
  return 0;
}

static int seven_refs_with_keys() {
  const int w = 320, h = 192;
  std::vector<Frame420> pics;
  for (int i = 0; i < 9; i++) pics.push_back(scene_frame(w, h, i * 3, -i, 7));
  CudaEngine cuda(w, h, 64);
  CpuEngine cpu(w, h, 64, 4);
  for (int first = 1; first <= 2; first++) {  // one reference new to the store on the second pass
    std::vector<const Frame420*> refs;
    std::vector<long long> keys;
    for (int i = first; i < first + 7; i++) refs.push_back(&pics[i]), keys.push_back(i);
    CHECK(identical(run(cuda, pics[0], refs, 90, keys), run(cpu, pics[0], refs, 90, keys)));
  }
  return 0;
}

static int prepared_sequence_matches_cpu() {
  const int w = 416, h = 240;
  std::vector<Frame420> f;
  for (int i = 0; i < 6; i++) f.push_back(scene_frame(w, h, 2 * i, i, 3));
  CudaEngine cuda(w, h, 64);
  CpuEngine cpu(w, h, 64, 8);
  for (size_t i = 2; i < f.size(); i++) {  // tools/engine_bench.cpp:44-57
    std::vector<const Frame420*> refs{&f[i - 1], &f[i - 2]};
    std::vector<long long> keys{static_cast<long long>(i - 1), static_cast<long long>(i - 2)};
    DecisionMap dm;
    RowGate gate;
    cuda.launch(f[i], refs, 120, dm, keys, static_cast<long long>(i));
    if (i + 1 < f.size()) cuda.prepare(f[i + 1], static_cast<long long>(i + 1));
    cuda.collect(dm, gate);
    CHECK(identical(dm, run(cpu, f[i], refs, 120)));
  }
  return 0;
}

static int rows_publish_before_collect_ends() {
  const Frame420 src = scene_frame(640, 360, 3, 2), prev = scene_frame(640, 360);
  CudaEngine cuda(640, 360, 64);
  cuda.set_row_streams(2);
  DecisionMap dm;
  cuda.launch(src, &prev, 120, dm);
  RowGate gate;
  std::exception_ptr err;
  std::thread collector([&] {
    try {
      cuda.collect(dm, gate);
    } catch (...) {
      err = std::current_exception();
    }
  });
  int first = -1;
  gate.wait_row(0);
  first = gate.ready_rows();
  collector.join();
  if (err) std::rethrow_exception(err);
  CHECK(first >= 1);
  CHECK_EQ(gate.ready_rows(), dm.sb_rows);
  return 0;
}

static int no_intra_block_wider_than_32() {
  for (const auto& wh : {std::pair<int, int>{640, 360}, std::pair<int, int>{202, 122}}) {
    Frame420 flat = make_frame(wh.first, wh.second);
    std::fill(flat.y.begin(), flat.y.end(), uint8_t{128});
    CudaEngine cuda(wh.first, wh.second, 64);
    for (const DecisionMap& dm : {cuda.decide_intra(flat, 120), cuda.decide_inter(flat, flat, 120)})
      for (const auto& sb : dm.sbs)
        for (const auto& b : sb.blocks) CHECK(b.w4 <= (b.inter ? 16 : 8) && b.h4 <= (b.inter ? 16 : 8));
  }
  return 0;
}

static int errors_as_the_reference() {
  bool threw = false;
  try {
    CudaEngine bad(0, 0, 64);
  } catch (const std::runtime_error&) {
    threw = true;
  }
  CHECK(threw);
  threw = false;
  try {
    CudaEngine bad(64, 64, 128);
  } catch (const std::runtime_error&) {
    threw = true;
  }
  CHECK(threw);
  const Frame420 f = scene_frame(64, 64), other = scene_frame(32, 32);
  CudaEngine cuda(64, 64, 64);
  DecisionMap dm;
  threw = false;
  try {
    cuda.launch(f, std::vector<const Frame420*>(8, &f), 120, dm);
  } catch (const std::runtime_error&) {
    threw = true;
  }
  CHECK(threw);
  threw = false;
  try {
    cuda.launch(f, {&f, &f}, 120, dm, {1});
  } catch (const std::invalid_argument&) {
    threw = true;
  }
  CHECK(threw);
  threw = false;
  try {
    cuda.launch(other, {}, 120, dm);
  } catch (const std::runtime_error&) {
    threw = true;
  }
  CHECK(threw);
  CHECK(identical(cuda.decide_inter(f, f, 120), decide_inter_ref(f, f, 64, 120)));  // still usable
  return 0;
}

// The leaves of a mini-GOP through launch_group / collect_group (what Pipeline::code_group,
// src/pipeline.cpp:328-384, would call) against the CpuEngine deciding them one by one.
static int group_matches_cpu_per_frame() {
  const int w = 416, h = 240;
  std::vector<Frame420> f;
  for (int i = 0; i < 9; i++) f.push_back(scene_frame(w, h, 2 * i, -i, 3));
  CudaEngine cuda(w, h, 64);
  CpuEngine cpu(w, h, 64, 8);
  // anchor and middle first (ordinary launches, keyed), then the leaves as one group
  const std::vector<std::vector<int>> leaves_refs{{0, 2, 4}, {2, 4, 0}, {4, 6, 2}, {6, 8, 4}};
  for (int pass = 0; pass < 2; pass++) {  // the second pass finds its keyed references stored
    std::vector<const Frame420*> srcs;
    std::vector<std::vector<const Frame420*>> refs;
    std::vector<std::vector<long long>> keys;
    for (size_t i = 0; i < leaves_refs.size(); i++) {
      srcs.push_back(&f[2 * i + 1]);
      refs.emplace_back();
      keys.emplace_back();
      for (int r : leaves_refs[i]) refs.back().push_back(&f[r]), keys.back().push_back(r);
    }
    std::vector<int> q{120, 90, 150, 120};
    std::vector<DecisionMap> dms;
    cuda.launch_group(srcs, refs, keys, q, dms);
    std::vector<RowGate> gates(srcs.size());
    std::vector<RowGate*> gp;
    for (RowGate& g : gates) gp.push_back(&g);
    cuda.collect_group(dms, gp);
    for (size_t i = 0; i < srcs.size(); i++) {
      CHECK_EQ(gates[i].ready_rows(), dms[i].sb_rows);
      CHECK(identical(dms[i], run(cpu, *srcs[i], refs[i], q[i])));
    }
    // an ordinary launch in between, with a key the group path stored
    CHECK(identical(run(cuda, f[3], {&f[2], &f[4]}, 120, {2, 4}), run(cpu, f[3], {&f[2], &f[4]}, 120)));
  }
  // without keys, and a KEY frame among inter frames
  std::vector<DecisionMap> dms;
  cuda.launch_group({&f[5], &f[7]}, {{}, {&f[6], &f[8]}}, {}, {120, 120}, dms);
  std::vector<RowGate> gates(2);
  cuda.collect_group(dms, {&gates[0], &gates[1]});
  CHECK(identical(dms[0], run(cpu, f[5], {}, 120)));
  CHECK(identical(dms[1], run(cpu, f[7], {&f[6], &f[8]}, 120)));
  return 0;
}

int main() {
  int fails = 0;
  fails += RUN(cpu_engine_matches_cuda);
  fails += RUN(launch_collect_matches_decide);
  fails += RUN(multi_ref_matches_rules);
  fails += RUN(seven_refs_with_keys);
  fails += RUN(prepared_sequence_matches_cpu);
  fails += RUN(rows_publish_before_collect_ends);
  fails += RUN(no_intra_block_wider_than_32);
  fails += RUN(errors_as_the_reference);
  fails += RUN(group_matches_cpu_per_frame);
  if (fails) std::fprintf(stderr, "%d test(s) failed\n", fails);
  else std::printf("all adapter cases passed\n");
  return fails ? 1 : 0;
}
