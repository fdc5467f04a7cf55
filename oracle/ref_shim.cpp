// ref_shim.cpp: a C entry point into the REFERENCE's own decision engine, compiled together with
// the reference sources src/gpu/{kernels_ref,cpu_engine,decision_map}.cpp and src/io/y4m.cpp
// (oracle/Makefile). TEST INFRASTRUCTURE ONLY: it pins the C restatement (celv2_oracle.c) and
// times the reference CPU engine as the CPU baseline; the product never links it.
//
// lambda_q8 (src/core/quant.cpp:31-39) needs AVM's quantizer table, which is not available, so
// it is read from a table the harness sets (refx_set_lambda). Engine-to-engine parity does not
// depend on its values as long as every engine receives the same one.
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <vector>

#include "celv2_decision.h"
#include "gpu/cpu_engine.h"
#include "gpu/decision_map.h"
#include "gpu/kernels_ref.h"
#include "io/y4m.h"

namespace {
int64_t g_lambda[256];
thread_local char g_error[512];

int fail(const char* what) {
  std::snprintf(g_error, sizeof g_error, "%s", what);
  return -1;
}

Frame420 luma_frame(int width, int height, const uint8_t* y) {
  Frame420 f = make_frame(width, height);
  std::memcpy(f.y.data(), y, f.y.size());
  return f;
}

// The DecisionMap's superblock as the device record layout (the inverse of
// celv2::sb_out_to_decision, src/gpu/decision_map.cpp:65-105): MVs back to quarter pels.
void to_record(const SbDecision& d, celv2_sb_out* o) {
  std::memset(o, 0, sizeof *o);
  o->ntree = static_cast<int32_t>(d.tree.size());
  for (size_t k = 0; k < d.tree.size(); k++) o->tree[k] = static_cast<uint8_t>(d.tree[k]);
  o->nblocks = static_cast<int32_t>(d.blocks.size());
  for (size_t k = 0; k < d.blocks.size(); k++) {
    const BlockDecision& b = d.blocks[k];
    o->w4[k] = b.w4, o->h4[k] = b.h4;
    o->mode[k] = b.inter ? CELV2_NUM_MODES : static_cast<uint8_t>(b.intra);
    o->mvx[k] = static_cast<int16_t>(b.mv_col / 2), o->mvy[k] = static_cast<int16_t>(b.mv_row / 2);
    o->ref[k] = b.ref, o->ref2[k] = b.ref2;
    o->mv2x[k] = static_cast<int16_t>(b.mv2_col / 2), o->mv2y[k] = static_cast<int16_t>(b.mv2_row / 2);
  }
  for (size_t k = 0; k < d.cands.size() && k < CELV2_SB_BLOCKS; k++) {
    const BlockCandidates& c = d.cands[k];
    o->c_inter_cost[k] = c.inter_cost, o->c_intra_cost[k] = c.intra_cost;
    o->c_mvx[k] = static_cast<int16_t>(c.inter.mv_col / 2), o->c_mvy[k] = static_cast<int16_t>(c.inter.mv_row / 2);
    o->c_mv2x[k] = static_cast<int16_t>(c.inter.mv2_col / 2), o->c_mv2y[k] = static_cast<int16_t>(c.inter.mv2_row / 2);
    o->c_ref[k] = c.inter.ref, o->c_ref2[k] = c.inter.ref2, o->c_intra[k] = static_cast<uint8_t>(c.intra);
    for (int r = 0; r < CELV2_MAX_REFS; r++) {
      o->c_rcost[r][k] = c.ref_cost[r];
      o->c_rmvx[r][k] = static_cast<int16_t>(c.ref_mv_col[r] / 2), o->c_rmvy[r][k] = static_cast<int16_t>(c.ref_mv_row[r] / 2);
    }
  }
}

void to_records(const DecisionMap& dm, celv2_sb_out* out) {
  for (size_t i = 0; i < dm.sbs.size(); i++) to_record(dm.sbs[i], &out[i]);
}
}  // namespace

int64_t lambda_q8(int qindex) { return g_lambda[qindex < 0 ? 0 : qindex > 255 ? 255 : qindex]; }

extern "C" {

const char* refx_last_error() { return g_error; }

void refx_set_lambda(const int64_t* table256) { std::memcpy(g_lambda, table256, sizeof g_lambda); }

// decide_intra_ref / decide_inter_ref (src/gpu/kernels_ref.cpp:278-305): single-threaded rules.
int refx_decide_ref(int width, int height, const uint8_t* src_y, const uint8_t* const* ref_y, int nrefs, int qindex,
                    celv2_sb_out* out) {
  try {
    const Frame420 src = luma_frame(width, height, src_y);
    std::vector<Frame420> refs;
    std::vector<const Frame420*> rp;
    for (int r = 0; r < nrefs; r++) refs.push_back(luma_frame(width, height, ref_y[r]));
    for (const Frame420& f : refs) rp.push_back(&f);
    const DecisionMap dm = nrefs ? decide_inter_ref(src, rp, 64, qindex) : decide_intra_ref(src, 64, qindex);
    to_records(dm, out);
    return 0;
  } catch (const std::exception& e) {
    return fail(e.what());
  }
}

// The pyramid of build_pyramid_ref (src/gpu/kernels_ref.cpp:213-238), levels back to back.
int refx_build_pyramid(int width, int height, const uint8_t* y, int phases, uint8_t* out) {
  try {
    const RefPyramid p = build_pyramid_ref(luma_frame(width, height, y), phases != 0);
    size_t off = 0;
    for (int l = 0; l < celv2::kMeLevels; l++) {
      std::memcpy(out + off, p.px[l].data(), p.px[l].size());
      off += p.px[l].size();
    }
    return 0;
  } catch (const std::exception& e) {
    return fail(e.what());
  }
}

// Every level's field of one reference, coarsest level searched first (me_level_rows_ref,
// src/gpu/kernels_ref.cpp:240-251): out holds, per level 0..4, mvx then mvy (cols x rows each).
int refx_me_fields(int width, int height, const uint8_t* cur_y, const uint8_t* ref_y, int32_t* out) {
  try {
    const RefPyramid cur = build_pyramid_ref(luma_frame(width, height, cur_y));
    const RefPyramid ref = build_pyramid_ref(luma_frame(width, height, ref_y), true);
    std::vector<RefMvLevel> lv(celv2::kMeLevels);
    for (int l = celv2::kMeLevels - 1; l >= 0; l--) {
      RefMvLevel& o = lv[l];
      o.cols = (cur.plane[l].w + 7) / 8, o.rows = (cur.plane[l].h + 7) / 8;
      o.mvx.assign(static_cast<size_t>(o.cols) * o.rows, 0), o.mvy = o.mvx;
      me_level_rows_ref(cur, ref, l, l == celv2::kMeLevels - 1 ? nullptr : &lv[l + 1], 0, o.rows, o);
    }
    size_t off = 0;
    for (int l = 0; l < celv2::kMeLevels; l++) {
      for (int v : lv[l].mvx) out[off++] = v;
      for (int v : lv[l].mvy) out[off++] = v;
    }
    return 0;
  } catch (const std::exception& e) {
    return fail(e.what());
  }
}

// The reference CpuEngine (src/gpu/cpu_engine.cpp:11-128) behind a handle: launch, collect.
struct refx_engine {
  std::unique_ptr<CpuEngine> e;
  int width, height;
  DecisionMap dm;
};

refx_engine* refx_engine_new(int width, int height, int threads) {
  try {
    auto* h = new refx_engine{std::make_unique<CpuEngine>(width, height, 64, threads), width, height, {}};
    return h;
  } catch (const std::exception& e) {
    fail(e.what());
    return nullptr;
  }
}

void refx_engine_free(refx_engine* h) { delete h; }

// One frame decided end to end (launch, then collect with a RowGate), as tools/engine_bench.cpp:44-57
// does per frame; out (may be null) receives the records.
int refx_engine_decide(refx_engine* h, const uint8_t* src_y, const uint8_t* const* ref_y, int nrefs, int qindex,
                       celv2_sb_out* out) {
  try {
    const Frame420 src = luma_frame(h->width, h->height, src_y);
    std::vector<Frame420> refs;
    std::vector<const Frame420*> rp;
    for (int r = 0; r < nrefs; r++) refs.push_back(luma_frame(h->width, h->height, ref_y[r]));
    for (const Frame420& f : refs) rp.push_back(&f);
    RowGate gate;
    h->e->launch(src, rp, qindex, h->dm);
    h->e->collect(h->dm, gate);
    if (out) to_records(h->dm, out);
    return 0;
  } catch (const std::exception& e) {
    return fail(e.what());
  }
}

// The same with frames already held as Frame420 (no copies inside the timed call): the
// benchmark's CPU leg, which keeps the frames resident like the GPU leg keeps them in HBM.
struct refx_frames {
  std::vector<Frame420> f;
};
refx_frames* refx_frames_new(int width, int height, int n, const uint8_t* const* ys) {
  auto* s = new refx_frames;
  for (int i = 0; i < n; i++) s->f.push_back(luma_frame(width, height, ys[i]));
  return s;
}
void refx_frames_free(refx_frames* s) { delete s; }
int refx_engine_decide_idx(refx_engine* h, refx_frames* s, int src, const int* refs, int nrefs, int qindex) {
  try {
    std::vector<const Frame420*> rp;
    for (int r = 0; r < nrefs; r++) rp.push_back(&s->f[refs[r]]);
    RowGate gate;
    h->e->launch(s->f[src], rp, qindex, h->dm);
    h->e->collect(h->dm, gate);
    return 0;
  } catch (const std::exception& e) {
    return fail(e.what());
  }
}

// round_to_8bit (src/io/y4m.cpp:28-34) on a 10-bit luma plane.
int refx_round_to_8bit(int width, int height, const uint16_t* hy, uint8_t* y) {
  try {
    Frame420 f = make_frame(width, height, 10);
    std::memcpy(f.hy.data(), hy, f.hy.size() * 2);
    round_to_8bit(f);
    std::memcpy(y, f.y.data(), f.y.size());
    return 0;
  } catch (const std::exception& e) {
    return fail(e.what());
  }
}

}  // extern "C"
