// owl_api.cu -- libowl: plans, buffers and the C ABI of include/owl.h.
//
// Per squaring the engine launches two kernels (k_pass2 then k_pass1), the
// B200 counterpart of the reference's four-kernel chain fftMiddleIn ->
// tailSquare -> fftMiddleOut -> carryFused (src/Gpu.cpp:851-856, 903-932).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "owl.h"
#include "owl_kernels.cuh"
#include "owl_pass2_tc.cuh"
#include "owl_pack.cuh"
#include "owl_tables.hpp"
#include "owl_words.hpp"

using owl::C;

namespace {

thread_local std::string g_lastError;
thread_local const char* g_lastLiteral = nullptr;

struct OwlError {
  int code;
  std::string msg;
};

void fail(int code, const std::string& msg) { throw OwlError{code, msg}; }

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    fail(e == cudaErrorMemoryAllocation ? OWL_ERR_NOMEM : OWL_ERR_CUDA,
         std::string(what) + ": " + cudaGetErrorString(e));
  }
}

template <typename F> int guarded(F&& f) {
  try {
    f();
    return OWL_OK;
  } catch (const OwlError& e) {
    g_lastLiteral = nullptr;
    g_lastError = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    g_lastLiteral = "host allocation failed";
    return OWL_ERR_NOMEM;
  } catch (const std::exception& e) {
    g_lastLiteral = nullptr;
    g_lastError = e.what();
    return OWL_ERR_ARG;
  }
}

constexpr int kR = 2;                    // lines per pass-1 CTA
constexpr uint32_t kRoeCap = 1u << 16;   // per-launch ROE slots
constexpr double kDefaultMaxBpw = 19.2;  // at N = 256K; lowered 0.3 per doubling

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) { ck(cudaSetDevice(dev), "cudaSetDevice"); }
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) { cudaSetDevice(prev); }
  }
};

}  // namespace

namespace owl_detail {
void set_error_literal(const char* msg) { g_lastLiteral = msg; }
void set_error_string(const std::string& msg) {
  g_lastLiteral = nullptr;
  g_lastError = msg;
}
}  // namespace owl_detail

struct owl_plan {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint32_t E = 0, N = 0, W = 0, H = 0, hN = 0;
  owl::Args args{};
  C* F1 = nullptr;
  C* F2 = nullptr;
  void* tableMem = nullptr;
  void* scratch = nullptr;  // shuttle, flags, ctl, roe, small outputs
  int32_t* small = nullptr; // 64 gathered words
  unsigned long long* sum = nullptr;
  int* eq = nullptr;
  uint32_t roePos = 0;
  std::vector<int32_t*> bufs;
  // squaring blocks captured as CUDA graphs, keyed by (in, out, n, flags, with events)
  struct GraphEntry {
    const int32_t* in;
    int32_t* out;
    uint32_t n, flags;
    bool profiled;
    cudaGraphExec_t exec;
    uint64_t lastUse;
  };
  std::vector<GraphEntry> graphs;
  uint64_t useClock = 0;
  // column variant (owl::COL_V16 / COL_V8 / COL_V16_OCC2) and the device copies of its stage
  // tables (COL_V16_OCC2 shares COL_V16's)
  int colVariant = owl::COL_V16;
  const C* twHv16 = nullptr;
  const C* twHv8 = nullptr;
  // split-precision form: the column pass's (H = 2048 or 2560) DFT digit planes and stage tables; the
  // line pass's (W = 2048) digit planes are args.tc1B
  uint32_t split = 0;  // OWL_SPLIT_* flags
  const unsigned char* tcB = nullptr;
  const C* twHtc = nullptr;
  // device-side expand / compact: word staging (nWords + 1, zero padded), block carries, status
  uint32_t* dwords = nullptr;
  uint32_t* packBlk = nullptr;
  owl::PackCtl* packCtl = nullptr;
  uint32_t nw = 0, packBlocks = 0;
};

namespace {

// ---- kernel dispatch on the compile-time shape --------------------------------

template <int W, int M> void setp1attr() {
  size_t sm = (size_t)kR * owl::p1_line_stride<W, kR>() * sizeof(C);
  if constexpr (W == owl::kLtcW) {
    const int smx = (int)sm + owl::ltc_extra_smem();
    ck(cudaFuncSetAttribute(owl::k_pass1<W, kR, M, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smx),
       "cudaFuncSetAttribute(pass1 split)");
    if (M == owl::P1_FUSED) {
      ck(cudaFuncSetAttribute(owl::k_pass1<W, kR, M, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smx),
         "cudaFuncSetAttribute(pass1 split without round-off)");
    }
  }
  ck(cudaFuncSetAttribute(owl::k_pass1<W, kR, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm),
     "cudaFuncSetAttribute(pass1)");
  ck(cudaFuncSetAttribute(owl::k_pass1_group<W, kR, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm),
     "cudaFuncSetAttribute(pass1 group)");
  if (M == owl::P1_FUSED) {
    ck(cudaFuncSetAttribute(owl::k_pass1<W, kR, owl::P1_FUSED, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int)sm),
       "cudaFuncSetAttribute(pass1 without round-off)");
    ck(cudaFuncSetAttribute(owl::k_pass1_group<W, kR, owl::P1_FUSED, false>,
                            cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm),
       "cudaFuncSetAttribute(pass1 group without round-off)");
  }
}
template <int H, int M, int CV> void setp2attr_v() {
  constexpr int V = owl::col_vpt(CV), MB = owl::col_minb(CV);
  size_t sm = 2 * (size_t)owl::p2_col_stride<H, V>() * sizeof(C);
  ck(cudaFuncSetAttribute(owl::k_pass2<H, kR, M, V, MB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm),
     "cudaFuncSetAttribute(pass2)");
  if (M == owl::P2_SQUARE) {
    ck(cudaFuncSetAttribute(owl::k_pass2_group<H, kR, V, MB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm),
       "cudaFuncSetAttribute(pass2 group)");
  }
}
// every column variant built for H
template <int H, int M> void setp2attr() {
  setp2attr_v<H, M, owl::COL_V16>();
  if constexpr (owl::col_variant_ok(H, owl::COL_V8)) { setp2attr_v<H, M, owl::COL_V8>(); }
  if constexpr (owl::col_variant_ok(H, owl::COL_V16_OCC2)) { setp2attr_v<H, M, owl::COL_V16_OCC2>(); }
}

template <int H, int M> void setp2tcattr() {
  ck(cudaFuncSetAttribute(owl::k_pass2_tc<H, kR, M>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          owl::TcCfg<H>::SMEM),
     "cudaFuncSetAttribute(pass2 split)");
}

// Launches a pass kernel on the plan's stream. With `pdl` it is a programmatic dependent of the
// kernel before it (the pass kernels begin with griddep_wait()): its CTAs may be scheduled on SMs
// that the previous pass's last CTAs leave free, which hides the launch gap between the passes.
template <typename... KArgs, typename... Args>
void launch_on(cudaStream_t stream, bool pdl, void (*kernel)(KArgs...), dim3 grid, int threads, size_t smem,
               Args... args) {
  if (!pdl) {
    kernel<<<grid, threads, smem, stream>>>(args...);
    return;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  ck(cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...), "cudaLaunchKernelEx");
}
template <typename... KArgs, typename... Args>
void launch_pass(owl_plan* p, bool pdl, void (*kernel)(KArgs...), dim3 grid, int threads, size_t smem,
                 Args... args) {
  launch_on(p->stream, pdl, kernel, grid, threads, smem, args...);
}

template <int H> void p2launch_tc_h(owl_plan* p, int mode, C* F, const C* Fb, C* Fq, int ts, bool pdl) {
  dim3 grid(p->W / 2);
  constexpr int T = H / 8;
  auto k = (mode == owl::P2_SQUARE) ? owl::k_pass2_tc<H, kR, owl::P2_SQUARE>
           : (mode == owl::P2_FWD)  ? owl::k_pass2_tc<H, kR, owl::P2_FWD>
                                    : owl::k_pass2_tc<H, kR, owl::P2_MUL>;
  launch_pass(p, pdl, k, grid, T, owl::TcCfg<H>::SMEM, p->args, (const unsigned char*)p->tcB, (const C*)p->twHtc, F,
              Fb, Fq, ts);
}
void p2launch_tc(owl_plan* p, int mode, C* F, const C* Fb, C* Fq, int ts, bool pdl) {
  if (p->H == 2560) {
    p2launch_tc_h<2560>(p, mode, F, Fb, Fq, ts, pdl);
  } else {
    p2launch_tc_h<2048>(p, mode, F, Fb, Fq, ts, pdl);
  }
}

template <int W> void p1launch(owl_plan* p, int mode, C* F, int32_t* words, int roeSlot, int flags, int ts, bool pdl) {
  constexpr int T = kR * W / 16;
  size_t sm = (size_t)kR * owl::p1_line_stride<W, kR>() * sizeof(C);
  dim3 grid(p->H / kR);
  if constexpr (W == owl::kLtcW) {
    if (p->split & OWL_SPLIT_LINES) {
      // the split-precision line pass (its GEMM stages on the tensor cores)
      auto k = (mode == owl::P1_FUSED) ? (roeSlot >= 0 ? owl::k_pass1<W, kR, owl::P1_FUSED, true, true>
                                                       : owl::k_pass1<W, kR, owl::P1_FUSED, false, true>)
               : (mode == owl::P1_IN)  ? owl::k_pass1<W, kR, owl::P1_IN, true, true>
                                       : owl::k_pass1<W, kR, owl::P1_OUT, true, true>;
      launch_pass(p, pdl, k, grid, T, sm + owl::ltc_extra_smem(), p->args, F, words, roeSlot, flags, ts);
      return;
    }
  }
  // a fused pass with no round-off slot runs the build without the measurement
  auto k = (mode == owl::P1_FUSED) ? (roeSlot >= 0 ? owl::k_pass1<W, kR, owl::P1_FUSED>
                                                   : owl::k_pass1<W, kR, owl::P1_FUSED, false>)
           : (mode == owl::P1_IN)  ? owl::k_pass1<W, kR, owl::P1_IN>
                                   : owl::k_pass1<W, kR, owl::P1_OUT>;
  launch_pass(p, pdl, k, grid, T, sm, p->args, F, words, roeSlot, flags, ts);
}

template <int H, int CV> void p2launch_v(owl_plan* p, int mode, C* F, const C* Fb, C* Fq, int ts, bool pdl) {
  constexpr int V = owl::col_vpt(CV), MB = owl::col_minb(CV);
  constexpr int T = 2 * H / V;
  size_t sm = 2 * (size_t)owl::p2_col_stride<H, V>() * sizeof(C);
  dim3 grid(p->W / 2);
  auto k = (mode == owl::P2_SQUARE) ? owl::k_pass2<H, kR, owl::P2_SQUARE, V, MB>
           : (mode == owl::P2_FWD)  ? owl::k_pass2<H, kR, owl::P2_FWD, V, MB>
                                    : owl::k_pass2<H, kR, owl::P2_MUL, V, MB>;
  launch_pass(p, pdl, k, grid, T, sm, p->args, F, Fb, Fq, ts);
}
// the plan's column variant (checked against H when it was set)
template <int H> void p2launch(owl_plan* p, int mode, C* F, const C* Fb, C* Fq, int ts, bool pdl) {
  if constexpr (owl::col_variant_ok(H, owl::COL_V8)) {
    if (p->colVariant == owl::COL_V8) { return p2launch_v<H, owl::COL_V8>(p, mode, F, Fb, Fq, ts, pdl); }
  }
  if constexpr (owl::col_variant_ok(H, owl::COL_V16_OCC2)) {
    if (p->colVariant == owl::COL_V16_OCC2) {
      return p2launch_v<H, owl::COL_V16_OCC2>(p, mode, F, Fb, Fq, ts, pdl);
    }
  }
  p2launch_v<H, owl::COL_V16>(p, mode, F, Fb, Fq, ts, pdl);
}

#define OWL_FOR_SIZES(X) X(64) X(128) X(256) X(512) X(1024) X(2048) X(4096)
// column heights: the powers of two, and 5 * 2^k (radix-5 middle stage) for the 5 * 2^m FFT lengths
#define OWL_FOR_H_SIZES(X) OWL_FOR_SIZES(X) X(640) X(1280) X(2560)

void set_attrs(uint32_t W, uint32_t H) {
  switch (W) {
#define CASE_W(n)                  \
  case n:                          \
    setp1attr<n, owl::P1_FUSED>(); \
    setp1attr<n, owl::P1_IN>();    \
    setp1attr<n, owl::P1_OUT>();   \
    break;
    OWL_FOR_SIZES(CASE_W)
#undef CASE_W
    default:
      fail(OWL_ERR_ARG, "unsupported W");
  }
  switch (H) {
#define CASE_H(n)                   \
  case n:                           \
    setp2attr<n, owl::P2_SQUARE>(); \
    setp2attr<n, owl::P2_FWD>();    \
    setp2attr<n, owl::P2_MUL>();    \
    break;
    OWL_FOR_H_SIZES(CASE_H)
#undef CASE_H
    default:
      fail(OWL_ERR_ARG, "unsupported H");
  }
  if (H == 2048) {
    setp2tcattr<2048, owl::P2_SQUARE>();
    setp2tcattr<2048, owl::P2_FWD>();
    setp2tcattr<2048, owl::P2_MUL>();
  } else if (H == 2560) {
    setp2tcattr<2560, owl::P2_SQUARE>();
    setp2tcattr<2560, owl::P2_FWD>();
    setp2tcattr<2560, owl::P2_MUL>();
  }
}

constexpr int kNoRoe = -2;  // pass1's fixedSlot for a line pass that measures no round-off

void pass1(owl_plan* p, int mode, C* F, int32_t* words, int flags, int fixedSlot = -1, int ts = -1,
           bool pdl = false) {
  int slot = -1;
  if (mode != owl::P1_IN && fixedSlot != kNoRoe) {
    if (fixedSlot >= 0) {
      slot = std::min(fixedSlot, (int)kRoeCap - 1);
      p->roePos = std::max(p->roePos, (uint32_t)slot + 1);
    } else {
      slot = (int)std::min(p->roePos, kRoeCap - 1);
      if (p->roePos < kRoeCap) { ++p->roePos; }
    }
  }
  switch (p->W) {
#define CASE_W(n)                                \
  case n:                                        \
    p1launch<n>(p, mode, F, words, slot, flags, ts, pdl); \
    break;
    OWL_FOR_SIZES(CASE_W)
#undef CASE_W
    default:
      fail(OWL_ERR_ARG, "unsupported W");
  }
  ck(cudaGetLastError(), "pass1 launch");
}

void pass2(owl_plan* p, int mode, C* F, const C* Fb, C* Fq, int ts = -1, bool pdl = false) {
  if (p->split & OWL_SPLIT_COLUMNS) {
    p2launch_tc(p, mode, F, Fb, Fq, ts, pdl);
    ck(cudaGetLastError(), "pass2 split launch");
    return;
  }
  switch (p->H) {
#define CASE_H(n)                       \
  case n:                               \
    p2launch<n>(p, mode, F, Fb, Fq, ts, pdl); \
    break;
    OWL_FOR_H_SIZES(CASE_H)
#undef CASE_H
    default:
      fail(OWL_ERR_ARG, "unsupported H");
  }
  ck(cudaGetLastError(), "pass2 launch");
}

// the block-exit line pass, then the (normally empty) queue of leftover carries
void pass1_out(owl_plan* p, int32_t* words, int flags, int fixedSlot = -1, int ts = -1, bool pdl = false) {
  pass1(p, owl::P1_OUT, p->F1, words, flags, fixedSlot, ts, pdl);
  owl::k_carry_fixup<<<1, 32, 0, p->stream>>>(p->args, words);
  ck(cudaGetLastError(), "fixup launch");
}

constexpr uint32_t kTsCap = 4096;  // launch-timestamp slots (profiled blocks of up to 2047 squarings)

// Enqueues n squarings in -> out on the plan's stream: entry line pass, n x
// (column pass, line pass), exit fixup. ROE slot k holds squaring k's
// round-off. With `stamp`, launch i records its first CTA start and last CTA
// end in timestamp slot i (launch 0 is the entry pass, 2k+1 / 2k+2 are
// squaring k's column and line passes).
void enqueue_square(owl_plan* p, int32_t* out, const int32_t* in, uint32_t n, uint32_t flags, bool stamp) {
  const int ll = (flags & OWL_SQ_LL) ? owl::FL_LL : 0;
  const int mul3 = (flags & OWL_SQ_MUL3) ? owl::FL_MUL3 : 0;
  const bool roe = !(flags & OWL_SQ_NO_ROE);
  int li = 0;
  auto ts = [&] { return stamp ? li++ : -1; };
  if (stamp) {
    const size_t cnt = 2 * (size_t)n + 1;
    ck(cudaMemsetAsync(p->args.tsStart, 0xff, cnt * sizeof(unsigned long long), p->stream), "memset ts");
    ck(cudaMemsetAsync(p->args.tsEnd, 0, cnt * sizeof(unsigned long long), p->stream), "memset ts");
  }
  // the passes after the entry pass are programmatic dependents of the pass before them, except
  // the line pass after the split-precision column pass (8 us slower per iteration at 8M that way)
  const bool pdl = !(p->split & OWL_SPLIT_COLUMNS);
  pass1(p, owl::P1_IN, p->F1, const_cast<int32_t*>(in), 0, -1, ts());
  for (uint32_t k = 0; k < n; ++k) {
    pass2(p, owl::P2_SQUARE, p->F1, nullptr, nullptr, ts(), true);
    if (k + 1 < n) {
      pass1(p, owl::P1_FUSED, p->F1, nullptr, ll, roe ? (int)k : kNoRoe, ts(), pdl);
    } else {
      pass1_out(p, out, ll | mul3, roe ? (int)k : kNoRoe, ts(), pdl);
    }
  }
}

// ---- grouped launches: the same pass of several plans of one shape in one launch ----

template <int W> void p1group(cudaStream_t st, int mode, bool roe, const owl::GroupArgs& ga, uint32_t cnt, uint32_t H,
                              int roeSlot, int flags) {
  constexpr int T = kR * W / 16;
  const size_t sm = (size_t)kR * owl::p1_line_stride<W, kR>() * sizeof(C);
  const dim3 grid(H / kR, cnt);
  auto k = (mode == owl::P1_FUSED) ? (roe ? owl::k_pass1_group<W, kR, owl::P1_FUSED>
                                          : owl::k_pass1_group<W, kR, owl::P1_FUSED, false>)
           : (mode == owl::P1_IN)  ? owl::k_pass1_group<W, kR, owl::P1_IN>
                                   : owl::k_pass1_group<W, kR, owl::P1_OUT>;
  launch_on(st, mode != owl::P1_IN, k, grid, T, sm, ga, roeSlot, flags);
}
template <int H, int CV> void p2group_v(cudaStream_t st, const owl::GroupArgs& ga, uint32_t cnt, uint32_t W) {
  constexpr int V = owl::col_vpt(CV), MB = owl::col_minb(CV);
  const size_t sm = 2 * (size_t)owl::p2_col_stride<H, V>() * sizeof(C);
  launch_on(st, true, owl::k_pass2_group<H, kR, V, MB>, dim3(W / 2, cnt), 2 * H / V, sm, ga);
}
template <int H> void p2group(cudaStream_t st, const owl::GroupArgs& ga, uint32_t cnt, uint32_t W, int cv) {
  if constexpr (owl::col_variant_ok(H, owl::COL_V8)) {
    if (cv == owl::COL_V8) { return p2group_v<H, owl::COL_V8>(st, ga, cnt, W); }
  }
  if constexpr (owl::col_variant_ok(H, owl::COL_V16_OCC2)) {
    if (cv == owl::COL_V16_OCC2) { return p2group_v<H, owl::COL_V16_OCC2>(st, ga, cnt, W); }
  }
  p2group_v<H, owl::COL_V16>(st, ga, cnt, W);
}

// n squarings of each plan's buffer (in place) as grouped launches on `st`: plans of one plain
// (not split-precision) shape and column variant, at most kGroupMax
void enqueue_square_group(cudaStream_t st, const std::vector<owl_plan*>& plans, const std::vector<int32_t*>& bufs,
                          uint32_t n, uint32_t flags) {
  const uint32_t cnt = (uint32_t)plans.size();
  const uint32_t W = plans[0]->W, H = plans[0]->H;
  const int cv = plans[0]->colVariant;
  owl::GroupArgs ga{};
  for (uint32_t i = 0; i < cnt; ++i) {
    ga.a[i] = plans[i]->args;
    ga.F[i] = plans[i]->F1;
    ga.words[i] = bufs[i];
  }
  const int ll = (flags & OWL_SQ_LL) ? owl::FL_LL : 0;
  const int mul3 = (flags & OWL_SQ_MUL3) ? owl::FL_MUL3 : 0;
  const bool roe = !(flags & OWL_SQ_NO_ROE);
  auto p1 = [&](int mode, int slot, int fl) {
    switch (W) {
#define CASE_W(x)                                                   \
  case x:                                                           \
    p1group<x>(st, mode, slot >= 0, ga, cnt, H, slot, fl);          \
    break;
      OWL_FOR_SIZES(CASE_W)
#undef CASE_W
      default:
        fail(OWL_ERR_ARG, "unsupported W");
    }
  };
  auto p2 = [&]() {
    switch (H) {
#define CASE_H(x)                            \
  case x:                                    \
    p2group<x>(st, ga, cnt, W, cv);          \
    break;
      OWL_FOR_H_SIZES(CASE_H)
#undef CASE_H
      default:
        fail(OWL_ERR_ARG, "unsupported H");
    }
  };
  p1(owl::P1_IN, -1, 0);
  for (uint32_t k = 0; k < n; ++k) {
    p2();
    const int slot = roe ? (int)std::min(k, kRoeCap - 1) : -1;
    p1(k + 1 < n ? owl::P1_FUSED : owl::P1_OUT, slot, k + 1 < n ? ll : (ll | mul3));
  }
  owl::k_carry_fixup_group<<<cnt, 32, 0, st>>>(ga);
  ck(cudaGetLastError(), "grouped launch");
}

constexpr uint32_t kGraphMinIters = 16;
constexpr size_t kGraphCacheMax = 8;

// the cached graph for this block, captured on first use
owl_plan::GraphEntry& graph_for(owl_plan* p, int32_t* out, const int32_t* in, uint32_t n, uint32_t flags,
                                bool profiled) {
  ++p->useClock;
  for (auto& g : p->graphs) {
    if (g.in == in && g.out == out && g.n == n && g.flags == flags && g.profiled == profiled) {
      g.lastUse = p->useClock;
      return g;
    }
  }
  if (p->graphs.size() >= kGraphCacheMax) {
    auto lru = std::min_element(p->graphs.begin(), p->graphs.end(),
                                [](const auto& a, const auto& b) { return a.lastUse < b.lastUse; });
    cudaGraphExecDestroy(lru->exec);
    p->graphs.erase(lru);
  }
  owl_plan::GraphEntry g{in, out, n, flags, profiled, nullptr, p->useClock};
  cudaGraph_t graph = nullptr;
  ck(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
  try {
    enqueue_square(p, out, in, n, flags, profiled);
  } catch (...) {
    cudaStreamEndCapture(p->stream, &graph);
    if (graph) { cudaGraphDestroy(graph); }
    throw;
  }
  ck(cudaStreamEndCapture(p->stream, &graph), "cudaStreamEndCapture");
  cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
  cudaGraphDestroy(graph);
  ck(e, "cudaGraphInstantiate");
  p->graphs.push_back(std::move(g));
  return p->graphs.back();
}

void run_square(owl_plan* p, int32_t* out, const int32_t* in, uint32_t n, uint32_t flags) {
  if (n < kGraphMinIters) {
    enqueue_square(p, out, in, n, flags, false);
    return;
  }
  auto& g = graph_for(p, out, in, n, flags, false);
  ck(cudaGraphLaunch(g.exec, p->stream), "cudaGraphLaunch");
  if (!(flags & OWL_SQ_NO_ROE)) { p->roePos = std::max(p->roePos, std::min(n, kRoeCap)); }
}

void check_plan(const owl_plan* p) {
  if (!p) { fail(OWL_ERR_ARG, "null plan"); }
}

void check_buf(const owl_plan* p, const int32_t* b) {
  if (!b) { fail(OWL_ERR_ARG, "null buffer"); }
  if (std::find(p->bufs.begin(), p->bufs.end(), b) == p->bufs.end()) {
    fail(OWL_ERR_ARG, "buffer does not belong to this plan");
  }
}

// reads and clears the device error word; throws on a recorded wait timeout
void sync_and_check(owl_plan* p) {
  ck(cudaStreamSynchronize(p->stream), "cudaStreamSynchronize");
  uint32_t err = 0;
  ck(cudaMemcpy(&err, &p->args.ctl->error, sizeof(err), cudaMemcpyDeviceToHost), "read error word");
  if (err) {
    // reset the carry-chain state so that the plan stays usable
    uint32_t G = p->H / kR;
    ck(cudaMemset(p->args.ctl, 0, sizeof(owl::Ctl)), "reset ctl");
    ck(cudaMemset(p->args.flags, 0, G * sizeof(uint32_t)), "reset flags");
    ck(cudaMemset(p->args.shuttle, 0, (size_t)G * p->W * sizeof(long long)), "reset carry words");
    fail(OWL_ERR_TIMEOUT, "device-side carry wait timed out");
  }
}

static_assert(OWL_COL_AUTO == owl::COL_AUTO && OWL_COL_V16 == owl::COL_V16 && OWL_COL_V8 == owl::COL_V8 &&
                  OWL_COL_V16_OCC2 == owl::COL_V16_OCC2,
              "column variant numbers of owl.h and the kernels");

// the column variant's kernels and stage tables (the variant checked against H by the caller)
void apply_col_variant(owl_plan* p, int cv) {
  p->colVariant = cv;
  p->args.twH = (cv == owl::COL_V8) ? p->twHv8 : p->twHv16;
}

template <typename T> T* carve(char*& cur, size_t count) {
  size_t off = (reinterpret_cast<uintptr_t>(cur) + 255) & ~uintptr_t(255);
  T* r = reinterpret_cast<T*>(off);
  cur = reinterpret_cast<char*>(off + count * sizeof(T));
  return r;
}

void plan_create(int device, uint32_t E, uint32_t W, uint32_t H, owl_plan** out) {
  if (!out) { fail(OWL_ERR_ARG, "null out"); }
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    fail(OWL_ERR_NODEV, "no CUDA device " + std::to_string(device));
  }
  if (E < 1000 || E % 2 == 0) { fail(OWL_ERR_ARG, "exponent must be odd and >= 1000"); }
  if (W == 0 && H == 0) {
    uint32_t N;
    if (owl_fft_choose(E, 0, &N, &W, &H) != OWL_OK) { fail(OWL_ERR_ARG, "no FFT shape for this exponent"); }
  }
  if (!owl::shape_supported(W, H)) {
    fail(OWL_ERR_ARG, "W must be a power of two in [64, 4096]; H a power of two in [64, 4096] or 640, 1280, 2560");
  }
  const uint32_t N = 2 * W * H;
  // below ~8 bits per word the sloppy carry-in of a line group can overflow a
  // digit; above ~21 the FP64 round-off can reach 0.5 at any size built here
  if (E / N < 8 || (double)E / N > 21.0) { fail(OWL_ERR_ARG, "bits per word out of range for this FFT"); }

  owl::Tables t = owl::make_tables(E, W, H);

  DeviceGuard dg(device);
  std::unique_ptr<owl_plan> p(new owl_plan());
  p->device = device;
  p->E = E;
  p->N = N;
  p->W = W;
  p->H = H;
  p->hN = W * H;
  set_attrs(W, H);
  ck(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking), "cudaStreamCreate");

  // tables: one allocation
  static_assert(kR == owl::kLinesPerBlock, "table layout and launch disagree on lines per block");
  const bool tcShape = owl::tc_height((int)H);
  const std::vector<owl::HostC> twHtc =
      H == 2048 ? owl::stage_tables(H, 8, owl::TcCfg<2048>::R1)
                : (H == 2560 ? owl::stage_tables(H, 8, owl::TcCfg<2560>::R1) : std::vector<owl::HostC>());
  const std::vector<uint8_t> tcB =
      H == 2048 ? owl::tc_dft_digits<2048>() : (H == 2560 ? owl::tc_dft_digits<2560>() : std::vector<uint8_t>());
  const std::vector<uint8_t> tc1B = W == (uint32_t)owl::kLtcW ? owl::line_tc_dft_digits() : std::vector<uint8_t>();
  const std::vector<owl::HostC> twH8 =
      owl::col_variant_ok((int)H, owl::COL_V8) ? owl::col_stage_tables(H, owl::COL_V8) : std::vector<owl::HostC>();
  size_t nC = t.twW.size() + t.twH.size() + twH8.size() + t.rootH.size() + t.twLo.size() + t.twHi.size() +
              twHtc.size();
  size_t bytes = 256 * 20 + nC * sizeof(C) + (t.wt1.size() * 2 + t.wt2.size() * 2) * sizeof(double) +
                 (t.x1.size() + t.x2.size() + t.p1masks.size()) * sizeof(uint32_t) + tcB.size() + tc1B.size();
  ck(cudaMalloc(&p->tableMem, bytes), "cudaMalloc(tables)");
  std::vector<char> host(bytes, 0);
  char* hcur = host.data();
  auto put = [&](const void* src, size_t n) -> size_t {
    size_t off = ((size_t)(hcur - host.data()) + 255) & ~size_t(255);
    std::memcpy(host.data() + off, src, n);
    hcur = host.data() + off + n;
    return off;
  };
  char* dbase = static_cast<char*>(p->tableMem);
  p->args.twW = reinterpret_cast<const C*>(dbase + put(t.twW.data(), t.twW.size() * sizeof(C)));
  p->twHv16 = reinterpret_cast<const C*>(dbase + put(t.twH.data(), t.twH.size() * sizeof(C)));
  if (!twH8.empty()) { p->twHv8 = reinterpret_cast<const C*>(dbase + put(twH8.data(), twH8.size() * sizeof(C))); }
  p->args.rootH = reinterpret_cast<const C*>(dbase + put(t.rootH.data(), t.rootH.size() * sizeof(C)));
  p->args.twLo = reinterpret_cast<const C*>(dbase + put(t.twLo.data(), t.twLo.size() * sizeof(C)));
  p->args.twHi = reinterpret_cast<const C*>(dbase + put(t.twHi.data(), t.twHi.size() * sizeof(C)));
  p->args.wt1 = reinterpret_cast<const double*>(dbase + put(t.wt1.data(), t.wt1.size() * sizeof(double)));
  p->args.iwt1 = reinterpret_cast<const double*>(dbase + put(t.iwt1.data(), t.iwt1.size() * sizeof(double)));
  p->args.x1 = reinterpret_cast<const uint32_t*>(dbase + put(t.x1.data(), t.x1.size() * sizeof(uint32_t)));
  p->args.wt2 = reinterpret_cast<const double*>(dbase + put(t.wt2.data(), t.wt2.size() * sizeof(double)));
  p->args.iwt2 = reinterpret_cast<const double*>(dbase + put(t.iwt2.data(), t.iwt2.size() * sizeof(double)));
  p->args.x2 = reinterpret_cast<const uint32_t*>(dbase + put(t.x2.data(), t.x2.size() * sizeof(uint32_t)));
  p->args.p1masks = reinterpret_cast<const uint2*>(dbase + put(t.p1masks.data(), t.p1masks.size() * sizeof(uint32_t)));
  if (tcShape) {
    p->twHtc = reinterpret_cast<const C*>(dbase + put(twHtc.data(), twHtc.size() * sizeof(C)));
    p->tcB = reinterpret_cast<const unsigned char*>(dbase + put(tcB.data(), tcB.size()));
  }
  if (!tc1B.empty()) { p->args.tc1B = reinterpret_cast<const unsigned char*>(dbase + put(tc1B.data(), tc1B.size())); }
  ck(cudaMemcpy(p->tableMem, host.data(), bytes, cudaMemcpyHostToDevice), "upload tables");

  // FFT work buffers
  ck(cudaMalloc(&p->F1, (size_t)p->hN * sizeof(C)), "cudaMalloc(F1)");
  ck(cudaMalloc(&p->F2, (size_t)p->hN * sizeof(C)), "cudaMalloc(F2)");

  // scratch: carry shuttle, flags, control word, ROE slots, small outputs
  const uint32_t G = H / kR;
  const uint32_t nw = owl::n_words(E), packBlocks = (N + owl::kPackDigits - 1) / owl::kPackDigits;
  size_t sbytes = 256 * 14 + (size_t)G * W * sizeof(long long) + G * sizeof(uint32_t) + sizeof(owl::Ctl) +
                  (size_t)(nw + 2) * sizeof(uint32_t) + packBlocks * sizeof(uint32_t) + sizeof(owl::PackCtl) +
                  2 * owl::kPendingCap * sizeof(long long) + 2 * kTsCap * sizeof(unsigned long long) +
                  kRoeCap * sizeof(float) + 64 * sizeof(int32_t) + sizeof(unsigned long long) + sizeof(int);
  ck(cudaMalloc(&p->scratch, sbytes), "cudaMalloc(scratch)");
  ck(cudaMemset(p->scratch, 0, sbytes), "memset(scratch)");
  char* cur = static_cast<char*>(p->scratch);
  p->args.shuttle = carve<long long>(cur, (size_t)G * W);
  p->args.flags = carve<uint32_t>(cur, G);
  p->args.ctl = carve<owl::Ctl>(cur, 1);
  p->args.pending = carve<long long>(cur, 2 * owl::kPendingCap);
  p->args.tsStart = carve<unsigned long long>(cur, kTsCap);
  p->args.tsEnd = carve<unsigned long long>(cur, kTsCap);
  p->args.roe = carve<float>(cur, kRoeCap);
  p->small = carve<int32_t>(cur, 64);
  p->sum = carve<unsigned long long>(cur, 1);
  p->eq = carve<int>(cur, 1);
  p->dwords = carve<uint32_t>(cur, nw + 2);
  p->packBlk = carve<uint32_t>(cur, packBlocks);
  p->packCtl = carve<owl::PackCtl>(cur, 1);
  p->nw = nw;
  p->packBlocks = packBlocks;

  p->args.E = E;
  p->args.N = N;
  p->args.W = W;
  p->args.H = H;
  p->args.hN = p->hN;
  p->args.bitsLo = E / N;
  p->args.eModN = E % N;
  p->args.scaleLo = std::ldexp(1.0, (int)(E / N));
  p->args.iscaleLo = std::ldexp(1.0, -(int)(E / N));
  p->args.loShift = t.loShift;
  p->args.timeoutNs = 2000000000ull;
  apply_col_variant(p.get(), owl::default_col_variant(W, H));
  *out = p.release();
}

void plan_destroy(owl_plan* p) {
  DeviceGuard dg(p->device);
  if (p->stream) { cudaStreamSynchronize(p->stream); }
  for (auto& g : p->graphs) { cudaGraphExecDestroy(g.exec); }
  for (int32_t* b : p->bufs) { cudaFree(b); }
  cudaFree(p->F1);
  cudaFree(p->F2);
  cudaFree(p->tableMem);
  cudaFree(p->scratch);
  if (p->stream) { cudaStreamDestroy(p->stream); }
  delete p;
}

// compact words (host) -> balanced digits in buf, on the device (reference expandBits)
void expand_on_device(owl_plan* p, int32_t* buf, const uint32_t* words) {
  ck(cudaMemcpyAsync(p->dwords, words, (size_t)p->nw * sizeof(uint32_t), cudaMemcpyHostToDevice, p->stream),
     "upload words");
  owl::k_pack_summary<true><<<p->packBlocks, owl::kPackThreads, 0, p->stream>>>(p->dwords, nullptr, p->nw, p->E,
                                                                                 p->N, p->packBlk);
  owl::k_pack_chain<<<1, owl::kPackThreads, 0, p->stream>>>(p->packBlk, p->packBlocks, p->packCtl);
  owl::k_expand_digits<<<p->packBlocks, owl::kPackThreads, 0, p->stream>>>(p->dwords, p->nw, p->E, p->N, p->packBlk,
                                                                             p->packCtl, buf);
  ck(cudaGetLastError(), "expand launch");
  sync_and_check(p);
}

// The words as little-endian u64 (the device sum's view) summed mod 2^64 on the host. The pass over
// the readout is bound by host memory bandwidth (17 MB at 8M), so large readouts are split over up
// to 8 threads: about 1 ms instead of 3 on 8 cores.
unsigned long long host_sum64(const uint32_t* words, uint32_t nw) {
  const size_t n2 = nw / 2;
  auto sum_range = [words](size_t lo, size_t hi) {
    unsigned long long acc = 0;
    for (size_t i = lo; i < hi; ++i) {
      uint64_t v;
      std::memcpy(&v, words + 2 * i, sizeof(v));
      acc += v;
    }
    return acc;
  };
  unsigned nt = std::thread::hardware_concurrency();
  nt = (n2 < (1u << 20) || nt < 2) ? 1u : std::min(nt, 8u);
  unsigned long long total = 0;
  if (nt == 1) {
    total = sum_range(0, n2);
  } else {
    std::vector<unsigned long long> part(nt, 0);
    std::vector<std::thread> th;
    th.reserve(nt - 1);
    for (unsigned k = 1; k < nt; ++k) {
      th.emplace_back([&, k] { part[k] = sum_range(n2 * k / nt, n2 * (k + 1) / nt); });
    }
    part[0] = sum_range(0, n2 / nt);
    for (auto& x : th) { x.join(); }
    for (unsigned long long v : part) { total += v; }
  }
  if (nw & 1u) { total += words[nw - 1]; }
  return total;
}

// balanced digits in buf -> compact words (host), on the device (reference compactBits), read back
// with a device checksum compared on the host (reference readChecked, src/Gpu.cpp:677-705)
void compact_on_device(owl_plan* p, const int32_t* buf, uint32_t* words) {
  for (int attempt = 0; attempt < 3; ++attempt) {
    ck(cudaMemsetAsync(p->dwords, 0, (size_t)(p->nw + 2) * sizeof(uint32_t), p->stream), "memset words");
    owl::k_pack_summary<false><<<p->packBlocks, owl::kPackThreads, 0, p->stream>>>(nullptr, buf, p->nw, p->E, p->N,
                                                                                    p->packBlk);
    owl::k_pack_chain<<<1, owl::kPackThreads, 0, p->stream>>>(p->packBlk, p->packBlocks, p->packCtl);
    owl::k_compact_words<<<p->packBlocks, owl::kPackThreads, 0, p->stream>>>(buf, p->nw, p->E, p->N, p->packBlk,
                                                                               p->packCtl, p->dwords);
    owl::k_compact_finish<<<1, 32, 0, p->stream>>>(p->packCtl, p->nw, p->dwords);
    ck(cudaMemsetAsync(p->sum, 0, sizeof(unsigned long long), p->stream), "memset sum");
    owl::k_sum64<<<296, 256, 0, p->stream>>>(reinterpret_cast<const unsigned long long*>(p->dwords), (p->nw + 1) / 2,
                                             p->sum);
    ck(cudaGetLastError(), "compact launch");
    unsigned long long gpuSum = 0;
    owl::PackCtl ctl{};
    ck(cudaMemcpyAsync(&gpuSum, p->sum, sizeof(gpuSum), cudaMemcpyDeviceToHost, p->stream), "read sum");
    ck(cudaMemcpyAsync(&ctl, p->packCtl, sizeof(ctl), cudaMemcpyDeviceToHost, p->stream), "read status");
    ck(cudaMemcpyAsync(words, p->dwords, (size_t)p->nw * sizeof(uint32_t), cudaMemcpyDeviceToHost, p->stream),
       "read words");
    sync_and_check(p);
    if (ctl.error) { fail(OWL_ERR_READ, "digit out of range"); }
    if (host_sum64(words, p->nw) == gpuSum) { return; }
  }
  fail(OWL_ERR_READ, "GPU persistent read errors");
}

}  // namespace

extern "C" {

int owl_abi_version(void) { return OWL_ABI_VERSION; }

const char* owl_error_string(int status) {
  switch (status) {
    case OWL_OK: return "ok";
    case OWL_ERR_ARG: return "bad argument";
    case OWL_ERR_NOMEM: return "out of memory";
    case OWL_ERR_CUDA: return "CUDA error";
    case OWL_ERR_TIMEOUT: return "device wait timeout";
    case OWL_ERR_NODEV: return "no such device";
    case OWL_ERR_READ: return "persistent read errors";
    default: return "unknown status";
  }
}

const char* owl_last_error(void) { return g_lastLiteral ? g_lastLiteral : g_lastError.c_str(); }

int owl_device_count(int* count) {
  return guarded([&] {
    if (!count) { fail(OWL_ERR_ARG, "null count"); }
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    *count = (e == cudaSuccess) ? n : 0;
  });
}

int owl_device_info(int ordinal, char* name, size_t name_len, size_t* total_mem, char* pci, size_t pci_len) {
  return guarded([&] {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, ordinal) != cudaSuccess) { fail(OWL_ERR_NODEV, "no such device"); }
    if (name && name_len) { std::snprintf(name, name_len, "%s", prop.name); }
    if (total_mem) { *total_mem = prop.totalGlobalMem; }
    if (pci && pci_len) { ck(cudaDeviceGetPCIBusId(pci, (int)pci_len, ordinal), "cudaDeviceGetPCIBusId"); }
  });
}

int owl_fft_choose(uint32_t E, double max_bpw, uint32_t* N, uint32_t* W, uint32_t* H) {
  return guarded([&] {
    if (!N || !W || !H) { fail(OWL_ERR_ARG, "null output"); }
    // FFT lengths in increasing order: 5 * 2^(lg-3) (between 2^(lg-1) and 2^lg), then 2^lg
    for (uint32_t lg = 13; lg <= 25; ++lg) {
      for (int five = 1; five >= 0; --five) {
        uint32_t n = five ? 5u << (lg - 3) : 1u << lg;
        double lim = max_bpw > 0 ? max_bpw : kDefaultMaxBpw - 0.3 * (std::log2((double)n) - 18.0);
        if ((double)E / n > lim) { continue; }
        uint32_t w = 0, h = 0;
        if (!owl::shape_for(n, &w, &h)) { continue; }
        *N = n;
        *W = w;
        *H = h;
        return;
      }
    }
    fail(OWL_ERR_ARG, "exponent outside the supported FFT range");
  });
}

int owl_plan_create(int device, uint32_t E, uint32_t W, uint32_t H, owl_plan** out) {
  return guarded([&] { plan_create(device, E, W, H, out); });
}

int owl_plan_destroy(owl_plan* plan) {
  return guarded([&] {
    check_plan(plan);
    plan_destroy(plan);
  });
}

int owl_plan_shape(const owl_plan* plan, uint32_t* N, uint32_t* W, uint32_t* H) {
  return guarded([&] {
    check_plan(plan);
    if (N) { *N = plan->N; }
    if (W) { *W = plan->W; }
    if (H) { *H = plan->H; }
  });
}

int owl_plan_set_timeout(owl_plan* plan, uint64_t ns) {
  return guarded([&] {
    check_plan(plan);
    if (ns == 0) { fail(OWL_ERR_ARG, "timeout must be positive"); }
    plan->args.timeoutNs = ns;
  });
}

int owl_plan_set_split(owl_plan* plan, int flags) {
  return guarded([&] {
    check_plan(plan);
    const uint32_t f = (uint32_t)flags;
    if (f & ~(OWL_SPLIT_COLUMNS | OWL_SPLIT_LINES)) { fail(OWL_ERR_ARG, "unknown split flags"); }
    if ((f & OWL_SPLIT_COLUMNS) && !owl::tc_height((int)plan->H)) {
      fail(OWL_ERR_ARG, "the split-precision column pass needs H = 2048 or 2560");
    }
    if ((f & OWL_SPLIT_LINES) && plan->W != (uint32_t)owl::kLtcW) {
      fail(OWL_ERR_ARG, "the split-precision line pass needs W = 2048");
    }
    DeviceGuard dg(plan->device);
    ck(cudaStreamSynchronize(plan->stream), "cudaStreamSynchronize");
    for (auto& g : plan->graphs) { cudaGraphExecDestroy(g.exec); }
    plan->graphs.clear();
    plan->split = f;
  });
}

int owl_plan_set_column_variant(owl_plan* plan, uint32_t variant) {
  return guarded([&] {
    check_plan(plan);
    const int cv = variant == OWL_COL_AUTO ? owl::default_col_variant(plan->W, plan->H) : (int)variant;
    if (variant > OWL_COL_V16_OCC2 || !owl::col_variant_ok((int)plan->H, cv)) {
      fail(OWL_ERR_ARG, "column variant not built for this height");
    }
    DeviceGuard dg(plan->device);
    ck(cudaStreamSynchronize(plan->stream), "cudaStreamSynchronize");
    for (auto& g : plan->graphs) { cudaGraphExecDestroy(g.exec); }
    plan->graphs.clear();
    apply_col_variant(plan, cv);
  });
}

int owl_plan_column_variant(const owl_plan* plan, uint32_t* variant) {
  return guarded([&] {
    check_plan(plan);
    if (!variant) { fail(OWL_ERR_ARG, "null out"); }
    *variant = (uint32_t)plan->colVariant;
  });
}

int owl_column_variant_supported(uint32_t H, uint32_t variant) {
  return variant >= OWL_COL_V16 && variant <= OWL_COL_V16_OCC2 && owl::col_variant_ok((int)H, (int)variant) ? 1 : 0;
}

int owl_buf_alloc(owl_plan* plan, int32_t** buf) {
  return guarded([&] {
    check_plan(plan);
    if (!buf) { fail(OWL_ERR_ARG, "null out"); }
    DeviceGuard dg(plan->device);
    int32_t* b = nullptr;
    ck(cudaMalloc(&b, (size_t)plan->N * sizeof(int32_t)), "cudaMalloc(words)");
    cudaError_t e = cudaMemsetAsync(b, 0, (size_t)plan->N * sizeof(int32_t), plan->stream);
    if (e != cudaSuccess) {
      cudaFree(b);
      ck(e, "memset(words)");
    }
    plan->bufs.push_back(b);
    *buf = b;
  });
}

int owl_buf_free(owl_plan* plan, int32_t* buf) {
  return guarded([&] {
    check_plan(plan);
    check_buf(plan, buf);
    DeviceGuard dg(plan->device);
    ck(cudaStreamSynchronize(plan->stream), "sync");
    plan->bufs.erase(std::find(plan->bufs.begin(), plan->bufs.end(), buf));
    ck(cudaFree(buf), "cudaFree");
  });
}

int owl_buf_copy(owl_plan* plan, int32_t* dst, const int32_t* src) {
  return guarded([&] {
    check_plan(plan);
    check_buf(plan, dst);
    check_buf(plan, src);
    DeviceGuard dg(plan->device);
    ck(cudaMemcpyAsync(dst, src, (size_t)plan->N * sizeof(int32_t), cudaMemcpyDeviceToDevice, plan->stream),
       "copy");
  });
}

int owl_buf_set(owl_plan* plan, int32_t* buf, uint32_t value) {
  return guarded([&] {
    check_plan(plan);
    check_buf(plan, buf);
    std::vector<uint32_t> w(owl::n_words(plan->E), 0);
    w[0] = value;
    std::vector<int32_t> d(plan->N);
    if (!owl::expand_bits(w.data(), plan->N, plan->E, d.data())) { fail(OWL_ERR_ARG, "expand failed"); }
    DeviceGuard dg(plan->device);
    ck(cudaMemcpyAsync(buf, d.data(), (size_t)plan->N * sizeof(int32_t), cudaMemcpyHostToDevice, plan->stream),
       "upload");
    ck(cudaStreamSynchronize(plan->stream), "sync");
  });
}

int owl_write_digits(owl_plan* plan, int32_t* buf, const int32_t* host) {
  return guarded([&] {
    check_plan(plan);
    check_buf(plan, buf);
    if (!host) { fail(OWL_ERR_ARG, "null host"); }
    DeviceGuard dg(plan->device);
    ck(cudaMemcpyAsync(buf, host, (size_t)plan->N * sizeof(int32_t), cudaMemcpyHostToDevice, plan->stream),
       "upload");
    ck(cudaStreamSynchronize(plan->stream), "sync");
  });
}

int owl_read_digits(owl_plan* plan, const int32_t* buf, int32_t* host) {
  return guarded([&] {
    check_plan(plan);
    check_buf(plan, buf);
    if (!host) { fail(OWL_ERR_ARG, "null host"); }
    DeviceGuard dg(plan->device);
    ck(cudaMemcpyAsync(host, buf, (size_t)plan->N * sizeof(int32_t), cudaMemcpyDeviceToHost, plan->stream),
       "download");
    sync_and_check(plan);
  });
}

int owl_write_words(owl_plan* plan, int32_t* buf, const uint32_t* words) {
  return guarded([&] {
    check_plan(plan);
    check_buf(plan, buf);
    if (!words) { fail(OWL_ERR_ARG, "null words"); }
    if (plan->E % 32 == 0) { fail(OWL_ERR_ARG, "expandBits failed"); }
    DeviceGuard dg(plan->device);
    expand_on_device(plan, buf, words);
  });
}

int owl_read_words(owl_plan* plan, const int32_t* buf, uint32_t* words) {
  return guarded([&] {
    check_plan(plan);
    check_buf(plan, buf);
    if (!words) { fail(OWL_ERR_ARG, "null words"); }
    DeviceGuard dg(plan->device);
    compact_on_device(plan, buf, words);
  });
}

int owl_square(owl_plan* plan, int32_t* out, const int32_t* in, uint32_t n, uint32_t flags) {
  return guarded([&] {
    check_plan(plan);
    check_buf(plan, out);
    check_buf(plan, in);
    if (n == 0) {
      if (out != in) { owl_buf_copy(plan, out, in); }
      return;
    }
    DeviceGuard dg(plan->device);
    run_square(plan, out, in, n, flags & (OWL_SQ_LL | OWL_SQ_MUL3 | OWL_SQ_NO_ROE));
  });
}

int owl_modmul(owl_plan* plan, int32_t* io_a, const int32_t* in_b, int mul3) {
  return guarded([&] {
    check_plan(plan);
    check_buf(plan, io_a);
    check_buf(plan, in_b);
    DeviceGuard dg(plan->device);
    pass1(plan, owl::P1_IN, plan->F2, const_cast<int32_t*>(in_b), 0);
    pass2(plan, owl::P2_FWD, plan->F2, nullptr, plan->F2);
    pass1(plan, owl::P1_IN, plan->F1, io_a, 0);
    pass2(plan, owl::P2_MUL, plan->F1, plan->F2, nullptr);
    pass1_out(plan, io_a, mul3 ? owl::FL_MUL3 : 0);
  });
}

int owl_exp_mul(owl_plan* plan, int32_t* io_a, uint64_t h, const int32_t* in_b) {
  return guarded([&] {
    check_plan(plan);
    check_buf(plan, io_a);
    check_buf(plan, in_b);
    if (io_a == in_b) { fail(OWL_ERR_ARG, "A and B must be different buffers"); }
    DeviceGuard dg(plan->device);
    if (h == 0) {
      ck(cudaMemcpyAsync(io_a, in_b, (size_t)plan->N * sizeof(int32_t), cudaMemcpyDeviceToDevice, plan->stream),
         "copy");
      sync_and_check(plan);
      return;
    }
    // left-to-right binary powering with the base's column spectrum kept in F2
    pass1(plan, owl::P1_IN, plan->F2, io_a, 0);
    pass2(plan, owl::P2_FWD, plan->F2, nullptr, plan->F2);
    pass1(plan, owl::P1_IN, plan->F1, io_a, 0);
    int top = 63;
    while (!((h >> top) & 1)) { --top; }
    for (int b = top - 1; b >= 0; --b) {
      pass2(plan, owl::P2_SQUARE, plan->F1, nullptr, nullptr);
      pass1(plan, owl::P1_FUSED, plan->F1, nullptr, 0);
      if ((h >> b) & 1) {
        pass2(plan, owl::P2_MUL, plan->F1, plan->F2, nullptr);
        pass1(plan, owl::P1_FUSED, plan->F1, nullptr, 0);
      }
    }
    // times B
    pass1(plan, owl::P1_IN, plan->F2, const_cast<int32_t*>(in_b), 0);
    pass2(plan, owl::P2_FWD, plan->F2, nullptr, plan->F2);
    pass2(plan, owl::P2_MUL, plan->F1, plan->F2, nullptr);
    pass1_out(plan, io_a, 0);
    sync_and_check(plan);
  });
}

int owl_is_equal(owl_plan* plan, const int32_t* a, const int32_t* b, int* equal) {
  return guarded([&] {
    check_plan(plan);
    check_buf(plan, a);
    check_buf(plan, b);
    if (!equal) { fail(OWL_ERR_ARG, "null out"); }
    DeviceGuard dg(plan->device);
    int one = 1;
    ck(cudaMemcpyAsync(plan->eq, &one, sizeof(int), cudaMemcpyHostToDevice, plan->stream), "set eq");
    owl::k_is_equal<<<296, 256, 0, plan->stream>>>(a, b, plan->N, plan->eq);
    ck(cudaGetLastError(), "isEqual launch");
    int r = 0;
    ck(cudaMemcpyAsync(&r, plan->eq, sizeof(int), cudaMemcpyDeviceToHost, plan->stream), "read eq");
    sync_and_check(plan);
    *equal = r;
  });
}

int owl_res64(owl_plan* plan, const int32_t* buf, uint64_t* res64) {
  return guarded([&] {
    check_plan(plan);
    check_buf(plan, buf);
    if (!res64) { fail(OWL_ERR_ARG, "null out"); }
    DeviceGuard dg(plan->device);
    owl::k_gather_residue<<<1, 64, 0, plan->stream>>>(buf, plan->N, plan->small);
    ck(cudaGetLastError(), "gather launch");
    int32_t w[64];
    ck(cudaMemcpyAsync(w, plan->small, sizeof(w), cudaMemcpyDeviceToHost, plan->stream), "read residue words");
    sync_and_check(plan);
    bool decided = false;
    uint64_t r = owl::residue_from_wrap(w, plan->N, plan->E, &decided);
    if (!decided) {
      std::vector<uint32_t> words(owl::n_words(plan->E));
      compact_on_device(plan, buf, words.data());
      r = (uint64_t)words[0] | ((words.size() > 1 ? (uint64_t)words[1] : 0) << 32);
    }
    *res64 = r;
  });
}

int owl_sum64(owl_plan* plan, const int32_t* buf, uint64_t* sum) {
  return guarded([&] {
    check_plan(plan);
    check_buf(plan, buf);
    if (!sum) { fail(OWL_ERR_ARG, "null out"); }
    DeviceGuard dg(plan->device);
    ck(cudaMemsetAsync(plan->sum, 0, sizeof(unsigned long long), plan->stream), "memset sum");
    owl::k_sum64<<<296, 256, 0, plan->stream>>>(reinterpret_cast<const unsigned long long*>(buf), plan->N / 2,
                                                 plan->sum);
    ck(cudaGetLastError(), "sum64 launch");
    unsigned long long s = 0;
    ck(cudaMemcpyAsync(&s, plan->sum, sizeof(s), cudaMemcpyDeviceToHost, plan->stream), "read sum");
    sync_and_check(plan);
    *sum = s;
  });
}

int owl_read_roe(owl_plan* plan, float* out, uint32_t cap, uint32_t* n) {
  return guarded([&] {
    check_plan(plan);
    if (!n) { fail(OWL_ERR_ARG, "null out"); }
    DeviceGuard dg(plan->device);
    uint32_t cnt = plan->roePos;
    std::vector<float> host(cnt);
    if (cnt) {
      ck(cudaMemcpyAsync(host.data(), plan->args.roe, cnt * sizeof(float), cudaMemcpyDeviceToHost, plan->stream),
         "read roe");
      ck(cudaMemsetAsync(plan->args.roe, 0, cnt * sizeof(float), plan->stream), "clear roe");
    }
    sync_and_check(plan);
    plan->roePos = 0;
    uint32_t m = std::min(cnt, cap);
    if (out && m) { std::memcpy(out, host.data(), m * sizeof(float)); }
    *n = out ? m : cnt;
  });
}

int owl_sync(owl_plan* plan) {
  return guarded([&] {
    check_plan(plan);
    DeviceGuard dg(plan->device);
    sync_and_check(plan);
  });
}

int owl_plan_stream(owl_plan* plan, void** stream) {
  return guarded([&] {
    check_plan(plan);
    if (!stream) { fail(OWL_ERR_ARG, "null out"); }
    *stream = (void*)plan->stream;
  });
}

int owl_profile_square(owl_plan* plan, int32_t* buf, uint32_t n, uint32_t flags, float* ms, uint32_t* launches) {
  return guarded([&] {
    check_plan(plan);
    check_buf(plan, buf);
    if (!ms || !launches || n == 0 || 2 * n + 1 > kTsCap) { fail(OWL_ERR_ARG, "bad argument"); }
    DeviceGuard dg(plan->device);
    flags &= OWL_SQ_LL | OWL_SQ_MUL3 | OWL_SQ_NO_ROE;
    auto& g = graph_for(plan, buf, buf, n, flags, true);
    ck(cudaGraphLaunch(g.exec, plan->stream), "cudaGraphLaunch");
    if (!(flags & OWL_SQ_NO_ROE)) { plan->roePos = std::max(plan->roePos, std::min(n, kRoeCap)); }
    const size_t cnt = 2 * (size_t)n + 1;
    std::vector<unsigned long long> t0(cnt), t1(cnt);
    ck(cudaMemcpyAsync(t0.data(), plan->args.tsStart, cnt * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                       plan->stream), "read ts");
    ck(cudaMemcpyAsync(t1.data(), plan->args.tsEnd, cnt * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                       plan->stream), "read ts");
    sync_and_check(plan);
    double t2ms = 0, t1ms = 0, tems = 0;
    for (size_t i = 0; i < cnt; ++i) {
      double d = (t1[i] > t0[i]) ? (double)(t1[i] - t0[i]) * 1e-6 : 0.0;
      if (i == 0 || i + 1 == cnt) { tems += d; } else if (i % 2 == 1) { t2ms += d; } else { t1ms += d; }
    }
    ms[0] = (float)t2ms;
    ms[1] = (float)t1ms;
    ms[2] = (float)tems;
    launches[0] = n;
    launches[1] = n - 1;
    launches[2] = 2;
  });
}

}  // extern "C"

struct owl_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::vector<owl_plan*> plans;
  cudaEvent_t fork = nullptr, done = nullptr;
  std::vector<cudaEvent_t> joins;
  struct Entry {
    std::vector<int32_t*> bufs;
    uint32_t n, flags;
    cudaGraphExec_t exec;
  };
  std::vector<Entry> graphs;
};

namespace {

void batch_destroy(owl_batch* b) {
  DeviceGuard dg(b->device);
  if (b->stream) { cudaStreamSynchronize(b->stream); }
  for (auto& g : b->graphs) { cudaGraphExecDestroy(g.exec); }
  for (auto e : b->joins) { cudaEventDestroy(e); }
  if (b->fork) { cudaEventDestroy(b->fork); }
  if (b->done) { cudaEventDestroy(b->done); }
  if (b->stream) { cudaStreamDestroy(b->stream); }
  delete b;
}

cudaGraphExec_t batch_graph(owl_batch* b, int32_t* const* bufs, uint32_t n, uint32_t flags) {
  std::vector<int32_t*> key(bufs, bufs + b->plans.size());
  for (auto& g : b->graphs) {
    if (g.n == n && g.flags == flags && g.bufs == key) { return g.exec; }
  }
  if (b->graphs.size() >= 4) {
    cudaGraphExecDestroy(b->graphs.front().exec);
    b->graphs.erase(b->graphs.begin());
  }
  cudaGraph_t graph = nullptr;
  // plans of one plain shape run as grouped launches (one branch per group of up to kGroupMax, on
  // its first plan's stream); split-precision plans and shapes of one plan get a branch each
  std::vector<std::vector<size_t>> branches;
  {
    std::vector<std::pair<uint64_t, size_t>> order;
    for (size_t i = 0; i < b->plans.size(); ++i) {
      const owl_plan* p = b->plans[i];
      const uint64_t key =
          p->split ? (1ull << 63) | i : ((uint64_t)p->W << 32) | ((uint64_t)p->H << 4) | (uint64_t)p->colVariant;
      order.push_back({key, i});
    }
    std::stable_sort(order.begin(), order.end());
    for (size_t i = 0; i < order.size();) {
      size_t j = i;
      std::vector<size_t> g;
      while (j < order.size() && order[j].first == order[i].first && g.size() < (size_t)owl::kGroupMax) {
        g.push_back(order[j].second);
        ++j;
      }
      branches.push_back(g);
      i = j;
    }
  }
  ck(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
  try {
    ck(cudaEventRecord(b->fork, b->stream), "fork");
    for (size_t bi = 0; bi < branches.size(); ++bi) {
      const auto& g = branches[bi];
      owl_plan* p = b->plans[g[0]];
      ck(cudaStreamWaitEvent(p->stream, b->fork, 0), "fork wait");
      if (g.size() == 1) {
        enqueue_square(p, bufs[g[0]], bufs[g[0]], n, flags, false);
      } else {
        std::vector<owl_plan*> gp;
        std::vector<int32_t*> gb;
        for (size_t i : g) {
          gp.push_back(b->plans[i]);
          gb.push_back(bufs[i]);
        }
        enqueue_square_group(p->stream, gp, gb, n, flags);
      }
      ck(cudaEventRecord(b->joins[bi], p->stream), "join");
      ck(cudaStreamWaitEvent(b->stream, b->joins[bi], 0), "join wait");
    }
  } catch (...) {
    cudaStreamEndCapture(b->stream, &graph);
    if (graph) { cudaGraphDestroy(graph); }
    throw;
  }
  ck(cudaStreamEndCapture(b->stream, &graph), "cudaStreamEndCapture");
  cudaGraphExec_t exec = nullptr;
  cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  ck(e, "cudaGraphInstantiate");
  b->graphs.push_back({key, n, flags, exec});
  return exec;
}

}  // namespace

extern "C" {

int owl_batch_create(int device, uint32_t count, owl_plan* const* plans, owl_batch** out) {
  return guarded([&] {
    if (!out || !plans || count == 0) { fail(OWL_ERR_ARG, "bad argument"); }
    *out = nullptr;
    for (uint32_t i = 0; i < count; ++i) {
      check_plan(plans[i]);
      if (plans[i]->device != device) { fail(OWL_ERR_ARG, "all plans of a batch must be on its device"); }
    }
    DeviceGuard dg(device);
    std::unique_ptr<owl_batch, void (*)(owl_batch*)> b(new owl_batch(), batch_destroy);
    b->device = device;
    b->plans.assign(plans, plans + count);
    ck(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    ck(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "cudaEventCreate");
    ck(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming), "cudaEventCreate");
    b->joins.resize(count);
    for (auto& e : b->joins) { ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate"); }
    *out = b.release();
  });
}

int owl_batch_square(owl_batch* b, int32_t* const* bufs, uint32_t n, uint32_t flags) {
  return guarded([&] {
    if (!b || !bufs) { fail(OWL_ERR_ARG, "bad argument"); }
    if (n == 0) { return; }
    for (size_t i = 0; i < b->plans.size(); ++i) { check_buf(b->plans[i], bufs[i]); }
    DeviceGuard dg(b->device);
    // the batch starts after each plan's pending work, and each plan's later work after the batch
    for (size_t i = 0; i < b->plans.size(); ++i) {
      ck(cudaEventRecord(b->joins[i], b->plans[i]->stream), "record");
      ck(cudaStreamWaitEvent(b->stream, b->joins[i], 0), "wait");
    }
    flags &= OWL_SQ_LL | OWL_SQ_MUL3 | OWL_SQ_NO_ROE;
    cudaGraphExec_t exec = batch_graph(b, bufs, n, flags);
    ck(cudaGraphLaunch(exec, b->stream), "cudaGraphLaunch");
    ck(cudaEventRecord(b->done, b->stream), "record");
    for (owl_plan* p : b->plans) {
      ck(cudaStreamWaitEvent(p->stream, b->done, 0), "wait");
      if (!(flags & OWL_SQ_NO_ROE)) { p->roePos = std::max(p->roePos, std::min(n, kRoeCap)); }
    }
  });
}

int owl_batch_sync(owl_batch* b) {
  return guarded([&] {
    if (!b) { fail(OWL_ERR_ARG, "null batch"); }
    DeviceGuard dg(b->device);
    ck(cudaStreamSynchronize(b->stream), "cudaStreamSynchronize");
    for (owl_plan* p : b->plans) { sync_and_check(p); }
  });
}

int owl_batch_destroy(owl_batch* b) {
  return guarded([&] {
    if (!b) { fail(OWL_ERR_ARG, "null batch"); }
    batch_destroy(b);
  });
}

int owl_probe_wait_timeout(owl_plan* plan) {
  return guarded([&] {
    check_plan(plan);
    DeviceGuard dg(plan->device);
    // an index past the line groups' flags that nothing ever sets: the flags
    // array is followed by the control block, so use the Ctl padding word
    owl::Args a = plan->args;
    a.flags = &plan->args.ctl->pad[0];
    ck(cudaMemsetAsync(a.flags, 0, sizeof(uint32_t), plan->stream), "clear probe flag");
    owl::k_wait_probe<<<1, 32, 0, plan->stream>>>(a, 0);
    ck(cudaGetLastError(), "probe launch");
    sync_and_check(plan);
  });
}

int owl_probe_tc_wait_timeout(owl_plan* plan) {
  return guarded([&] {
    check_plan(plan);
    DeviceGuard dg(plan->device);
    owl::k_tc_wait_probe<<<1, 32, 0, plan->stream>>>(plan->args);
    ck(cudaGetLastError(), "probe launch");
    sync_and_check(plan);
  });
}

}  // extern "C"
