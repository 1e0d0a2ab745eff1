// owl_noalloc.cu -- owl_square_noalloc: n squarings of a caller's word buffer
// with no allocation at all.
//
// Some callers of this library cannot allocate device memory: a host that has
// handed all device memory to its own pool allocator (a cudaMalloc would fail,
// or take memory the pool counts on), a real-time loop that must not enter the
// allocator (cudaMalloc and cudaFree can block on the device and take an
// unbounded time), and plug-ins whose host forbids them to allocate. For them
// this entry point keeps every piece of scratch the squaring needs -- the FFT
// state, the carry rows and flags, the control word, the twiddle and weight
// tables -- in one file-scope device array of a fixed size, so the library
// never calls cudaMalloc, cudaFree or any other allocating routine on this path
// (the tables are computed on the device).
//
// Limits and rules:
//   - N = 2 W H <= kNoAllocMaxWords (W <= 128, H <= 256) and at most 19 bits
//     per word (exponents up to about 1.24 million); anything else returns
//     OWL_ERR_ARG;
//   - the array (kNoAllocScratchBytes) lives on every GPU that loads libowl
//     until the process exits;
//   - every call shares that one array and it keeps the last call's contents;
//     the call clears what must start at zero, but calls that overlap on the
//     GPU (other streams, other host threads) race on it and corrupt each other;
//   - the first call on a device looks up the array's device address (with
//     that device current) and caches it; make that first call before any
//     stream capture;
//   - the call waits for its work on `stream` and reads back the device-side
//     status and the round-off maximum.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <cstdint>
#include <mutex>

#include "owl.h"
#include "owl_kernels.cuh"

namespace owl_detail {
// owl_last_error() text for this thread; takes a string literal, allocates nothing
void set_error_literal(const char* msg);
}

namespace {

constexpr uint32_t kNoAllocMaxWords = 1u << 16;
constexpr uint32_t kNoAllocMaxW = 128;
constexpr uint32_t kNoAllocMaxH = 256;
constexpr size_t kNoAllocScratchBytes = 1u << 20;
constexpr int kR = 2;
constexpr uint32_t kRoeSlots = 16;
constexpr double kNoAllocMaxBpw = 19.0;
// a round-off above this means the FFT was too short for the exponent; the call fails
constexpr float kNoAllocMaxRoe = 0.4f;

// The scratch array. Its name is a host-side stand-in in host code: kernels
// get the address looked up with cudaGetSymbolAddress, never &g_noalloc_scratch.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

size_t up256(size_t x) { return (x + 255) & ~size_t(255); }

// byte layout of the scratch for one shape; returns the total size
struct Layout {
  size_t F, shuttle, pending, flags, ctl, roe, twW, twH, rootH, twLo, twHi, wt1, iwt1, x1, wt2, iwt2, x2, masks, total;
};
Layout layout(uint32_t W, uint32_t H, uint32_t loShift) {
  const uint32_t hN = W * H, G = H / kR;
  const int vH = owl::col_vpt(owl::COL_V16);  // the default column variant's kernels
  const int twWn = owl::tw_offsets((int)W, 16 / kR).total, twHn = owl::tw_offsets((int)H, vH / 2, 0, vH).total;
  Layout L{};
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t at = o; o = up256(o + bytes); return at; };
  L.F = take((size_t)hN * sizeof(owl::C));
  L.shuttle = take((size_t)G * W * sizeof(long long));
  L.pending = take(2 * owl::kPendingCap * sizeof(long long));
  L.flags = take(G * sizeof(uint32_t));
  L.ctl = take(sizeof(owl::Ctl));
  L.roe = take(kRoeSlots * sizeof(float));
  L.twW = take(twWn * sizeof(owl::C));
  L.twH = take(twHn * sizeof(owl::C));
  L.rootH = take(H * sizeof(owl::C));
  L.twLo = take((size_t(1) << loShift) * sizeof(owl::C));
  L.twHi = take((hN >> loShift) * sizeof(owl::C) + sizeof(owl::C));
  L.wt1 = take(W * sizeof(double));
  L.iwt1 = take(W * sizeof(double));
  L.x1 = take(W * sizeof(uint32_t));
  L.wt2 = take(2 * H * sizeof(double));
  L.iwt2 = take(2 * H * sizeof(double));
  L.x2 = take(2 * H * sizeof(uint32_t));
  L.masks = take((size_t)G * (kR * W / 16) * sizeof(uint2));
  L.total = o;
  return L;
}

__device__ owl::C droot(uint32_t n, uint64_t k) {
  double s, c;
  sincospi(2.0 * (double)(k % n) / (double)n, &s, &c);
  return owl::mk(c, -s);
}

// Fills the tables of (E, W, H) in the scratch (same layouts as the host-built
// tables of owl_plan_create), and clears the carry-chain control state.
__global__ void k_noalloc_tables(owl::Args a, uint32_t twWn, uint32_t twHn) {
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
  const uint32_t W = a.W, H = a.H, N = a.N;
  auto stage = [&](owl::C* tab, uint32_t n, uint32_t rl, uint32_t vmax, uint32_t i) {
    const owl::TwOffsets o = owl::tw_offsets((int)n, (int)rl, 0, (int)vmax);
    const uint32_t r1 = owl::plan_r1(n, rl, 0, vmax), m1 = owl::plan_m1(n, rl, 0, vmax),
                   m2 = owl::plan_m2(n, rl, 0, vmax);
    // which stage table does entry i belong to
    int off;
    uint32_t R, NS;
    if (m1 > 1 && (int)i >= o.aM1 && (int)i < o.aM2) { off = o.aM1; R = m1; NS = r1; }
    else if (m2 > 1 && (int)i >= o.aM2 && (int)i < o.aRL) { off = o.aM2; R = m2; NS = r1 * m1; }
    else if ((int)i >= o.aRL && (int)i < o.bM2) { off = o.aRL; R = rl; NS = n / rl; }
    else if (m2 > 1 && (int)i >= o.bM2 && (int)i < o.bM1) { off = o.bM2; R = m2; NS = rl; }
    else if (m1 > 1 && (int)i >= o.bM1 && (int)i < o.bR1) { off = o.bM1; R = m1; NS = rl * m2; }
    else { off = o.bR1; R = r1; NS = n / r1; }
    const uint32_t e = i - off, r = e / NS, k = e % NS;
    tab[i] = droot(R * NS, (uint64_t)r * k);
  };
  const uint32_t vH = (uint32_t)owl::col_vpt(owl::COL_V16);
  for (uint32_t i = tid; i < twWn; i += nth) { stage(const_cast<owl::C*>(a.twW), W, 16 / kR, 16, i); }
  for (uint32_t i = tid; i < twHn; i += nth) { stage(const_cast<owl::C*>(a.twH), H, vH / 2, vH, i); }
  for (uint32_t i = tid; i < H; i += nth) { const_cast<owl::C*>(a.rootH)[i] = droot(H, i); }
  const uint32_t S = 1u << a.loShift;
  for (uint32_t i = tid; i < S; i += nth) { const_cast<owl::C*>(a.twLo)[i] = droot(a.hN, i); }
  for (uint32_t i = tid; i <= (a.hN >> a.loShift); i += nth) {
    const_cast<owl::C*>(a.twHi)[i] = droot(a.hN, (uint64_t)i << a.loShift);
  }
  const uint64_t step = N - (a.E % N);
  for (uint32_t j1 = tid; j1 < W; j1 += nth) {
    uint32_t X = (uint32_t)((step * 2 * H * (uint64_t)j1) % N);
    const_cast<uint32_t*>(a.x1)[j1] = X;
    const_cast<double*>(a.wt1)[j1] = exp2((double)X / N);
    const_cast<double*>(a.iwt1)[j1] = exp2(-(double)X / N);
  }
  for (uint32_t i = tid; i < 2 * H; i += nth) {
    uint32_t X = (uint32_t)((step * (uint64_t)i) % N);
    const_cast<uint32_t*>(a.x2)[i] = X;
    const_cast<double*>(a.wt2)[i] = exp2((double)X / N);
    const_cast<double*>(a.iwt2)[i] = exp2(-(double)X / N) / (4.0 * (double)a.hN);
  }
  // pass-1 word classes (the host-side word_masks, from the same X1 / X2 formulas)
  {
    constexpr uint32_t RL = 16 / kR;
    const uint32_t T = kR * W / 16, G = H / kR;
    for (uint32_t i = tid; i < G * T; i += nth) {
      const uint32_t g = i / T, th = i % T;
      uint32_t big = 0, wrap = 0;
      for (uint32_t r = 0; r < RL; ++r) {
        const uint32_t j1 = th + (W / RL) * r;
        const uint32_t X1 = (uint32_t)((step * 2 * H * (uint64_t)j1) % N);
        for (uint32_t ll = 0; ll < kR; ++ll) {
          for (uint32_t e = 0; e < 2; ++e) {
            const uint32_t bit = (r * kR + ll) * 2 + e;
            const uint32_t X = X1 + (uint32_t)((step * (uint64_t)(2 * (g * kR + ll) + e)) % N);
            const bool w = X >= N;
            if (w) { wrap |= 1u << bit; }
            if ((w ? X - N : X) < a.E % N) { big |= 1u << bit; }
          }
        }
      }
      const_cast<uint2*>(a.p1masks)[i] = make_uint2(big, wrap);
    }
  }
  for (uint32_t i = tid; i < H / kR; i += nth) { a.flags[i] = 0; }
  // carry words: 0 = consumed (a call that stopped on an error may have left some set)
  for (uint32_t i = tid; i < (H / kR) * W; i += nth) { a.shuttle[i] = 0; }
  if (tid == 0) {
    a.ctl->ticket = 0;
    a.ctl->error = 0;
    a.ctl->npending = 0;
  }
  for (uint32_t i = tid; i < kRoeSlots; i += nth) { a.roe[i] = 0.0f; }
}

template <int W> void p1(const owl::Args& a, int mode, owl::C* F, int32_t* words, int flags, cudaStream_t s) {
  constexpr int T = kR * W / 16;
  const size_t sm = (size_t)kR * owl::p1_line_stride<W, kR>() * sizeof(owl::C);
  const dim3 grid(a.H / kR);
  const int slot = (int)(kRoeSlots - 1);
  if (mode == owl::P1_IN) {
    owl::k_pass1<W, kR, owl::P1_IN><<<grid, T, sm, s>>>(a, F, words, slot, flags, -1);
  } else if (mode == owl::P1_FUSED) {
    owl::k_pass1<W, kR, owl::P1_FUSED><<<grid, T, sm, s>>>(a, F, words, slot, flags, -1);
  } else {
    owl::k_pass1<W, kR, owl::P1_OUT><<<grid, T, sm, s>>>(a, F, words, slot, flags, -1);
  }
}
template <int H> void p2(const owl::Args& a, owl::C* F, cudaStream_t s) {
  const size_t sm = 2 * (size_t)owl::p2_col_stride<H>() * sizeof(owl::C);
  owl::k_pass2<H, kR, owl::P2_SQUARE><<<a.W / 2, H / 8, sm, s>>>(a, F, nullptr, nullptr, -1);
}

void launch_p1(const owl::Args& a, int mode, owl::C* F, int32_t* words, int flags, cudaStream_t s) {
  if (a.W == 64) { p1<64>(a, mode, F, words, flags, s); } else { p1<128>(a, mode, F, words, flags, s); }
}
void launch_p2(const owl::Args& a, owl::C* F, cudaStream_t s) {
  if (a.H == 64) { p2<64>(a, F, s); } else if (a.H == 128) { p2<128>(a, F, s); } else { p2<256>(a, F, s); }
}

int fail(int code, const char* msg) {
  owl_detail::set_error_literal(msg);
  return code;
}

}  // namespace

extern "C" int owl_square_noalloc(int device, uint32_t E, uint32_t W, uint32_t H, int32_t* words, uint32_t n,
                                  uint32_t flags, void* stream) {
  if (!words) { return fail(OWL_ERR_ARG, "null word buffer"); }
  if (W == 0 && H == 0) {
    // smallest shape of this path with at most 19 bits per word
    const uint32_t shapes[4][2] = {{64, 64}, {64, 128}, {128, 128}, {128, 256}};
    for (const auto& sh : shapes) {
      if ((double)E / (2.0 * sh[0] * sh[1]) <= kNoAllocMaxBpw) {
        W = sh[0];
        H = sh[1];
        break;
      }
    }
    if (W == 0) { return fail(OWL_ERR_ARG, "no-alloc path: exponent too large for its fixed scratch (N <= 65536)"); }
  }
  if ((W != 64 && W != 128) || W > kNoAllocMaxW) { return fail(OWL_ERR_ARG, "no-alloc path: W must be 64 or 128"); }
  if ((H != 64 && H != 128 && H != 256) || H > kNoAllocMaxH) {
    return fail(OWL_ERR_ARG, "no-alloc path: H must be 64, 128 or 256");
  }
  const uint32_t N = 2 * W * H;
  if (N > kNoAllocMaxWords) { return fail(OWL_ERR_ARG, "no-alloc path: FFT larger than its fixed scratch (N <= 65536)"); }
  // the same 19-bit limit as the automatic choice: these small transforms are not shown to keep the
  // round-off safe above it
  if (E < 1000 || E % 2 == 0 || E / N < 8 || (double)E / N > kNoAllocMaxBpw) {
    return fail(OWL_ERR_ARG, "no-alloc path: exponent out of range for this FFT (8 to 19 bits per word)");
  }
  if (device < 0 || device >= kMaxDevices) { return fail(OWL_ERR_NODEV, "device ordinal out of range"); }
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) { return fail(OWL_ERR_CUDA, "cudaGetDevice failed"); }
  if (prev != device && cudaSetDevice(device) != cudaSuccess) { return fail(OWL_ERR_NODEV, "cudaSetDevice failed"); }
  struct Restore {
    int prev, dev;
    ~Restore() { if (prev >= 0 && prev != dev) { cudaSetDevice(prev); } }
  } restore{prev, device};
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (s != nullptr && s != cudaStreamLegacy && s != cudaStreamPerThread) {
    int sdev = -1;
    if (cudaStreamGetDevice(s, &sdev) != cudaSuccess) { return fail(OWL_ERR_ARG, "no-alloc path: invalid stream"); }
    if (sdev != device) { return fail(OWL_ERR_ARG, "no-alloc path: stream belongs to another device"); }
  }

  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[device]) {
      void* ptr = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess || !ptr) { return fail(OWL_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed"); }
      g_scratch_ptr[device] = ptr;
    }
    base = static_cast<unsigned char*>(g_scratch_ptr[device]);
  }

  uint32_t hN = W * H, loShift = 0;
  while ((1u << loShift) < hN) { ++loShift; }
  loShift = (loShift + 1) / 2;
  const Layout L = layout(W, H, loShift);
  if (L.total > kNoAllocScratchBytes) { return fail(OWL_ERR_ARG, "no-alloc path: shape does not fit the scratch"); }

  owl::Args a{};
  a.twW = reinterpret_cast<const owl::C*>(base + L.twW);
  a.twH = reinterpret_cast<const owl::C*>(base + L.twH);
  a.rootH = reinterpret_cast<const owl::C*>(base + L.rootH);
  a.twLo = reinterpret_cast<const owl::C*>(base + L.twLo);
  a.twHi = reinterpret_cast<const owl::C*>(base + L.twHi);
  a.wt1 = reinterpret_cast<const double*>(base + L.wt1);
  a.iwt1 = reinterpret_cast<const double*>(base + L.iwt1);
  a.x1 = reinterpret_cast<const uint32_t*>(base + L.x1);
  a.wt2 = reinterpret_cast<const double*>(base + L.wt2);
  a.iwt2 = reinterpret_cast<const double*>(base + L.iwt2);
  a.x2 = reinterpret_cast<const uint32_t*>(base + L.x2);
  a.p1masks = reinterpret_cast<const uint2*>(base + L.masks);
  a.shuttle = reinterpret_cast<long long*>(base + L.shuttle);
  a.pending = reinterpret_cast<long long*>(base + L.pending);
  a.flags = reinterpret_cast<uint32_t*>(base + L.flags);
  a.ctl = reinterpret_cast<owl::Ctl*>(base + L.ctl);
  a.roe = reinterpret_cast<float*>(base + L.roe);
  a.E = E;
  a.N = N;
  a.W = W;
  a.H = H;
  a.hN = hN;
  a.bitsLo = E / N;
  a.eModN = E % N;
  a.scaleLo = std::ldexp(1.0, (int)(E / N));
  a.iscaleLo = std::ldexp(1.0, -(int)(E / N));
  a.loShift = loShift;
  a.timeoutNs = 2000000000ull;
  owl::C* F = reinterpret_cast<owl::C*>(base + L.F);

  const int vH = owl::col_vpt(owl::COL_V16);  // the default column variant's kernels
  const int twWn = owl::tw_offsets((int)W, 16 / kR).total, twHn = owl::tw_offsets((int)H, vH / 2, 0, vH).total;
  k_noalloc_tables<<<64, 256, 0, s>>>(a, (uint32_t)twWn, (uint32_t)twHn);
  if (n > 0) {
    const int ll = (flags & OWL_SQ_LL) ? owl::FL_LL : 0;
    const int mul3 = (flags & OWL_SQ_MUL3) ? owl::FL_MUL3 : 0;
    launch_p1(a, owl::P1_IN, F, words, 0, s);
    for (uint32_t k = 0; k < n; ++k) {
      launch_p2(a, F, s);
      launch_p1(a, (k + 1 < n) ? owl::P1_FUSED : owl::P1_OUT, F, words, (k + 1 < n) ? ll : (ll | mul3), s);
    }
    owl::k_carry_fixup<<<1, 32, 0, s>>>(a, words);
  }
  if (cudaGetLastError() != cudaSuccess) { return fail(OWL_ERR_CUDA, "launch failed"); }
  // the device-side status word and the round-off slots are read back in one copy (the control
  // word comes first in the scratch, the round-off slots right after it)
  static_assert(sizeof(owl::Ctl) <= 256, "control word layout");
  unsigned char back[256 + kRoeSlots * sizeof(float)];
  if (L.roe != L.ctl + 256 ||
      cudaMemcpyAsync(back, base + L.ctl, sizeof(back), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess) {
    return fail(OWL_ERR_CUDA, "synchronize failed");
  }
  owl::Ctl ctl;
  float roe[kRoeSlots];
  std::memcpy(&ctl, back, sizeof(ctl));
  std::memcpy(roe, back + 256, sizeof(roe));
  if (ctl.error & owl::DEVERR_WAIT) { return fail(OWL_ERR_TIMEOUT, "device-side carry wait timed out"); }
  if (ctl.error & owl::DEVERR_PENDING) {
    return fail(OWL_ERR_CUDA, "no-alloc path: the leftover-carry queue of the last pass overflowed");
  }
  if (n > 0 && !(roe[kRoeSlots - 1] <= kNoAllocMaxRoe)) {
    return fail(OWL_ERR_ARG, "no-alloc path: round-off above 0.4, the FFT is too short for this exponent");
  }
  return OWL_OK;
}
