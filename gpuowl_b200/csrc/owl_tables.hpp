// owl_tables.hpp -- host-side tables for one (E, W, H) shape: twiddles, the
// IBDWT weights factored per column and per line, and the big-word data.
//
// Word model (reference src/state.h:14-17): N = 2 W H words, step = N - E mod N,
// extra(k) = step k mod N, word k is big (one more bit) iff extra(k) < E mod N,
// weight(k) = 2^(extra(k)/N) (src/Gpu.cpp:42-56). Complex element j = j2 + H j1
// (line j2, column j1) holds words 2j and 2j+1 (src/Gpu.cpp:40 kAt), so
// extra(2j+e) = (X1[j1] + X2[2 j2 + e]) mod N with X1 = step 2H j1 mod N and
// X2 = step (2 j2 + e) mod N; the weight is the product of the two table
// factors, halved when X1 + X2 >= N.
//
// Twiddles are evaluated in long double after an exact octant reduction of the
// angle and rounded once to double (the reference builds its tables in long
// double too, src/TrigBufCache.cpp:22-120).
#pragma once
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <utility>
#include <vector>

#include "owl_dft.cuh"

namespace owl {

struct HostC {
  double x, y;
};

// cos and sin of 2 pi k / n
inline void root_ld(uint64_t n, uint64_t k, long double* c, long double* s) {
  const long double PI_L = 3.141592653589793238462643383279502884L;
  uint64_t q = 8 * n, p = 8 * (k % n);
  bool negS = false, negC = false, swp = false;
  if (2 * p > q) { p = q - p; negS = true; }
  if (4 * p > q) { p = q / 2 - p; negC = true; }
  if (8 * p > q) { p = q / 4 - p; swp = true; }
  long double a = 2.0L * PI_L * (long double)p / (long double)q;
  long double cc = cosl(a), ss = sinl(a);
  if (swp) { std::swap(cc, ss); }
  if (negC) { cc = -cc; }
  if (negS) { ss = -ss; }
  *c = cc;
  *s = ss;
}

// forward root w_n^k = exp(-2 pi i k / n)
inline HostC root(uint64_t n, uint64_t k) {
  long double c, s;
  root_ld(n, k, &c, &s);
  return HostC{(double)c, (double)-s};
}

inline bool is_pow2(uint32_t x) { return x && !(x & (x - 1)); }
inline uint32_t log2u(uint32_t x) {
  uint32_t r = 0;
  while ((1u << r) < x) { ++r; }
  return r;
}

// the stage twiddle tables of a length-n line FFT in the tw_offsets(n, rl) layout
inline std::vector<HostC> stage_tables(uint32_t n, uint32_t rl, uint32_t r1f = 0, uint32_t vmax = 16) {
  const TwOffsets o = tw_offsets((int)n, (int)rl, (int)r1f, (int)vmax);
  const uint32_t r1 = plan_r1(n, rl, r1f, vmax), m1 = plan_m1(n, rl, r1f, vmax), m2 = plan_m2(n, rl, r1f, vmax);
  std::vector<HostC> t(o.total);
  auto fill = [&](int off, uint32_t R, uint32_t NS) {
    for (uint32_t r = 0; r < R; ++r) {
      for (uint32_t k = 0; k < NS; ++k) { t[off + r * NS + k] = root((uint64_t)R * NS, (uint64_t)r * k); }
    }
  };
  if (m1 > 1) { fill(o.aM1, m1, r1); }
  if (m2 > 1) { fill(o.aM2, m2, r1 * m1); }
  fill(o.aRL, rl, n / rl);
  if (m2 > 1) { fill(o.bM2, m2, rl); }
  if (m1 > 1) { fill(o.bM1, m1, rl * m2); }
  fill(o.bR1, r1, n / r1);
  return t;
}

// the column FFT's stage tables for a column variant (its values a thread V: tw_offsets(H, V/2, 0, V))
inline std::vector<HostC> col_stage_tables(uint32_t H, int variant) {
  const uint32_t v = (uint32_t)col_vpt(variant);
  return stage_tables(H, v / 2, 0, v);
}

// The column variant a plan of shape W x H starts with: the fastest of the variants built for H as
// measured on B200 by gpuowl_b200.tune --variants (time per squaring of 1,000-squaring blocks; the
// reference's built-in tune defaults play the same part, src/TuneEntry.cpp); owl_plan_set_column_variant
// overrides it. 8 values a thread won at 128 x 256 (10.4 against 10.7 us), 256 x 256 (10.8-10.9
// against 11.6-11.8) and 512 x 512 (14.1 against 14.3); two CTAs per SM at 4096 x 2560 (381.3-381.6
// against 384.0-384.8); every other measured shape keeps 16 values a thread.
inline int default_col_variant(uint32_t W, uint32_t H) {
  if ((W == 128 && H == 256) || (W == 256 && H == 256) || (W == 512 && H == 512)) { return COL_V8; }
  if (W == 4096 && H == 2560) { return COL_V16_OCC2; }
  return COL_V16;
}

struct Tables {
  uint32_t E = 0, N = 0, W = 0, H = 0, hN = 0, loShift = 0;
  std::vector<HostC> twW, twH, rootH, twLo, twHi;
  std::vector<double> wt1, iwt1, wt2, iwt2;
  std::vector<uint32_t> x1, x2;
  std::vector<uint32_t> p1masks;  // (bigmask, wrapmask) per (line group, pass-1 thread)
};

// lines per pass-1 block; the width FFT's cross-line radix is 16 / kLinesPerBlock
constexpr uint32_t kLinesPerBlock = 2;

// Shapes the library supports: W a power of two in [64, 4096]; H a power of two in
// [64, 4096], or 5 * 2^k in {640, 1280, 2560} (a radix-5 stage in the column FFT).
inline bool h_supported(uint32_t H) {
  return (is_pow2(H) && H >= 64 && H <= 4096) || H == 640 || H == 1280 || H == 2560;
}
inline bool shape_supported(uint32_t W, uint32_t H) { return is_pow2(W) && W >= 64 && W <= 4096 && h_supported(H); }

// The default W x H split of an FFT of n words: for 2^lg, W = 2^((lg-1)/2) <= H;
// for 5 * 2^k the supported H that makes the shape closest to square (ties to the larger H).
inline bool shape_for(uint32_t n, uint32_t* W, uint32_t* H) {
  const uint32_t hN = n / 2;
  if (is_pow2(n)) {
    const uint32_t w = 1u << ((log2u(n) - 1) / 2), h = hN / w;
    if (!shape_supported(w, h)) { return false; }
    *W = w;
    *H = h;
    return true;
  }
  bool found = false;
  double best = 0;
  for (uint32_t h : {2560u, 1280u, 640u}) {
    if (hN % h) { continue; }
    const uint32_t w = hN / h;
    if (!shape_supported(w, h)) { continue; }
    const double d = std::fabs(std::log((double)w / h));
    if (!found || d < best - 1e-9) {
      found = true;
      best = d;
      *W = w;
      *H = h;
    }
  }
  return found;
}

// The big-word and wrap bits of every pass-1 thread's words: thread t of line group g holds
// column j1 = t + (W/RL) r (r < RL = 16/R) of lines j2 = g R + ll (ll < R), words e = 0, 1;
// bit (r R + ll) 2 + e. With X = X1[j1] + X2[2 j2 + e], the weight wraps when X >= N and the
// word is big when X mod N < E mod N.
inline std::vector<uint32_t> word_masks(uint32_t E, uint32_t W, uint32_t H, const uint32_t* x1, const uint32_t* x2) {
  const uint32_t R = kLinesPerBlock, RL = 16 / R, T = R * W / 16, G = H / R, N = 2 * W * H;
  std::vector<uint32_t> m(2 * (size_t)G * T);
  for (uint32_t g = 0; g < G; ++g) {
    for (uint32_t th = 0; th < T; ++th) {
      uint32_t big = 0, wrap = 0;
      for (uint32_t r = 0; r < RL; ++r) {
        const uint32_t j1 = th + (W / RL) * r;
        for (uint32_t ll = 0; ll < R; ++ll) {
          const uint32_t j2 = g * R + ll;
          for (uint32_t e = 0; e < 2; ++e) {
            const uint32_t bit = (r * R + ll) * 2 + e;
            const uint32_t X = x1[j1] + x2[2 * j2 + e];
            const bool w = X >= N;
            if (w) { wrap |= 1u << bit; }
            if ((w ? X - N : X) < E % N) { big |= 1u << bit; }
          }
        }
      }
      m[2 * ((size_t)g * T + th)] = big;
      m[2 * ((size_t)g * T + th) + 1] = wrap;
    }
  }
  return m;
}

inline Tables make_tables(uint32_t E, uint32_t W, uint32_t H) {
  if (!shape_supported(W, H)) { throw std::invalid_argument("unsupported W x H shape"); }
  Tables t;
  t.E = E;
  t.W = W;
  t.H = H;
  t.hN = W * H;
  t.N = 2 * W * H;
  const uint32_t N = t.N;
  t.loShift = (log2u(t.hN) + 1) / 2;
  t.twW = stage_tables(W, 16 / kLinesPerBlock);
  t.twH = col_stage_tables(H, COL_V16);
  t.rootH.resize(H);
  for (uint32_t i = 0; i < H; ++i) { t.rootH[i] = root(H, i); }
  uint32_t S = 1u << t.loShift;
  t.twLo.resize(S);
  for (uint32_t i = 0; i < S; ++i) { t.twLo[i] = root(t.hN, i); }
  uint32_t nHi = (t.hN + S - 1) / S;
  t.twHi.resize(nHi);
  for (uint32_t i = 0; i < nHi; ++i) { t.twHi[i] = root(t.hN, (uint64_t)i * S); }

  const uint64_t step = N - (E % N);
  t.x1.resize(W);
  t.wt1.resize(W);
  t.iwt1.resize(W);
  for (uint32_t j1 = 0; j1 < W; ++j1) {
    uint32_t X = (uint32_t)((step * 2 * H * (uint64_t)j1) % N);
    t.x1[j1] = X;
    t.wt1[j1] = (double)exp2l((long double)X / N);
    t.iwt1[j1] = (double)exp2l(-(long double)X / N);
  }
  t.x2.resize(2 * H);
  t.wt2.resize(2 * H);
  t.iwt2.resize(2 * H);
  const long double norm = 1.0L / (4.0L * (long double)t.hN);
  for (uint32_t i = 0; i < 2 * H; ++i) {
    uint32_t X = (uint32_t)((step * (uint64_t)i) % N);
    t.x2[i] = X;
    t.wt2[i] = (double)exp2l((long double)X / N);
    t.iwt2[i] = (double)(exp2l(-(long double)X / N) * norm);
  }
  t.p1masks = word_masks(E, W, H, t.x1.data(), t.x2.data());
  return t;
}

}  // namespace owl
