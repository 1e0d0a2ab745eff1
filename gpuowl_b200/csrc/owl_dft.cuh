// owl_dft.cuh -- FP64 complex arithmetic and small DFTs in registers, plus the
// shared-memory Stockham stage helpers used by the two pass kernels.
//
// Conventions: forward DFT X[k] = sum_n x[n] w^(nk) with w = exp(-2 pi i / n);
// INV selects w = exp(+2 pi i / n) (unnormalised). All small DFTs take and
// return natural order.
#pragma once
#include <cstdint>
#include "owl_compat.cuh"

namespace owl {

typedef double2 C;

__device__ __forceinline__ C mk(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ C cneg(C a) { return mk(-a.x, -a.y); }
__device__ __forceinline__ C cconj(C a) { return mk(a.x, -a.y); }
__device__ __forceinline__ C cmul(C a, C b) {
  return mk(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ C cmulc(C a, C b) {
  return mk(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ C csq(C a) { return mk(fma(a.x, a.x, -a.y * a.y), 2.0 * a.x * a.y); }
// multiply by i
__device__ __forceinline__ C cmuli(C a) { return mk(-a.y, a.x); }
// multiply by -i
__device__ __forceinline__ C cmulmi(C a) { return mk(a.y, -a.x); }

template <bool INV> __device__ __forceinline__ C cmulw(C a, C w) { return INV ? cmulc(a, w) : cmul(a, w); }

// w4 = -i (forward) / +i (inverse)
template <bool INV> __device__ __forceinline__ C mul_w4(C a) { return INV ? cmuli(a) : cmulmi(a); }

constexpr double kC1 = 0.92387953251128675613;  // cos(pi/8)
constexpr double kS1 = 0.38268343236508977173;  // sin(pi/8)
constexpr double kSQ = 0.70710678118654752440;  // sqrt(1/2)

// a * w16^M, M a compile-time constant in [0, 16)
template <bool INV, int M> __device__ __forceinline__ C mul_w16(C a) {
  constexpr int m = M & 15;
  if constexpr (m == 0) {
    return a;
  } else if constexpr (m == 8) {
    return cneg(a);
  } else if constexpr (m == 4) {
    return mul_w4<INV>(a);
  } else if constexpr (m == 12) {
    return mul_w4<!INV>(a);
  } else if constexpr (m == 2 || m == 6 || m == 10 || m == 14) {
    // (+-1 +- i) sqrt(1/2): forward w16^2 = (1 - i)/sqrt2
    constexpr int q = m / 2;  // 1,3,5,7 -> w8^q
    C b = a;
    if constexpr (q == 3) { b = mul_w4<INV>(a); }
    if constexpr (q == 5) { b = cneg(a); }
    if constexpr (q == 7) { b = mul_w4<!INV>(a); }
    // b * w8^1
    if constexpr (!INV) {
      return mk((b.x + b.y) * kSQ, (b.y - b.x) * kSQ);
    } else {
      return mk((b.x - b.y) * kSQ, (b.x + b.y) * kSQ);
    }
  } else {
    // odd m: full complex multiply by (cos 2pi m/16, -+sin 2pi m/16)
    constexpr int k = m % 4;     // 1 or 3
    constexpr int quad = m / 4;  // rotation by w4^quad
    constexpr double c = (k == 1) ? kC1 : kS1;
    constexpr double s = (k == 1) ? kS1 : kC1;
    C b = a;
    if constexpr (quad == 1) { b = mul_w4<INV>(a); }
    if constexpr (quad == 2) { b = cneg(a); }
    if constexpr (quad == 3) { b = mul_w4<!INV>(a); }
    // forward: (c - i s), inverse: (c + i s)
    if constexpr (!INV) {
      return mk(fma(b.x, c, b.y * s), fma(b.y, c, -b.x * s));
    } else {
      return mk(fma(b.x, c, -b.y * s), fma(b.y, c, b.x * s));
    }
  }
}

// a * w8^r for r known after unrolling
template <bool INV> __device__ __forceinline__ C mul_w8(C a, int r) {
  switch (r & 7) {
    case 0: return a;
    case 1: return mul_w16<INV, 2>(a);
    case 2: return mul_w16<INV, 4>(a);
    case 3: return mul_w16<INV, 6>(a);
    case 4: return mul_w16<INV, 8>(a);
    case 5: return mul_w16<INV, 10>(a);
    case 6: return mul_w16<INV, 12>(a);
    default: return mul_w16<INV, 14>(a);
  }
}

template <bool INV> __device__ __forceinline__ void dft2(C* v) {
  C a = v[0];
  v[0] = cadd(a, v[1]);
  v[1] = csub(a, v[1]);
}

template <bool INV> __device__ __forceinline__ void dft4s(C& x0, C& x1, C& x2, C& x3) {
  C a = cadd(x0, x2), b = csub(x0, x2), c = cadd(x1, x3), d = mul_w4<INV>(csub(x1, x3));
  x0 = cadd(a, c);
  x2 = csub(a, c);
  x1 = cadd(b, d);
  x3 = csub(b, d);
}

template <bool INV> __device__ __forceinline__ void dft4(C* v) { dft4s<INV>(v[0], v[1], v[2], v[3]); }

// 8 = 4 (over n1, stride 2) x 2
template <bool INV> __device__ __forceinline__ void dft8(C* v) {
  C y0 = v[0], y2 = v[2], y4 = v[4], y6 = v[6];
  C y1 = v[1], y3 = v[3], y5 = v[5], y7 = v[7];
  dft4s<INV>(y0, y2, y4, y6);  // Y0[k1], k1 = 0..3 in (y0, y2, y4, y6)
  dft4s<INV>(y1, y3, y5, y7);  // Y1[k1]
  y3 = mul_w16<INV, 2>(y3);
  y5 = mul_w16<INV, 4>(y5);
  y7 = mul_w16<INV, 6>(y7);
  v[0] = cadd(y0, y1);
  v[4] = csub(y0, y1);
  v[1] = cadd(y2, y3);
  v[5] = csub(y2, y3);
  v[2] = cadd(y4, y5);
  v[6] = csub(y4, y5);
  v[3] = cadd(y6, y7);
  v[7] = csub(y6, y7);
}

// 16 = 4 (over n1, stride 4) x 4
template <bool INV> __device__ __forceinline__ void dft16(C* v) {
  C y[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) { y[i] = v[i]; }
  // step 1: for n2: DFT4 over n1 of x[4 n1 + n2]; result k1 kept at index n2 + 4 k1
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) { dft4s<INV>(y[n2], y[n2 + 4], y[n2 + 8], y[n2 + 12]); }
  // step 2: twiddle w16^(n2 k1)
  y[1 + 4 * 1] = mul_w16<INV, 1>(y[1 + 4 * 1]);
  y[1 + 4 * 2] = mul_w16<INV, 2>(y[1 + 4 * 2]);
  y[1 + 4 * 3] = mul_w16<INV, 3>(y[1 + 4 * 3]);
  y[2 + 4 * 1] = mul_w16<INV, 2>(y[2 + 4 * 1]);
  y[2 + 4 * 2] = mul_w16<INV, 4>(y[2 + 4 * 2]);
  y[2 + 4 * 3] = mul_w16<INV, 6>(y[2 + 4 * 3]);
  y[3 + 4 * 1] = mul_w16<INV, 3>(y[3 + 4 * 1]);
  y[3 + 4 * 2] = mul_w16<INV, 6>(y[3 + 4 * 2]);
  y[3 + 4 * 3] = mul_w16<INV, 9>(y[3 + 4 * 3]);
  // step 3: for k1: DFT4 over n2 -> X[k1 + 4 k2]
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    C a = y[0 + 4 * k1], b = y[1 + 4 * k1], c = y[2 + 4 * k1], d = y[3 + 4 * k1];
    dft4s<INV>(a, b, c, d);
    v[k1 + 0] = a;
    v[k1 + 4] = b;
    v[k1 + 8] = c;
    v[k1 + 12] = d;
  }
}

constexpr double kC51 = 0.30901699437494742410;   // cos(2 pi / 5)
constexpr double kC52 = -0.80901699437494742410;  // cos(4 pi / 5)
constexpr double kS51 = 0.95105651629515357212;   // sin(2 pi / 5)
constexpr double kS52 = 0.58778525229247312917;   // sin(4 pi / 5)

// 5-point DFT: with t1 = x1 + x4, t2 = x2 + x3, t3 = x1 - x4, t4 = x2 - x3,
// X1,4 = x0 + c1 t1 + c2 t2 -/+ i (s1 t3 + s2 t4), X2,3 = x0 + c2 t1 + c1 t2 -/+ i (s2 t3 - s1 t4)
// (signs of the i terms flipped for the inverse)
template <bool INV> __device__ __forceinline__ void dft5(C* v) {
  const C x0 = v[0];
  const C t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
  const C t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
  const C a1 = mk(x0.x + kC51 * t1.x + kC52 * t2.x, x0.y + kC51 * t1.y + kC52 * t2.y);
  const C a2 = mk(x0.x + kC52 * t1.x + kC51 * t2.x, x0.y + kC52 * t1.y + kC51 * t2.y);
  const C b1 = mk(kS51 * t3.x + kS52 * t4.x, kS51 * t3.y + kS52 * t4.y);
  const C b2 = mk(kS52 * t3.x - kS51 * t4.x, kS52 * t3.y - kS51 * t4.y);
  const C ib1 = INV ? cmulmi(b1) : cmuli(b1);
  const C ib2 = INV ? cmulmi(b2) : cmuli(b2);
  v[0] = cadd(x0, cadd(t1, t2));
  v[1] = csub(a1, ib1);
  v[4] = cadd(a1, ib1);
  v[2] = csub(a2, ib2);
  v[3] = cadd(a2, ib2);
}

template <int R, bool INV> __device__ __forceinline__ void dftR(C* v) {
  if constexpr (R == 5) {
    dft5<INV>(v);
  } else if constexpr (R == 2) {
    dft2<INV>(v);
  } else if constexpr (R == 4) {
    dft4<INV>(v);
  } else if constexpr (R == 8) {
    dft8<INV>(v);
  } else {
    static_assert(R == 16, "radix");
    dft16<INV>(v);
  }
}

// shared-memory index padding: one 16-byte pad per 2^PS elements
template <int PS> __device__ __forceinline__ int pad(int i) { return i + (i >> PS); }

constexpr int ilog2(int x) { return x <= 1 ? 0 : 1 + ilog2(x / 2); }

// ---- Stockham stage helpers for one line of N complex values held by N/VPT
// threads, VPT (16 or 8) values per thread. Stage radix R (R divides VPT, or 5):
// thread `tl` runs butterflies j = tl + (N/VPT) b, b < VPT/R, inputs x[j + r N/R],
// twiddle w_(NS R)^(r (j mod NS)), outputs y[(j/NS) NS R + j mod NS + r NS].

// butterflies per thread of a radix-R stage (radix 5 leaves the last one to some threads only)
template <int R, int VPT = 16> constexpr int st_nb() { return (VPT + R - 1) / R; }
template <int R, int N, int VPT = 16> __device__ __forceinline__ bool st_has(int j) {
  return (VPT % R == 0) || j < N / R;
}
// j mod NS and j / NS for j >= 0 (mask and shift when NS is a power of two)
template <int NS> __device__ __forceinline__ int smod(int j) {
  if constexpr ((NS & (NS - 1)) == 0) { return j & (NS - 1); } else { return (int)((unsigned)j % (unsigned)NS); }
}
template <int NS> __device__ __forceinline__ int sdiv(int j) { return (int)((unsigned)j / (unsigned)NS); }

template <int R, int N, int PS, int VPT = 16> __device__ __forceinline__ void st_load(const C* buf, int tl, C* v) {
#pragma unroll
  for (int b = 0; b < st_nb<R, VPT>(); ++b) {
    int j = tl + (N / VPT) * b;
    if (!st_has<R, N, VPT>(j)) { continue; }
#pragma unroll
    for (int r = 0; r < R; ++r) { v[b * R + r] = buf[pad<PS>(j + r * (N / R))]; }
  }
}

// tab: this stage's [r][k] table, entry r * NS + k = w_(R NS)^(r k). For
// radix 8 and 16 only the rows r = 1 and r = 4 are read; the other powers come
// from at most three products of those two correctly rounded values (each
// within a few ulp), which keeps the L1 data path free for the exchanges.
template <bool INV> __device__ __forceinline__ void twmul(C& v, C w) { v = cmulw<INV>(v, w); }

template <int R, int N, int NS, bool INV, int VPT = 16>
__device__ __forceinline__ void st_twiddle(int tl, C* v, const C* __restrict__ tab) {
  if constexpr (NS > 1) {
#pragma unroll
    for (int b = 0; b < st_nb<R, VPT>(); ++b) {
      int j = tl + (N / VPT) * b;
      if (!st_has<R, N, VPT>(j)) { continue; }
      int k = smod<NS>(j);
      C* x = v + b * R;
      if constexpr (R >= 8) {
        const C w1 = __ldg(tab + 1 * NS + k);
        const C w4 = __ldg(tab + 4 * NS + k);
        const C w2 = csq(w1);
        const C w3 = cmul(w2, w1);
        twmul<INV>(x[1], w1);
        twmul<INV>(x[2], w2);
        twmul<INV>(x[3], w3);
        twmul<INV>(x[4], w4);
        twmul<INV>(x[5], cmul(w4, w1));
        twmul<INV>(x[6], cmul(w4, w2));
        twmul<INV>(x[7], cmul(w4, w3));
        if constexpr (R == 16) {
          const C w8 = csq(w4);
          const C w12 = cmul(w8, w4);
          twmul<INV>(x[8], w8);
          twmul<INV>(x[9], cmul(w8, w1));
          twmul<INV>(x[10], cmul(w8, w2));
          twmul<INV>(x[11], cmul(w8, w3));
          twmul<INV>(x[12], w12);
          twmul<INV>(x[13], cmul(w12, w1));
          twmul<INV>(x[14], cmul(w12, w2));
          twmul<INV>(x[15], cmul(w12, w3));
        }
      } else {
#pragma unroll
        for (int r = 1; r < R; ++r) { twmul<INV>(x[r], __ldg(tab + r * NS + k)); }
      }
    }
  }
}

template <int R, bool INV, int VPT = 16> __device__ __forceinline__ void st_dft(C* v) {
#pragma unroll
  for (int b = 0; b < st_nb<R, VPT>(); ++b) { dftR<R, INV>(v + b * R); }
}

template <int R, int N, int NS, int PS, int VPT = 16> __device__ __forceinline__ void st_store(C* buf, int tl, const C* v) {
#pragma unroll
  for (int b = 0; b < st_nb<R, VPT>(); ++b) {
    int j = tl + (N / VPT) * b;
    if (!st_has<R, N, VPT>(j)) { continue; }
    int base = sdiv<NS>(j) * NS * R + smod<NS>(j);
#pragma unroll
    for (int r = 0; r < R; ++r) { buf[pad<PS>(base + r * NS)] = v[b * R + r]; }
  }
}

// Radix plan for a line of N points whose last inverse / first forward stage
// (radix RL) is split across lines or columns: N = R1 * M1 * M2 * RL.
// "A order" runs the stages R1, M1, M2, RL; "B order" runs RL, M2, M1, R1.
// n = 2^a or 5 * 2^a; the factor 5 becomes the M2 stage. r1f != 0 forces the
// first radix (the split-precision column pass runs a 32-point first stage).
// vmax: the largest radix (the values per thread).
constexpr int plan_r1(int n, int rl, int r1f = 0, int vmax = 16) {
  return r1f ? r1f : (n / rl >= vmax ? vmax : n / rl);
}
constexpr int plan_rest2(int n, int rl, int r1f = 0, int vmax = 16) { return n / rl / plan_r1(n, rl, r1f, vmax); }
constexpr int plan_m1(int n, int rl, int r1f = 0, int vmax = 16) {
  return plan_rest2(n, rl, r1f, vmax) % 5 == 0
             ? plan_rest2(n, rl, r1f, vmax) / 5
             : (plan_rest2(n, rl, r1f, vmax) >= vmax ? vmax : plan_rest2(n, rl, r1f, vmax));
}
constexpr int plan_m2(int n, int rl, int r1f = 0, int vmax = 16) {
  return plan_rest2(n, rl, r1f, vmax) / plan_m1(n, rl, r1f, vmax);
}

// Column-pass tile variants, chosen per plan (owl_plan_set_column_variant; gpuowl_b200.tune times
// them per shape): the values a thread holds (which fixes the radix plan and the threads of a CTA)
// and the CTAs per SM that the launch bounds ask for.
//   COL_V16       16 values a thread, H/8 threads a CTA: every H
//   COL_V8         8 values a thread, H/4 threads (twice the threads at half the registers; the radix
//                  plan 8 x ... x 4): H a power of two up to 2048, 640 and 1280
//   COL_V16_OCC2  16 values a thread at two CTAs per SM (102 registers, a few spilled): H = 2560,
//                  whose default runs one 320-thread CTA of 168 registers per SM
// COL_AUTO (0) stands for the shape's default (owl_tables.hpp: default_col_variant).
enum : int { COL_AUTO = 0, COL_V16 = 1, COL_V8 = 2, COL_V16_OCC2 = 3 };
__host__ __device__ constexpr bool col_variant_ok(int H, int v) {
  return v == COL_V16 || (v == COL_V8 && ((((H & (H - 1)) == 0) && H <= 2048) || H == 640 || H == 1280)) ||
         (v == COL_V16_OCC2 && H == 2560);
}
__host__ __device__ constexpr int col_vpt(int v) { return v == COL_V8 ? 8 : 16; }
// the CTAs per SM of the column pass's launch bounds (0: the kernel's own rule)
__host__ __device__ constexpr int col_minb(int v) { return v == COL_V16_OCC2 ? 2 : 0; }

// CTAs per SM that the pass kernels' launch bounds ask for: enough for 16 resident warps at most
// 128 registers a thread (T threads a CTA; at most 32 CTAs an SM). Without the hint the kernels of
// the small FFTs (32- to 128-thread CTAs) took 200-255 registers, which left 8-10 warps on an SM.
constexpr int occ_blocks(int T) {
  return T >= 512 ? 1 : (16 / ((T + 31) / 32) > 32 ? 32 : 16 / ((T + 31) / 32));
}

// Stage twiddle tables, one per stage with twiddles, each laid out [r][k]:
// entry r * NS + k = w_(R NS)^(r k) (forward sign), so that a warp's threads
// (consecutive k) read one contiguous run per r. Offsets in complex elements.
struct TwOffsets {
  int aM1, aM2, aRL, bM2, bM1, bR1, total;
};
constexpr TwOffsets tw_offsets(int n, int rl, int r1f = 0, int vmax = 16) {
  const int r1 = plan_r1(n, rl, r1f, vmax), m1 = plan_m1(n, rl, r1f, vmax), m2 = plan_m2(n, rl, r1f, vmax);
  TwOffsets o{};
  o.aM1 = 0;
  o.aM2 = o.aM1 + (m1 > 1 ? m1 * r1 : 0);
  o.aRL = o.aM2 + (m2 > 1 ? m2 * r1 * m1 : 0);
  o.bM2 = o.aRL + n;
  o.bM1 = o.bM2 + (m2 > 1 ? m2 * rl : 0);
  o.bR1 = o.bM1 + (m1 > 1 ? m1 * rl * m2 : 0);
  o.total = o.bR1 + n;
  return o;
}

template <int N, int RL, int R1F = 0, int VPT = 16> struct Plan {
  static constexpr int R1 = plan_r1(N, RL, R1F, VPT);
  static constexpr int M1 = plan_m1(N, RL, R1F, VPT);
  static constexpr int M2 = plan_m2(N, RL, R1F, VPT);
  static constexpr TwOffsets TW = tw_offsets(N, RL, R1F, VPT);
  static_assert(R1 * M1 * M2 * RL == N, "plan");
  static_assert(M2 >= 1 && M2 <= VPT, "plan depth");
  static_assert(M1 <= VPT && (VPT % M1 == 0), "plan: first middle radix must divide the values per thread");
  static_assert(M2 == 5 || (VPT % M2 == 0), "plan: second middle radix 5 or a divisor of the values per thread");
  static_assert(R1 >= 4, "first radix too small for conflict-free padding");
};

}  // namespace owl
