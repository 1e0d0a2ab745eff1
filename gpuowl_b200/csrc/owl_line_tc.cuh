// owl_line_tc.cuh -- the split-precision form of the line pass's GEMM stage: the first inverse and
// the last forward radix-16 stage of the 2048-point width FFT as INT8 GEMMs on the tensor cores
// (tcgen05.mma kind::i8), the same Ozaki-style digit splitting as the column pass's
// (owl_pass2_tc.cuh): 7 balanced base-256 digit planes of each row scaled below 2^54, the 28 digit
// products with i + j <= 6 accumulated exactly per diagonal in INT32 tensor memory, recombined in
// FP64 by Horner's rule. owl_kernels.cuh includes this file after Args and before the line-pass
// kernels, whose body (owl_pass1_body.inc) calls line_tc_dft in place of the FP64 radix-16 stage.
//
// A CTA of the 2048-point line pass holds R = 2 lines of 128 sub-vectors each, x[j + 128 r],
// r < 16: the 256 rows of the GEMM (row = the thread index t, so line t % 2, sub-vector t / 2),
// K = 16 complex inputs (32 int8 values, one k-step), N = 16 complex outputs (32 values). It runs
// as two M = 128 tiles (rows 0-127, then 128-255) through the same 7 x 32 accumulator columns of
// tensor memory, 256 columns per CTA, so that two CTAs share an SM's 512 columns.
//
// The operands use the no-swizzle K-major layout (core matrices of 8 rows x 16 bytes, LBO = 128
// between the two 16-byte halves of K, SBO = 256 between groups of 8 rows): 32-byte rows cost half
// the shared memory of the 64-byte swizzled layout, which keeps the line pass at two CTAs per SM.
// The data digit planes (7 x 8 KiB) overlay the line buffers; the DFT digit planes (7 x 32 rows,
// plane after plane, so that one MMA multiplies data plane i by DFT planes 0 .. 6-i), the row
// exponents, the barrier and the tensor-memory base follow the line buffers.
#pragma once

namespace owl {

constexpr int kLtcW = 2048;                     // line width of the split-precision line pass
constexpr int kLtcRows = 256;                   // 2 lines x 128 sub-vectors
constexpr int kLtcK = 32;                       // int8 inputs a row (16 complex)
constexpr int kLtcN = 32;                       // int8 outputs a row (16 complex)
constexpr uint32_t kLtcLbo = 128, kLtcSbo = 256;
constexpr int kLtcAPlane = kLtcRows * kLtcK;    // 8 KiB
constexpr int kLtcBBytes = 7 * kLtcN * kLtcK;   // 7 KiB
constexpr uint32_t kLtcTmemCols = 256;
constexpr long long kLtcBias = 0x0000808080808080LL;

// byte offset of (row, K byte kb) in a no-swizzle K-major operand with 32-byte rows
__host__ __device__ constexpr uint32_t ltc_off(int row, int kb) {
  return (uint32_t)((row / 8) * kLtcSbo + (kb / 16) * kLtcLbo + (row % 8) * 16 + kb % 16);
}

// shared memory of the split line pass beyond its line buffers (lineBytes): DFT planes, exponents,
// barrier, tensor-memory base, and 128 bytes of slack to align the operands
__host__ __device__ constexpr int ltc_extra_smem() { return kLtcBBytes + kLtcRows * 4 + 16 + 128; }

struct LineTc {
  unsigned char* sA;  // data digit planes (overlay the line buffers)
  unsigned char* sB;  // DFT digit planes
  int* sExp;
  uint64_t* sBar;
  uint32_t taddr, aBase, bBase, phase;
};

// 4 int8 values of Z = Y + bias bytes -> 7 digit words (word 6 - p holds byte p of each)
__device__ __forceinline__ void ltc_words(long long z0, long long z1, long long z2, long long z3, uint32_t (&wd)[7]) {
  const uint32_t l0 = (uint32_t)z0, l1 = (uint32_t)z1, l2 = (uint32_t)z2, l3 = (uint32_t)z3;
  const uint32_t h0 = (uint32_t)(z0 >> 32), h1 = (uint32_t)(z1 >> 32), h2 = (uint32_t)(z2 >> 32),
                 h3 = (uint32_t)(z3 >> 32);
#pragma unroll
  for (int p = 0; p < 7; ++p) {
    const uint32_t a0 = p < 4 ? l0 : h0, a1 = p < 4 ? l1 : h1, a2 = p < 4 ? l2 : h2, a3 = p < 4 ? l3 : h3;
    const int q = p & 3;
    const uint32_t lo = __byte_perm(a0, a1, (uint32_t)(q | ((q + 4) << 4)));
    const uint32_t hi = __byte_perm(a2, a3, (uint32_t)(q | ((q + 4) << 4)));
    uint32_t word = __byte_perm(lo, hi, 0x5410u);
    if (p < 6) { word ^= 0x80808080u; }
    wd[6 - p] = word;
  }
}

// Sets up the split stage: carves the operands out of shared memory (line buffers of lineBytes
// bytes first), allocates the tensor memory (warp 0) and initialises the barrier. Every thread calls
// it; a barrier follows inside.
__device__ __forceinline__ LineTc ltc_setup(unsigned char* smemBytes, int lineBytes, const unsigned char* tcB) {
  LineTc L;
  const uint32_t pad = (uint32_t)(128 - (tc::smem_addr(smemBytes) & 127u)) & 127u;
  L.sA = smemBytes + pad;
  L.sB = smemBytes + pad + ((lineBytes + 127) / 128) * 128;
  L.sExp = reinterpret_cast<int*>(L.sB + kLtcBBytes);
  L.sBar = reinterpret_cast<uint64_t*>(L.sB + kLtcBBytes + kLtcRows * 4);
  uint32_t* sTaddr = reinterpret_cast<uint32_t*>(L.sB + kLtcBBytes + kLtcRows * 4 + 8);
  const int t = threadIdx.x;
  if ((t >> 5) == 0) {
    tc::tmem_alloc(sTaddr, kLtcTmemCols);
    tc::tmem_relinquish();
  }
  if (t == 0) { tc::mbar_init(L.sBar, 1); }
  {
    const uint4* src = reinterpret_cast<const uint4*>(tcB);
    uint4* dst = reinterpret_cast<uint4*>(L.sB);
    for (int i = t; i < kLtcBBytes / 16; i += (int)blockDim.x) { dst[i] = __ldg(src + i); }
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  L.taddr = *sTaddr;
  L.aBase = tc::smem_addr(L.sA);
  L.bBase = tc::smem_addr(L.sB);
  L.phase = 0;
  return L;
}

// releases the tensor memory (every thread calls it, after the last GEMM)
__device__ __forceinline__ void ltc_release(const LineTc& L) {
  tc::fence_before();
  __syncthreads();
  if ((threadIdx.x >> 5) == 0) { tc::tmem_dealloc(L.taddr, kLtcTmemCols); }
}

// The 16-point DFT (inverse when INV) of the 256 rows: thread t passes in row t's 16 inputs (x) and
// receives, for tile tau = 0, 1, the outputs 8 (warp / 4) + k, k < 8, of row 128 tau + 32 (warp % 4)
// + lane in y[8 tau + k]. The caller must not touch the line buffers between this call's first
// barrier and its return (the data planes overlay them). Returns false on a tensor-core timeout.
template <bool INV>
__device__ __forceinline__ bool line_tc_dft(const Args& a, LineTc& L, const C* x, C* y) {
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  double m = 0.0;
#pragma unroll
  for (int i = 0; i < 16; ++i) { m = fmax(m, fmax(fabs(x[i].x), fabs(x[i].y))); }
  int ex = 0;
  if (m > 0.0) { ex = (int)((__double_as_longlong(m) >> 52) & 0x7ff) - 1022; }  // m < 2^ex
  if (ex < -900) { ex = -900; }
  __syncthreads();  // the digit planes overlay the line buffers
  L.sExp[t] = ex;
  const double sc = tc::exp2i(54 - ex);
#pragma unroll
  for (int q = 0; q < 2; ++q) {  // 8 complex values = 16 bytes of K per plane
    uint32_t wd[4][7];
#pragma unroll
    for (int wi = 0; wi < 4; ++wi) {
      const C v0 = x[8 * q + 2 * wi], v1 = x[8 * q + 2 * wi + 1];
      ltc_words(__double2ll_rn(v0.x * sc) + kLtcBias, __double2ll_rn((INV ? -v0.y : v0.y) * sc) + kLtcBias,
                __double2ll_rn(v1.x * sc) + kLtcBias, __double2ll_rn((INV ? -v1.y : v1.y) * sc) + kLtcBias, wd[wi]);
    }
#pragma unroll
    for (int s = 0; s < 7; ++s) {
      *reinterpret_cast<uint4*>(L.sA + s * kLtcAPlane + ltc_off(t, 16 * q)) =
          make_uint4(wd[0][s], wd[1][s], wd[2][s], wd[3][s]);
    }
  }
  tc::fence_proxy_async();
  __syncthreads();
  bool ok = true;
  const int qd = w & 3, cs = (w >> 2) * 16;
#pragma unroll 1
  for (int tau = 0; tau < 2; ++tau) {
    if (t == 0) {
      tc::fence_after();
      const uint64_t bd = tc::smem_desc(L.bBase, kLtcLbo, kLtcSbo, 0);
#pragma unroll
      for (int i = 0; i < 7; ++i) {
        const uint64_t ad = tc::smem_desc(L.aBase + (uint32_t)(i * kLtcAPlane + tau * (128 / 8) * kLtcSbo), kLtcLbo,
                                          kLtcSbo, 0);
        tc::mma_s8(L.taddr + (uint32_t)(i * kLtcN), ad, bd, tc::idesc_s8(128, kLtcN * (7 - i)), i > 0);
      }
      tc::commit(L.sBar);
    }
    ok &= tc::mbar_wait(L.sBar, L.phase & 1u, a.timeoutNs);
    ++L.phase;
    tc::fence_after();
    const int drow = 128 * tau + 32 * qd + lane;
    const double post = tc::exp2i(L.sExp[drow] - 60);
    // D_d < (d + 1) 2^19: D0 256 + D1, D2 256 + D3 and D4 256 + D5 are exact in INT32; the rest of
    // Horner's rule runs in FP64
#pragma unroll
    for (int g = 0; g < 2; ++g) {
      const uint32_t tb = L.taddr + ((uint32_t)(32 * qd) << 16) + (uint32_t)(cs + 8 * g);
      uint32_t ra[8], rb[8];
      int32_t p01[8], p23[8], p45[8];
      tc::tmem_ld8(tb + 0 * kLtcN, ra);
      tc::tmem_ld8(tb + 1 * kLtcN, rb);
      tc::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 8; ++i) { p01[i] = (int32_t)ra[i] * 256 + (int32_t)rb[i]; }
      tc::tmem_ld8(tb + 2 * kLtcN, ra);
      tc::tmem_ld8(tb + 3 * kLtcN, rb);
      tc::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 8; ++i) { p23[i] = (int32_t)ra[i] * 256 + (int32_t)rb[i]; }
      tc::tmem_ld8(tb + 4 * kLtcN, ra);
      tc::tmem_ld8(tb + 5 * kLtcN, rb);
      tc::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 8; ++i) { p45[i] = (int32_t)ra[i] * 256 + (int32_t)rb[i]; }
      tc::tmem_ld8(tb + 6 * kLtcN, ra);
      tc::tmem_wait_ld();
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        double v2[2];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int i = 2 * k + e;
          double acc = fma(tc::i32_to_f64(p01[i]), 65536.0, tc::i32_to_f64(p23[i]));
          acc = fma(acc, 65536.0, tc::i32_to_f64(p45[i]));
          v2[e] = fma(acc, 256.0, tc::i32_to_f64((int32_t)ra[i])) * post;
        }
        y[8 * tau + 4 * g + k] = mk(v2[0], INV ? -v2[1] : v2[1]);
      }
    }
    tc::fence_before();
    __syncthreads();  // accumulators read before the next tile overwrites them
  }
  return ok;
}

}  // namespace owl

#include <vector>

#include "owl_tables.hpp"

namespace owl {

// Host: the 7 digit planes of the 16-point DFT matrix (32 output values n = 2 m + {re, im} x 32
// inputs kb = 2 r + {re, im}; cos / sin of 2 pi r m / 16 scaled by 2^54 and rounded once), plane j
// at rows 32 j .. of one no-swizzle K-major operand.
inline std::vector<uint8_t> line_tc_dft_digits() {
  std::vector<uint8_t> out(kLtcBBytes, 0);
  for (int n = 0; n < kLtcN; ++n) {
    for (int kb = 0; kb < kLtcK; ++kb) {
      const int m = n / 2, cn = n & 1, r = kb / 2, ck = kb & 1;
      long double cs, sn;
      root_ld(16, (uint64_t)((r * m) % 16), &cs, &sn);
      const long double v = cn == 0 ? (ck == 0 ? cs : sn) : (ck == 0 ? -sn : cs);
      const long long Z = llrintl(ldexpl(v, 54)) + kLtcBias;
      for (int p = 0; p < 7; ++p) {
        uint8_t b = (uint8_t)((unsigned long long)Z >> (8 * p));
        if (p < 6) { b ^= 0x80; }
        out[ltc_off(32 * (6 - p) + n, kb)] = b;
      }
    }
  }
  return out;
}

}  // namespace owl
