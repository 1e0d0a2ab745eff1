// owl_pass2_tc.cuh -- the split-precision form of the column pass (k_pass2) for
// 2048-point columns: its first forward and last inverse radix-32 stages run as
// INT8 GEMMs on the tensor cores (tcgen05.mma kind::i8, INT32 accumulators in
// tensor memory), every other step stays FP64.
//
// The column FFT is 2048 = 32 (GEMM) x 8 x 8 (the cross-column radix-8 stage of
// k_pass2). A CTA owns two columns, i.e. 2 x 64 sub-vectors x[j + 64 r],
// r < 32: the 128 rows of one GEMM whose K dimension is the 32 complex inputs
// (64 int8 values: re, im interleaved) and whose N dimension is the 32 complex
// outputs (64 values).
//
// Ozaki-style splitting: each row is scaled by its own power of two so that
// its largest component is below 2^54, rounded to an integer Y, and Y is cut
// into 7 signed base-256 digits (balanced, so the top digit is within +-64):
// Y = sum_i d_i 256^(6-i). The DFT matrix (entries cos, sin scaled by 2^54)
// is cut the same way on the host. The digit products with i + j <= 6 are
// accumulated exactly in INT32 per diagonal d = i + j (7 accumulators,
// |D_d| < 2^25), and recombined in FP64 by Horner's rule,
// sum_d D_d 256^(6-d), times 2^(e - 60) for the row exponent e. Dropped
// products (i + j >= 7) and the 2^-55 rounding of both operands put the
// relative error of a GEMM output near 2^-51 of its row's largest input.
// The IBDWT weights, the inter-pass twiddles, the pair squaring, the
// rounding and the carry are untouched (they run in k_pass1 / FP64 here).
//
// The inverse stage uses the same digit matrix: IDFT(x) = conj(DFT(conj x)).
#pragma once
#include "owl_kernels.cuh"
#include "owl_tc.cuh"

namespace owl {

constexpr int kTcH = 2048;                      // column length of the split-precision pass
constexpr int kTcR1 = 32;                       // first forward / last inverse radix, as GEMMs
constexpr int kTcSlices = 7;                    // base-256 digits per operand
constexpr int kTcRows = 128;                    // GEMM M: 2 columns x 64 sub-vectors
constexpr int kTcK = 2 * kTcR1;                 // int8 inputs per row
constexpr int kTcN = 2 * kTcR1;                 // outputs per row
constexpr int kTcNHalf = 32;                    // N of one MMA batch
constexpr int kTcASlice = kTcRows * kTcK;       // bytes of one data digit plane (8 KiB)
constexpr int kTcBSlice = kTcN * kTcK;          // bytes of one DFT digit plane (4 KiB)
constexpr int kTcBBytes = kTcSlices * kTcBSlice;
// The DFT digit planes are stored per N half: the 32 output rows of the half, plane after plane,
// as one K-major operand of 7 x 32 = 224 rows (row q = 32 j + n for plane j, output row n of the
// half). One MMA then multiplies data plane i by planes 0 .. 6-i at once (N = 32 (7 - i)), and its
// output column 32 (i + j) + n is accumulator d = i + j: each data plane is read once per k-step
// instead of once per diagonal.
constexpr int kTcBRows = kTcSlices * kTcNHalf;  // 224
constexpr int kTcBHalf = kTcBRows * kTcK;       // bytes of one half's operand (14 KiB)
constexpr uint32_t kTcTmemCols = 256;           // 7 accumulators x 32 columns, rounded to a power of two
constexpr long long kTcBias = 0x0000808080808080LL;  // 128 in each of the 6 low digit positions
// Both operands are K-major with 64-byte rows (the 64 int8 inputs of a GEMM row) in the 64-byte
// swizzled layout (tc::sw64_off: 512-byte atoms of 8 rows, SBO = 512; one MMA's K = 32 bytes stays
// inside a row, so LBO is unused); a k-step starts 32 bytes into the rows.
constexpr uint32_t kTcSbo = 512;

// dynamic shared memory: two column buffers (the data digit planes overlay
// them), the DFT digit planes, row exponents, the MMA barrier, the TMEM base;
// the two operands start 1024-byte aligned (the swizzle is on address bits 4-8),
// which the kernel arranges at run time inside the 1 KiB of slack (kTcAlign)
constexpr int kTcAlign = 1024;
constexpr int kTcColStride = p2_col_stride<kTcH>();
constexpr int kTcOffB = (2 * kTcColStride * (int)sizeof(C) + kTcAlign - 1) / kTcAlign * kTcAlign;
constexpr int kTcOffExp = kTcOffB + kTcBBytes;
constexpr int kTcOffBar = kTcOffExp + kTcRows * 4;
constexpr int kTcOffTaddr = kTcOffBar + 8;
constexpr int kTcSmem = kTcOffTaddr + 8 + kTcAlign;
static_assert(kTcSlices * kTcASlice <= kTcOffB, "data digit planes must fit in the column buffers");
static_assert(kTcASlice % kTcAlign == 0 && kTcBHalf % kTcAlign == 0, "operand planes keep the swizzle alignment");
static_assert(kTcBBytes == 2 * kTcBHalf, "DFT digit planes: two N halves");
static_assert(kTcOffB % 16 == 0 && kTcOffBar % 8 == 0, "alignment");

// byte offset of data digit plane s, GEMM row `row`, K index kb
__host__ __device__ constexpr uint32_t tc_off_a(int s, int row, int kb) {
  return (uint32_t)(s * kTcASlice) + tc::sw64_off(row, kb);
}
// byte offset of DFT digit plane s, output row n (< 64), K index kb in the per-half operands
__host__ __device__ constexpr uint32_t tc_off_b(int s, int n, int kb) {
  return (uint32_t)((n / kTcNHalf) * kTcBHalf) + tc::sw64_off(s * kTcNHalf + n % kTcNHalf, kb);
}

// the 7 digits of one value v (|v| < 2^54 after scaling), byte p of Z = Y + bias is digit 6 - p
__device__ __forceinline__ long long tc_digits_src(double v) { return __double2ll_rn(v) + kTcBias; }

// writes the digit planes of 16 complex inputs (elements 16 hh .. 16 hh + 15 of GEMM row `row`)
template <bool CONJ>
__device__ __forceinline__ void tc_put_digits(unsigned char* sA, int row, int hh, const C* x, double sc) {
#pragma unroll
  for (int qq = 0; qq < 2; ++qq) {
    uint32_t wd[kTcSlices][4];
#pragma unroll
    for (int wi = 0; wi < 4; ++wi) {
      const C v0 = x[8 * qq + 2 * wi], v1 = x[8 * qq + 2 * wi + 1];
      const long long z0 = tc_digits_src(v0.x * sc), z1 = tc_digits_src((CONJ ? -v0.y : v0.y) * sc);
      const long long z2 = tc_digits_src(v1.x * sc), z3 = tc_digits_src((CONJ ? -v1.y : v1.y) * sc);
      const uint32_t l0 = (uint32_t)z0, l1 = (uint32_t)z1, l2 = (uint32_t)z2, l3 = (uint32_t)z3;
      const uint32_t h0 = (uint32_t)(z0 >> 32), h1 = (uint32_t)(z1 >> 32), h2 = (uint32_t)(z2 >> 32),
                     h3 = (uint32_t)(z3 >> 32);
      // bytes p = 0..3 from the low words, 4..6 from the high words
#pragma unroll
      for (int p = 0; p < 7; ++p) {
        const uint32_t a0 = p < 4 ? l0 : h0, a1 = p < 4 ? l1 : h1, a2 = p < 4 ? l2 : h2, a3 = p < 4 ? l3 : h3;
        const int q = p & 3;
        const uint32_t lo = __byte_perm(a0, a1, (uint32_t)(q | ((q + 4) << 4)));
        const uint32_t hi = __byte_perm(a2, a3, (uint32_t)(q | ((q + 4) << 4)));
        uint32_t word = __byte_perm(lo, hi, 0x5410u);
        if (p < 6) { word ^= 0x80808080u; }
        wd[6 - p][wi] = word;
      }
    }
    const int q = 2 * hh + qq;
#pragma unroll
    for (int s = 0; s < kTcSlices; ++s) {
      *reinterpret_cast<uint4*>(sA + tc_off_a(s, row, 16 * q)) = make_uint4(wd[s][0], wd[s][1], wd[s][2], wd[s][3]);
    }
  }
}

// issues the 14 MMAs of one N half: accumulator d (TMEM columns 32 d ..) gets sum_{i+j=d} A_i B_j^T.
// MMA (ks, i) multiplies data plane i by DFT planes 0 .. 6-i (N = 32 (7 - i)) into columns 32 i ..;
// the first one (ks = 0, i = 0) covers all 7 accumulators and initialises them.
__device__ __forceinline__ void tc_issue(uint32_t aBase, uint32_t bBase, uint32_t taddr, int half) {
#pragma unroll
  for (int ks = 0; ks < kTcK / 32; ++ks) {
    const uint64_t bd = tc::smem_desc(bBase + half * kTcBHalf + ks * 32, 16, kTcSbo, 4);
#pragma unroll
    for (int i = 0; i < kTcSlices; ++i) {
      const uint64_t ad = tc::smem_desc(aBase + i * kTcASlice + ks * 32, 16, kTcSbo, 4);
      tc::mma_s8(taddr + (uint32_t)(i * kTcNHalf), ad, bd, tc::idesc_s8(kTcRows, kTcNHalf * (kTcSlices - i)),
                 i > 0 || ks > 0);
    }
  }
}

// The 32-point DFT (inverse when INV) of the 128 GEMM rows. This thread passes in
// elements 16 hh + i of row `row` (x) and receives 16 outputs of row
// drow = 32 (warp % 4) + lane: y[k] = X[8 (warp / 4) + k], y[8 + k] = X[16 + 8 (warp / 4) + k].
// Returns false if the tensor cores did not finish within the plan's timeout.
template <bool INV>
__device__ __forceinline__ bool tc_dft32(const Args& a, unsigned char* sA, int* sExp, uint64_t* sBar, uint32_t aBase,
                                         uint32_t bBase, uint32_t taddr, uint32_t& phase, int row, int hh, const C* x,
                                         C* y) {
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  double m = 0.0;
#pragma unroll
  for (int i = 0; i < 16; ++i) { m = fmax(m, fmax(fabs(x[i].x), fabs(x[i].y))); }
  m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 16));
  int ex = 0;
  if (m > 0.0) { ex = (int)((__double_as_longlong(m) >> 52) & 0x7ff) - 1022; }  // m < 2^ex
  if (ex < -900) { ex = -900; }
  __syncthreads();  // the digit planes overlay the column buffers the inputs were read from
  if (hh == 0) { sExp[row] = ex; }
  tc_put_digits<INV>(sA, row, hh, x, tc::exp2i(54 - ex));
  tc::fence_proxy_async();
  __syncthreads();

  bool ok = true;
  const int q = w & 3, cs = (w >> 2) * 16;
  const int drow = 32 * q + lane;
  const double post = tc::exp2i(sExp[drow] - 60);
#pragma unroll 1
  for (int half = 0; half < 2; ++half) {
    if (t == 0) {
      tc::fence_after();
      tc_issue(aBase, bBase, taddr, half);
      tc::commit(sBar);
    }
    ok &= tc::mbar_wait(sBar, phase & 1u, a.timeoutNs);
    ++phase;
    tc::fence_after();
    // D_d < (d + 1) 2^20, so D0 256 + D1, D2 256 + D3 and D4 256 + D5 are exact in INT32; the
    // rest of Horner's rule runs in FP64 (exact up to the last two steps, one rounding each)
#pragma unroll
    for (int g = 0; g < 2; ++g) {
      const uint32_t tb = taddr + ((uint32_t)(32 * q) << 16) + (uint32_t)(cs + 8 * g);
      uint32_t ra[8], rb[8];
      int32_t p01[8], p23[8], p45[8];
      tc::tmem_ld8(tb + 0 * kTcNHalf, ra);
      tc::tmem_ld8(tb + 1 * kTcNHalf, rb);
      tc::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 8; ++i) { p01[i] = (int32_t)ra[i] * 256 + (int32_t)rb[i]; }
      tc::tmem_ld8(tb + 2 * kTcNHalf, ra);
      tc::tmem_ld8(tb + 3 * kTcNHalf, rb);
      tc::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 8; ++i) { p23[i] = (int32_t)ra[i] * 256 + (int32_t)rb[i]; }
      tc::tmem_ld8(tb + 4 * kTcNHalf, ra);
      tc::tmem_ld8(tb + 5 * kTcNHalf, rb);
      tc::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 8; ++i) { p45[i] = (int32_t)ra[i] * 256 + (int32_t)rb[i]; }
      tc::tmem_ld8(tb + 6 * kTcNHalf, ra);
      tc::tmem_wait_ld();
      double v[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        double acc = fma(tc::i32_to_f64(p01[i]), 65536.0, tc::i32_to_f64(p23[i]));
        acc = fma(acc, 65536.0, tc::i32_to_f64(p45[i]));
        v[i] = fma(acc, 256.0, tc::i32_to_f64((int32_t)ra[i])) * post;
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) { y[half * 8 + 4 * g + k] = mk(v[2 * k], INV ? -v[2 * k + 1] : v[2 * k + 1]); }
    }
    tc::fence_before();
    __syncthreads();  // all accumulator reads done before the next batch overwrites them
  }
  return ok;
}

template <int R, int MODE>
__global__ void __launch_bounds__(kTcH / 8, 2)
    k_pass2_tc(Args a, const unsigned char* __restrict__ tcB, const C* __restrict__ twT, C* __restrict__ F,
               const C* __restrict__ Fb, C* __restrict__ Fq, int tslot) {
  constexpr int H = kTcH;
  constexpr int T = H / 8;
  constexpr int TC = H / 16;
  using P = Plan<H, 8, kTcR1>;
  static_assert(P::R1 == 32 && P::M1 == 8 && P::M2 == 1, "split-precision column plan");
  constexpr int CS = kTcColStride;
  OWL_DYN_SHARED(C, smem);
  unsigned char* sm8 = reinterpret_cast<unsigned char*>(smem);
  // the operands 1024-byte aligned: the data planes overlay the column buffers from the first
  // aligned address; everything from the DFT planes on moves by the same amount
  const uint32_t alignPad = (uint32_t)(kTcAlign - (tc::smem_addr(sm8) & (kTcAlign - 1))) & (kTcAlign - 1);
  unsigned char* sA = sm8 + alignPad;
  unsigned char* sB = sm8 + alignPad + kTcOffB;
  int* sExp = reinterpret_cast<int*>(sm8 + alignPad + kTcOffExp);
  uint64_t* sBar = reinterpret_cast<uint64_t*>(sm8 + alignPad + kTcOffBar);
  uint32_t* sTaddr = reinterpret_cast<uint32_t*>(sm8 + alignPad + kTcOffTaddr);

  const uint32_t W = a.W;
  const uint32_t c = blockIdx.x;
  griddep_wait();
  griddep_launch();
  ts_begin(a, tslot);
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int col = t / TC;
  const int tc = t % TC;
  const uint32_t kA = c, kB = (c == 0) ? W / 2 : W - c;
  C* cbuf = smem + col * CS;
  // GEMM input role of this thread: row (column gcol, sub-vector gj), elements 16 ghh ..
  const int gcol = (lane >> 1) & 1;
  const int gj = (w << 3) | (((lane >> 2) & 3) << 1) | (lane & 1);
  const int ghh = lane >> 4;
  const int grow = gcol * 64 + gj;
  // GEMM output role: row drow (column dcol, sub-vector dj), outputs m = dm0 + k, 16 + dm0 + k
  const int drow = 32 * (w & 3) + lane;
  const int dcol = drow >> 6, dj = drow & 63, dm0 = (w >> 2) * 8;
  const unsigned long long pol = l2_keep_policy();

  if (w == 0) {
    tc::tmem_alloc(sTaddr, kTcTmemCols);
    tc::tmem_relinquish();
  }
  if (t == 0) { tc::mbar_init(sBar, 1); }
  {
    const uint4* src = reinterpret_cast<const uint4*>(tcB);
    uint4* dst = reinterpret_cast<uint4*>(sB);
    for (int i = t; i < kTcBBytes / 16; i += T) { dst[i] = __ldg(src + i); }
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t taddr = *sTaddr;
  const uint32_t aBase = tc::smem_addr(sA), bBase = tc::smem_addr(sB);
  uint32_t phase = 0;
  bool ok = true;

  C u[16];
  C y[16];
  // ---- forward: inputs from HBM (the line pass applied the w_hN^(k1 j2) twiddle) ----
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    const int r = 16 * ghh + i;
    const uint32_t j2 = (uint32_t)(gj + 64 * r);
    u[i] = ld_state(F + faddr<R>(W, j2, c, gcol), pol);
  }
  ok &= tc_dft32<false>(a, sA, sExp, sBar, aBase, bBase, taddr, phase, grow, ghh, u, y);
  {
    C* db = smem + dcol * CS;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      db[pad<5>(dj * 32 + dm0 + k)] = y[k];
      db[pad<5>(dj * 32 + 16 + dm0 + k)] = y[8 + k];
    }
  }
  __syncthreads();
  // ---- radix-8 middle stage (NS = 32) ----
  st_load<8, H, 5>(cbuf, tc, u);
  st_twiddle<8, H, 32, false>(tc, u, twT + P::TW.aM1);
  st_dft<8, false>(u);
  __syncthreads();
  st_store<8, H, 32, 4>(cbuf, tc, u);
  __syncthreads();
  // ---- last forward stage (radix 8, NS = T): A butterfly t, B butterfly T-1-t ----
  const int jB = T - 1 - t;
  C* bufA = smem;
  C* bufB = smem + CS;
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    u[r] = bufA[pad<4>(t + r * T)];
    u[8 + r] = bufB[pad<4>(jB + r * T)];
  }
#pragma unroll
  for (int r = 1; r < 8; ++r) {
    u[r] = cmul(u[r], __ldg(twT + P::TW.aRL + r * T + t));
    u[8 + r] = cmul(u[8 + r], __ldg(twT + P::TW.aRL + r * T + jB));
  }
  dft8<false>(u);
  dft8<false>(u + 8);

  if constexpr (MODE == P2_FWD) {
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      uint32_t kA2 = t + T * r, kB2 = jB + T * r;
      Fq[faddr<R>(W, kA2, c, 0)] = u[r];
      Fq[faddr<R>(W, kB2, c, 1)] = u[8 + r];
    }
  } else {
    if (c != 0) {
      const C base2 = cmul(bigtw(a, kA), __ldg(a.rootH + t));
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        uint32_t k2 = t + T * r;
        C t2 = mul_w8<false>(base2, r);
        if constexpr (MODE == P2_SQUARE) {
          pair_sq(u[r], u[15 - r], t2);
        } else {
          C cA = Fb[faddr<R>(W, k2, c, 0)];
          C cB = Fb[faddr<R>(W, H - 1 - k2, c, 1)];
          pair_mul(u[r], u[15 - r], cA, cB, t2);
        }
      }
    } else {
      __syncthreads();
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        bufA[t + T * r] = u[r];
        bufB[jB + T * r] = u[8 + r];
      }
      __syncthreads();
      const C baseA = __ldg(a.rootH + t);
      const C baseB = cmul(bigtw(a, W / 2), __ldg(a.rootH + jB));
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        uint32_t kA2 = t + T * r;
        uint32_t pA = (kA2 == 0) ? 0u : H - kA2;
        uint32_t kB2 = jB + T * r;
        uint32_t pB = H - 1 - kB2;
        C t2A = mul_w8<false>(baseA, r);
        C t2B = mul_w8<false>(baseB, r);
        if constexpr (MODE == P2_SQUARE) {
          u[r] = one_sq(u[r], bufA[pA], t2A);
          u[8 + r] = one_sq(u[8 + r], bufB[pB], t2B);
        } else {
          C cA = Fb[faddr<R>(W, kA2, 0, 0)], dA = Fb[faddr<R>(W, pA, 0, 0)];
          C cB = Fb[faddr<R>(W, kB2, 0, 1)], dB = Fb[faddr<R>(W, pB, 0, 1)];
          u[r] = one_mul(u[r], bufA[pA], cA, dA, t2A);
          u[8 + r] = one_mul(u[8 + r], bufB[pB], cB, dB, t2B);
        }
      }
    }
    // ---- inverse: radix 8 (NS = 1) from registers, radix 8 (NS = 8), then the GEMM stage ----
    dft8<true>(u);
    dft8<true>(u + 8);
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      bufA[pad<3>(t * 8 + r)] = u[r];
      bufB[pad<3>(jB * 8 + r)] = u[8 + r];
    }
    __syncthreads();
    st_load<8, H, 3>(cbuf, tc, u);
    st_twiddle<8, H, 8, true>(tc, u, twT + P::TW.bM1);
    st_dft<8, true>(u);
    __syncthreads();
    st_store<8, H, 8, 4>(cbuf, tc, u);
    __syncthreads();
    {
      const C* gb = smem + gcol * CS;
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int r = 16 * ghh + i;
        u[i] = cmulc(gb[pad<4>(gj + 64 * r)], __ldg(twT + P::TW.bR1 + r * 64 + gj));
      }
    }
    ok &= tc_dft32<true>(a, sA, sExp, sBar, aBase, bBase, taddr, phase, grow, ghh, u, y);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const int mm = (k < 8) ? dm0 + k : 16 + dm0 + (k - 8);
      const uint32_t j2 = (uint32_t)(dj + 64 * mm);
      st_state(F + faddr<R>(W, j2, c, dcol), y[k], pol);
    }
  }
  if (!ok && threadIdx.x == 0) { atomicOr(&a.ctl->error, DEVERR_WAIT); }
  tc::fence_before();
  __syncthreads();
  if (w == 0) { tc::tmem_dealloc(taddr, kTcTmemCols); }
  ts_end(a, tslot);
}

// timeout probe of the tensor-core completion wait: an mbarrier that no MMA commit ever arrives on
static __global__ void k_tc_wait_probe(Args a) {
  OWL_SHARED(uint64_t, bar);
  if (threadIdx.x == 0) { tc::mbar_init(&bar, 1); }
  __syncthreads();
  const bool ok = tc::mbar_wait(&bar, 0, a.timeoutNs);
  if (!ok && threadIdx.x == 0) { atomicOr(&a.ctl->error, DEVERR_WAIT); }
}

}  // namespace owl

#include <vector>

#include "owl_tables.hpp"

namespace owl {

// Host: the 7 digit planes of the 32-point DFT matrix in the per-half swizzled K-major
// layout of tc_off_b (64 output rows n = 2 m + {re, im}, 64 inputs kb = 2 r + {re, im}),
// entries cos / sin of 2 pi r m / 32 scaled by 2^54 and rounded once.
inline std::vector<uint8_t> tc_dft_digits() {
  std::vector<uint8_t> out(kTcBBytes);
  for (int n = 0; n < kTcN; ++n) {
    for (int kb = 0; kb < kTcK; ++kb) {
      const int m = n / 2, cn = n & 1, r = kb / 2, ck = kb & 1;
      long double cs, sn;
      root_ld(kTcR1, (uint64_t)((r * m) % kTcR1), &cs, &sn);
      const long double v = cn == 0 ? (ck == 0 ? cs : sn) : (ck == 0 ? -sn : cs);
      const long long Y = llrintl(ldexpl(v, 54));
      const long long Z = Y + kTcBias;
      for (int p = 0; p < 7; ++p) {
        uint8_t b = (uint8_t)((unsigned long long)Z >> (8 * p));
        if (p < 6) { b ^= 0x80; }
        out[tc_off_b(6 - p, n, kb)] = b;
      }
    }
  }
  return out;
}

}  // namespace owl
