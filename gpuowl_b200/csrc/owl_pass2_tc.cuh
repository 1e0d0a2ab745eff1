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

constexpr int kTcSlices = 7;                    // base-256 digits per operand
constexpr int kTcRows = 128;                    // GEMM M: 2 columns x 64 sub-vectors
constexpr int kTcPanel = kTcRows * 64;          // bytes of one 64-byte-wide K panel of a data plane (8 KiB)
constexpr int kTcAlign = 1024;
// Both operands are K-major in the 64-byte swizzled layout (tc::sw64_off: 512-byte atoms of 8 rows
// of 64 bytes, SBO = 512). K beyond 64 bytes goes to a second panel of the same layout; a k-step
// (32 bytes of K) starts 32 bytes into a panel's rows or at the next panel.
constexpr uint32_t kTcSbo = 512;
constexpr uint32_t kTcTmemCols = 256;           // 7 accumulators x 32 columns, rounded to a power of two
constexpr long long kTcBias = 0x0000808080808080LL;  // 128 in each of the 6 low digit positions

// heights with a split-precision column pass
constexpr bool tc_height(int H) { return H == 2048 || H == 2560; }

// The per-height constants. The DFT digit planes are stored per output chunk: the chunk's NC output
// values (re / im of NC / 2 outputs), plane after plane, as one K-major operand of 7 NC rows (row
// q = NC j + n for plane j, output value n of the chunk). One MMA then multiplies data plane i by
// planes 0 .. 6-i at once (N = NC (7 - i)), and its output column NC (i + j) + n is accumulator
// d = i + j: each data plane is read once per k-step and chunk instead of once per diagonal.
template <int H> struct TcCfg {
  static_assert(tc_height(H), "split-precision heights: 2048, 2560");
  static constexpr int R1 = H == 2048 ? 32 : 40;        // GEMM radix
  static constexpr int KP = H == 2048 ? 64 : 96;        // K bytes, padded to k-steps of 32
  static constexpr int KSTEPS = KP / 32;
  static constexpr int PANELS = (KP + 63) / 64;
  static constexpr int NCH = H == 2048 ? 2 : 3;         // output chunks
  static constexpr int nc(int c) { return c < 2 ? 32 : 16; }  // output values of chunk c
  static constexpr int voff(int c) { return c == 0 ? 0 : voff(c - 1) + nc(c - 1); }
  static constexpr int bpanel(int c) { return kTcSlices * nc(c) * 64; }  // bytes of one K panel of chunk c
  static constexpr int boff(int c) { return c == 0 ? 0 : boff(c - 1) + PANELS * bpanel(c - 1); }
  static constexpr int BBYTES = boff(NCH);
  static constexpr int APLANE = PANELS * kTcPanel;      // bytes of one data digit plane
  static constexpr int NV = R1 / 2;                     // complex inputs a thread writes (2 threads a row)
  static constexpr int NY = R1 / 2;                     // complex outputs a thread drains
  static constexpr int CS = p2_col_stride<H>();
  static constexpr int COLBUF = 2 * CS * (int)sizeof(C);
  // dynamic shared memory: the region of the two column buffers, which the data digit planes overlay
  // (grown to hold them), the DFT digit planes, row exponents, the MMA barrier, the TMEM base; the
  // operands start 1024-byte aligned (the swizzle is on address bits 4-8), which the kernel arranges
  // at run time inside the 1 KiB of slack (kTcAlign)
  static constexpr int AREG0 = COLBUF > kTcSlices * APLANE ? COLBUF : kTcSlices * APLANE;
  static constexpr int OFFB = (AREG0 + kTcAlign - 1) / kTcAlign * kTcAlign;
  static constexpr int OFFEXP = OFFB + BBYTES;
  static constexpr int OFFBAR = OFFEXP + kTcRows * 4;
  static constexpr int OFFTADDR = OFFBAR + 8;
  static constexpr int SMEM = OFFTADDR + 8 + kTcAlign;
  static_assert(APLANE % kTcAlign == 0 && bpanel(NCH - 1) % kTcAlign == 0, "operand panels keep the swizzle alignment");
  static_assert(OFFB % 16 == 0 && OFFBAR % 8 == 0, "alignment");
  static_assert(SMEM <= 227 * 1024, "shared memory");
  static_assert(7 * nc(0) <= (int)kTcTmemCols, "accumulators of a chunk fit the tensor-memory allocation");
  static_assert(nc(0) == 32 && nc(1) == 32 && (NCH == 2 || nc(2) == 16), "chunks: 32, 32 (, 16) values");
};

// byte offset of data digit plane s, GEMM row `row`, K index kb
template <int H> __host__ __device__ constexpr uint32_t tc_off_a(int s, int row, int kb) {
  return (uint32_t)(s * TcCfg<H>::APLANE + (kb / 64) * kTcPanel) + tc::sw64_off(row, kb % 64);
}
// byte offset of DFT digit plane s, output value n (< 2 R1), K index kb in the per-chunk operands
template <int H> __host__ __device__ constexpr uint32_t tc_chunk_of(int n) {
  return (uint32_t)(n < 32 ? 0 : (n < 64 ? 1 : 2));
}
template <int H> __host__ __device__ constexpr uint32_t tc_off_b(int s, int n, int kb) {
  using G = TcCfg<H>;
  const int c = (int)tc_chunk_of<H>(n), nn = n - G::voff(c);
  return (uint32_t)(G::boff(c) + (kb / 64) * G::bpanel(c)) + tc::sw64_off(s * G::nc(c) + nn, kb % 64);
}

// the 7 digits of one value v (|v| < 2^54 after scaling), byte p of Z = Y + bias is digit 6 - p
__device__ __forceinline__ long long tc_digits_src(double v) { return __double2ll_rn(v) + kTcBias; }

// the 7 digit words of 4 int8 values each: word[6 - p] holds byte p of the four Z values
__device__ __forceinline__ void tc_digit_words(long long z0, long long z1, long long z2, long long z3,
                                               uint32_t (&wd)[kTcSlices]) {
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
    wd[6 - p] = word;
  }
}

// writes the digit planes of this thread's NV complex inputs (elements NV hh .. NV hh + NV - 1 of GEMM
// row `row`): 16-byte stores where the run is 16-byte aligned (H = 2048), 8-byte stores otherwise
template <int H, bool CONJ>
__device__ __forceinline__ void tc_put_digits(unsigned char* sA, int row, int hh, const C* x, double sc) {
  constexpr int NV = TcCfg<H>::NV;
  constexpr int G4 = (NV % 8 == 0) ? 2 : 1;  // groups of 4 complex values per store (16 or 8 bytes)
  static_assert(NV % (4 * G4) == 0, "digit stores of 4 or 8 complex values");
#pragma unroll
  for (int q = 0; q < NV / (4 * G4); ++q) {
    uint32_t wd[2 * G4][kTcSlices];
#pragma unroll
    for (int wi = 0; wi < 2 * G4; ++wi) {
      const C v0 = x[4 * G4 * q + 2 * wi], v1 = x[4 * G4 * q + 2 * wi + 1];
      tc_digit_words(tc_digits_src(v0.x * sc), tc_digits_src((CONJ ? -v0.y : v0.y) * sc), tc_digits_src(v1.x * sc),
                     tc_digits_src((CONJ ? -v1.y : v1.y) * sc), wd[wi]);
    }
    const int kb = 2 * (NV * hh + 4 * G4 * q);  // first K byte of these complex values
#pragma unroll
    for (int s = 0; s < kTcSlices; ++s) {
      if constexpr (G4 == 2) {
        *reinterpret_cast<uint4*>(sA + tc_off_a<H>(s, row, kb)) = make_uint4(wd[0][s], wd[1][s], wd[2][s], wd[3][s]);
      } else {
        *reinterpret_cast<uint2*>(sA + tc_off_a<H>(s, row, kb)) = make_uint2(wd[0][s], wd[1][s]);
      }
    }
  }
}

// issues the 7 KSTEPS MMAs of an output chunk of NC values whose DFT planes start at bChunk:
// accumulator d (TMEM columns NC d ..) gets sum_{i+j=d} A_i B_j^T. MMA (ks, i) multiplies data plane i
// by DFT planes 0 .. 6-i (N = NC (7 - i)) into columns NC i ..; the first one (ks = 0, i = 0) covers
// all 7 accumulators and initialises them.
template <int H, int NC> __device__ __forceinline__ void tc_issue(uint32_t aBase, uint32_t bChunk, uint32_t taddr) {
  using G = TcCfg<H>;
  constexpr uint32_t bPanel = (uint32_t)(kTcSlices * NC * 64);
#pragma unroll
  for (int ks = 0; ks < G::KSTEPS; ++ks) {
    const uint32_t kofs = (uint32_t)((ks % 2) * 32);  // k-steps 0, 1 in panel 0; 2 in panel 1
    const uint64_t bd = tc::smem_desc(bChunk + (uint32_t)(ks / 2) * bPanel + kofs, 16, kTcSbo, 4);
#pragma unroll
    for (int i = 0; i < kTcSlices; ++i) {
      const uint64_t ad =
          tc::smem_desc(aBase + (uint32_t)(i * G::APLANE + (ks / 2) * kTcPanel) + kofs, 16, kTcSbo, 4);
      tc::mma_s8(taddr + (uint32_t)(i * NC), ad, bd, tc::idesc_s8(kTcRows, NC * (kTcSlices - i)), i > 0 || ks > 0);
    }
  }
}

// drains an NC-value chunk's accumulators for this thread's GEMM output row (32 (warp % 4) + lane):
// the warp's half (warp / 4) of the chunk's columns, 4 complex outputs per 8 columns, into y[y0 ..]
template <int NC, bool INV>
__device__ __forceinline__ void tc_drain(uint32_t taddr, int w, double post, C* y, int y0) {
  const int q = w & 3, cs = (w >> 2) * (NC / 2);
  // D_d < (d + 1) 2^22, so D0 256 + D1, D2 256 + D3 and D4 256 + D5 are exact in INT32; the
  // rest of Horner's rule runs in FP64 (exact up to the last two steps, one rounding each)
#pragma unroll
  for (int g = 0; g < NC / 16; ++g) {
    const uint32_t tb = taddr + ((uint32_t)(32 * q) << 16) + (uint32_t)(cs + 8 * g);
    uint32_t ra[8], rb[8];
    int32_t p01[8], p23[8], p45[8];
    tc::tmem_ld8(tb + 0 * NC, ra);
    tc::tmem_ld8(tb + 1 * NC, rb);
    tc::tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < 8; ++i) { p01[i] = (int32_t)ra[i] * 256 + (int32_t)rb[i]; }
    tc::tmem_ld8(tb + 2 * NC, ra);
    tc::tmem_ld8(tb + 3 * NC, rb);
    tc::tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < 8; ++i) { p23[i] = (int32_t)ra[i] * 256 + (int32_t)rb[i]; }
    tc::tmem_ld8(tb + 4 * NC, ra);
    tc::tmem_ld8(tb + 5 * NC, rb);
    tc::tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < 8; ++i) { p45[i] = (int32_t)ra[i] * 256 + (int32_t)rb[i]; }
    tc::tmem_ld8(tb + 6 * NC, ra);
    tc::tmem_wait_ld();
    double v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      double acc = fma(tc::i32_to_f64(p01[i]), 65536.0, tc::i32_to_f64(p23[i]));
      acc = fma(acc, 65536.0, tc::i32_to_f64(p45[i]));
      v[i] = fma(acc, 256.0, tc::i32_to_f64((int32_t)ra[i])) * post;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) { y[y0 + 4 * g + k] = mk(v[2 * k], INV ? -v[2 * k + 1] : v[2 * k + 1]); }
  }
}

// one chunk: issue, wait for the tensor cores, drain (warps 0-7), and the barrier after which the
// accumulators may be overwritten
template <int H, int NC, bool INV>
__device__ __forceinline__ bool tc_chunk(const Args& a, uint64_t* sBar, uint32_t aBase, uint32_t bChunk, uint32_t taddr,
                                         uint32_t& phase, bool role, int w, double post, C* y, int y0) {
  if (threadIdx.x == 0) {
    tc::fence_after();
    tc_issue<H, NC>(aBase, bChunk, taddr);
    tc::commit(sBar);
  }
  const bool ok = tc::mbar_wait(sBar, phase & 1u, a.timeoutNs);
  ++phase;
  tc::fence_after();
  if (role) { tc_drain<NC, INV>(taddr, w, post, y, y0); }
  tc::fence_before();
  __syncthreads();  // all accumulator reads done before the next chunk overwrites them
  return ok;
}

// output index (within the R1-point DFT) of y[k] for a drain warp w: chunk by chunk, the warp's half
// of the chunk's outputs
template <int H> __device__ __forceinline__ int tc_out_index(int w, int k) {
  using G = TcCfg<H>;
  int base = 0;
#pragma unroll
  for (int c = 0; c < G::NCH; ++c) {
    const int per = G::nc(c) / 4;  // outputs of this warp in chunk c
    if (k < base + per) { return G::voff(c) / 2 + (w >> 2) * per + (k - base); }
    base += per;
  }
  return -1;
}

// The R1-point DFT (inverse when INV) of the 128 GEMM rows. Threads of warps 0-7 pass in elements
// NV hh + i of row `row` (x) and receive NY outputs of row drow = 32 (warp % 4) + lane, y[k] =
// X[tc_out_index(warp, k)]; warps 8 and up (H = 2560) only keep the barriers. The two 32-value
// chunks run as one loop (y indexed at run time), a 16-value third chunk after it.
// Returns false if the tensor cores did not finish within the plan's timeout.
template <int H, bool INV>
__device__ __forceinline__ bool tc_dft(const Args& a, unsigned char* sA, int* sExp, uint64_t* sBar, uint32_t aBase,
                                       uint32_t bBase, uint32_t taddr, uint32_t& phase, int row, int hh, const C* x,
                                       C* y) {
  using G = TcCfg<H>;
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const bool role = w < 8;
  int ex = 0;
  if (role) {
    double m = 0.0;
#pragma unroll
    for (int i = 0; i < G::NV; ++i) { m = fmax(m, fmax(fabs(x[i].x), fabs(x[i].y))); }
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 16));
    if (m > 0.0) { ex = (int)((__double_as_longlong(m) >> 52) & 0x7ff) - 1022; }  // m < 2^ex
    if (ex < -900) { ex = -900; }
  }
  __syncthreads();  // the digit planes overlay the column buffers the inputs were read from
  if (role) {
    if (hh == 0) { sExp[row] = ex; }
    tc_put_digits<H, INV>(sA, row, hh, x, tc::exp2i(54 - ex));
  }
  tc::fence_proxy_async();
  __syncthreads();
  const int drow = 32 * (w & 3) + lane;
  const double post = tc::exp2i(sExp[drow] - 60);
  bool ok = true;
#pragma unroll 1
  for (int c = 0; c < 2; ++c) {
    ok &= tc_chunk<H, 32, INV>(a, sBar, aBase, bBase + (uint32_t)(c * G::PANELS * kTcSlices * 32 * 64), taddr, phase,
                               role, w, post, y, 8 * c);
  }
  if constexpr (G::NCH == 3) {
    ok &= tc_chunk<H, 16, INV>(a, sBar, aBase, bBase + (uint32_t)G::boff(2), taddr, phase, role, w, post, y, 16);
  }
  return ok;
}

template <int H, int R, int MODE>
__global__ void __launch_bounds__(H / 8, H == 2048 ? 2 : 1)
    k_pass2_tc(Args a, const unsigned char* __restrict__ tcB, const C* __restrict__ twT, C* __restrict__ F,
               const C* __restrict__ Fb, C* __restrict__ Fq, int tslot) {
  using G = TcCfg<H>;
  constexpr int T = H / 8;
  constexpr int TC = H / 16;
  constexpr int R1 = G::R1;
  using P = Plan<H, 8, R1>;
  static_assert(P::R1 == R1 && P::M1 == 8 && P::M2 == 1 && H / R1 == 64, "split-precision column plan");
  constexpr int CS = G::CS;
  constexpr int PS1 = ilog2(R1);
  OWL_DYN_SHARED(C, smem);
  unsigned char* sm8 = reinterpret_cast<unsigned char*>(smem);
  // the operands 1024-byte aligned: the data planes overlay the column buffers from the first
  // aligned address; everything from the DFT planes on moves by the same amount
  const uint32_t alignPad = (uint32_t)(kTcAlign - (tc::smem_addr(sm8) & (kTcAlign - 1))) & (kTcAlign - 1);
  unsigned char* sA = sm8 + alignPad;
  unsigned char* sB = sm8 + alignPad + G::OFFB;
  int* sExp = reinterpret_cast<int*>(sm8 + alignPad + G::OFFEXP);
  uint64_t* sBar = reinterpret_cast<uint64_t*>(sm8 + alignPad + G::OFFBAR);
  uint32_t* sTaddr = reinterpret_cast<uint32_t*>(sm8 + alignPad + G::OFFTADDR);

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
  // GEMM input role (warps 0-7): row (column gcol, sub-vector gj), elements NV ghh ..
  const bool role = w < 8;
  const int gcol = (lane >> 1) & 1;
  const int gj = ((w & 7) << 3) | (((lane >> 2) & 3) << 1) | (lane & 1);
  const int ghh = lane >> 4;
  const int grow = gcol * 64 + gj;
  // GEMM output role (warps 0-7): row drow (column dcol, sub-vector dj), outputs tc_out_index(w, k)
  const int drow = 32 * (w & 3) + lane;
  const int dcol = drow >> 6, dj = drow & 63;
  const unsigned long long pol = l2_keep_policy();

  if (w == 0) {
    tc::tmem_alloc(sTaddr, kTcTmemCols);
    tc::tmem_relinquish();
  }
  if (t == 0) { tc::mbar_init(sBar, 1); }
  {
    const uint4* src = reinterpret_cast<const uint4*>(tcB);
    uint4* dst = reinterpret_cast<uint4*>(sB);
    for (int i = t; i < G::BBYTES / 16; i += T) { dst[i] = __ldg(src + i); }
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t taddr = *sTaddr;
  const uint32_t aBase = tc::smem_addr(sA), bBase = tc::smem_addr(sB);
  uint32_t phase = 0;
  bool ok = true;

  C u[G::NV > 16 ? G::NV : 16];
  C y[G::NY];
  // ---- forward: inputs from HBM (the line pass applied the w_hN^(k1 j2) twiddle) ----
  if (role) {
#pragma unroll
    for (int i = 0; i < G::NV; ++i) {
      const int r = G::NV * ghh + i;
      const uint32_t j2 = (uint32_t)(gj + 64 * r);
      u[i] = ld_state(F + faddr<R>(W, j2, c, gcol), pol);
    }
  }
  ok &= tc_dft<H, false>(a, sA, sExp, sBar, aBase, bBase, taddr, phase, grow, ghh, u, y);
  if (role) {
    C* db = smem + dcol * CS;
#pragma unroll
    for (int k = 0; k < G::NY; ++k) { db[pad<PS1>(dj * R1 + tc_out_index<H>(w, k))] = y[k]; }
  }
  __syncthreads();
  // ---- radix-8 middle stage (NS = R1) ----
  st_load<8, H, PS1>(cbuf, tc, u);
  st_twiddle<8, H, R1, false>(tc, u, twT + P::TW.aM1);
  st_dft<8, false>(u);
  __syncthreads();
  st_store<8, H, R1, 4>(cbuf, tc, u);
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
    if (role) {
      const C* gb = smem + gcol * CS;
#pragma unroll
      for (int i = 0; i < G::NV; ++i) {
        const int r = G::NV * ghh + i;
        u[i] = cmulc(gb[pad<4>(gj + 64 * r)], __ldg(twT + P::TW.bR1 + r * 64 + gj));
      }
    }
    ok &= tc_dft<H, true>(a, sA, sExp, sBar, aBase, bBase, taddr, phase, grow, ghh, u, y);
    if (role) {
#pragma unroll
      for (int k = 0; k < G::NY; ++k) {
        const uint32_t j2 = (uint32_t)(dj + 64 * tc_out_index<H>(w, k));
        st_state(F + faddr<R>(W, j2, c, dcol), y[k], pol);
      }
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

// Host: the 7 digit planes of the R1-point DFT matrix in the per-chunk swizzled K-major layout of
// tc_off_b (2 R1 output values n = 2 m + {re, im}, K indices kb = 2 r + {re, im} < 2 R1, zero up to
// KP), entries cos / sin of 2 pi r m / R1 scaled by 2^54 and rounded once.
template <int H> inline std::vector<uint8_t> tc_dft_digits() {
  using G = TcCfg<H>;
  std::vector<uint8_t> out(G::BBYTES, 0);
  for (int n = 0; n < 2 * G::R1; ++n) {
    for (int kb = 0; kb < G::KP; ++kb) {
      long long Y = 0;
      if (kb < 2 * G::R1) {
        const int m = n / 2, cn = n & 1, r = kb / 2, ck = kb & 1;
        long double cs, sn;
        root_ld(G::R1, (uint64_t)((r * m) % G::R1), &cs, &sn);
        const long double v = cn == 0 ? (ck == 0 ? cs : sn) : (ck == 0 ? -sn : cs);
        Y = llrintl(ldexpl(v, 54));
      }
      const long long Z = Y + kTcBias;
      for (int p = 0; p < 7; ++p) {
        uint8_t b = (uint8_t)((unsigned long long)Z >> (8 * p));
        if (p < 6) { b ^= 0x80; }
        out[tc_off_b<H>(6 - p, n, kb)] = b;
      }
    }
  }
  return out;
}

}  // namespace owl
