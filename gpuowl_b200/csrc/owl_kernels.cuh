// owl_kernels.cuh -- the IBDWT squaring passes for sm_100a.
//
// One iteration x <- x^2 (-2) mod 2^E-1 over N = 2*W*H FP64 words is two HBM
// passes over the hN = W*H complex state F (packing z[j] = x[2j] + i x[2j+1],
// the reference's kAt(), src/Gpu.cpp:40):
//
//   pass 2 ("column" pass, k_pass2): for each column pair (k1, W-k1) of the
//     W x H matrix A[k1][j2]: twiddle by w_hN^(k1 j2), forward length-H DFT,
//     real-signal squaring of Z[k] with Z[hN-k] (reference tailSquare /
//     pairSq, src/cl/tailsquare.cl:35-74), inverse DFT, untwiddle.
//   pass 1 ("line" pass, k_pass1): for each group of R lines j2: inverse
//     length-W DFT, inverse weight, round, balanced-digit carry, publish the
//     line group's carry-out, take the predecessor's carry-in (decoupled
//     lookback with a bounded wait), weight, forward length-W DFT (reference
//     carryFused, src/cl/carryfused.cl:21-231).
//
// Layout of F in HBM: tiles of R lines x one column pair. Element (column k1,
// line j2) lives at (((j2/R) * (W/2) + c) * 2 + s) * R + j2 % R where the pair
// index c and side s are c = k1, s = 0 for 0 < k1 < W/2; c = W-k1, s = 1 for
// k1 > W/2; (0,0) for k1 = 0 and (0,1) for k1 = W/2. Pass 1 reads one
// contiguous block of R*W elements; pass 2 reads 2*R contiguous elements per
// line group, and each 32-byte sector it touches is used whole.
#pragma once
#include "owl_compat.cuh"
#include "owl_dft.cuh"

namespace owl {

struct Ctl {
  uint32_t ticket;    // line-group ticket for the carry chain (reset by the last taker)
  uint32_t error;     // DEVERR_* bits, sticky until the host clears them
  uint32_t npending;  // carries left over at the end of a thread's word chain (block exit only)
  uint32_t pad[29];
};

enum : uint32_t { DEVERR_WAIT = 1u, DEVERR_PENDING = 2u };
constexpr uint32_t kPendingCap = 1024;

struct Args {
  // the carry's two FP64 constants first, as a 16-byte-aligned pair (with them at offset 184 the
  // 8M line pass spilled a register and ran 1.8 us slower)
  double scaleLo;      // 2^bitsLo
  double iscaleLo;     // 2^-bitsLo
  const C* twW;    // stage tables of the width FFT (tw_offsets(W, 16/R) layout)
  const C* twH;    // stage tables of the height FFT (tw_offsets(H, V / 2, 0, V) layout, V = col_vpt(variant))
  const C* rootH;  // w_H^i, i < H
  const C* twLo;   // w_hN^i, i < 2^loShift
  const C* twHi;   // w_hN^(i << loShift)
  const double* wt1;   // per column j1: 2^(X1/N)
  const double* iwt1;  // per column j1: 2^(-X1/N)
  const uint32_t* x1;  // per column j1: X1 = step*2H*j1 mod N
  const double* wt2;   // per (line j2, e): 2^(X2/N)
  const double* iwt2;  // per (line j2, e): 2^(-X2/N) / (4 hN)
  const uint32_t* x2;  // per (line j2, e): X2 = step*(2 j2 + e) mod N
  const uint2* p1masks; // per (line group g, pass-1 thread t): the big-word and wrap bits of the thread's
                        // 32 words, bit (r R + ll) 2 + e for column t + (W/RL) r, line g R + ll, word e
  long long* shuttle;  // carry words, (H/R) x W; 0 = consumed, else the carry encoded (kCarryOffset)
  long long* pending;  // (word index, carry) pairs, kPendingCap entries
  uint32_t* flags;     // per line group
  Ctl* ctl;
  float* roe;          // per-launch max round-off slots
  unsigned long long* tsStart;  // per-launch earliest CTA start (%globaltimer), profiling only
  unsigned long long* tsEnd;    // per-launch latest CTA end
  uint32_t E, N, W, H, hN;
  uint32_t bitsLo;     // E / N
  uint32_t eModN;      // E % N (a word is big iff its extra < E % N)
  uint32_t loShift;
  unsigned long long timeoutNs;
  const unsigned char* tc1B;  // the split line pass's 16-point DFT digit planes (W = 2048), else null
};

enum : int { P1_FUSED = 0, P1_IN = 1, P1_OUT = 2 };

}  // namespace owl
#include "owl_tc.cuh"
#include "owl_line_tc.cuh"
namespace owl {

// smem strides: room for the largest padding used (one pad per 2^PS elements,
// PS >= 2), rounded so that consecutive lines start 4 elements apart mod 8
template <int W, int R> constexpr int p1_line_stride() {
  constexpr int ps = ilog2(16 / R) < ilog2(Plan<W, 16 / R>::R1) ? ilog2(16 / R) : ilog2(Plan<W, 16 / R>::R1);
  return W + (W >> ps) + 4;
}
// room for the smallest padding the column pass uses (one pad per RL = VPT/2 elements)
template <int H, int VPT = 16> constexpr int p2_col_stride() { return H + (H >> ilog2(VPT / 2)) + 4; }
enum : int { P2_SQUARE = 0, P2_FWD = 1, P2_MUL = 2 };
enum : int { FL_MUL3 = 1, FL_LL = 2 };

template <int R> __device__ __forceinline__ uint32_t faddr(uint32_t W, uint32_t j2, uint32_t c, uint32_t s) {
  return (((j2 / R) * (W / 2) + c) * 2 + s) * R + (j2 % R);
}
// pair index and side of column k1
__device__ __forceinline__ void colpair(uint32_t W, uint32_t k1, uint32_t& c, uint32_t& s) {
  if (k1 == 0) {
    c = 0; s = 0;
  } else if (k1 == W / 2) {
    c = 0; s = 1;
  } else if (k1 < W / 2) {
    c = k1; s = 0;
  } else {
    c = W - k1; s = 1;
  }
}

// w_hN^m, m < hN, from the two-level table (one rounding in the product)
__device__ __forceinline__ C bigtw(const Args& a, uint32_t m) {
  C lo = __ldg(a.twLo + (m & ((1u << a.loShift) - 1)));
  C hi = __ldg(a.twHi + (m >> a.loShift));
  return cmul(lo, hi);
}

__device__ __forceinline__ long long sext_low(long long x, uint32_t bits) {
  return (long long)((unsigned long long)x << (64 - bits)) >> (64 - bits);
}

constexpr double RNDVAL = 3.0 * 2251799813685248.0;  // 3 * 2^51
// offset of an integer carry word in the carry rows (words are never 0: 0 marks a consumed word)
constexpr long long kCarryOffset = 1ll << 62;

// launch timestamps for the profiler: slot < 0 turns them off
__device__ __forceinline__ void ts_begin(const Args& a, int slot) {
  if (slot >= 0 && threadIdx.x == 0) { atomicMin(a.tsStart + slot, gtimer()); }
}
__device__ __forceinline__ void ts_end(const Args& a, int slot) {
  if (slot >= 0 && threadIdx.x == 0) { atomicMax(a.tsEnd + slot, gtimer()); }
}

// weight line ll of a pass-1 group: digits dgl[r][e] of column j1 = t + (W/RL) r
// times 2^(extra/N), halved where the two table exponents wrap past N
template <int W, int R>
__device__ __forceinline__ void p1_weight_line(const Args& a, int t, uint32_t g, int ll, const double (&dgl)[16 / R][2],
                                               uint32_t wrapmask, C* v) {
  constexpr int RL = 16 / R;
  const uint32_t j2 = g * R + ll;
  const double w20 = __ldg(a.wt2 + 2 * j2), w21 = __ldg(a.wt2 + 2 * j2 + 1);
#pragma unroll
  for (int r = 0; r < RL; ++r) {
    const uint32_t j1 = t + (W / RL) * r;
    const double w1 = __ldg(a.wt1 + j1);
    double y0 = dgl[r][0] * (w1 * w20);
    double y1 = dgl[r][1] * (w1 * w21);
    if ((wrapmask >> ((r * R + ll) * 2 + 0)) & 1u) { y0 *= 0.5; }
    if ((wrapmask >> ((r * R + ll) * 2 + 1)) & 1u) { y1 *= 0.5; }
    v[ll * RL + r] = mk(y0, y1);
  }
}

// first forward width stage (radix 16/R, NS = 1) of one line, from registers to
// shared memory
template <int W, int R> __device__ __forceinline__ void p1_fwd_first(C* ln, int t, C* vl) {
  constexpr int RL = 16 / R;
  dftR<RL, false>(vl);
#pragma unroll
  for (int r = 0; r < RL; ++r) { ln[pad<ilog2(RL)>(t * RL + r)] = vl[r]; }
}

// Pass 1 (the line pass) runs R lines of W points per CTA, R*W/16 threads, 16 values per thread:
// its body is owl_pass1_body.inc, its kernels k_pass1 / k_pass1_group follow the column pass below.

// ---------------------------------------------------------------------------
// Pass 2: one column pair (A: k1 = c, B: k1 = W - c; pair 0 is (0, W/2)) of H
// points per CTA, H/8 threads. Per-column stages use threads [0, H/16) for A
// and [H/16, H/8) for B; the last forward / first inverse stage (radix 8) runs
// butterfly j = t of A and j = H/8-1-t of B in the same thread, so that the
// thread ends up holding A[k2] and its partner B[H-1-k2] (src/cl/tailsquare.cl
// pairs lines k and H-k the same way, 225-313).

// real-signal squaring of the pair (a = Z[k], b = Z[hN-k]) with t2 = w_hN^k:
// returns 4 W[k] in a and 4 W[hN-k] in b.
__device__ __forceinline__ void pair_sq(C& a, C& b, C t2) {
  C bc = cconj(b);
  C e2 = cadd(a, bc);
  C o2 = cmulmi(csub(a, bc));
  C s = cadd(csq(e2), cmul(t2, csq(o2)));
  C p = cmuli(cmul(e2, o2));
  p = mk(2.0 * p.x, 2.0 * p.y);
  a = cadd(s, p);
  b = cconj(csub(s, p));
}

// product of two signals: (a, b) pair of the first, (c, d) of the second
__device__ __forceinline__ void pair_mul(C& a, C& b, C c, C d, C t2) {
  C bc = cconj(b), dc = cconj(d);
  C e2a = cadd(a, bc), o2a = cmulmi(csub(a, bc));
  C e2b = cadd(c, dc), o2b = cmulmi(csub(c, dc));
  C s = cadd(cmul(e2a, e2b), cmul(t2, cmul(o2a, o2b)));
  C p = cmuli(cadd(cmul(e2a, o2b), cmul(o2a, e2b)));
  a = cadd(s, p);
  b = cconj(csub(s, p));
}

// one-sided version for the self-paired columns 0 and W/2 (a = Z[k], b = Z[partner])
__device__ __forceinline__ C one_sq(C a, C b, C t2) {
  C bc = cconj(b);
  C e2 = cadd(a, bc);
  C o2 = cmulmi(csub(a, bc));
  C s = cadd(csq(e2), cmul(t2, csq(o2)));
  C p = cmuli(cmul(e2, o2));
  return cadd(s, mk(2.0 * p.x, 2.0 * p.y));
}
__device__ __forceinline__ C one_mul(C a, C b, C c, C d, C t2) {
  C bc = cconj(b), dc = cconj(d);
  C e2a = cadd(a, bc), o2a = cmulmi(csub(a, bc));
  C e2b = cadd(c, dc), o2b = cmulmi(csub(c, dc));
  C s = cadd(cmul(e2a, e2b), cmul(t2, cmul(o2a, o2b)));
  C p = cmuli(cadd(cmul(e2a, o2b), cmul(o2a, e2b)));
  return cadd(s, p);
}

// VPT: values per thread (16, or 8 for twice the threads at half the registers); the
// cross-column last stage has radix RL = VPT/2 (A and B butterflies in one thread).
// Occupancy hint (MINB = 0): 2 CTAs per SM for the 256-thread (and 512-thread VPT 8) columns; 3 for
// the 160-thread H = 1280 columns, which otherwise take 243 registers and run one 5-warp CTA per SM
// (5M: 45.5 -> 32.6 us per column pass with a few spilled registers). The 320-thread H = 2560
// columns take one CTA, or two with MINB = 2 (the COL_V16_OCC2 variant: 102 registers).

// ---------------------------------------------------------------------------
// The pass kernels: one plan (k_pass1, k_pass2), or the same pass of up to kGroupMax plans of one
// shape in one launch (blockIdx.y = plan), which a batch of exponents uses so that one launch per
// pass and shape replaces a launch per plan.

// ROE: measure the round-off |x - rint(x)| into roe[roeSlot]. The reference measures it on a
// sample of iterations only, with a separate kernel build (kCarryFusedROE vs kCarryFused,
// src/Gpu.cpp:592-596); the fused line pass without it runs about 0.8 us faster at 8M.
// SPLIT (W = 2048 only): the first inverse and last forward radix-16 stages as INT8 tensor-core
// GEMMs (owl_line_tc.cuh), the split-precision form of the line pass.
template <int W, int R, int MODE, bool ROE = true, bool SPLIT = false>
__global__ void __launch_bounds__(R * W / 16, (R * W / 16 == 256) ? 2 : 1)
    k_pass1(Args a, C* __restrict__ F, int32_t* __restrict__ words, int roeSlot, int flags, int tslot) {
  constexpr bool REGBOUND = false;
  const uint32_t blk = blockIdx.x;
#include "owl_pass1_body.inc"
}

template <int H, int R, int MODE, int VPT = 16, int MINB = 0>
__global__ void __launch_bounds__(2 * H / VPT,
                                  MINB ? MINB
                                       : (((2 * H / VPT == 256) || (VPT == 8 && 2 * H / VPT == 512)) ? 2
                                                                                                     : (H == 1280 ? 3 : 1)))
    k_pass2(Args a, C* __restrict__ F, const C* __restrict__ Fb, C* __restrict__ Fq, int tslot) {
  const uint32_t blk = blockIdx.x;
#include "owl_pass2_body.inc"
}

constexpr int kGroupMax = 16;
// the plans of a grouped launch: their arguments, FFT state and word buffers (in place)
struct GroupArgs {
  Args a[kGroupMax];
  C* F[kGroupMax];
  int32_t* words[kGroupMax];
};

// The grouped kernels run many CTAs of several plans at once, so they are built for occupancy
// (occ_blocks: 16 resident warps at most 128 registers); the one-plan kernels of the small FFTs run
// few CTAs, latency-bound, and keep all the registers they want (a single 256K plan: 0.0157 ->
// 0.0142 ms/iter without the occupancy bound; the 64-exponent batch: 90.6k -> 163.6k iter/s with
// grouping and the bound, measured on one box).
template <int W, int R, int MODE, bool ROE = true>
__global__ void __launch_bounds__(R * W / 16, occ_blocks(R * W / 16))
    k_pass1_group(const __grid_constant__ GroupArgs ga, int roeSlot, int flags) {
  constexpr bool SPLIT = false;
  constexpr bool REGBOUND = true;
  const Args& a = ga.a[blockIdx.y];
  C* __restrict__ F = ga.F[blockIdx.y];
  int32_t* __restrict__ words = ga.words[blockIdx.y];
  const int tslot = -1;
  const uint32_t blk = blockIdx.x;
#include "owl_pass1_body.inc"
}

template <int H, int R, int VPT = 16, int MINB = 0>
__global__ void __launch_bounds__(2 * H / VPT,
                                  MINB ? MINB
                                       : ((VPT == 8 && 2 * H / VPT == 512)
                                              ? 2
                                              : (H == 1280 ? 3 : (H == 2560 ? 1 : occ_blocks(2 * H / VPT)))))
    k_pass2_group(const __grid_constant__ GroupArgs ga) {
  constexpr int MODE = P2_SQUARE;
  const Args& a = ga.a[blockIdx.y];
  C* __restrict__ F = ga.F[blockIdx.y];
  const C* __restrict__ Fb = nullptr;
  C* __restrict__ Fq = nullptr;
  const int tslot = -1;
  const uint32_t blk = blockIdx.x;
#include "owl_pass2_body.inc"
}

// ---------------------------------------------------------------------------
// small helpers

// out[0] &= (a == b) over n int32 (outEq must hold 1 on entry)
static __global__ void k_is_equal(const int32_t* __restrict__ a, const int32_t* __restrict__ b, size_t n, int* outEq) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  size_t stride = (size_t)gridDim.x * blockDim.x;
  bool eq = true;
  for (; i < n; i += stride) { eq &= (a[i] == b[i]); }
  if (!__all_sync(0xffffffffu, eq)) {
    if ((threadIdx.x & 31) == 0) { atomicAnd(outEq, 0); }
  }
}

// 64-bit checksum of n int32 taken as n/2 u64 (reference sum64, src/cl/etc.cl:19-29)
static __global__ void k_sum64(const unsigned long long* __restrict__ in, size_t n64, unsigned long long* out) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  size_t stride = (size_t)gridDim.x * blockDim.x;
  unsigned long long s = 0;
  for (; i < n64; i += stride) { s += in[i]; }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) { s += __shfl_xor_sync(0xffffffffu, s, o); }
  if ((threadIdx.x & 31) == 0) { atomicAdd(out, s); }
}

// words around the wrap: out[i] = data[(N - 32 + i) mod N], i < 64
static __global__ void k_gather_residue(const int32_t* __restrict__ data, uint32_t N, int32_t* out) {
  int i = threadIdx.x;
  if (i < 64) { out[i] = data[(N - 32 + i) % N]; }
}

// Applies the carries queued by a block-exit line pass, one after the other,
// each propagated word by word (with wrap-around) until it is absorbed.
__device__ __forceinline__ void carry_fixup(const Args& a, int32_t* __restrict__ words) {
  uint32_t n = a.ctl->npending;
  if (n > kPendingCap) { n = kPendingCap; }
  const uint64_t step = a.N - a.E % a.N;
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t w = (uint32_t)a.pending[2 * i];
    long long c = a.pending[2 * i + 1];
    for (uint32_t k = 0; c != 0 && k < a.N; ++k) {
      uint32_t extra = (uint32_t)((step * w) % a.N);
      uint32_t bits = a.bitsLo + (extra < a.eModN ? 1u : 0u);
      long long xx = (long long)words[w] + c;
      long long dd = sext_low(xx, bits);
      c = (xx - dd) >> bits;
      words[w] = (int32_t)dd;
      w = (w + 1 == a.N) ? 0 : w + 1;
    }
  }
  a.ctl->npending = 0;
}
static __global__ void k_carry_fixup(Args a, int32_t* __restrict__ words) {
  if (threadIdx.x != 0 || blockIdx.x != 0) { return; }
  carry_fixup(a, words);
}
// one plan per CTA
static __global__ void k_carry_fixup_group(const __grid_constant__ GroupArgs ga) {
  if (threadIdx.x != 0) { return; }
  carry_fixup(ga.a[blockIdx.x], ga.words[blockIdx.x]);
}

// timeout probe: wait on a flag that is never set, with the pass-1 wait loop
static __global__ void k_wait_probe(Args a, uint32_t flagIndex) {
  if (threadIdx.x == 0) {
    unsigned long long t0 = gtimer();
    bool ok = false;
    for (uint32_t it = 0; it < (1u << 30); ++it) {
      if (ld_acquire(a.flags + flagIndex) != 0u) { ok = true; break; }
      if ((it & 255u) == 255u && gtimer() - t0 > a.timeoutNs) { break; }
      spin_pause();
    }
    if (!ok) { atomicOr(&a.ctl->error, DEVERR_WAIT); }
  }
}

}  // namespace owl
