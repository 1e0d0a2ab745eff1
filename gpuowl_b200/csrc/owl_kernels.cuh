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
  const C* twH;    // stage tables of the height FFT (tw_offsets(H, 8) layout)
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
  long long* shuttle;  // carry rows, (H/R) x W
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
};

enum : int { P1_FUSED = 0, P1_IN = 1, P1_OUT = 2 };

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

// ---------------------------------------------------------------------------
// Pass 1: R lines of W points per CTA, R*W/16 threads, 16 values per thread.
template <int W, int R, int MODE>
__global__ void __launch_bounds__(R * W / 16, (R * W / 16 == 256) ? 2 : 1)
    k_pass1(Args a, C* __restrict__ F, int32_t* __restrict__ words, int roeSlot, int flags, int tslot) {
  constexpr int T = R * W / 16;
  constexpr int RL = 16 / R;
  using P = Plan<W, RL>;
  constexpr int PS_R1 = ilog2(P::R1);
  constexpr int PS_RL = ilog2(RL);
  constexpr int LS = p1_line_stride<W, R>();  // line stride in smem (elements), == 4 mod 8
  OWL_DYN_SHARED(C, smem);
  OWL_SHARED(uint32_t, s_g);
  OWL_SHARED_ARR(float, s_roe, 32);

  // Launched as a programmatic dependent of the column pass, a CTA may start before that pass has
  // completed. It then takes its ticket and reads its tables (nothing that pass writes) before
  // griddep_wait(), and the state after it. The ticket stays this launch's: the column pass's CTAs
  // call griddep_launch() only after their own griddep_wait(), so this pass starts no CTA before
  // the previous line pass, which took and reset the same counter, has completed.
  const int t = threadIdx.x;
  const uint32_t G = a.H / R;
  uint32_t g;
  if (MODE == P1_IN) {
    g = blockIdx.x;
  } else {
    if (t == 0) {
      uint32_t tk = atomicAdd(&a.ctl->ticket, 1u);
      if (tk == G - 1) { atomicExch(&a.ctl->ticket, 0u); }
      s_g = tk;
    }
    __syncthreads();
    g = s_g;
  }

  const unsigned long long pol = l2_keep_policy();
  const C* __restrict__ twW = a.twW;  // the width stage tables, read-only for the whole pass
  // The inter-pass twiddle w_hN^(k1 j2) of this group's lines is applied here, on the way out
  // (forward) and on the way in (inverse), not in the column pass: that pass is held by its FP64
  // pipe, this one by latency. With k1 = j + (W/R1) r it is base(j) * step(line)^r; the steps of
  // the R lines are tabulated per CTA (made visible by a barrier that the state loads overlap).
  OWL_SHARED_ARR(C, s_tw, 2 * 16);
  static_assert(R <= 2 && P::R1 <= 16, "line-pass twiddle table size");
  for (int i = t; i < R * P::R1; i += T) {
    const int ll = i / P::R1, rr = i % P::R1;
    s_tw[rr * R + ll] = bigtw(a, (uint32_t)(W / P::R1) * (uint32_t)rr * (g * R + ll));  // lines adjacent
  }
  // word classes of this thread's 32 words (fixed per shape, tabulated on the host)
  const uint2 wmask = __ldg(a.p1masks + (size_t)g * T + t);
  griddep_wait();
  griddep_launch();
  ts_begin(a, tslot);
  // per-line mapping for the inner stages
  const int l = t % R;
  const int tl = t / R;
  C* line = smem + l * LS;

  C v[16];  // cross-line layout: v[ll * RL + r] = line ll, column j1 = t + (W/RL) r
  float roe = 0.0f;

  if constexpr (MODE != P1_IN) {
    // ---- inverse width DFT ----
    {
      C u[16];
#pragma unroll
      for (int b = 0; b < 16 / P::R1; ++b) {
        int j = tl + (W / 16) * b;
#pragma unroll
        for (int r = 0; r < P::R1; ++r) {
          uint32_t k1 = j + r * (W / P::R1), c, s;
          colpair(W, k1, c, s);
          u[b * P::R1 + r] = ld_state(F + faddr<R>(W, g * R + l, c, s), pol);
        }
      }
      __syncthreads();  // s_tw
#pragma unroll
      for (int b = 0; b < 16 / P::R1; ++b) {
        const int j = tl + (W / 16) * b;
        const C base = bigtw(a, (uint32_t)j * (g * R + l));
#pragma unroll
        for (int r = 0; r < P::R1; ++r) { u[b * P::R1 + r] = cmulc(u[b * P::R1 + r], cmul(base, s_tw[r * R + l])); }
      }
      st_dft<P::R1, true>(u);
      st_store<P::R1, W, 1, PS_R1>(line, tl, u);
      __syncthreads();
      constexpr int NS2 = P::R1;
      constexpr int PS_AFTER_M1 = (P::M1 > 1) ? 4 : PS_R1;
      if constexpr (P::M1 > 1) {
        st_load<P::M1, W, PS_R1>(line, tl, u);
        st_twiddle<P::M1, W, NS2, true>(tl, u, twW + P::TW.aM1);
        st_dft<P::M1, true>(u);
        __syncthreads();
        st_store<P::M1, W, NS2, 4>(line, tl, u);
        __syncthreads();
      }
      constexpr int NS3 = NS2 * P::M1;
      constexpr int PS_AFTER_M2 = (P::M2 > 1) ? 4 : PS_AFTER_M1;
      if constexpr (P::M2 > 1) {
        st_load<P::M2, W, PS_AFTER_M1>(line, tl, u);
        st_twiddle<P::M2, W, NS3, true>(tl, u, twW + P::TW.aM2);
        st_dft<P::M2, true>(u);
        __syncthreads();
        st_store<P::M2, W, NS3, 4>(line, tl, u);
        __syncthreads();
      }
      // last stage, radix RL, across the R lines: butterfly j = t of every line
      constexpr int NSL = W / RL;
#pragma unroll
      for (int ll = 0; ll < R; ++ll) {
        const C* ln = smem + ll * LS;
#pragma unroll
        for (int r = 0; r < RL; ++r) { v[ll * RL + r] = ln[pad<PS_AFTER_M2>(t + r * NSL)]; }
        if constexpr (NSL > 1) {
#pragma unroll
          for (int r = 1; r < RL; ++r) { v[ll * RL + r] = cmulw<true>(v[ll * RL + r], __ldg(twW + P::TW.aRL + r * NSL + t)); }
        }
        dftR<RL, true>(v + ll * RL);
      }
    }
  }

  // ---- words: inverse weight, round, carry (or load digits for P1_IN) ----
  // Fused mode keeps the digits as doubles: with power-of-two scales the split
  // x = q 2^b + d, q = rint(x 2^-b), is exact in FP64 for |x| < 2^51, so no
  // integer conversion is needed. The block entry/exit modes use exact integers
  // (the exit mode must produce the canonical balanced digits).
  double dg[R][RL][2];
  long long dig[R][RL][2];
  const uint32_t bigmask = wmask.x;   // bit (r*R + ll)*2 + e: word is big
  const uint32_t wrapmask = wmask.y;  // bit (r*R + ll)*2 + e: X1 + X2 >= N (weight halved)
#pragma unroll
  for (int r = 0; r < RL; ++r) {
    const uint32_t j1 = t + (W / RL) * r;
    if constexpr (MODE == P1_IN) {
      // digits in natural word order: word 2(H j1 + j2) + e
#pragma unroll
      for (int ll = 0; ll < R; ++ll) {
        uint32_t j2 = g * R + ll;
        int2 w2 = *reinterpret_cast<const int2*>(words + 2 * ((size_t)a.H * j1 + j2));
        dg[ll][r][0] = (double)w2.x;
        dg[ll][r][1] = (double)w2.y;
      }
    } else {
      const double iw1 = __ldg(a.iwt1 + j1);
      const bool ll0 = (flags & FL_LL) && g == 0 && j1 == 0;
      double fcarry = ll0 ? -2.0 : 0.0;
      long long carry = ll0 ? -2 : 0;
#pragma unroll
      for (int ll = 0; ll < R; ++ll) {
        uint32_t j2 = g * R + ll;
        C z = v[ll * RL + r];
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int bit = (r * R + ll) * 2 + e;
          const bool wrap = (wrapmask >> bit) & 1u;
          const bool big = (bigmask >> bit) & 1u;
          double iw = iw1 * __ldg(a.iwt2 + 2 * j2 + e);
          if (wrap) { iw *= 2.0; }
          double x = e ? z.y : z.x;
          double d = fma(x, iw, RNDVAL);
          double rv = d - RNDVAL;
          roe = fmaxf(roe, (float)fabs(fma(x, iw, -rv)));
          if constexpr (MODE == P1_FUSED) {
            const double sc = big ? 2.0 * a.scaleLo : a.scaleLo;
            const double isc = big ? 0.5 * a.iscaleLo : a.iscaleLo;
            double xx = rv + fcarry;
            double q = fma(xx, isc, RNDVAL) - RNDVAL;
            dg[ll][r][e] = fma(q, -sc, xx);
            fcarry = q;
          } else {
            uint32_t bits = a.bitsLo + (big ? 1 : 0);
            long long n = __double_as_longlong(d) - __double_as_longlong(RNDVAL);
            if (flags & FL_MUL3) { n *= 3; }
            long long xx = n + carry;
            long long dd = sext_low(xx, bits);
            carry = (xx - dd) >> bits;
            dig[ll][r][e] = dd;
          }
        }
      }
      if constexpr (MODE == P1_FUSED) {
        a.shuttle[(size_t)g * W + j1] = __double_as_longlong(fcarry);
      } else {
        a.shuttle[(size_t)g * W + j1] = carry;
      }
    }
  }

  if constexpr (MODE == P1_IN) {
#pragma unroll
    for (int ll = 0; ll < R; ++ll) { p1_weight_line<W, R>(a, t, g, ll, dg[ll], wrapmask, v); }
#pragma unroll
    for (int ll = 0; ll < R; ++ll) { p1_fwd_first<W, R>(smem + ll * LS, t, v + ll * RL); }
    __syncthreads();
  } else {
    // publish this group's carry row: the barrier below orders every thread's shuttle stores
    // before thread 0's fence and release of the flag (one fence per CTA, as in a grid barrier)
    constexpr unsigned WMASK = (T >= 32) ? 0xffffffffu : ((1u << T) - 1u);
#pragma unroll
    for (int o = (T >= 32 ? 16 : T / 2); o > 0; o >>= 1) { roe = fmaxf(roe, __shfl_xor_sync(WMASK, roe, o)); }
    if ((t & 31) == 0) { s_roe[t >> 5] = roe; }
    __syncthreads();  // carries stored; the inverse DFT's shared-memory reads are done
    if (t == 0) {
      __threadfence();
      st_release(a.flags + g, 1u);
      float m = 0.0f;
      for (int i = 0; i < (T + 31) / 32; ++i) { m = fmaxf(m, s_roe[i]); }
      if (a.roe != nullptr && roeSlot >= 0) { atomicMax(reinterpret_cast<unsigned int*>(a.roe) + roeSlot, __float_as_uint(m)); }
    }
    if constexpr (MODE == P1_FUSED) {
      // lines 1..R-1 never see the carry-in in this mode: weight them and run
      // their first forward stage while the predecessor's carries arrive
#pragma unroll
      for (int ll = 1; ll < R; ++ll) {
        p1_weight_line<W, R>(a, t, g, ll, dg[ll], wrapmask, v);
        p1_fwd_first<W, R>(smem + ll * LS, t, v + ll * RL);
      }
    }
    // take the predecessor's carry row (bounded wait, decoupled lookback)
    if (t == 0) {
      const uint32_t prev = (g == 0) ? G - 1 : g - 1;
      unsigned long long t0 = gtimer();
      bool ok = false;
      for (uint32_t it = 0; it < (1u << 30); ++it) {
        if (ld_acquire(a.flags + prev) != 0u) { ok = true; break; }
        if ((it & 255u) == 255u && gtimer() - t0 > a.timeoutNs) { break; }
        spin_pause();
      }
      if (ok) {
        a.flags[prev] = 0u;
      } else {
        atomicOr(&a.ctl->error, DEVERR_WAIT);
      }
    }
    __syncthreads();
    // carry-in for line 0 of this group; column j1 of the last group wraps to
    // column j1 + 1 of group 0 (and the top word's carry to word 0)
    const uint32_t prevg = (g == 0) ? G - 1 : g - 1;
#pragma unroll
    for (int r = 0; r < RL; ++r) {
      const uint32_t j1 = t + (W / RL) * r;
      uint32_t src = (g == 0) ? (j1 == 0 ? W - 1 : j1 - 1) : j1;
      long long cin = __ldcg(a.shuttle + (size_t)prevg * W + src);
      if constexpr (MODE == P1_FUSED) {
        // sloppy: two words only, the digits feed the next FFT (carryFinal,
        // src/cl/carryinc.cl:18-23)
        const bool big0 = (bigmask >> ((r * R + 0) * 2 + 0)) & 1u;
        const double sc = big0 ? 2.0 * a.scaleLo : a.scaleLo;
        const double isc = big0 ? 0.5 * a.iscaleLo : a.iscaleLo;
        double xx = dg[0][r][0] + __longlong_as_double(cin);
        double q = fma(xx, isc, RNDVAL) - RNDVAL;
        dg[0][r][0] = fma(q, -sc, xx);
        dg[0][r][1] += q;
      } else {
        // block exit: propagate through the thread's whole chain so that every
        // digit is balanced -- the canonical form isEqual compares (carryB,
        // src/cl/carryb.cl:5-32); a carry that survives the chain is queued
        long long c = cin;
#pragma unroll
        for (int ll = 0; ll < R; ++ll) {
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            uint32_t bits = a.bitsLo + ((bigmask >> ((r * R + ll) * 2 + e)) & 1u);
            long long xx = dig[ll][r][e] + c;
            long long dd = sext_low(xx, bits);
            c = (xx - dd) >> bits;
            dig[ll][r][e] = dd;
          }
        }
        if (c != 0) {
          uint32_t i = atomicAdd(&a.ctl->npending, 1u);
          if (i < kPendingCap) {
            uint64_t next = 2ull * ((uint64_t)a.H * j1 + g * R + R);
            a.pending[2 * i] = (long long)(next % a.N);
            a.pending[2 * i + 1] = c;
          } else {
            atomicOr(&a.ctl->error, DEVERR_PENDING);
          }
        }
      }
    }
    if constexpr (MODE == P1_OUT) {
      // digits to natural word order
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        const uint32_t j1 = t + (W / RL) * r;
#pragma unroll
        for (int ll = 0; ll < R; ++ll) {
          uint32_t j2 = g * R + ll;
          int2 w2 = make_int2((int)dig[ll][r][0], (int)dig[ll][r][1]);
          *reinterpret_cast<int2*>(words + 2 * ((size_t)a.H * j1 + j2)) = w2;
        }
      }
      ts_end(a, tslot);
      return;
    } else {
      p1_weight_line<W, R>(a, t, g, 0, dg[0], wrapmask, v);
      p1_fwd_first<W, R>(smem, t, v);
      __syncthreads();
    }
  }

  if constexpr (MODE != P1_OUT) {
    // ---- rest of the forward width DFT ----
    C u[16];
    constexpr int NSa = RL;
    constexpr int PS_A = (P::M2 > 1) ? 4 : PS_RL;
    if constexpr (P::M2 > 1) {
      st_load<P::M2, W, PS_RL>(line, tl, u);
      st_twiddle<P::M2, W, NSa, false>(tl, u, twW + P::TW.bM2);
      st_dft<P::M2, false>(u);
      __syncthreads();
      st_store<P::M2, W, NSa, 4>(line, tl, u);
      __syncthreads();
    }
    constexpr int NSb = NSa * P::M2;
    constexpr int PS_B = (P::M1 > 1) ? 4 : PS_A;
    if constexpr (P::M1 > 1) {
      st_load<P::M1, W, PS_A>(line, tl, u);
      st_twiddle<P::M1, W, NSb, false>(tl, u, twW + P::TW.bM1);
      st_dft<P::M1, false>(u);
      __syncthreads();
      st_store<P::M1, W, NSb, 4>(line, tl, u);
      __syncthreads();
    }
    constexpr int NSc = NSb * P::M1;  // == W / R1
    st_load<P::R1, W, PS_B>(line, tl, u);
    st_twiddle<P::R1, W, NSc, false>(tl, u, twW + P::TW.bR1);
    st_dft<P::R1, false>(u);
    // outputs k1 = j + r (W/R1) straight to HBM
#pragma unroll
    for (int b = 0; b < 16 / P::R1; ++b) {
      int j = tl + (W / 16) * b;
      const C base = bigtw(a, (uint32_t)j * (g * R + l));
#pragma unroll
      for (int r = 0; r < P::R1; ++r) {
        uint32_t k1 = j + r * (W / P::R1), c, s;
        colpair(W, k1, c, s);
        st_state(F + faddr<R>(W, g * R + l, c, s), cmul(u[b * P::R1 + r], cmul(base, s_tw[r * R + l])), pol);
      }
    }
    ts_end(a, tslot);
  }
}

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
// Occupancy hint: 2 CTAs per SM for the 256-thread (and 512-thread VPT 8) columns; 3 for the
// 160-thread H = 1280 columns, which otherwise take 243 registers and run one 5-warp CTA per SM
// (5M: 45.5 -> 32.6 us per column pass with a few spilled registers). The 320-thread H = 2560
// columns stay at one CTA: two would cap them at 102 registers.
template <int H, int R, int MODE, int VPT = 16>
__global__ void __launch_bounds__(2 * H / VPT,
                                  ((2 * H / VPT == 256) || (VPT == 8 && 2 * H / VPT == 512)) ? 2 : (H == 1280 ? 3 : 1))
    k_pass2(Args a, C* __restrict__ F, const C* __restrict__ Fb, C* __restrict__ Fq, int tslot) {
  constexpr int RL = VPT / 2;
  constexpr int T = H / RL;
  constexpr int TC = H / VPT;  // threads per column in the per-column stages
  using P = Plan<H, RL, 0, VPT>;
  constexpr int PS_R1 = ilog2(P::R1);
  constexpr int PS_RL = ilog2(RL);
  constexpr int CS = p2_col_stride<H, VPT>();
  OWL_DYN_SHARED(C, smem);

  const uint32_t W = a.W;
  const uint32_t c = blockIdx.x;
  griddep_wait();
  griddep_launch();
  ts_begin(a, tslot);
  const int t = threadIdx.x;
  const int col = t / TC;
  const int tc = t % TC;
  const uint32_t kA = c, kB = (c == 0) ? W / 2 : W - c;
  (void)a.E;
  C* cbuf = smem + col * CS;
  // the HBM-facing first (forward) and last (inverse) stages interleave the two
  // columns across lanes, so that a warp's request covers whole 64-byte runs
  // (both columns of R lines of one line group) of the tile layout
  const int colI = (t >> 1) & 1;
  const int tcI = ((t >> 2) << 1) | (t & 1);
  C* cbufI = smem + colI * CS;

  const unsigned long long pol = l2_keep_policy();

  C u[VPT + 4];  // VPT values per thread; a radix-5 stage may run one butterfly more
  // ---- forward column DFT, first stage from HBM (the line pass applied the w_hN^(k1 j2) twiddle) ----
#pragma unroll
  for (int b = 0; b < VPT / P::R1; ++b) {
    int j = tcI + TC * b;
#pragma unroll
    for (int r = 0; r < P::R1; ++r) {
      uint32_t j2 = j + r * (H / P::R1);
      u[b * P::R1 + r] = ld_state(F + faddr<R>(W, j2, c, colI), pol);
    }
  }
  st_dft<P::R1, false, VPT>(u);
  st_store<P::R1, H, 1, PS_R1, VPT>(cbufI, tcI, u);
  __syncthreads();
  constexpr int PS_AFTER_M1 = (P::M1 > 1) ? 4 : PS_R1;
  if constexpr (P::M1 > 1) {
    st_load<P::M1, H, PS_R1, VPT>(cbuf, tc, u);
    st_twiddle<P::M1, H, P::R1, false, VPT>(tc, u, a.twH + P::TW.aM1);
    st_dft<P::M1, false, VPT>(u);
    __syncthreads();
    st_store<P::M1, H, P::R1, 4, VPT>(cbuf, tc, u);
    __syncthreads();
  }
  constexpr int PS_AFTER_M2 = (P::M2 > 1) ? 4 : PS_AFTER_M1;
  if constexpr (P::M2 > 1) {
    st_load<P::M2, H, PS_AFTER_M1, VPT>(cbuf, tc, u);
    st_twiddle<P::M2, H, P::R1 * P::M1, false, VPT>(tc, u, a.twH + P::TW.aM2);
    st_dft<P::M2, false, VPT>(u);
    __syncthreads();
    st_store<P::M2, H, P::R1 * P::M1, 4, VPT>(cbuf, tc, u);
    __syncthreads();
  }
  // last forward stage (radix RL, NS = H/RL = T): A butterfly t, B butterfly T-1-t
  const int jB = T - 1 - t;
  C* bufA = smem;
  C* bufB = smem + CS;
#pragma unroll
  for (int r = 0; r < RL; ++r) {
    u[r] = bufA[pad<PS_AFTER_M2>(t + r * T)];
    u[RL + r] = bufB[pad<PS_AFTER_M2>(jB + r * T)];
  }
  if constexpr (T > 1) {
#pragma unroll
    for (int r = 1; r < RL; ++r) {
      u[r] = cmul(u[r], __ldg(a.twH + P::TW.aRL + r * T + t));
      u[RL + r] = cmul(u[RL + r], __ldg(a.twH + P::TW.aRL + r * T + jB));
    }
  }
  dftR<RL, false>(u);
  dftR<RL, false>(u + RL);
  // now u[r] = ZA[t + T r], u[RL + r] = ZB[jB + T r]

  if constexpr (MODE == P2_FWD) {
#pragma unroll
    for (int r = 0; r < RL; ++r) {
      uint32_t kA2 = t + T * r, kB2 = jB + T * r;
      Fq[faddr<R>(W, kA2, c, 0)] = u[r];
      Fq[faddr<R>(W, kB2, c, 1)] = u[RL + r];
    }
    ts_end(a, tslot);
    return;
  } else {
    if (c != 0) {
      // w_hN^(c + W k2) with k2 = t + (H/RL) r is w_hN^c w_H^t w_RL^r
      const C base2 = cmul(bigtw(a, kA), __ldg(a.rootH + t));
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        uint32_t k2 = t + T * r;  // A index; partner is B[H-1-k2] = u[RL + RL-1 - r]
        C t2 = mul_w8<false>(base2, r * (8 / RL));
        if constexpr (MODE == P2_SQUARE) {
          pair_sq(u[r], u[2 * RL - 1 - r], t2);
        } else {
          C cA = Fb[faddr<R>(W, k2, c, 0)];
          C cB = Fb[faddr<R>(W, H - 1 - k2, c, 1)];
          pair_mul(u[r], u[2 * RL - 1 - r], cA, cB, t2);
        }
      }
    } else {
      // columns 0 and W/2 pair with themselves: exchange through smem
      __syncthreads();
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        bufA[t + T * r] = u[r];
        bufB[jB + T * r] = u[RL + r];
      }
      __syncthreads();
      const C baseA = __ldg(a.rootH + t);
      const C baseB = cmul(bigtw(a, W / 2), __ldg(a.rootH + jB));
#pragma unroll
      for (int r = 0; r < RL; ++r) {
        uint32_t kA2 = t + T * r;
        uint32_t pA = (kA2 == 0) ? 0u : H - kA2;
        uint32_t kB2 = jB + T * r;
        uint32_t pB = H - 1 - kB2;
        C t2A = mul_w8<false>(baseA, r * (8 / RL));
        C t2B = mul_w8<false>(baseB, r * (8 / RL));
        if constexpr (MODE == P2_SQUARE) {
          u[r] = one_sq(u[r], bufA[pA], t2A);
          u[RL + r] = one_sq(u[RL + r], bufB[pB], t2B);
        } else {
          C cA = Fb[faddr<R>(W, kA2, 0, 0)], dA = Fb[faddr<R>(W, pA, 0, 0)];
          C cB = Fb[faddr<R>(W, kB2, 0, 1)], dB = Fb[faddr<R>(W, pB, 0, 1)];
          u[r] = one_mul(u[r], bufA[pA], cA, dA, t2A);
          u[RL + r] = one_mul(u[RL + r], bufB[pB], cB, dB, t2B);
        }
      }
    }
    // ---- inverse column DFT: first stage (radix RL, NS = 1) from registers ----
    dftR<RL, true>(u);
    dftR<RL, true>(u + RL);
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RL; ++r) {
      bufA[pad<PS_RL>(t * RL + r)] = u[r];
      bufB[pad<PS_RL>(jB * RL + r)] = u[RL + r];
    }
    __syncthreads();
    constexpr int PS_I1 = (P::M2 > 1) ? 4 : PS_RL;
    if constexpr (P::M2 > 1) {
      st_load<P::M2, H, PS_RL, VPT>(cbuf, tc, u);
      st_twiddle<P::M2, H, RL, true, VPT>(tc, u, a.twH + P::TW.bM2);
      st_dft<P::M2, true, VPT>(u);
      __syncthreads();
      st_store<P::M2, H, RL, 4, VPT>(cbuf, tc, u);
      __syncthreads();
    }
    constexpr int NSi = RL * P::M2;
    constexpr int PS_I2 = (P::M1 > 1) ? 4 : PS_I1;
    if constexpr (P::M1 > 1) {
      st_load<P::M1, H, PS_I1, VPT>(cbuf, tc, u);
      st_twiddle<P::M1, H, NSi, true, VPT>(tc, u, a.twH + P::TW.bM1);
      st_dft<P::M1, true, VPT>(u);
      __syncthreads();
      st_store<P::M1, H, NSi, 4, VPT>(cbuf, tc, u);
      __syncthreads();
    }
    constexpr int NSl = NSi * P::M1;  // == H / R1
    st_load<P::R1, H, PS_I2, VPT>(cbufI, tcI, u);
    st_twiddle<P::R1, H, NSl, true, VPT>(tcI, u, a.twH + P::TW.bR1);
    st_dft<P::R1, true, VPT>(u);
#pragma unroll
    for (int b = 0; b < VPT / P::R1; ++b) {
      int j = tcI + TC * b;
#pragma unroll
      for (int r = 0; r < P::R1; ++r) {
        uint32_t j2 = j + r * (H / P::R1);
        st_state(F + faddr<R>(W, j2, c, colI), u[b * P::R1 + r], pol);
      }
    }
    ts_end(a, tslot);
  }
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
static __global__ void k_carry_fixup(Args a, int32_t* __restrict__ words) {
  if (threadIdx.x != 0 || blockIdx.x != 0) { return; }
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
