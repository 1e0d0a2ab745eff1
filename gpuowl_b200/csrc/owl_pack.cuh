// owl_pack.cuh -- device-side conversion between the compact E-bit form (nWords
// 32-bit words, little-endian) and the balanced digits the engine works on, the
// same results bit for bit as the host restatements in owl_words.hpp of the
// reference's expandBits (src/state.cpp:93-115) and compactBits (26-69).
//
// Word k holds bits [off(k), off(k+1)) with off(k) = ceil(k E / N) (the word
// model of src/state.h:14-17 in closed form). Both conversions are a carry
// chain with carries in {0, 1} (expand) or borrows in {0, -1} (compact). Each
// digit either kills the incoming carry, generates one, or propagates it, so
// the chain is a scan of the operator compose(lower, upper) = upper unless
// upper propagates. Three launches: per-block summaries of 1024 digits, a
// one-thread pass over the block summaries, then the digits (or packed words)
// with each digit's carry taken from the scan inside its block.
#pragma once
#include <cstdint>

#include "owl_compat.cuh"

namespace owl {

constexpr int kPackDigits = 1024;  // digits per CTA
constexpr int kPackThreads = 256;  // 4 digits per thread
enum : uint32_t { ST_KILL = 0, ST_GEN = 1, ST_PROP = 2 };

struct PackCtl {
  uint32_t carryOut;  // carry (expand) or borrow flag (compact) out of the top digit
  uint32_t error;     // compact: a digit outside [-2^bits, 2^bits)
};

__device__ __forceinline__ uint64_t pk_off(uint64_t k, uint32_t E, uint32_t N) { return (k * E + N - 1) / N; }
__device__ __forceinline__ uint32_t pk_compose(uint32_t lower, uint32_t upper) {
  return upper == ST_PROP ? lower : upper;
}

// bits [off, off + len) of the word array, len <= 32
__device__ __forceinline__ uint32_t pk_bits(const uint32_t* w, uint32_t nw, uint64_t off, uint32_t len) {
  const uint32_t i = (uint32_t)(off >> 5), s = (uint32_t)(off & 31);
  uint64_t v = w[i];
  if (i + 1 < nw) { v |= (uint64_t)w[i + 1] << 32; }
  return (uint32_t)((v >> s) & ((1ull << len) - 1));
}

// expand: status of raw digit v of len bits (carry in c gives v + c; out = [v + c >= 2^(len-1)])
__device__ __forceinline__ uint32_t pk_expand_status(uint32_t v, uint32_t len) {
  const uint32_t half = 1u << (len - 1);
  return v >= half ? ST_GEN : (v + 1 == half ? ST_PROP : ST_KILL);
}
// compact: borrow out of digit d (borrow in b gives d + b; out = [d + b < 0])
__device__ __forceinline__ uint32_t pk_compact_status(int32_t d) {
  return d < 0 ? ST_GEN : (d > 0 ? ST_KILL : ST_PROP);
}

// status of the digits [k0, k0 + 4) of this thread, in increasing order
template <bool EXPAND>
__device__ __forceinline__ uint32_t pk_thread_status(const uint32_t* words, const int32_t* digits, uint32_t nw,
                                                     uint32_t E, uint32_t N, uint32_t k0, uint32_t* st) {
  uint32_t agg = ST_PROP;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint32_t k = k0 + i;
    uint32_t s = ST_PROP;
    if (k < N) {
      if constexpr (EXPAND) {
        const uint64_t o = pk_off(k, E, N);
        const uint32_t len = (uint32_t)(pk_off(k + 1, E, N) - o);
        s = pk_expand_status(pk_bits(words, nw, o, len), len);
      } else {
        s = pk_compact_status(digits[k]);
      }
    }
    st[i] = s;
    agg = pk_compose(agg, s);
  }
  return agg;
}

// K1: one status per block of 1024 digits
template <bool EXPAND>
__global__ void __launch_bounds__(kPackThreads) k_pack_summary(const uint32_t* __restrict__ words,
                                                                const int32_t* __restrict__ digits, uint32_t nw,
                                                                uint32_t E, uint32_t N, uint32_t* __restrict__ blk) {
  OWL_SHARED_ARR(uint32_t, s_st, kPackThreads);
  const uint32_t t = threadIdx.x;
  uint32_t st[4];
  s_st[t] = pk_thread_status<EXPAND>(words, digits, nw, E, N, blockIdx.x * kPackDigits + 4 * t, st);
  __syncthreads();
  if (t == 0) {
    uint32_t agg = ST_PROP;
    for (int i = 0; i < kPackThreads; ++i) { agg = pk_compose(agg, s_st[i]); }
    blk[blockIdx.x] = agg;
  }
}

// K2: block carries in, in order; blk[b] becomes the carry into block b (0/1). One CTA of
// kPackThreads threads: each thread composes the statuses of its run of consecutive blocks, the runs'
// statuses are scanned in shared memory (Hillis-Steele with pk_compose, which is associative), and
// each thread then walks its run with the carry into it. A single thread walking all the blocks
// would make one dependent global load per 1,024 digits (8,192 in a row at 8M).
static __global__ void __launch_bounds__(kPackThreads) k_pack_chain(uint32_t* __restrict__ blk, uint32_t nblocks,
                                                                    PackCtl* ctl) {
  OWL_SHARED_ARR(uint32_t, s_run, kPackThreads);
  const uint32_t t = threadIdx.x;
  const uint32_t per = (nblocks + kPackThreads - 1) / kPackThreads;
  const uint32_t lo = (t * per < nblocks) ? t * per : nblocks;
  const uint32_t hi = (lo + per < nblocks) ? lo + per : nblocks;
  uint32_t agg = ST_PROP;  // an empty run propagates
  for (uint32_t b = lo; b < hi; ++b) { agg = pk_compose(agg, blk[b]); }
  s_run[t] = agg;
  __syncthreads();
  for (uint32_t off = 1; off < kPackThreads; off <<= 1) {
    const uint32_t v = (t >= off) ? pk_compose(s_run[t - off], s_run[t]) : s_run[t];
    __syncthreads();
    s_run[t] = v;
    __syncthreads();
  }
  // carry into this run: the composed status of all runs below; none below, or all propagating: 0
  uint32_t c = (t == 0) ? (uint32_t)ST_KILL : s_run[t - 1];
  if (c == ST_PROP) { c = ST_KILL; }
  for (uint32_t b = lo; b < hi; ++b) {
    const uint32_t st = blk[b];
    blk[b] = c;
    c = (st == ST_PROP) ? c : st;
  }
  if (lo < hi && hi == nblocks) { ctl->carryOut = c; }
  if (t == 0) { ctl->error = 0; }
}

// carry into this thread's first digit: the nearest non-propagating thread below, else the block's
__device__ __forceinline__ uint32_t pk_carry_in(const uint32_t* s_st, uint32_t t, uint32_t blockCarry) {
  for (int j = (int)t - 1; j >= 0; --j) {
    if (s_st[j] != ST_PROP) { return s_st[j]; }
  }
  return blockCarry;
}

// K3 (expand): balanced digits; digit 0 also takes the carry out of the top digit and any bits above E
static __global__ void __launch_bounds__(kPackThreads) k_expand_digits(const uint32_t* __restrict__ words, uint32_t nw,
                                                                       uint32_t E, uint32_t N,
                                                                       const uint32_t* __restrict__ blk,
                                                                       const PackCtl* ctl, int32_t* __restrict__ out) {
  OWL_SHARED_ARR(uint32_t, s_st, kPackThreads);
  const uint32_t t = threadIdx.x;
  const uint32_t k0 = blockIdx.x * kPackDigits + 4 * t;
  uint32_t st[4];
  s_st[t] = pk_thread_status<true>(words, nullptr, nw, E, N, k0, st);
  __syncthreads();
  uint32_t c = pk_carry_in(s_st, t, blk[blockIdx.x]);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint32_t k = k0 + i;
    if (k >= N) { break; }
    const uint64_t o = pk_off(k, E, N);
    const uint32_t len = (uint32_t)(pk_off(k + 1, E, N) - o);
    const int64_t w = (int64_t)pk_bits(words, nw, o, len) + c;
    const int64_t half = 1ll << (len - 1);
    int32_t d;
    if (w >= half) {
      d = (int32_t)(w - (1ll << len));
      c = 1;
    } else {
      d = (int32_t)w;
      c = 0;
    }
    if (k == 0) { d += (int32_t)(ctl->carryOut + (words[nw - 1] >> (E % 32))); }
    out[k] = d;
  }
}

// K3 (compact): digits made non-negative with the borrow chain, packed into
// the (zeroed) word array; interior words of the block are stored, the two
// words shared with the neighbouring blocks are OR-ed in atomically
static __global__ void __launch_bounds__(kPackThreads) k_compact_words(const int32_t* __restrict__ digits, uint32_t nw,
                                                                       uint32_t E, uint32_t N,
                                                                       const uint32_t* __restrict__ blk, PackCtl* ctl,
                                                                       uint32_t* __restrict__ out) {
  OWL_SHARED_ARR(uint32_t, s_st, kPackThreads);
  OWL_SHARED_ARR(uint32_t, s_w, kPackDigits + 2);
  const uint32_t t = threadIdx.x;
  const uint32_t kb = blockIdx.x * kPackDigits;
  const uint32_t k0 = kb + 4 * t;
  const uint32_t kEnd = (kb + kPackDigits < N) ? kb + kPackDigits : N;
  const uint64_t bit0 = pk_off(kb, E, N), bitEnd = pk_off(kEnd, E, N);
  const uint32_t w0 = (uint32_t)(bit0 >> 5), wLast = (uint32_t)((bitEnd - 1) >> 5);
  for (uint32_t i = t; i < kPackDigits + 2; i += kPackThreads) { s_w[i] = 0; }
  uint32_t st[4];
  s_st[t] = pk_thread_status<false>(nullptr, digits, nw, E, N, k0, st);
  __syncthreads();
  // borrow in {0, -1}, carried as 0 / ST_GEN
  uint32_t b = pk_carry_in(s_st, t, blk[blockIdx.x]);
  bool bad = false;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint32_t k = k0 + i;
    if (k >= N) { break; }
    const uint64_t o = pk_off(k, E, N);
    const uint32_t len = (uint32_t)(pk_off(k + 1, E, N) - o);
    int64_t w = (int64_t)digits[k] - (b ? 1 : 0);
    b = 0;
    if (w < 0) {
      w += 1ll << len;
      b = ST_GEN;
    }
    if (w < 0 || w >= (1ll << len)) {
      bad = true;
      w = 0;
    }
    const uint64_t rel = o - ((uint64_t)w0 << 5);
    const uint64_t sh = (uint64_t)w << (rel & 31);
    const uint32_t wi = (uint32_t)(rel >> 5);
    atomicOr(&s_w[wi], (uint32_t)sh);
    if ((uint32_t)(sh >> 32)) { atomicOr(&s_w[wi + 1], (uint32_t)(sh >> 32)); }
  }
  if (bad) { atomicOr(&ctl->error, 1u); }
  __syncthreads();
  for (uint32_t i = w0 + t; i <= wLast; i += kPackThreads) {
    const uint32_t v = s_w[i - w0];
    if (i == w0 || i == wLast) {
      if (v) { atomicOr(&out[i], v); }
    } else {
      out[i] = v;
    }
  }
}

// K4 (compact): the borrow out of the top digit is subtracted at bit 0 (2^E == 1)
static __global__ void k_compact_finish(const PackCtl* ctl, uint32_t nw, uint32_t* __restrict__ out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) { return; }
  int64_t borrow = ctl->carryOut ? -1 : 0;
  for (uint32_t p = 0; borrow && p < nw; ++p) {
    const int64_t v = (int64_t)out[p] + borrow;
    out[p] = (uint32_t)v;
    borrow = v >> 32;
  }
}

}  // namespace owl
