// owl_words.hpp -- host-side digit packing for libowl.
//
// compact_bits restates the reference's compactBits (src/state.cpp:26-69):
// balanced digits are made non-negative from word 0 upward with a borrow in
// {0,-1}, packed little-endian at bitlen(k) bits each, and the final borrow is
// added at bit 0 (2^E == 1 mod 2^E-1). expand_bits restates expandBits
// (src/state.cpp:93-115): take bitlen(k) bits as a signed digit, a negative
// digit borrows one from the remaining bits, and the leftover bucket bit goes
// back into word 0. Both are needed bit-for-bit because savefiles, proofs and
// res64 are defined on the compact form.
#pragma once
#include <cstdint>
#include <cstring>
#include <vector>

namespace owl {

inline uint32_t n_words(uint32_t E) { return (E - 1) / 32 + 1; }
inline uint32_t word_step(uint32_t N, uint32_t E) { return N - (E % N); }
inline uint32_t word_extra(uint32_t N, uint32_t E, uint32_t k) {
  return (uint32_t)(((uint64_t)word_step(N, E) * k) % N);
}
inline uint32_t word_bits(uint32_t N, uint32_t E, uint32_t k) {
  return E / N + ((word_extra(N, E, k) + word_step(N, E) < N) ? 1u : 0u);
}

// returns false if a digit is out of range for its word
inline bool compact_bits(const int32_t* data, uint32_t N, uint32_t E, uint32_t* out) {
  const uint32_t nw = n_words(E);
  std::memset(out, 0, nw * sizeof(uint32_t));
  const uint32_t step = word_step(N, E);
  const uint32_t lo = E / N;
  uint32_t extra = 0;  // extra(p), advanced incrementally
  int borrow = 0;
  uint64_t acc = 0;
  int have = 0;
  uint32_t o = 0;
  for (uint32_t p = 0; p < N; ++p) {
    const int nb = (int)(lo + ((extra + step < N) ? 1 : 0));
    extra += step;
    if (extra >= N) { extra -= N; }
    int64_t w = (int64_t)data[p] + borrow;
    borrow = 0;
    if (w < 0) {
      w += (int64_t)1 << nb;
      borrow = -1;
    }
    if (w < 0 || w >= ((int64_t)1 << nb)) { return false; }
    acc |= (uint64_t)w << have;
    have += nb;
    while (have >= 32) {
      if (o >= nw) { return false; }
      out[o++] = (uint32_t)acc;
      acc >>= 32;
      have -= 32;
    }
  }
  if (have) {
    if (o >= nw) { return false; }
    out[o++] = (uint32_t)acc;
  }
  if (o != nw) { return false; }
  for (uint32_t p = 0; borrow && p < nw; ++p) {
    int64_t v = (int64_t)out[p] + borrow;
    out[p] = (uint32_t)v;
    borrow = (int)(v >> 32);
  }
  return true;
}

inline bool expand_bits(const uint32_t* words, uint32_t N, uint32_t E, int32_t* out) {
  if (E % 32 == 0) { return false; }
  const uint32_t nw = n_words(E);
  const uint32_t step = word_step(N, E);
  const uint32_t lo = E / N;
  uint32_t extra = 0;
  uint64_t bits = 0;
  uint32_t size = 0, it = 0;
  for (uint32_t p = 0; p < N; ++p) {
    const uint32_t len = lo + ((extra + step < N) ? 1 : 0);
    extra += step;
    if (extra >= N) { extra -= N; }
    if (size < len) {
      if (it >= nw) { return false; }
      bits += (uint64_t)words[it++] << size;
      size += 32;
    }
    int64_t b = (int64_t)(bits << (64 - len)) >> (64 - len);
    bits >>= len;
    size -= len;
    if (b < 0) { bits += 1; }
    out[p] = (int32_t)b;
  }
  if (it != nw) { return false; }
  out[0] += (int32_t)bits;
  return true;
}

// Gpu::bufResidue (src/Gpu.cpp:955-975) on words64[i] = data[(N-32+i) mod N].
// *decided is false when the top 32 words are all zero, the one case where the
// borrow into word 0 depends on words further down.
inline uint64_t residue_from_wrap(const int32_t* words64, uint32_t N, uint32_t E, bool* decided) {
  bool allZero = true;
  for (int i = 0; i < 32; ++i) { allZero &= (words64[i] == 0); }
  *decided = !allZero;
  int carry = 0;
  for (int i = 0; i < 32; ++i) { carry = (words64[i] + carry < 0) ? -1 : 0; }
  uint64_t res = 0;
  int has = 0;
  for (int k = 0; k < 32 && has < 64; ++k) {
    uint32_t len = word_bits(N, E, (uint32_t)k);
    int64_t w = (int64_t)words64[32 + k] + carry;
    carry = (w < 0) ? -1 : 0;
    if (w < 0) { w += (int64_t)1 << len; }
    res |= (uint64_t)w << has;
    has += (int)len;
  }
  return res;
}

}  // namespace owl
