/*
 * words.c -- oracle: word model, digit packing, residue readout, exponent choice.
 *
 * TEST INFRASTRUCTURE ONLY (see owl_oracle.h). Each function restates the
 * reference behaviour it cites; the restatement is pinned against the
 * reference's own state.cpp compiled into oracle/_ref (tests/test_oracle.py).
 */
#include "owl_oracle.h"

#include <stdlib.h>
#include <string.h>

/* src/state.h:14 -- step(N,E) = N - E mod N */
uint32_t oracle_step(uint32_t N, uint32_t E) { return N - (E % N); }

/* src/state.h:15 -- extra(k) = step*k mod N. This is N*ceil(kE/N) - kE, so the
   IBDWT weight of word k is 2^(extra(k)/N). */
uint32_t oracle_extra(uint32_t N, uint32_t E, uint32_t k) {
  return (uint32_t)(((uint64_t)oracle_step(N, E) * k) % N);
}

/* src/state.h:16 -- a word is big (one extra bit) iff extra(k)+step < N */
int oracle_is_big_word(uint32_t N, uint32_t E, uint32_t k) {
  return oracle_extra(N, E, k) + oracle_step(N, E) < N;
}

/* src/state.h:17 */
uint32_t oracle_bitlen(uint32_t N, uint32_t E, uint32_t k) {
  return E / N + (uint32_t)oracle_is_big_word(N, E, k);
}

uint32_t oracle_nwords(uint32_t E) { return (E - 1) / 32 + 1; }

/* src/state.cpp:26-69 (compactBits) with unbalance() from src/state.cpp:13-24.
   Digits are made non-negative from the bottom up with a borrow in {0,-1}; the
   final borrow wraps to bit 0 because 2^E == 1 mod 2^E-1. */
int oracle_compact_bits(const int32_t* data, uint32_t N, uint32_t E, uint32_t* out) {
  uint32_t nw = oracle_nwords(E);
  memset(out, 0, nw * sizeof(uint32_t));
  int carry = 0;
  uint64_t acc = 0;    /* pending bits */
  int have = 0;
  uint32_t o = 0;
  for (uint32_t p = 0; p < N; ++p) {
    int nb = (int)oracle_bitlen(N, E, p);
    int64_t w = (int64_t)data[p] + carry;
    carry = 0;
    if (w < 0) { w += ((int64_t)1 << nb); carry = -1; }
    if (w < 0 || w >= ((int64_t)1 << nb)) { return -1; }
    acc |= (uint64_t)w << have;
    have += nb;
    while (have >= 32) {
      if (o >= nw) { return -1; }
      out[o++] = (uint32_t)acc;
      acc >>= 32;
      have -= 32;
    }
  }
  if (have) {
    if (o >= nw) { return -1; }
    out[o++] = (uint32_t)acc;
  }
  if (o != nw) { return -1; }
  /* wrap-around borrow: add -1 at bit 0 */
  for (uint32_t p = 0; carry && p < nw; ++p) {
    int64_t v = (int64_t)out[p] + carry;
    out[p] = (uint32_t)v;
    carry = (int)(v >> 32);
  }
  return 0;
}

/* src/state.cpp:93-115 (expandBits): pop `bitlen` signed bits per word; a
   negative digit borrows one from the rest; the final bucket carry (0 or 1)
   is added to word 0 (wrap-around). */
int oracle_expand_bits(const uint32_t* words, uint32_t N, uint32_t E, int32_t* out) {
  if (E % 32 == 0) { return -1; }
  uint32_t nw = oracle_nwords(E);
  uint64_t bits = 0;
  uint32_t size = 0;
  uint32_t it = 0;
  for (uint32_t p = 0; p < N; ++p) {
    uint32_t len = oracle_bitlen(N, E, p);
    if (size < len) {
      if (it >= nw) { return -1; }
      bits += (uint64_t)words[it++] << size;
      size += 32;
    }
    /* low `len` bits as a signed value */
    int64_t b = (int64_t)(bits << (64 - len)) >> (64 - len);
    bits >>= len;
    size -= len;
    if (b < 0) { bits += 1; }
    out[p] = (int32_t)b;
  }
  if (it != nw) { return -1; }
  out[0] += (int32_t)bits;
  return 0;
}

/* src/Gpu.cpp:955-975 (bufResidue): the carry into word 0 is taken from the
   sign of the top 32 words; then the low words are made non-negative and
   packed until 64 bits are collected. words64[i] = data[(N-32+i) mod N]. */
uint64_t oracle_buf_residue(const int32_t* words64, uint32_t N, uint32_t E) {
  int carry = 0;
  for (int i = 0; i < 32; ++i) { carry = (words64[i] + carry < 0) ? -1 : 0; }
  uint64_t res = 0;
  int has = 0;
  for (int k = 0; k < 32 && has < 64; ++k) {
    uint32_t len = oracle_bitlen(N, E, (uint32_t)k);
    int64_t w = (int64_t)words64[32 + k] + carry;
    carry = (w < 0) ? -1 : 0;
    if (w < 0) { w += ((int64_t)1 << len); }
    res |= (uint64_t)w << has;
    has += (int)len;
  }
  return res;
}

/* src/Primes.cpp: trial division by odd primes up to 50,000 (enough for
   n < 2.5e9, the range every exponent here lives in). */
int oracle_is_prime(uint32_t n) {
  if (n < 2) { return 0; }
  if (n % 2 == 0) { return n == 2; }
  for (uint64_t d = 3; d * d <= n; d += 2) {
    if (n % d == 0) { return 0; }
  }
  return 1;
}

/* src/Primes.cpp:46-54: the smallest prime strictly greater than n */
uint32_t oracle_next_prime(uint32_t n) {
  ++n;
  if (n <= 2) { return 2; }
  if (n % 2 == 0) { ++n; }
  while (!oracle_is_prime(n)) { n += 2; }
  return n;
}

/* splitmix64 (Steele, Lea, Flood 2014), the published generator */
uint64_t oracle_splitmix64(uint64_t* state) {
  uint64_t z = (*state += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

uint32_t oracle_seeded_prime(uint64_t seed, uint32_t lo, uint32_t hi) {
  uint64_t s = seed;
  uint64_t u = oracle_splitmix64(&s);
  uint32_t n = lo + (uint32_t)(u % ((uint64_t)hi - lo + 1));
  return oracle_next_prime(n);
}
