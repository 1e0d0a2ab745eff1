// ref_shim.cpp -- C entry points onto the REFERENCE's own host code, compiled
// from its sources where they lie (see oracle/Makefile `ref`), so that tests can
// pin the oracle's and libowl's restatements against the reference itself.
// TEST INFRASTRUCTURE ONLY; the output goes to oracle/_ref/ and is never shipped.
#include <cstdint>
#include <vector>

#include "Primes.h"
#include "common.h"
#include "state.h"

extern "C" {

// reference compactBits (src/state.cpp:26-69); returns the number of words written
int ref_compact_bits(const int32_t* data, uint32_t N, uint32_t E, uint32_t* out) {
  std::vector<int> d(data, data + N);
  std::vector<u32> w = compactBits(d, E);
  for (size_t i = 0; i < w.size(); ++i) { out[i] = w[i]; }
  return (int)w.size();
}

// reference expandBits (src/state.cpp:93-115)
int ref_expand_bits(const uint32_t* words, uint32_t N, uint32_t E, int32_t* out) {
  std::vector<u32> w(words, words + nWords(E));
  std::vector<int> d = expandBits(w, N, E);
  for (uint32_t i = 0; i < N; ++i) { out[i] = d[i]; }
  return 0;
}

uint32_t ref_bitlen(uint32_t N, uint32_t E, uint32_t k) { return bitlen(N, E, k); }
uint32_t ref_extra(uint32_t N, uint32_t E, uint32_t k) { return extra(N, E, k); }

// reference Primes::nextPrime (src/Primes.cpp:46-54)
uint32_t ref_next_prime(uint32_t n) {
  static Primes primes;
  return primes.nextPrime(n);
}

// reference crc32 (src/common.cpp), the savefile checksum
uint32_t ref_crc32(const void* data, size_t size) { return crc32(data, size); }
}
