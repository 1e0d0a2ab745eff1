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

// ---- the reference's Saver (src/Saver.cpp), for savefile format parity ----
#include <unistd.h>

#include "Saver.h"

namespace {
struct Cwd {
  std::string old;
  explicit Cwd(const char* dir) {
    char buf[4096];
    old = getcwd(buf, sizeof(buf)) ? buf : ".";
    if (chdir(dir) != 0) { throw "chdir"; }
  }
  ~Cwd() { (void)!chdir(old.c_str()); }
};
}  // namespace

extern "C" {

// Saver<PRPState>::save in <dir>/<E>/ (the reference's cwd-relative layout)
int ref_prp_save(const char* dir, uint32_t E, uint32_t k, uint32_t block, uint64_t res64, const uint32_t* check,
                 uint32_t nErrors, double elapsed) {
  try {
    Cwd cwd(dir);
    Saver<PRPState> s(E, block, 4);
    s.save(PRPState{E, k, block, res64, std::vector<u32>(check, check + nWords(E)), nErrors, elapsed});
    return 0;
  } catch (...) {
    return -1;
  }
}

int ref_prp_load(const char* dir, uint32_t E, uint32_t block, uint32_t* k, uint32_t* blockOut, uint64_t* res64,
                 uint32_t* check, uint32_t* nErrors) {
  try {
    Cwd cwd(dir);
    Saver<PRPState> s(E, block, 4);
    PRPState st = s.load();
    *k = st.k;
    *blockOut = st.blockSize;
    *res64 = st.res64;
    *nErrors = st.nErrors;
    for (size_t i = 0; i < st.check.size(); ++i) { check[i] = st.check[i]; }
    return 0;
  } catch (...) {
    return -1;
  }
}

int ref_ll_save(const char* dir, uint32_t E, uint32_t k, const uint32_t* data) {
  try {
    Cwd cwd(dir);
    Saver<LLState> s(E, 1000, 4);
    s.save(LLState{E, k, std::vector<u32>(data, data + nWords(E)), 0});
    return 0;
  } catch (...) {
    return -1;
  }
}

int ref_ll_load(const char* dir, uint32_t E, uint32_t* k, uint32_t* data) {
  try {
    Cwd cwd(dir);
    Saver<LLState> s(E, 1000, 4);
    LLState st = s.load();
    *k = st.k;
    for (size_t i = 0; i < st.data.size(); ++i) { data[i] = st.data[i]; }
    return 0;
  } catch (...) {
    return -1;
  }
}
}
