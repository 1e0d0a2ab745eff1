// ref_proof_shim.cpp -- C entry points onto the REFERENCE's own proof code (src/Proof.cpp with
// src/sha3.cpp and src/md5.cpp), compiled from its sources where they lie (oracle/Makefile `ref`),
// so that tests can exchange PRP proofs with it: a proof written by libowl must load and verify
// with the reference's Proof::load / Proof::verify, and a proof the reference computes and saves
// must pass libowl's verifier. The reference's Gpu is replaced by oracle/ref_stub/Gpu.h, whose
// arithmetic is the GMP oracle (exact, on the CPU).
// TEST INFRASTRUCTURE ONLY; the output goes to oracle/_ref/ and is never shipped.
#include <unistd.h>

#include <array>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "Gpu.h"
#include "Proof.h"
#include "common.h"

extern "C" {
int oracle_gmp_square_words(uint32_t E, const uint32_t* in, uint32_t n, int ll, uint32_t* out);
int oracle_gmp_mul_words(uint32_t E, const uint32_t* a, const uint32_t* b, int mul3, uint32_t* out);
}

namespace {
Words sq(u32 E, const Words& a, u32 n) {
  Words out(nWords(E));
  oracle_gmp_square_words(E, a.data(), n, 0, out.data());
  return out;
}
Words mul(u32 E, const Words& a, const Words& b) {
  Words out(nWords(E));
  oracle_gmp_mul_words(E, a.data(), b.data(), 0, out.data());
  return out;
}
// A^h, left-to-right binary powering
Words power(u32 E, const Words& A, u64 h) {
  if (h == 0) { return makeWords(E, 1); }
  int p = 63;
  while (!((h >> p) & 1)) { --p; }
  Words x = A;
  for (--p; p >= 0; --p) {
    x = sq(E, x, 1);
    if ((h >> p) & 1) { x = mul(E, x, A); }
  }
  return x;
}

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

Words Gpu::expMul(const Words& A, u64 h, const Words& B, bool doSquareB) {
  return mul(E, power(E, A, h), doSquareB ? sq(E, B, 1) : B);
}
void Gpu::expMul(Buffer<i32>& A, u64 h, Buffer<i32>& B) { A.words = mul(E, power(E, A.words, h), B.words); }
Words Gpu::expExp2(const Words& A, u32 n) { return sq(E, A, n); }

extern "C" {

// the reference's Proof::load + Proof::verify of `path`; 1 valid, 0 invalid, -1 load error.
// *isPrime is set from B == 9 (probable prime).
int ref_proof_verify(const char* path, int* isPrime) {
  try {
    Proof proof = Proof::load(path);
    Gpu gpu{proof.E};
    if (isPrime) { *isPrime = proof.B == makeWords(proof.E, 9); }
    return proof.verify(&gpu) ? 1 : 0;
  } catch (...) {
    return -1;
  }
}

// the reference's proof::hashWords(E, words)[0] and the whole 32-byte hash
void ref_proof_hash_words(uint32_t E, const uint32_t* words, uint64_t* hash4) {
  Words w(words, words + nWords(E));
  auto h = proof::hashWords(E, w);
  for (int i = 0; i < 4; ++i) { hash4[i] = h[i]; }
}

// the reference's ProofSet::save of one residue (into `dir`/<E>/proof/<k>)
int ref_proofset_save(const char* dir, uint32_t E, uint32_t power, uint32_t k, const uint32_t* words) {
  try {
    Cwd cwd{dir};
    ProofSet set{E, power};
    set.save(k, Words(words, words + nWords(E)));
    return 0;
  } catch (...) {
    return -1;
  }
}

// the reference's ProofSet::load of the residue at proof point k (CRC checked); 0 ok, -1 error
int ref_proofset_load(const char* dir, uint32_t E, uint32_t power, uint32_t k, uint32_t* out) {
  try {
    if (!ProofSet::isInPoints(E, power, k)) { return -1; }
    Cwd cwd{dir};
    const Words w = ProofSet::load(E, power, k);
    for (size_t i = 0; i < w.size(); ++i) { out[i] = w[i]; }
    return 0;
  } catch (...) {
    return -1;
  }
}

// the reference's ProofSet::computeProof from the residues under `dir`/<E>/proof/, then
// Proof::save into `dir`; the file name goes to `outPath` (capacity `cap`)
int ref_proof_compute_and_save(const char* dir, uint32_t E, uint32_t power, char* outPath, size_t cap) {
  try {
    Cwd cwd{dir};
    ProofSet set{E, power};
    Gpu gpu{E};
    auto [proof, hashes] = set.computeProof(&gpu);
    fs::path f = proof.file(".");
    proof.save(f);
    std::string s = (fs::path(dir) / f).string();
    if (s.size() + 1 > cap) { return -1; }
    std::memcpy(outPath, s.c_str(), s.size() + 1);
    return 0;
  } catch (...) {
    return -1;
  }
}

// the reference's ProofSet points (src/Proof.cpp:136-159): up to `cap` of them into `out`
int ref_proof_points(uint32_t E, uint32_t power, uint32_t* out, uint32_t cap) {
  std::vector<u32> pts;
  for (u32 k = 1; k <= E; ++k) {
    if (ProofSet::isInPoints(E, power, k)) { pts.push_back(k); }
  }
  if (pts.size() > cap) { return -1; }
  for (size_t i = 0; i < pts.size(); ++i) { out[i] = pts[i]; }
  return (int)pts.size();
}
}
