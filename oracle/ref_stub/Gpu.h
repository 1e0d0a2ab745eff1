// Gpu.h (stand-in) -- TEST INFRASTRUCTURE ONLY. Found before the reference's own Gpu.h when
// the reference's src/Proof.cpp is compiled by `make -C oracle ref` (the -I- include order), so
// that Proof.cpp builds without OpenCL. It declares only what Proof.cpp calls on its Gpu
// (src/Proof.cpp:84-126 verify, 262-297 computeProof); oracle/ref_proof_shim.cpp implements
// those calls with the GMP oracle (oracle/gmp_loop.c) on the CPU.
#pragma once

// the standard headers the reference's Gpu.h brings in, which Proof.cpp relies on
#include <cmath>
#include <filesystem>
#include <memory>
#include <vector>

#include "common.h"

struct OracleArgs {
  bool verbose = false;
};

// a device buffer of the reference holds the words on the CPU here
template <typename T> struct Buffer {
  Words words;
};

class Gpu {
public:
  explicit Gpu(u32 E) : E{E} {}
  const u32 E;
  OracleArgs args;

  // A^h * (B or B^2), as the reference's Gpu::expMul (src/Gpu.cpp:838-845)
  Words expMul(const Words& A, u64 h, const Words& B, bool doSquareB);
  // A := A^h * B (src/Gpu.cpp:833-836)
  void expMul(Buffer<i32>& A, u64 h, Buffer<i32>& B);
  // A^(2^n)
  Words expExp2(const Words& A, u32 n);
  vector<Buffer<i32>> makeBufVector(u32 size) { return vector<Buffer<i32>>(size); }
  void writeIn(Buffer<i32>& buf, const Words& w) { buf.words = w; }
  Words readAndCompress(Buffer<i32>& buf) { return buf.words; }
};
