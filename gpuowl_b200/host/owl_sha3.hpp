// owl_sha3.hpp -- SHA3-256 (FIPS 202): the Keccak-f[1600] permutation in a
// sponge of rate 136 bytes, domain padding 0x06 ... 0x80. It hashes the PRP
// proof residues the way the reference does (src/Proof.cpp:22-28 through
// src/Sha3Hash.h: SHA3-256 of the first (E-1)/8+1 bytes of the words, chained
// by prefixing the previous 32-byte digest). Written from the standard: the
// round constants are the LFSR outputs of FIPS 202 3.2.5 and the rotation
// offsets those of 3.2.2, both generated below rather than tabulated.
#pragma once
#include <array>
#include <cstddef>
#include <cstdint>
#include <cstring>

namespace owl {

class Sha3_256 {
 public:
  Sha3_256() { std::memset(s_, 0, sizeof(s_)); }

  Sha3_256& update(const void* data, size_t n) {
    const uint8_t* p = static_cast<const uint8_t*>(data);
    while (n) {
      const size_t take = std::min(n, kRate - fill_);
      for (size_t i = 0; i < take; ++i) { xor_byte(fill_ + i, p[i]); }
      fill_ += take;
      p += take;
      n -= take;
      if (fill_ == kRate) {
        permute();
        fill_ = 0;
      }
    }
    return *this;
  }

  // the 32-byte digest, also as four little-endian 64-bit words
  std::array<uint64_t, 4> finish() {
    xor_byte(fill_, 0x06);
    xor_byte(kRate - 1, 0x80);
    permute();
    return {s_[0], s_[1], s_[2], s_[3]};
  }

  static void digest_bytes(const std::array<uint64_t, 4>& h, uint8_t out[32]) {
    for (int i = 0; i < 32; ++i) { out[i] = (uint8_t)(h[i / 8] >> (8 * (i % 8))); }
  }

 private:
  static constexpr size_t kRate = 136;  // 1600 - 2 * 256 bits
  uint64_t s_[25];
  size_t fill_ = 0;

  void xor_byte(size_t i, uint8_t b) { s_[i / 8] ^= (uint64_t)b << (8 * (i % 8)); }
  static uint64_t rotl(uint64_t x, unsigned r) { return r ? (x << r) | (x >> (64 - r)) : x; }

  struct Consts {
    uint64_t rc[24];
    unsigned rho[25];
    Consts() {
      // round constants: bit 2^j - 1 of RC[i] is rc(j + 7 i), rc from the LFSR x^8 + x^6 + x^5 + x^4 + 1
      uint8_t r = 1;
      auto lfsr = [&]() {
        const bool out = r & 1;
        r = (r & 0x80) ? (uint8_t)((r << 1) ^ 0x71) : (uint8_t)(r << 1);
        return out;
      };
      for (int i = 0; i < 24; ++i) {
        rc[i] = 0;
        for (int j = 0; j < 7; ++j) {
          if (lfsr()) { rc[i] |= 1ull << ((1u << j) - 1); }
        }
      }
      // rotation offsets: walk (x, y) -> (y, 2x + 3y) from (1, 0), offset (t + 1)(t + 2)/2 mod 64
      std::memset(rho, 0, sizeof(rho));
      int x = 1, y = 0;
      for (int t = 0; t < 24; ++t) {
        rho[x + 5 * y] = (unsigned)(((t + 1) * (t + 2) / 2) % 64);
        const int nx = y, ny = (2 * x + 3 * y) % 5;
        x = nx;
        y = ny;
      }
    }
  };

  void permute() {
    static const Consts K;
    uint64_t c[5], b[25];
    for (int round = 0; round < 24; ++round) {
      // theta
      for (int x = 0; x < 5; ++x) { c[x] = s_[x] ^ s_[x + 5] ^ s_[x + 10] ^ s_[x + 15] ^ s_[x + 20]; }
      for (int x = 0; x < 5; ++x) {
        const uint64_t d = c[(x + 4) % 5] ^ rotl(c[(x + 1) % 5], 1);
        for (int y = 0; y < 5; ++y) { s_[x + 5 * y] ^= d; }
      }
      // rho and pi: B[y, 2x + 3y] = rot(A[x, y], rho[x, y])
      for (int x = 0; x < 5; ++x) {
        for (int y = 0; y < 5; ++y) { b[y + 5 * ((2 * x + 3 * y) % 5)] = rotl(s_[x + 5 * y], K.rho[x + 5 * y]); }
      }
      // chi
      for (int y = 0; y < 5; ++y) {
        for (int x = 0; x < 5; ++x) {
          s_[x + 5 * y] = b[x + 5 * y] ^ (~b[(x + 1) % 5 + 5 * y] & b[(x + 2) % 5 + 5 * y]);
        }
      }
      // iota
      s_[0] ^= K.rc[round];
    }
  }
};

}  // namespace owl
