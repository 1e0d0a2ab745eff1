/*
 * owl_oracle.h -- CPU oracle for the PRP/LL IBDWT squaring path.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product (gpuowl_b200/, include/)
 * links, loads or calls this library. Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline arm use it, and only as the checker or the timed
 * CPU baseline. It is never the thing measured on the GPU, and never a fallback.
 *
 * Parity pins:
 *   - word model, expandBits/compactBits, bufResidue: restated from the
 *     reference (src/state.h:14-17, src/state.cpp:26-115, src/Gpu.cpp:955-975)
 *     and cross-checked against the reference's own state.cpp compiled into
 *     oracle/_ref/libref_state.so (see oracle/Makefile);
 *   - x <- x^2 (-2) mod 2^E-1: GMP 6.3.0 (libgmp.so.10, runtime only; the
 *     prototypes below are our own because gmp.h is not installed);
 *   - IBDWT squaring: a scalar restatement of the reference's weights,
 *     real-signal squaring, rounding and carry (see ibdwt.c for citations).
 */
#ifndef OWL_ORACLE_H
#define OWL_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- word model: src/state.h:14-17 ---- */
uint32_t oracle_step(uint32_t N, uint32_t E);
uint32_t oracle_extra(uint32_t N, uint32_t E, uint32_t k);
int      oracle_is_big_word(uint32_t N, uint32_t E, uint32_t k);
uint32_t oracle_bitlen(uint32_t N, uint32_t E, uint32_t k);

/* ---- packing: src/state.cpp:26-115 ---- */
uint32_t oracle_nwords(uint32_t E);                         /* (E-1)/32+1, src/common.h */
/* balanced digits (N int32) -> E-bit little-endian u32 words; returns 0 or -1 (digit out of range) */
int oracle_compact_bits(const int32_t* data, uint32_t N, uint32_t E, uint32_t* out);
/* E-bit words -> balanced digits; returns 0 or -1 */
int oracle_expand_bits(const uint32_t* words, uint32_t N, uint32_t E, int32_t* out);
/* res64 from the 64 words around the wrap (words[i] = data[(N-32+i) % N]), src/Gpu.cpp:955-975 */
uint64_t oracle_buf_residue(const int32_t* words64, uint32_t N, uint32_t E);

/* ---- exponent choice: src/Primes.cpp:46-54 semantics (smallest prime > n) ---- */
uint32_t oracle_next_prime(uint32_t n);
int      oracle_is_prime(uint32_t n);
uint64_t oracle_splitmix64(uint64_t* state);
/* first splitmix64 output of `seed` mapped to [lo, hi], then next_prime */
uint32_t oracle_seeded_prime(uint64_t seed, uint32_t lo, uint32_t hi);

/* ---- GMP exact loop ---- */
/* x <- x^2 mod M (ll: x^2-2) `iters` times starting from `start` (3 for PRP, 4 for LL);
   res64 of x after every `step` iterations goes to res_out[i] (iters/step entries).
   If progress_path is non-NULL, each checkpoint is appended to it as "k res64\n".
   Returns 0. */
int oracle_gmp_run(uint32_t E, uint32_t start, int ll, uint32_t iters, uint32_t step,
                   uint64_t* res_out, const char* progress_path);
/* words (nwords(E) u32) -> square n times mod M (ll: x^2-2) -> words */
int oracle_gmp_square_words(uint32_t E, const uint32_t* in, uint32_t n, int ll, uint32_t* out);
/* out = a*b mod M (mul3: *3) */
int oracle_gmp_mul_words(uint32_t E, const uint32_t* a, const uint32_t* b, int mul3, uint32_t* out);
/* ms per squaring over `iters` iterations at exponent E (timing helper for the CPU baseline) */
double oracle_gmp_ms_per_iter(uint32_t E, uint32_t iters);

/* ---- IBDWT restatement (CPU, FP64) ---- */
typedef struct oracle_ibdwt oracle_ibdwt;
oracle_ibdwt* oracle_ibdwt_create(uint32_t E, uint32_t N, int threads);
void          oracle_ibdwt_destroy(oracle_ibdwt* p);
/* io: N balanced digits. One squaring (mul3: result*3; ll: minus 2). max_roe: max |x-rint(x)|. */
int oracle_ibdwt_square(oracle_ibdwt* p, int32_t* io, int mul3, int ll, double* max_roe);
/* io <- io*b (mul3: *3) */
int oracle_ibdwt_mul(oracle_ibdwt* p, int32_t* io, const int32_t* b, int mul3, double* max_roe);

#ifdef __cplusplus
}
#endif
#endif
