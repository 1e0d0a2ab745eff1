/*
 * gmp_loop.c -- oracle: exact x <- x^2 (-2) mod 2^E-1 with GMP.
 *
 * TEST INFRASTRUCTURE ONLY (see owl_oracle.h). This is the independent exact
 * oracle for every res64 the GPU path reports: PRP starts from 3 and LL from 4
 * (reference src/Saver.cpp:164-166), res64 is the low 64 bits of the canonical
 * residue (reference src/common.h res64(), src/Gpu.cpp:955-975).
 *
 * gmp.h is not installed, only the runtime libgmp.so.10 (GMP 6.3.0). The mpz
 * layout and the handful of entry points used are declared here from GMP's
 * public documentation.
 */
#include "owl_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef struct { int alloc; int size; unsigned long* d; } mpz_struct;
typedef mpz_struct mpz_t[1];

extern void __gmpz_init(mpz_struct*);
extern void __gmpz_clear(mpz_struct*);
extern void __gmpz_set_ui(mpz_struct*, unsigned long);
extern void __gmpz_set(mpz_struct*, const mpz_struct*);
extern void __gmpz_mul(mpz_struct*, const mpz_struct*, const mpz_struct*);
extern void __gmpz_mul_ui(mpz_struct*, const mpz_struct*, unsigned long);
extern void __gmpz_add(mpz_struct*, const mpz_struct*, const mpz_struct*);
extern void __gmpz_sub(mpz_struct*, const mpz_struct*, const mpz_struct*);
extern void __gmpz_sub_ui(mpz_struct*, const mpz_struct*, unsigned long);
extern void __gmpz_tdiv_q_2exp(mpz_struct*, const mpz_struct*, unsigned long);
extern void __gmpz_tdiv_r_2exp(mpz_struct*, const mpz_struct*, unsigned long);
extern int  __gmpz_cmp(const mpz_struct*, const mpz_struct*);
extern void __gmpz_setbit(mpz_struct*, unsigned long);
extern void __gmpz_import(mpz_struct*, size_t, int, size_t, int, size_t, const void*);
extern void* __gmpz_export(void*, size_t*, int, size_t, int, size_t, const mpz_struct*);

typedef struct {
  uint32_t E;
  mpz_t M, hi, lo;
} modctx;

static void ctx_init(modctx* c, uint32_t E) {
  c->E = E;
  __gmpz_init(c->M);
  __gmpz_init(c->hi);
  __gmpz_init(c->lo);
  __gmpz_setbit(c->M, E);
  __gmpz_sub_ui(c->M, c->M, 1);
}

static void ctx_clear(modctx* c) {
  __gmpz_clear(c->M);
  __gmpz_clear(c->hi);
  __gmpz_clear(c->lo);
}

/* x (0 <= x < 2^(2E+2)) -> x mod M in [0, M) using 2^E == 1 */
static void reduce(modctx* c, mpz_struct* x) {
  for (int i = 0; i < 2; ++i) {
    __gmpz_tdiv_q_2exp(c->hi, x, c->E);
    __gmpz_tdiv_r_2exp(c->lo, x, c->E);
    __gmpz_add(x, c->hi, c->lo);
  }
  while (__gmpz_cmp(x, c->M) >= 0) { __gmpz_sub(x, x, c->M); }
}

static uint64_t low64(const mpz_struct* x) {
  if (x->size == 0) { return 0; }
  return (uint64_t)x->d[0];
}

static void square_step(modctx* c, mpz_struct* x, int ll) {
  __gmpz_mul(x, x, x);
  if (ll) {
    /* x^2 - 2 could go negative only for x < 2; add M first to stay >= 0 */
    __gmpz_add(x, x, c->M);
    __gmpz_sub_ui(x, x, 2);
  }
  reduce(c, x);
}

int oracle_gmp_run(uint32_t E, uint32_t start, int ll, uint32_t iters, uint32_t step,
                   uint64_t* res_out, const char* progress_path) {
  modctx c;
  ctx_init(&c, E);
  mpz_t x;
  __gmpz_init(x);
  __gmpz_set_ui(x, start);
  uint32_t n = 0;
  for (uint32_t k = 1; k <= iters; ++k) {
    square_step(&c, x, ll);
    if (step && k % step == 0) {
      uint64_t r = low64(x);
      if (res_out) { res_out[n] = r; }
      ++n;
      if (progress_path) {
        FILE* f = fopen(progress_path, "a");
        if (f) {
          fprintf(f, "%u %016llx\n", k, (unsigned long long)r);
          fclose(f);
        }
      }
    }
  }
  __gmpz_clear(x);
  ctx_clear(&c);
  return 0;
}

static void import_words(mpz_struct* x, const uint32_t* w, uint32_t E) {
  __gmpz_import(x, oracle_nwords(E), -1, sizeof(uint32_t), 0, 0, w);
}

static void export_words(const mpz_struct* x, uint32_t E, uint32_t* out) {
  uint32_t nw = oracle_nwords(E);
  memset(out, 0, nw * sizeof(uint32_t));
  size_t cnt = 0;
  if (x->size == 0) { return; }
  uint32_t* tmp = (uint32_t*)__gmpz_export(NULL, &cnt, -1, sizeof(uint32_t), 0, 0, x);
  for (size_t i = 0; i < cnt && i < nw; ++i) { out[i] = tmp[i]; }
  free(tmp);
}

int oracle_gmp_square_words(uint32_t E, const uint32_t* in, uint32_t n, int ll, uint32_t* out) {
  modctx c;
  ctx_init(&c, E);
  mpz_t x;
  __gmpz_init(x);
  import_words(x, in, E);
  reduce(&c, x);
  for (uint32_t k = 0; k < n; ++k) { square_step(&c, x, ll); }
  export_words(x, E, out);
  __gmpz_clear(x);
  ctx_clear(&c);
  return 0;
}

int oracle_gmp_mul_words(uint32_t E, const uint32_t* a, const uint32_t* b, int mul3, uint32_t* out) {
  modctx c;
  ctx_init(&c, E);
  mpz_t x, y;
  __gmpz_init(x);
  __gmpz_init(y);
  import_words(x, a, E);
  import_words(y, b, E);
  __gmpz_mul(x, x, y);
  reduce(&c, x);
  if (mul3) {
    __gmpz_mul_ui(x, x, 3);
    reduce(&c, x);
  }
  export_words(x, E, out);
  __gmpz_clear(x);
  __gmpz_clear(y);
  ctx_clear(&c);
  return 0;
}

double oracle_gmp_ms_per_iter(uint32_t E, uint32_t iters) {
  modctx c;
  ctx_init(&c, E);
  mpz_t x;
  __gmpz_init(x);
  __gmpz_set_ui(x, 3);
  /* warm up into the uniformly distributed regime (3^(2^k) has E bits after log2(E) squarings) */
  for (int k = 0; k < 40; ++k) { square_step(&c, x, 0); }
  struct timespec t0, t1;
  clock_gettime(CLOCK_MONOTONIC, &t0);
  for (uint32_t k = 0; k < iters; ++k) { square_step(&c, x, 0); }
  clock_gettime(CLOCK_MONOTONIC, &t1);
  __gmpz_clear(x);
  ctx_clear(&c);
  double s = (double)(t1.tv_sec - t0.tv_sec) + 1e-9 * (double)(t1.tv_nsec - t0.tv_nsec);
  return 1e3 * s / (double)(iters ? iters : 1);
}
