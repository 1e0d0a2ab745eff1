/*
 * ibdwt.c -- oracle: a scalar CPU restatement of the reference's IBDWT
 * squaring, used as a cross-check of the word model and as the timed CPU
 * "port" baseline.
 *
 * TEST INFRASTRUCTURE ONLY (see owl_oracle.h). Follows:
 *   - weights 2^(extra(k)/N) on word k (reference src/Gpu.cpp:42-56, src/state.h:14-17);
 *   - packing of words 2j, 2j+1 as one complex value (src/Gpu.cpp:40 kAt);
 *   - real-signal squaring of the half-length complex transform, pairing
 *     Z[k] with Z[hN-k] under the twiddle w_hN^k (src/cl/tailsquare.cl:35-74);
 *     for the product of two signals the same pairing (src/cl/tailmul.cl:19-34);
 *   - inverse weight, rounding to the nearest integer with the round-off
 *     |x - rint(x)| recorded, MUL3 applied to the rounded value, LL's -2
 *     added at word 0, balanced-digit carry with the carry out of the top word
 *     wrapping to word 0 (src/cl/carryutil.cl:56-149, src/cl/carryinc.cl);
 *     here the carry is propagated fully and sequentially, which is one valid
 *     representative of the reference's sloppy carries (the number is the same).
 * The FFT itself is a plain iterative radix-2 transform in FP64 with twiddles
 * from a long-double table; only the rounded integers are compared.
 */
#include "owl_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double re, im; } cplx;

struct oracle_ibdwt {
  uint32_t E, N, hN, lg;
  int threads;
  double* w;    /* weight of word k */
  double* iw;   /* 1 / (weight * 4 hN) */
  uint8_t* bits;
  cplx* tw;     /* w_hN^k, k < hN */
  cplx* a;
  cplx* b;
  uint32_t* rev;
};

static void root(uint64_t n, uint64_t k, cplx* out) {
  const long double PI = 3.141592653589793238462643383279502884L;
  long double a = 2.0L * PI * (long double)(k % n) / (long double)n;
  out->re = (double)cosl(a);
  out->im = (double)-sinl(a);
}

oracle_ibdwt* oracle_ibdwt_create(uint32_t E, uint32_t N, int threads) {
  if (N < 4 || (N & (N - 1))) { return NULL; }
  oracle_ibdwt* p = (oracle_ibdwt*)calloc(1, sizeof(*p));
  p->E = E;
  p->N = N;
  p->hN = N / 2;
  p->lg = 0;
  while ((1u << p->lg) < p->hN) { ++p->lg; }
  p->threads = threads > 0 ? threads : 1;
  p->w = (double*)malloc(sizeof(double) * N);
  p->iw = (double*)malloc(sizeof(double) * N);
  p->bits = (uint8_t*)malloc(N);
  p->tw = (cplx*)malloc(sizeof(cplx) * p->hN);
  p->a = (cplx*)malloc(sizeof(cplx) * p->hN);
  p->b = (cplx*)malloc(sizeof(cplx) * p->hN);
  p->rev = (uint32_t*)malloc(sizeof(uint32_t) * p->hN);
  const long double norm = 1.0L / (4.0L * (long double)p->hN);
  for (uint32_t k = 0; k < N; ++k) {
    uint32_t ex = oracle_extra(N, E, k);
    p->w[k] = (double)exp2l((long double)ex / N);
    p->iw[k] = (double)(exp2l(-(long double)ex / N) * norm);
    p->bits[k] = (uint8_t)oracle_bitlen(N, E, k);
  }
  for (uint32_t k = 0; k < p->hN; ++k) { root(p->hN, k, &p->tw[k]); }
  for (uint32_t i = 0; i < p->hN; ++i) {
    uint32_t r = 0;
    for (uint32_t b = 0; b < p->lg; ++b) { r |= ((i >> b) & 1u) << (p->lg - 1 - b); }
    p->rev[i] = r;
  }
  return p;
}

void oracle_ibdwt_destroy(oracle_ibdwt* p) {
  if (!p) { return; }
  free(p->w); free(p->iw); free(p->bits); free(p->tw); free(p->a); free(p->b); free(p->rev);
  free(p);
}

/* in-place radix-2 DIT FFT of length hN; inv selects the conjugate twiddles */
static void fft(oracle_ibdwt* p, cplx* x, int inv) {
  const uint32_t n = p->hN;
#pragma omp parallel for num_threads(p->threads) schedule(static)
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t r = p->rev[i];
    if (r > i) { cplx t = x[i]; x[i] = x[r]; x[r] = t; }
  }
  for (uint32_t len = 2; len <= n; len <<= 1) {
    const uint32_t half = len / 2, stride = n / len;
#pragma omp parallel for num_threads(p->threads) schedule(static)
    for (uint32_t blk = 0; blk < n / 2; ++blk) {
      uint32_t g = blk / half, j = blk % half;
      uint32_t i0 = g * len + j, i1 = i0 + half;
      cplx t = p->tw[(uint64_t)j * stride];
      if (inv) { t.im = -t.im; }
      cplx u = x[i0], v = x[i1];
      cplx vt = {v.re * t.re - v.im * t.im, v.re * t.im + v.im * t.re};
      x[i0].re = u.re + vt.re; x[i0].im = u.im + vt.im;
      x[i1].re = u.re - vt.re; x[i1].im = u.im - vt.im;
    }
  }
}

static void load(oracle_ibdwt* p, const int32_t* d, cplx* x) {
#pragma omp parallel for num_threads(p->threads) schedule(static)
  for (uint32_t j = 0; j < p->hN; ++j) {
    x[j].re = d[2 * j] * p->w[2 * j];
    x[j].im = d[2 * j + 1] * p->w[2 * j + 1];
  }
}

static inline cplx cm(cplx a, cplx b) { cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static inline cplx ca(cplx a, cplx b) { cplx r = {a.re + b.re, a.im + b.im}; return r; }
static inline cplx cs(cplx a, cplx b) { cplx r = {a.re - b.re, a.im - b.im}; return r; }
static inline cplx cj(cplx a) { cplx r = {a.re, -a.im}; return r; }
static inline cplx mi(cplx a) { cplx r = {a.im, -a.re}; return r; }   /* -i a */
static inline cplx pi_(cplx a) { cplx r = {-a.im, a.re}; return r; }  /*  i a */

/* 4 W[k] for the product of signals with spectra (Z, Y); squaring when Y == Z */
static void pair_products(oracle_ibdwt* p, const cplx* Z, const cplx* Y, cplx* out) {
#pragma omp parallel for num_threads(p->threads) schedule(static)
  for (uint32_t k = 0; k < p->hN; ++k) {
    uint32_t q = (p->hN - k) % p->hN;
    cplx e2a = ca(Z[k], cj(Z[q])), o2a = mi(cs(Z[k], cj(Z[q])));
    cplx e2b = ca(Y[k], cj(Y[q])), o2b = mi(cs(Y[k], cj(Y[q])));
    cplx s = ca(cm(e2a, e2b), cm(p->tw[k], cm(o2a, o2b)));
    cplx t = pi_(ca(cm(e2a, o2b), cm(o2a, e2b)));
    out[k] = ca(s, t);
  }
}

static int round_and_carry(oracle_ibdwt* p, const cplx* x, int32_t* io, int mul3, int ll, double* max_roe) {
  const uint32_t N = p->N;
  double roe = 0;
  int64_t* v = (int64_t*)malloc(sizeof(int64_t) * N);
#pragma omp parallel for num_threads(p->threads) schedule(static) reduction(max : roe)
  for (uint32_t k = 0; k < N; ++k) {
    double y = ((k & 1) ? x[k / 2].im : x[k / 2].re) * p->iw[k];
    double r = rint(y);
    double e = fabs(y - r);
    if (e > roe) { roe = e; }
    v[k] = (int64_t)r * (mul3 ? 3 : 1);
  }
  if (ll) { v[0] -= 2; }
  int64_t carry = 0;
  for (int pass = 0; pass < 8; ++pass) {
    for (uint32_t k = 0; k < N; ++k) {
      int64_t t = v[k] + carry;
      int b = p->bits[k];
      int64_t d = (int64_t)((uint64_t)t << (64 - b)) >> (64 - b);
      carry = (t - d) >> b;
      v[k] = d;
      if (pass > 0 && carry == 0) { break; }
    }
    if (carry == 0) { break; }
  }
  int ok = carry == 0;
  for (uint32_t k = 0; k < N; ++k) { io[k] = (int32_t)v[k]; }
  free(v);
  if (max_roe) { *max_roe = roe; }
  return ok ? 0 : -1;
}

int oracle_ibdwt_square(oracle_ibdwt* p, int32_t* io, int mul3, int ll, double* max_roe) {
  load(p, io, p->a);
  fft(p, p->a, 0);
  pair_products(p, p->a, p->a, p->b);
  fft(p, p->b, 1);
  return round_and_carry(p, p->b, io, mul3, ll, max_roe);
}

int oracle_ibdwt_mul(oracle_ibdwt* p, int32_t* io, const int32_t* b, int mul3, double* max_roe) {
  cplx* c = (cplx*)malloc(sizeof(cplx) * p->hN);
  load(p, io, p->a);
  load(p, b, c);
  fft(p, p->a, 0);
  fft(p, c, 0);
  pair_products(p, p->a, c, p->b);
  free(c);
  fft(p, p->b, 1);
  return round_and_carry(p, p->b, io, mul3, 0, max_roe);
}
