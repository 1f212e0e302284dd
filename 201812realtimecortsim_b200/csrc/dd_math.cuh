// dd_math.cuh -- correctly rounded exp/log in double-double arithmetic, and
// a logf bit-identical to the host C library's.
//
// The reference calls the C library's exp (LIFCA calcium decay,
// DPSNN_neuron_sim.c:705), log (NormDev, randdev.c:599) and logf (bath
// lapses, DPSNN_neuron_sim.c:850).  The engine reproduces them as follows:
//  * exp_cr / log_cr return the correctly rounded double.  They are built
//    only from IEEE +,-,*,/ and fma, so host and device give bit-identical
//    results (device code is compiled with --fmad=false, host code with
//    -ffp-contract=off).  exp: argument reduction by k*ln2, a Taylor series
//    on r/256 and eight squarings.  log: x = 2^e*m, m in [0.75,1.5), table
//    point c = round(64 m)/64, log m = log c + 2 atanh((m-c)/(m+c)); a short
//    evaluation with an error bound decides the rounding, the full series
//    only when it cannot.
//    The C library's exp/log differ from the correctly rounded value in about
//    0.08% of arguments by one ulp; the raster is bit-identical to the
//    reference until such a difference first changes a threshold decision.
//  * logf_ref(x) equals the C library's logf for every float in (0,1]: the
//    correctly rounded float logarithm, except at the inputs listed in a
//    fix-up table built on the host from the C library itself
//    (logf_fixup.c), where the C library's value is returned.
#pragma once
#include <stdint.h>
#include <math.h>
#include "dd_tables.h"

#ifdef __CUDACC__
#define DD_HD __host__ __device__ __forceinline__
#else
#define DD_HD static inline
#endif

static const double dd_inv_fact_h[DD_INV_FACT_N][2] = DD_INV_FACT_INIT;
static const double dd_inv_odd_h[DD_INV_ODD_N][2] = DD_INV_ODD_INIT;
static const double dd_log_j64_h[DD_LOG_J64_N][2] = DD_LOG_J64_INIT;
#ifdef __CUDACC__
static __constant__ double dd_inv_fact_d[DD_INV_FACT_N][2] = DD_INV_FACT_INIT;
static __constant__ double dd_inv_odd_d[DD_INV_ODD_N][2] = DD_INV_ODD_INIT;
static __constant__ double dd_log_j64_d[DD_LOG_J64_N][2] = DD_LOG_J64_INIT;
#endif
#if defined(__CUDA_ARCH__)
#define DD_TAB(name) name##_d
#else
#define DD_TAB(name) name##_h
#endif

typedef struct { double hi, lo; } dd_t;

DD_HD dd_t dd_make(double hi, double lo) { dd_t r; r.hi = hi; r.lo = lo; return r; }
DD_HD dd_t two_sum(double a, double b) {
  double s = a + b, bb = s - a;
  return dd_make(s, (a - (s - bb)) + (b - bb));
}
DD_HD dd_t quick_two_sum(double a, double b) {
  double s = a + b;
  return dd_make(s, b - (s - a));
}
DD_HD dd_t two_prod(double a, double b) {
  double p = a * b;
  return dd_make(p, fma(a, b, -p));
}
DD_HD dd_t dd_add(dd_t a, dd_t b) {
  dd_t s = two_sum(a.hi, b.hi), t = two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = quick_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return quick_two_sum(s.hi, s.lo);
}
DD_HD dd_t dd_neg(dd_t a) { return dd_make(-a.hi, -a.lo); }
DD_HD dd_t dd_mul(dd_t a, dd_t b) {
  dd_t p = two_prod(a.hi, b.hi);
  p.lo += a.hi * b.lo + a.lo * b.hi;
  return quick_two_sum(p.hi, p.lo);
}
DD_HD dd_t dd_mul_d(dd_t a, double b) {
  dd_t p = two_prod(a.hi, b);
  p.lo += a.lo * b;
  return quick_two_sum(p.hi, p.lo);
}
DD_HD dd_t dd_div(dd_t a, dd_t b) {
  double q1 = a.hi / b.hi;
  dd_t r = dd_add(a, dd_neg(dd_mul_d(b, q1)));
  double q2 = r.hi / b.hi;
  r = dd_add(r, dd_neg(dd_mul_d(b, q2)));
  double q3 = r.hi / b.hi;
  dd_t q = quick_two_sum(q1, q2);
  return dd_add(q, dd_make(q3, 0.0));
}
DD_HD dd_t dd_tab(const double (*t)[2], int i) { return dd_make(t[i][0], t[i][1]); }

// Correctly rounded exp(x).
DD_HD double exp_cr(double x) {
  if (x != x) return x;
  if (x > 709.782712893384) return INFINITY;
  if (x < -745.1332191019412) return 0.0;
  if (x == 0.0) return 1.0;
  double k = rint(x * DD_INV_LN2);
  dd_t p = two_prod(k, DD_LN2_HI);
  dd_t r = two_sum(x - p.hi, -p.lo);          // x - p.hi is exact (Sterbenz)
  r = dd_add(r, dd_neg(two_prod(k, DD_LN2_LO)));
  r.hi *= 0x1p-8;
  r.lo *= 0x1p-8;
  const double (*f)[2] = DD_TAB(dd_inv_fact);
  dd_t e = dd_tab(f, DD_INV_FACT_N - 1);
  for (int i = DD_INV_FACT_N - 2; i >= 0; i--) e = dd_add(dd_mul(e, r), dd_tab(f, i));
  for (int i = 0; i < 8; i++) e = dd_mul(e, e);
  // round in the unscaled binade; scaling by 2^k is exact for normal results
  int ki = (int)k;
  int k1 = ki / 2, k2 = ki - k1;
  return ldexp(ldexp(e.hi + e.lo, k1), k2);
}

// Correctly rounded log(x) for x > 0: the full double-double series.
DD_HD double log_cr_dd(double x) {
  if (!(x > 0.0)) return (x == 0.0) ? -INFINITY : NAN;
  if (x == INFINITY) return x;
  int e = 0;
  double m = frexp(x, &e);   // m in [0.5,1)
  m *= 2.0;
  e -= 1;                    // m in [1,2)
  if (m >= 1.5) { m *= 0.5; e += 1; }
  double j = rint(m * 64.0);            // 48..96
  double c = j * 0x1p-6;
  double rn = m - c;                    // exact
  dd_t den = two_sum(m, c);
  dd_t s = dd_div(dd_make(rn, 0.0), den);
  dd_t s2 = dd_mul(s, s);
  const double (*o)[2] = DD_TAB(dd_inv_odd);
  dd_t poly = dd_tab(o, DD_INV_ODD_N - 1);
  for (int i = DD_INV_ODD_N - 2; i >= 0; i--) poly = dd_add(dd_mul(poly, s2), dd_tab(o, i));
  dd_t at = dd_mul(s, poly);
  at.hi *= 2.0;
  at.lo *= 2.0;
  dd_t res = dd_add(dd_tab(DD_TAB(dd_log_j64), (int)j - 48), at);
  if (e != 0) {
    dd_t el = dd_add(two_prod((double)e, DD_LN2_HI), two_prod((double)e, DD_LN2_LO));
    res = dd_add(el, res);
  }
  return res.hi + res.lo;
}

// Correctly rounded log(x) for x > 0.  The same reduction as log_cr_dd, but
// only the leading terms in double-double: 2s with s = (m-c)/(m+c) to about
// 2^-104, the table's log c and e*ln2; the rest of the atanh series
// (|s| < 0.0053, terms through s^13, the first omitted one below 2^-108 of
// 2|s|) in double.  The result carries an error bound; when both ends of it
// round to the same double that double is the correctly rounded log, else
// log_cr_dd decides (rare: the bound is about 2^-95 of the terms' size).
DD_HD double log_cr(double x) {
  if (!(x > 0.0)) return (x == 0.0) ? -INFINITY : NAN;
  if (x == INFINITY) return x;
  int e = 0;
  double m = frexp(x, &e);   // m in [0.5,1)
  m *= 2.0;
  e -= 1;                    // m in [1,2)
  if (m >= 1.5) { m *= 0.5; e += 1; }
  const double j = rint(m * 64.0);      // 48..96
  const double c = j * 0x1p-6;
  const double rn = m - c;              // exact
  const dd_t den = two_sum(m, c);
  const double sh = rn / den.hi;
  const dd_t p = two_prod(sh, den.hi);
  const double sl = (((rn - p.hi) - p.lo) - sh * den.lo) / den.hi;
  const double s2 = sh * sh;
  const double tail =
      sh * s2 *
      (2.0 / 3 + s2 * (2.0 / 5 + s2 * (2.0 / 7 + s2 * (2.0 / 9 + s2 * (2.0 / 11 + s2 * (2.0 / 13))))));
  const dd_t at = two_sum(2.0 * sh, 2.0 * sl + tail);
  const dd_t lc = dd_tab(DD_TAB(dd_log_j64), (int)j - 48);
  dd_t res = dd_add(lc, at);
  double mag = fabs(lc.hi) + fabs(at.hi);
  if (e != 0) {
    const dd_t el = dd_add(two_prod((double)e, DD_LN2_HI), two_prod((double)e, DD_LN2_LO));
    res = dd_add(el, res);
    mag += fabs(el.hi);
  }
  const double err = mag * 0x1p-95 + fabs(tail) * 0x1p-48;
  const double lo = res.hi + (res.lo - err), hi = res.hi + (res.lo + err);
  if (lo == hi) return lo;
  return log_cr_dd(x);
}

// Fix-up table of the C library's logf on (0,1]: sorted input bit patterns
// keys[] with the library's results vals[]; bucket[b] is the first entry
// whose key>>12 is >= b + LOGF_FIX_BASE, so the keys of one block of 4096
// floats are keys[bucket[b] .. bucket[b+1]).
#define LOGF_FIX_BASE (0x30000000u >> 12)
#define LOGF_FIX_NBUCKET ((0x3F800000u >> 12) - LOGF_FIX_BASE + 2)
typedef struct {
  const uint32_t *keys;
  const float *vals;
  const uint32_t *bucket;
  uint32_t n;
} logf_fixup_t;

// Correctly rounded float log, from a double log with at most one ulp of
// error when the rounding is unambiguous, else from log_cr.
DD_HD float logf_cr_from(float x, double y_approx) {
  float f1 = (float)(y_approx * (1.0 + 0x1p-49));
  float f2 = (float)(y_approx * (1.0 - 0x1p-49));
  if (f1 == f2) return f1;
  return (float)log_cr((double)x);
}
