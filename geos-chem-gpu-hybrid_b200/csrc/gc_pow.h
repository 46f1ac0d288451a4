/*
 * gc_pow.h -- the one pow(x, y) used by both the CPU oracle and the CUDA
 * kernels for the Rodas3 step-size factor  FacSafe / Err**(ONE/ros_ELO)
 * (gckpp_BatchIntegrator.F90:667).
 *
 * glibc's pow and CUDA's pow are different implementations that are not
 * guaranteed to agree in the last bit, and the whole step sequence of a cell
 * depends on that one value.  This file therefore computes x**y itself, from
 * plain IEEE operations that round identically on the host and the device:
 *
 *   - double-double arithmetic (Dekker 1971; the two-sum of Knuth, TAOCP
 *     vol. 2 4.2.2) with the exact product error obtained from one fused
 *     multiply-add (fma(a, b, -a*b) is exact; IEEE 754-2008 5.4.1);
 *   - ln(m), m in [sqrt(1/2), sqrt(2)), from the series
 *     ln m = 2 atanh(s) = 2 (s + s^3/3 + s^5/5 + ...), s = (m-1)/(m+1),
 *     evaluated in double-double to about 2^-100 relative;
 *   - exp(t) by t = k ln2 + r, |r| <= ln2/2, r scaled by 2^-8, Taylor series
 *     to order 14 in double-double, then squared 8 times, then scaled by 2^k.
 *
 * The result is the double nearest the double-double value, i.e. correctly
 * rounded except when x**y lies within ~2^-95 relative of a rounding
 * boundary.  It is only defined here for finite x > 0 and finite y with a
 * finite, normal result, which covers Err in [1e-10, DBL_MAX] and
 * y = 1/3; other arguments fall back to the IEEE special-case rules below.
 *
 * The constants are the mathematical values ln 2 (split into a double-double
 * pair) and the reciprocals 1/(2i+1), 1/i!; nothing here is taken from a
 * vendor library.
 */
#pragma once
#include <math.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define GC_HD __host__ __device__ __forceinline__
#else
#define GC_HD static inline
#endif

#if defined(__CUDA_ARCH__)
#define GC_FMA(a, b, c) __fma_rn((a), (b), (c))
#define GC_ADD(a, b) __dadd_rn((a), (b))
#define GC_SUB(a, b) __dsub_rn((a), (b))
#define GC_MUL(a, b) __dmul_rn((a), (b))
#define GC_DIV(a, b) __ddiv_rn((a), (b))
#else
#define GC_FMA(a, b, c) fma((a), (b), (c))
#define GC_ADD(a, b) ((a) + (b))
#define GC_SUB(a, b) ((a) - (b))
#define GC_MUL(a, b) ((a) * (b))
#define GC_DIV(a, b) ((a) / (b))
#endif

typedef struct { double hi, lo; } gc_dd;

GC_HD gc_dd gc_dd_make(double hi, double lo) { gc_dd r; r.hi = hi; r.lo = lo; return r; }

/* two-sum: s + e == a + b exactly */
GC_HD gc_dd gc_two_sum(double a, double b) {
  double s = GC_ADD(a, b);
  double bb = GC_SUB(s, a);
  double e = GC_ADD(GC_SUB(a, GC_SUB(s, bb)), GC_SUB(b, bb));
  return gc_dd_make(s, e);
}
/* fast two-sum, requires |a| >= |b| */
GC_HD gc_dd gc_fast_two_sum(double a, double b) {
  double s = GC_ADD(a, b);
  double e = GC_SUB(b, GC_SUB(s, a));
  return gc_dd_make(s, e);
}
GC_HD gc_dd gc_two_prod(double a, double b) {
  double p = GC_MUL(a, b);
  double e = GC_FMA(a, b, -p);
  return gc_dd_make(p, e);
}
GC_HD gc_dd gc_dd_add(gc_dd x, gc_dd y) {
  gc_dd s = gc_two_sum(x.hi, y.hi);
  gc_dd t = gc_two_sum(x.lo, y.lo);
  s.lo = GC_ADD(s.lo, t.hi);
  s = gc_fast_two_sum(s.hi, s.lo);
  s.lo = GC_ADD(s.lo, t.lo);
  return gc_fast_two_sum(s.hi, s.lo);
}
GC_HD gc_dd gc_dd_mul(gc_dd x, gc_dd y) {
  gc_dd p = gc_two_prod(x.hi, y.hi);
  double c = GC_FMA(x.hi, y.lo, GC_MUL(x.lo, y.hi));
  p.lo = GC_ADD(p.lo, c);
  return gc_fast_two_sum(p.hi, p.lo);
}
GC_HD gc_dd gc_dd_mul_d(gc_dd x, double y) {
  gc_dd p = gc_two_prod(x.hi, y);
  p.lo = GC_FMA(x.lo, y, p.lo);
  return gc_fast_two_sum(p.hi, p.lo);
}
/* x / y in double-double: one Newton correction of the double quotient */
GC_HD gc_dd gc_dd_div(gc_dd x, gc_dd y) {
  double q1 = GC_DIV(x.hi, y.hi);
  gc_dd r = gc_dd_add(x, gc_dd_mul_d(y, -q1));
  double q2 = GC_DIV(r.hi, y.hi);
  r = gc_dd_add(r, gc_dd_mul_d(y, -q2));
  double q3 = GC_DIV(r.hi, y.hi);
  gc_dd q = gc_fast_two_sum(q1, q2);
  return gc_dd_add(q, gc_dd_make(q3, 0.0));
}

/* ln 2 = 0.693147180559945309417232121458176568... as hi + lo */
#define GC_LN2_HI 6.93147180559945286226763982995180413126945495605468750e-01
#define GC_LN2_LO 2.31904681384629955842740722885893731112e-17

GC_HD uint64_t gc_bits(double x) { uint64_t u; memcpy(&u, &x, 8); return u; }
GC_HD double gc_from_bits(uint64_t u) { double x; memcpy(&x, &u, 8); return x; }

/* natural log of a finite positive normal double, in double-double */
GC_HD gc_dd gc_log_dd(double x) {
  uint64_t u = gc_bits(x);
  int e = (int)((u >> 52) & 0x7ff) - 1023;
  double m = gc_from_bits((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
  if (m > 1.4142135623730951) { m = GC_MUL(m, 0.5); e += 1; }
  /* s = (m-1)/(m+1) in double-double; m-1 and m+1 are exact for m in
     [0.7, 1.42) except m+1 which may round: use two-sum */
  gc_dd num = gc_two_sum(m, -1.0);
  gc_dd den = gc_two_sum(m, 1.0);
  gc_dd s = gc_dd_div(num, den);
  gc_dd s2 = gc_dd_mul(s, s);
  /* atanh series: sum_{i>=0} s^(2i)/(2i+1), |s| < 0.1716, s^2 < 0.02944;
     28 terms leave < 0.0295^28/57 ~ 1e-45 */
  gc_dd acc = gc_dd_make(1.0 / 57.0, 0.0);
  for (int i = 27; i >= 0; --i) {
    double inv_hi = GC_DIV(1.0, (double)(2 * i + 1));
    double inv_lo = GC_DIV(GC_FMA(-inv_hi, (double)(2 * i + 1), 1.0), (double)(2 * i + 1));
    acc = gc_dd_add(gc_dd_mul(acc, s2), gc_dd_make(inv_hi, inv_lo));
  }
  gc_dd lnm = gc_dd_mul(gc_dd_mul_d(s, 2.0), acc);
  gc_dd eln2 = gc_dd_mul_d(gc_dd_make(GC_LN2_HI, GC_LN2_LO), (double)e);
  return gc_dd_add(eln2, lnm);
}

/* exp of a double-double t with |t| < 700 */
GC_HD double gc_exp_dd(gc_dd t) {
  double kf = nearbyint(GC_DIV(t.hi, GC_LN2_HI));
  int k = (int)kf;
  /* r = t - k ln2 (k ln2 exact in double-double since |k| < 2^11) */
  gc_dd kl = gc_dd_mul_d(gc_dd_make(GC_LN2_HI, GC_LN2_LO), -kf);
  gc_dd r = gc_dd_add(t, kl);
  r = gc_dd_make(GC_MUL(r.hi, 0.00390625), GC_MUL(r.lo, 0.00390625)); /* /256 */
  /* Taylor: sum_{i=0}^{14} r^i / i!, |r| < 0.00136: 0.00136^15/15! ~ 1e-55 */
  gc_dd acc = gc_dd_make(1.0, 0.0);
  for (int i = 14; i >= 1; --i) {
    acc = gc_dd_mul(acc, r);
    double inv_hi = GC_DIV(1.0, (double)i);
    double inv_lo = GC_DIV(GC_FMA(-inv_hi, (double)i, 1.0), (double)i);
    acc = gc_dd_mul(acc, gc_dd_make(inv_hi, inv_lo));
    acc = gc_dd_add(acc, gc_dd_make(1.0, 0.0));
  }
  for (int i = 0; i < 8; ++i) acc = gc_dd_mul(acc, acc);
  double v = GC_ADD(acc.hi, acc.lo);
  /* scale by 2^k in two exact steps to stay clear of overflow in 2^k */
  int k1 = k / 2, k2 = k - k1;
  v = GC_MUL(v, gc_from_bits((uint64_t)(1023 + k1) << 52));
  v = GC_MUL(v, gc_from_bits((uint64_t)(1023 + k2) << 52));
  return v;
}

/* x**y for the integrator's step-size factor (see the file comment). */
GC_HD double gc_pow(double x, double y) {
  if (x != x || y != y) return x + y;          /* NaN in, NaN out */
  if (y == 0.0) return 1.0;
  if (x == 1.0) return 1.0;
  if (x == 0.0) return y > 0.0 ? 0.0 : 1.0 / 0.0;
  if (x < 0.0) return (x - x) / (x - x);       /* non-integer y assumed */
  if (x == 1.0 / 0.0) return y > 0.0 ? x : 0.0;
  uint64_t u = gc_bits(x);
  if (((u >> 52) & 0x7ff) == 0) {              /* subnormal: rescale by 2^64 */
    gc_dd l = gc_log_dd(GC_MUL(x, 18446744073709551616.0));
    l = gc_dd_add(l, gc_dd_mul_d(gc_dd_make(GC_LN2_HI, GC_LN2_LO), -64.0));
    gc_dd t = gc_dd_mul_d(l, y);
    if (t.hi > 709.0 || t.hi < -708.0) return t.hi > 0 ? 1.0 / 0.0 : 0.0;
    return gc_exp_dd(t);
  }
  gc_dd t = gc_dd_mul_d(gc_log_dd(x), y);
  if (t.hi > 709.0) return 1.0 / 0.0;
  if (t.hi < -708.0) return 0.0;               /* subnormal results flushed */
  return gc_exp_dd(t);
}
