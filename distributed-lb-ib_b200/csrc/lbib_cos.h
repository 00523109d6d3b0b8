/*
 * Correctly rounded double-precision cosine for the immersed-boundary delta
 * kernel, usable from host and device code.
 *
 * Why: the reference evaluates (1 + cos(pi/2 * r)) with the host C library
 * (cube_pthread/lbm_ib.c:1447, :2679-2683).  The LBM-IB run amplifies a
 * last-bit difference in any weight to ~1e-10 relative after ~1000 steps, so
 * the CUDA path needs cosine values that a CPU oracle can reproduce bit for
 * bit.  glibc's cos is not correctly rounded: on this argument range about
 * 0.13% of its values are 1 ulp off (tests/test_cos.py shows such cases), and
 * CUDA's cos carries a 2-ulp bound, so neither can be matched exactly by the
 * other.  A correctly rounded cosine is reproducible anywhere: the CUDA path
 * and the oracle built with this function agree bit for bit, and both stay
 * within 1e-10 of the reference's glibc-based run.  This is
 * not CUDA's algorithm: it is the double-double method of Dekker (1971) and
 * Knuth (TAOCP vol. 2, TwoSum) as used by the QD library (Hida, Li & Bailey,
 * 2001): reduce by k*pi/2 with a triple-double pi/2, then evaluate the Taylor
 * series of cos or sin in double-double and round the double-double once.
 * The double-double result carries ~100 correct bits, so the final rounding is
 * wrong only if the exact value lies within ~2^-100 relative of a rounding
 * boundary.  Constants were derived with Python's decimal module at 80 digits
 * (pi from Machin's formula, 1/(2n)! and 1/(2n+1)! exactly).
 *
 * Valid for |x| <= 4 (the delta kernel needs |x| <= pi).  The code must be
 * compiled without floating-point contraction or reassociation
 * (-fmad=false for nvcc, -ffp-contract=off for gcc); fma() is called
 * explicitly where the error-free product needs it.
 */
#ifndef LBIB_COS_H
#define LBIB_COS_H

#include <math.h>

#if defined(__CUDACC__)
#define LBIB_HD __host__ __device__ __forceinline__
#else
#define LBIB_HD static inline
#endif

typedef struct { double hi, lo; } lbib_dd;

LBIB_HD lbib_dd lbib_two_sum(double a, double b) {
  double s = a + b;
  double bb = s - a;
  double e = (a - (s - bb)) + (b - bb);
  lbib_dd r = {s, e};
  return r;
}

LBIB_HD lbib_dd lbib_quick_two_sum(double a, double b) {
  double s = a + b;
  double e = b - (s - a);
  lbib_dd r = {s, e};
  return r;
}

LBIB_HD lbib_dd lbib_dd_add(lbib_dd a, lbib_dd b) {
  lbib_dd s = lbib_two_sum(a.hi, b.hi);
  lbib_dd t = lbib_two_sum(a.lo, b.lo);
  s.lo += t.hi;
  s = lbib_quick_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return lbib_quick_two_sum(s.hi, s.lo);
}

LBIB_HD lbib_dd lbib_dd_mul(lbib_dd a, lbib_dd b) {
  double p = a.hi * b.hi;
  double e = fma(a.hi, b.hi, -p);
  e += a.hi * b.lo + a.lo * b.hi;
  return lbib_quick_two_sum(p, e);
}

/* pi/2 = P1 + P2 + P3 to ~160 bits. */
#define LBIB_PIO2_1 1.5707963267948966
#define LBIB_PIO2_2 6.123233995736766e-17
#define LBIB_PIO2_3 -1.4973849048591698e-33

LBIB_HD double lbib_cos(double x) {
  /* (-1)^n / (2n)!  and  (-1)^n / (2n+1)!  as double-doubles, n = 1..15 */
  const double CH[16] = {1.0, -0.5, 0.041666666666666664, -0.001388888888888889, 2.48015873015873e-05,
                         -2.755731922398589e-07, 2.08767569878681e-09, -1.1470745597729725e-11,
                         4.779477332387385e-14, -1.5619206968586225e-16, 4.110317623312165e-19,
                         -8.896791392450574e-22, 1.6117375710961184e-24, -2.4795962632247976e-27,
                         3.279889237069838e-30, -3.7699876288159054e-33};
  const double CL[16] = {0.0, 0.0, 2.3129646346357427e-18, 5.300543954373577e-20, 2.1511947866775882e-23,
                         -2.3767714622250297e-23, -1.20734505911326e-25, -2.0655512752830745e-28,
                         4.399205485834081e-31, -1.1910679660273754e-32, 1.4412973378659527e-36,
                         7.911402614872376e-38, -3.6846573564509766e-41, 1.2953730964765229e-43,
                         1.5117542744029879e-46, -2.5870347832750324e-49};
  const double SH[16] = {1.0, -0.16666666666666666, 0.008333333333333333, -0.0001984126984126984,
                         2.7557319223985893e-06, -2.505210838544172e-08, 1.6059043836821613e-10,
                         -7.647163731819816e-13, 2.8114572543455206e-15, -8.22063524662433e-18,
                         1.9572941063391263e-20, -3.868170170630684e-23, 6.446950284384474e-26,
                         -9.183689863795546e-29, 1.1309962886447716e-31, -1.216125041553518e-34};
  const double SL[16] = {0.0, -9.25185853854297e-18, 1.1564823173178714e-19, -1.7209558293420705e-22,
                         -1.858393274046472e-22, 1.448814070935912e-24, 1.2585294588752098e-26,
                         -7.03872877733453e-30, 1.6508842730861433e-31, -2.2141894119604265e-34,
                         -1.3643503830087908e-36, 8.843177655482344e-40, -1.9330404233703465e-42,
                         -1.4303150396787322e-45, 1.0498015412959506e-47, -5.586290567888806e-51};
  double kd = rint(x * 0.6366197723675814);
  int k = (int)kd;
  /* r = x - k*pi/2; k*P1, k*P2, k*P3 are exact for |k| <= 2 */
  lbib_dd r = lbib_two_sum(x, -kd * LBIB_PIO2_1);
  lbib_dd t2 = {-kd * LBIB_PIO2_2, 0.0};
  r = lbib_dd_add(r, t2);
  lbib_dd t3 = {-kd * LBIB_PIO2_3, 0.0};
  r = lbib_dd_add(r, t3);
  lbib_dd r2 = lbib_dd_mul(r, r);
  int odd = k & 1;
  const double* H = odd ? SH : CH;
  const double* L = odd ? SL : CL;
  lbib_dd acc = {H[15], L[15]};
  for (int n = 14; n >= 0; --n) {
    lbib_dd c = {H[n], L[n]};
    acc = lbib_dd_add(lbib_dd_mul(acc, r2), c);
  }
  if (odd) acc = lbib_dd_mul(acc, r);
  double v = acc.hi + acc.lo;
  int q = k & 3;  /* k mod 4 in two's complement */
  /* cos(r + k pi/2): q=0 cos r, q=1 -sin r, q=2 -cos r, q=3 sin r */
  return (q == 1 || q == 2) ? -v : v;
}

/* The same correctly rounded cosine in two phases (Ziv, "Fast evaluation of
 * elementary mathematical functions with correctly rounded last bit", ACM
 * TOMS 17(3), 1991; the quick/accurate split of CRlibm, Daramy-Loirat et
 * al., 2006).  Quick phase: the same reduction, then the series with its
 * first terms in double-double and its tail from the (2n)! / (2n+1)! term
 * n = 5 on in plain double, evaluated at z = r^2:
 *   cos r = 1 + z (c1 + z (c2 + z (c3 + z (c4 + z T(z))))),
 *   sin r = r (1 + z (s1 + z (s2 + z (s3 + z (s4 + z T'(z)))))).
 * For |r| <= pi/4 + 2^-50 (z <= 0.62): the tail term z^5 T is below 2^-25
 * and carries a relative error below 2^-48 from its seven double Horner
 * steps (alternating, fast-decreasing terms), i.e. below 2^-73 of the
 * result; the series truncated after n = 11 misses less than 2^-86; the
 * double-double steps, the reduction and z add less than 2^-98.  The
 * result (hi, lo) is thus within E < 2^-72 |hi| of the exact value.
 * Rounding test: with e = 2^-67 |hi| (> 2E plus the rounding of lo -/+ e),
 * hi + (lo - e) <= exact <= hi + (lo + e), and rounding is monotone, so if
 * both ends round to the same double that double is the correctly rounded
 * cosine.  Otherwise (about 1 evaluation in 6000) the accurate phase
 * lbib_cos decides.  Both phases return the correctly rounded value, so
 * this function and lbib_cos agree on every argument; the quick phase costs
 * about a fifth of lbib_cos's FP64 operations. */
LBIB_HD lbib_dd lbib_dd_mul_d(lbib_dd a, double b) {
  double p = a.hi * b;
  double e = fma(a.hi, b, -p);
  e += a.lo * b;
  return lbib_quick_two_sum(p, e);
}

/* The quick phase: 1 and the correctly rounded cosine in *out when the
 * rounding test decides, 0 otherwise. */
LBIB_HD int lbib_cos_quick(double x, double* out) {
  /* (-1)^n / (2n)!  and  (-1)^n / (2n+1)!: n = 1..4 as double-doubles,
     n = 5..11 as doubles */
  const double C1 = -0.5, C2H = 0.041666666666666664, C2L = 2.3129646346357427e-18,
               C3H = -0.001388888888888889, C3L = 5.300543954373577e-20, C4H = 2.48015873015873e-05,
               C4L = 2.1511947866775882e-23;
  const double S1H = -0.16666666666666666, S1L = -9.25185853854297e-18, S2H = 0.008333333333333333,
               S2L = 1.1564823173178714e-19, S3H = -0.0001984126984126984, S3L = -1.7209558293420705e-22,
               S4H = 2.7557319223985893e-06, S4L = -1.858393274046472e-22;
  const double CT[7] = {-2.755731922398589e-07, 2.08767569878681e-09, -1.1470745597729725e-11,
                        4.779477332387385e-14, -1.5619206968586225e-16, 4.110317623312165e-19,
                        -8.896791392450574e-22};
  const double ST[7] = {-2.505210838544172e-08, 1.6059043836821613e-10, -7.647163731819816e-13,
                        2.8114572543455206e-15, -8.22063524662433e-18, 1.9572941063391263e-20,
                        -3.868170170630684e-23};
  double kd = rint(x * 0.6366197723675814);
  int k = (int)kd;
  lbib_dd r = lbib_two_sum(x, -kd * LBIB_PIO2_1);
  lbib_dd t2 = {-kd * LBIB_PIO2_2, 0.0};
  r = lbib_dd_add(r, t2);
  lbib_dd t3 = {-kd * LBIB_PIO2_3, 0.0};
  r = lbib_dd_add(r, t3);
  lbib_dd z = lbib_dd_mul(r, r);
  int odd = k & 1;
  const double* T = odd ? ST : CT;
  double t = T[6];
  for (int n = 5; n >= 0; --n) t = T[n] + z.hi * t;
  lbib_dd acc = lbib_dd_mul_d(z, t);
  lbib_dd c4 = {odd ? S4H : C4H, odd ? S4L : C4L};
  acc = lbib_dd_add(c4, acc);
  lbib_dd c3 = {odd ? S3H : C3H, odd ? S3L : C3L};
  acc = lbib_dd_add(c3, lbib_dd_mul(z, acc));
  lbib_dd c2 = {odd ? S2H : C2H, odd ? S2L : C2L};
  acc = lbib_dd_add(c2, lbib_dd_mul(z, acc));
  lbib_dd c1 = {odd ? S1H : C1, odd ? S1L : 0.0};
  acc = lbib_dd_add(c1, lbib_dd_mul(z, acc));
  lbib_dd one = {1.0, 0.0};
  acc = lbib_dd_add(one, lbib_dd_mul(z, acc));
  if (odd) acc = lbib_dd_mul(acc, r);
  const double e = fabs(acc.hi) * 6.776263578034403e-21; /* 2^-67 */
  const double a = acc.hi + (acc.lo - e), b = acc.hi + (acc.lo + e);
  if (a != b) return 0;
  int q = k & 3;
  *out = (q == 1 || q == 2) ? -a : a;
  return 1;
}

LBIB_HD double lbib_cos_2phase(double x) {
  double v;
  return lbib_cos_quick(x, &v) ? v : lbib_cos(x);
}

#endif
