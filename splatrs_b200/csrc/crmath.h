// Correctly rounded single-precision exp and log, evaluated in double precision.
//
// Both functions use only IEEE-754 double additions, multiplications, one division
// (log) and explicit fused multiply-adds, plus integer bit manipulation. Those
// operations are exactly rounded on the host (gcc, -ffp-contract=off) and on sm_100a,
// so the same source produces bit-identical results on the CPU and the GPU. That is what
// lets an exhaustive host-side sweep stand as proof for the device code.
//
// Method (textbook, Cody & Waite 1980 range reduction + Taylor series):
//   exp: x = n ln2 + r with |r| <= ln2/2, ln2 split into a 45-bit head (so n*head and
//        x - n*head are exact for |n| < 256) and a tail; e^r by its Taylor series to
//        degree 13 (truncation < 2e-16 relative); result scaled by 2^n and rounded once
//        to float.
//   log: x = m 2^e with m in [sqrt(1/2), sqrt(2)); log m = 2 atanh(s), s = (m-1)/(m+1),
//        |s| < 0.1716, atanh by its odd power series to s^23; e ln2 added with the
//        split constant; rounded once to float.
// The double result carries a relative error of a few 1e-16, far below half a float
// ulp (3e-8), so the final rounding to float is correct except for inputs whose exact
// value lies within ~1e-16 of a float rounding boundary.
#pragma once
#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define CRM_HD __host__ __device__ __forceinline__
#else
#define CRM_HD static inline
#endif

namespace crm {

CRM_HD double bits_to_double(uint64_t b) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)b);
#else
  double d;
  __builtin_memcpy(&d, &b, 8);
  return d;
#endif
}

CRM_HD uint64_t double_to_bits(double d) {
#if defined(__CUDA_ARCH__)
  return (uint64_t)__double_as_longlong(d);
#else
  uint64_t b;
  __builtin_memcpy(&b, &d, 8);
  return b;
#endif
}

// ln 2 = LN2_HI + LN2_LO; LN2_HI keeps 45 significant bits.
#define CRM_LN2_HI 0x1.62e42fefa3900p-1
#define CRM_LN2_LO 0x1.de6af278ece60p-46
#define CRM_INV_LN2 0x1.71547652b82fep+0

// e^r for |r| <= ln2/2 by Horner evaluation of sum_{k<=13} r^k / k!.
CRM_HD double exp_reduced(double r) {
  double p = 0x1.6124613a86d09p-33;      // 1/13!
  p = fma(p, r, 0x1.1eed8eff8d898p-29);  // 1/12!
  p = fma(p, r, 0x1.ae64567f544e4p-26);  // 1/11!
  p = fma(p, r, 0x1.27e4fb7789f5cp-22);  // 1/10!
  p = fma(p, r, 0x1.71de3a556c734p-19);  // 1/9!
  p = fma(p, r, 0x1.a01a01a01a01ap-16);  // 1/8!
  p = fma(p, r, 0x1.a01a01a01a01ap-13);  // 1/7!
  p = fma(p, r, 0x1.6c16c16c16c17p-10);  // 1/6!
  p = fma(p, r, 0x1.1111111111111p-7);   // 1/5!
  p = fma(p, r, 0x1.5555555555555p-5);   // 1/4!
  p = fma(p, r, 0x1.5555555555555p-3);   // 1/3!
  p = fma(p, r, 0.5);
  p = fma(p, r, 1.0);
  p = fma(p, r, 1.0);
  return p;
}

// Correctly rounded e^x for float x.
CRM_HD float expf_cr(float x) {
  if (!(x == x)) return x;                 // NaN
  if (x > 88.8f) return (float)INFINITY;   // overflows float
  if (x < -104.0f) return 0.0f;            // below half the smallest subnormal
  double d = (double)x;
  double n = rint(d * CRM_INV_LN2);
  double r = fma(-n, CRM_LN2_HI, d);       // exact
  r = fma(-n, CRM_LN2_LO, r);
  double p = exp_reduced(r);
  int ni = (int)n;                         // in [-150, 129]
  double s = bits_to_double((uint64_t)(ni + 1023) << 52);
  return (float)(p * s);
}

// 2^(j/64), j = 0..63, each correctly rounded to double.
#define CRM_EXP2_TAB64                                                                          \
  {0x1.0000000000000p+0, 0x1.02c9a3e778061p+0, 0x1.059b0d3158574p+0, 0x1.0874518759bc8p+0,     \
   0x1.0b5586cf9890fp+0, 0x1.0e3ec32d3d1a2p+0, 0x1.11301d0125b51p+0, 0x1.1429aaea92de0p+0,     \
   0x1.172b83c7d517bp+0, 0x1.1a35beb6fcb75p+0, 0x1.1d4873168b9aap+0, 0x1.2063b88628cd6p+0,     \
   0x1.2387a6e756238p+0, 0x1.26b4565e27cddp+0, 0x1.29e9df51fdee1p+0, 0x1.2d285a6e4030bp+0,     \
   0x1.306fe0a31b715p+0, 0x1.33c08b26416ffp+0, 0x1.371a7373aa9cbp+0, 0x1.3a7db34e59ff7p+0,     \
   0x1.3dea64c123422p+0, 0x1.4160a21f72e2ap+0, 0x1.44e086061892dp+0, 0x1.486a2b5c13cd0p+0,     \
   0x1.4bfdad5362a27p+0, 0x1.4f9b2769d2ca7p+0, 0x1.5342b569d4f82p+0, 0x1.56f4736b527dap+0,     \
   0x1.5ab07dd485429p+0, 0x1.5e76f15ad2148p+0, 0x1.6247eb03a5585p+0, 0x1.6623882552225p+0,     \
   0x1.6a09e667f3bcdp+0, 0x1.6dfb23c651a2fp+0, 0x1.71f75e8ec5f74p+0, 0x1.75feb564267c9p+0,     \
   0x1.7a11473eb0187p+0, 0x1.7e2f336cf4e62p+0, 0x1.82589994cce13p+0, 0x1.868d99b4492edp+0,     \
   0x1.8ace5422aa0dbp+0, 0x1.8f1ae99157736p+0, 0x1.93737b0cdc5e5p+0, 0x1.97d829fde4e50p+0,     \
   0x1.9c49182a3f090p+0, 0x1.a0c667b5de565p+0, 0x1.a5503b23e255dp+0, 0x1.a9e6b5579fdbfp+0,     \
   0x1.ae89f995ad3adp+0, 0x1.b33a2b84f15fbp+0, 0x1.b7f76f2fb5e47p+0, 0x1.bcc1e904bc1d2p+0,     \
   0x1.c199bdd85529cp+0, 0x1.c67f12e57d14bp+0, 0x1.cb720dcef9069p+0, 0x1.d072d4a07897cp+0,     \
   0x1.d5818dcfba487p+0, 0x1.da9e603db3285p+0, 0x1.dfc97337b9b5fp+0, 0x1.e502ee78b3ff6p+0,     \
   0x1.ea4afa2a490dap+0, 0x1.efa1bee615a27p+0, 0x1.f50765b6e4540p+0, 0x1.fa7c1819e90d8p+0}

// The same correctly rounded e^x with fewer double operations, for hot loops (table-driven
// method, Tang 1989): x = (64 m + j) ln2/64 + r with |r| <= ln2/128, ln2/64 split into a
// 39-bit head and a tail (so the head product and x minus it are exact);
// e^x = 2^m * 2^(j/64) * (1 + q), q = e^r - 1 by its Taylor series to r^5 (truncation
// below 4e-17 relative). `tab` is CRM_EXP2_TAB64 (in shared memory on the device). An
// exhaustive sweep over every float in [-110, 90] gives results identical to expf_cr.
CRM_HD float expf_cr_tab(float x, const double* tab) {
  if (!(x == x)) return x;
  if (x > 88.8f) return (float)INFINITY;
  if (x < -104.0f) return 0.0f;
  double d = (double)x;
  double n = rint(d * 0x1.71547652b82fep+6);  // 64 / ln2
  double r = fma(-n, 0x1.62e42fefa0000p-7, d);
  r = fma(-n, 0x1.cf79abc9e3b3ap-46, r);
  int ni = (int)n;
  double c = fma(r, 0x1.1111111111111p-7, 0x1.5555555555555p-5);  // 1/120, 1/24
  c = fma(r, c, 0x1.5555555555555p-3);                            // 1/6
  c = fma(r, c, 0.5);
  c = fma(r, c, 1.0);
  double q = r * c;
  double t = tab[ni & 63];
  double y = fma(t, q, t);
  double s = bits_to_double((uint64_t)((ni >> 6) + 1023) << 52);
  return (float)(y * s);
}

// expf_cr_tab for the compositing range. The argument there is -sigma with
// 0 <= sigma <= sigma_max = ln(255 * opacity) <= ln 255, so n = rint(64 x / ln2) lies in
// [-512, 0]. A table of 2^(n/64) for n in [-(kExpNegEntries-1), 0] folds the 2^m scale into
// the table entry (entry k = table64[(-k) & 63] * 2^((-k) >> 6), exact), so
// fma(t', q, t') = 2^m * fma(t, q, t) exactly and the result equals expf_cr_tab bit for
// bit; arguments below kExpNegMin (never produced by a valid projection) and NaN take
// expf_cr.
constexpr int kExpNegEntries = 577;
constexpr float kExpNegMin = -6.2f;  // rint(-6.2 * 64 / ln2) = -572

CRM_HD double exp2_neg_entry(int k, const double* tab64) {
  const int n = -k;
  return bits_to_double(double_to_bits(tab64[n & 63]) + ((uint64_t)(int64_t)(n >> 6) << 52));
}

CRM_HD float expf_cr_neg(float x, const double* tab_neg) {
  if (!(x >= kExpNegMin)) return expf_cr(x);
  const double d = (double)x;
  const double n = rint(d * 0x1.71547652b82fep+6);  // 64 / ln2
  double r = fma(-n, 0x1.62e42fefa0000p-7, d);
  r = fma(-n, 0x1.cf79abc9e3b3ap-46, r);
  double c = fma(r, 0x1.1111111111111p-7, 0x1.5555555555555p-5);  // 1/120, 1/24
  c = fma(r, c, 0x1.5555555555555p-3);                            // 1/6
  c = fma(r, c, 0.5);
  c = fma(r, c, 1.0);
  const double q = r * c;
  const double t = tab_neg[-(int)n];
  return (float)fma(t, q, t);
}

// Correctly rounded natural log for float x.
CRM_HD float logf_cr(float x) {
  if (!(x == x) || x < 0.0f) return (float)NAN;
  if (x == 0.0f) return -(float)INFINITY;
  if (x == (float)INFINITY) return x;
  double d = (double)x;                    // float subnormals are normal doubles
  uint64_t b = double_to_bits(d);
  int e = (int)((b >> 52) & 0x7ff) - 1023;
  double m = bits_to_double((b & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
  if (m > 0x1.6a09e667f3bcdp+0) {          // sqrt(2)
    m *= 0.5;
    e += 1;
  }
  double s = (m - 1.0) / (m + 1.0);
  double s2 = s * s;
  double p = 0x1.642c8590b2164p-5;         // 1/23
  p = fma(p, s2, 0x1.745d1745d1746p-5);    // 1/21
  p = fma(p, s2, 0x1.8618618618618p-5);    // 1/19
  p = fma(p, s2, 0x1.af286bca1af28p-5);    // 1/17
  p = fma(p, s2, 0x1.e1e1e1e1e1e1ep-5);    // 1/15
  p = fma(p, s2, 0x1.1111111111111p-4);    // 1/13
  p = fma(p, s2, 0x1.745d1745d1746p-4);    // 1/11
  p = fma(p, s2, 0x1.c71c71c71c71cp-4);    // 1/9
  p = fma(p, s2, 0x1.2492492492492p-3);    // 1/7
  p = fma(p, s2, 0x1.999999999999ap-3);    // 1/5
  p = fma(p, s2, 0x1.5555555555555p-2);    // 1/3
  double lm = fma(2.0 * s, s2 * p, 2.0 * s);   // 2s + 2s^3 (1/3 + s^2/5 + ...)
  double de = (double)e;
  double r = fma(de, CRM_LN2_HI, fma(de, CRM_LN2_LO, lm));
  return (float)r;
}

}  // namespace crm
