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
