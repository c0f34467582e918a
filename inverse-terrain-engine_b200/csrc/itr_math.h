// itr_math.h — deterministic double-precision exp and log1p, host and device.
//
// The reference's objective J uses softplus(x) = log1p(exp(x)) from the pure-Rust `libm`
// crate 0.2.16 (crates/itr-core/src/objective.rs:70-75). That crate is not part of the
// reference tree. The incumbent early abort (`lb >= incumbent`, evaluator.rs:100-104) runs on
// the device, and the same decision must come out on the host checker, so both sides call
// THIS one implementation, compiled without FMA contraction (nvcc -fmad=false,
// gcc -ffp-contract=off): identical inputs give identical bits on the CPU and the GPU.
//
// Method (textbook, written from the mathematics):
//   exp:   x = k*ln2 + r with a two-part ln2 (Cody & Waite 1980 argument reduction),
//          |r| <= ln2/2, exp(r) by its Taylor series to degree 13 (truncation < 4e-18),
//          then an exact scaling by 2^k built from the exponent bits.
//   log1p: small |x|: 2*atanh(s), s = x/(2+x), as an odd power series in s.
//          otherwise: u = 1+x rounded, c = (x-(u-1))/u the first-order correction for that
//          rounding, u = m*2^e with m in [sqrt(1/2), sqrt(2)), log(m) = 2*atanh((m-1)/(m+1)).
// Accuracy is a few ulp (tested against the C library); these are not claimed to be
// correctly rounded, and the reference's libm values are matched only to that level.
#pragma once
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define ITR_HD __host__ __device__ __forceinline__
#else
#define ITR_HD inline
#endif

namespace itr_math {

ITR_HD double bits_to_f64(uint64_t b) {
#if defined(__CUDA_ARCH__)
  return __longlong_as_double((long long)b);
#else
  double d; memcpy(&d, &b, 8); return d;
#endif
}
ITR_HD uint64_t f64_to_bits(double d) {
#if defined(__CUDA_ARCH__)
  return (uint64_t)__double_as_longlong(d);
#else
  uint64_t b; memcpy(&b, &d, 8); return b;
#endif
}

// ln 2 = 0.693147180559945309417232121458176568... split so that k*LN2_HI is exact for
// |k| < 2^20: LN2_HI keeps the top 32 significant bits of the double nearest ln 2.
// LN2_LO = ln2 - LN2_HI, from the double nearest ln2 (0x3FE62E42FEFA39EF) plus its
// residual 2.3190468138462996e-17 (ln2 minus that double).
ITR_HD double ln2_hi() { return bits_to_f64(0x3FE62E42FEFA39EFull & ~((1ull << 21) - 1ull)); }
ITR_HD double ln2_lo() { return (bits_to_f64(0x3FE62E42FEFA39EFull) - ln2_hi()) + 2.3190468138462996e-17; }

// 2^k for -1022 <= k <= 1023.
ITR_HD double pow2i(int k) { return bits_to_f64((uint64_t)(k + 1023) << 52); }

ITR_HD double exp_ref(double x) {
  if (x != x) return x;
  if (x > 709.782712893384) return bits_to_f64(0x7FF0000000000000ull);
  if (x < -745.1332191019412) return 0.0;
  const double inv_ln2 = 1.4426950408889634;  // 1/ln 2 rounded; only picks k
  double kf = x * inv_ln2;
  kf = kf < 0.0 ? (double)(long long)(kf - 0.5) : (double)(long long)(kf + 0.5);
  int k = (int)kf;
  double r = (x - kf * ln2_hi()) - kf * ln2_lo();
  // Taylor coefficients 1/n!, n = 13 .. 2, in Horner form.
  double p = 1.0 / 6227020800.0;                 // 1/13!
  p = p * r + 1.0 / 479001600.0;                 // 1/12!
  p = p * r + 1.0 / 39916800.0;                  // 1/11!
  p = p * r + 1.0 / 3628800.0;                   // 1/10!
  p = p * r + 1.0 / 362880.0;                    // 1/9!
  p = p * r + 1.0 / 40320.0;                     // 1/8!
  p = p * r + 1.0 / 5040.0;                      // 1/7!
  p = p * r + 1.0 / 720.0;                       // 1/6!
  p = p * r + 1.0 / 120.0;                       // 1/5!
  p = p * r + 1.0 / 24.0;                        // 1/4!
  p = p * r + 1.0 / 6.0;                         // 1/3!
  p = p * r + 0.5;                               // 1/2!
  double e = 1.0 + (r + (r * r) * p);
  if (k > 1023) return (e * 2.0) * pow2i(k - 1);
  if (k < -1022) return (e * pow2i(k + 600)) * pow2i(-600);
  return e * pow2i(k);
}

// 2*atanh(s) = 2*(s + s^3/3 + s^5/5 + ...), |s| <= 0.18, 13 odd terms (remainder < 1e-19).
ITR_HD double two_atanh_series(double s) {
  double s2 = s * s;
  double p = 1.0 / 25.0;
  p = p * s2 + 1.0 / 23.0;
  p = p * s2 + 1.0 / 21.0;
  p = p * s2 + 1.0 / 19.0;
  p = p * s2 + 1.0 / 17.0;
  p = p * s2 + 1.0 / 15.0;
  p = p * s2 + 1.0 / 13.0;
  p = p * s2 + 1.0 / 11.0;
  p = p * s2 + 1.0 / 9.0;
  p = p * s2 + 1.0 / 7.0;
  p = p * s2 + 1.0 / 5.0;
  p = p * s2 + 1.0 / 3.0;
  return 2.0 * s + 2.0 * (s * (s2 * p));
}

ITR_HD double log1p_ref(double x) {
  if (x != x) return x;
  if (x == 0.0) return x;
  if (x < -1.0) return bits_to_f64(0x7FF8000000000000ull);
  if (x == -1.0) return -bits_to_f64(0x7FF0000000000000ull);
  if (x > 1.7976931348623157e308) return x;
  if (x > -0.25 && x < 0.25) return two_atanh_series(x / (2.0 + x));
  double u = 1.0 + x;
  double c = (x - (u - 1.0)) / u;
  uint64_t b = f64_to_bits(u);
  int e = (int)((b >> 52) & 0x7FF) - 1023;
  double m = bits_to_f64((b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);  // [1,2)
  if (m > 1.4142135623730951) { m = m * 0.5; e += 1; }
  double lm = two_atanh_series((m - 1.0) / (m + 1.0));
  double ef = (double)e;
  return ef * ln2_hi() + ((ef * ln2_lo() + lm) + c);
}

// softplus(x) = log(1 + e^x) with the reference's cut-offs (objective.rs:70-75).
ITR_HD double softplus(double x) {
  if (x > 30.0) return x;
  if (x < -30.0) return exp_ref(x);
  return log1p_ref(exp_ref(x));
}

}  // namespace itr_math
