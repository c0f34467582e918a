// itr_math.h — deterministic double-precision exp, log1p and sin, host and device.
//
// The reference's objective J uses softplus(x) = log1p(exp(x)) from the pure-Rust `libm`
// crate 0.2.16 (crates/itr-core/src/objective.rs:70-75). That crate is not part of the
// reference tree. The incumbent early abort (`lb >= incumbent`, evaluator.rs:100-104) runs on
// the device, and the same decision must come out of the host-side oracle, so both sides call
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
//   sin:   x = k*(pi/2) + r with a three-part pi/2 (Cody & Waite), |r| <= pi/4, then the
//          Taylor series of sin(r) to r^17 or of cos(r) to r^16 by the quadrant k mod 4.
// Accuracy is a few ulp (tested against the C library); these are not claimed to be
// correctly rounded, and the reference's libm values are matched only to that level.
// The f32 wrappers (sinf_ref, expf_ref, powf_ref) serve the headless scene render, whose
// shader leaves sin / exp / pow to the platform: with these the device image and the CPU
// oracle's agree bit for bit.
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

// pi/2 = 1.57079632679489661923132169163975144... in three parts: PIO2_1 and PIO2_2 keep 27
// and 25 significant bits, so k*PIO2_1 and k*PIO2_2 are exact for |k| < 2^26 (|x| < 1e8);
// PIO2_3 is the double nearest the remainder.
ITR_HD double sin_ref(double x) {
  if (!(x - x == 0.0)) return x - x;                 // NaN and +-inf give NaN
  if (x > 1e15 || x < -1e15) return 0.0;             // beyond the reduction's range
  const double PIO2_1 = bits_to_f64(0x3FF921FB54000000ull);
  const double PIO2_2 = bits_to_f64(0x3E110B4610000000ull);
  const double PIO2_3 = 5.721188726109832e-18;
  const double two_over_pi = 0.6366197723675814;     // only picks k
  double kf = x * two_over_pi;
  kf = kf < 0.0 ? (double)(long long)(kf - 0.5) : (double)(long long)(kf + 0.5);
  const double r = ((x - kf * PIO2_1) - kf * PIO2_2) - kf * PIO2_3;
  const int q = (int)((long long)kf & 3);
  const double r2 = r * r;
  // sin(r) = r + r^3 * P(r^2), coefficients (-1)^n / (2n+1)!, n = 8 .. 1
  double ps = 1.0 / 355687428096000.0;               // 1/17!
  ps = ps * r2 - 1.0 / 1307674368000.0;              // 1/15!
  ps = ps * r2 + 1.0 / 6227020800.0;                 // 1/13!
  ps = ps * r2 - 1.0 / 39916800.0;                   // 1/11!
  ps = ps * r2 + 1.0 / 362880.0;                     // 1/9!
  ps = ps * r2 - 1.0 / 5040.0;                       // 1/7!
  ps = ps * r2 + 1.0 / 120.0;                        // 1/5!
  ps = ps * r2 - 1.0 / 6.0;                          // 1/3!
  const double s = r + (r * r2) * ps;
  // cos(r) = 1 + r^2 * Q(r^2), coefficients (-1)^n / (2n)!, n = 8 .. 1
  double pc = 1.0 / 20922789888000.0;                // 1/16!
  pc = pc * r2 - 1.0 / 87178291200.0;                // 1/14!
  pc = pc * r2 + 1.0 / 479001600.0;                  // 1/12!
  pc = pc * r2 - 1.0 / 3628800.0;                    // 1/10!
  pc = pc * r2 + 1.0 / 40320.0;                      // 1/8!
  pc = pc * r2 - 1.0 / 720.0;                        // 1/6!
  pc = pc * r2 + 1.0 / 24.0;                         // 1/4!
  pc = pc * r2 - 0.5;                                // 1/2!
  const double c = 1.0 + r2 * pc;
  return q == 0 ? s : (q == 1 ? c : (q == 2 ? -s : -c));
}

// log(x) for x >= 0 through log1p_ref (x - 1 is exact for a float x in (0, 2]).
ITR_HD double log_ref(double x) {
  if (x == 0.0) return -bits_to_f64(0x7FF0000000000000ull);
  return log1p_ref(x - 1.0);
}

ITR_HD float sinf_ref(float x) { return (float)sin_ref((double)x); }
ITR_HD float expf_ref(float x) { return (float)exp_ref((double)x); }
// x^y for x >= 0 as exp(y log x) in double; y = 0 gives 1, x = 0 with y > 0 gives 0.
ITR_HD float powf_ref(float x, float y) {
  if (y == 0.0f) return 1.0f;
  return (float)exp_ref((double)y * log_ref((double)x));
}

// softplus(x) = log(1 + e^x) with the reference's cut-offs (objective.rs:70-75).
ITR_HD double softplus(double x) {
  if (x > 30.0) return x;
  if (x < -30.0) return exp_ref(x);
  return log1p_ref(exp_ref(x));
}

}  // namespace itr_math
