/*
 * rm_detmath.h - deterministic float transcendentals shared by host and device.
 *
 * The path tracer needs sin/cos (cosine-hemisphere and GGX azimuth sampling,
 * reference src/engine/pathtrace.metal:79, :208, :227), atan (the HSV "rainbow"
 * shader, pathtrace.metal:25, :194) and exp (the a-trous edge weights,
 * pathtrace.metal:1345-1348).  libm and the CUDA math library differ in the
 * last ulps, and a one-ulp change in a sampled direction can flip a later
 * bounce.  These functions use only IEEE-754 single-precision +, -, *, / and
 * floor, so any compiler that does not contract a*b+c into an FMA
 * (nvcc -fmad=false, gcc -ffp-contract=off) gives the same bits on the CPU and
 * on the GPU.
 *
 * Methods (all from the public literature, written from the mathematics):
 *  - argument reduction: Cody & Waite, "Software Manual for the Elementary
 *    Functions" (1980): subtract k*C with C split into parts with short
 *    mantissas so that k*C_hi is exact;
 *  - kernels: truncated Taylor series of sin, cos, atan and exp, evaluated
 *    with Horner's rule; every truncation error is below 2^-30 on the reduced
 *    interval, so the float rounding of the evaluation dominates.
 * The tests compare every function against double-precision libm.
 */
#ifndef RM_DETMATH_H
#define RM_DETMATH_H

#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define RM_HD __host__ __device__ __forceinline__
#else
#define RM_HD static inline
#endif

#ifdef __cplusplus
extern "C++" {
#endif

RM_HD float rm_bits_to_float(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f; memcpy(&f, &u, 4); return f;
#endif
}

RM_HD float rm_floorf(float x) {
#if defined(__CUDA_ARCH__)
  return floorf(x);
#else
  return __builtin_floorf(x);
#endif
}

/* sin(a) and cos(a) for |a| < 2^15.  Quadrant k = floor(a*2/pi + 1/2);
 * r = a - k*pi/2 with pi/2 = P1 + P2 + P3 (P1, P2 have 12 significant bits). */
RM_HD void rm_sincosf(float a, float* s_out, float* c_out) {
  const float kTwoOverPi = 0.6366197466850281f;
  const float P1 = 1.5703125f;
  const float P2 = 4.837512969970703125e-4f;
  const float P3 = 7.549790126404332e-08f;
  float k = rm_floorf(a * kTwoOverPi + 0.5f);
  float r = a - k * P1;
  r = r - k * P2;
  r = r - k * P3;
  float r2 = r * r;
  /* sin r = r - r^3/3! + ... - r^11/11!, cos r = 1 - r^2/2! + ... + r^12/12! */
  float ps = -2.5052108385441720e-08f;
  ps = ps * r2 + 2.7557319223985893e-06f;
  ps = ps * r2 + -1.9841269841269841e-04f;
  ps = ps * r2 + 8.3333333333333333e-03f;
  ps = ps * r2 + -1.6666666666666667e-01f;
  float sn = r + (r * r2) * ps;
  float pc = 2.0876756987868099e-09f;
  pc = pc * r2 + -2.7557319223985888e-07f;
  pc = pc * r2 + 2.4801587301587302e-05f;
  pc = pc * r2 + -1.3888888888888889e-03f;
  pc = pc * r2 + 4.1666666666666664e-02f;
  pc = pc * r2 + -0.5f;
  float cs = 1.0f + r2 * pc;
  int q = ((int)k) & 3;
  float s, c;
  if (q == 0) { s = sn; c = cs; }
  else if (q == 1) { s = cs; c = -sn; }
  else if (q == 2) { s = -sn; c = -cs; }
  else { s = -cs; c = sn; }
  *s_out = s;
  *c_out = c;
}

/* atan(x) for all finite and infinite x (NaN propagates). */
RM_HD float rm_atanf(float x) {
  const float kPio2 = 1.5707963705062866f;
  const float kPio4 = 0.7853981852531433f;
  const float kTanPi8 = 0.4142135679721832f;
  if (x != x) return x;
  float sgn = 1.0f;
  float t = x;
  if (t < 0.0f) { t = -t; sgn = -1.0f; }
  int inv = 0;
  if (t > 1.0f) { t = 1.0f / t; inv = 1; }
  float base = 0.0f;
  if (t > kTanPi8) { t = (t - 1.0f) / (t + 1.0f); base = kPio4; }
  /* atan u = u - u^3/3 + ... + u^17/17 for |u| <= tan(pi/8) */
  float u2 = t * t;
  float p = 1.0f / 17.0f;
  p = p * u2 - 1.0f / 15.0f;
  p = p * u2 + 1.0f / 13.0f;
  p = p * u2 - 1.0f / 11.0f;
  p = p * u2 + 1.0f / 9.0f;
  p = p * u2 - 1.0f / 7.0f;
  p = p * u2 + 1.0f / 5.0f;
  p = p * u2 - 1.0f / 3.0f;
  float at = base + (t + (t * u2) * p);
  if (inv) at = kPio2 - at;
  return sgn * at;
}

/* exp(x).  x*log2(e) = k + f, |f| <= 1/2; r = x - k*ln2 with ln2 = L1 + L2. */
RM_HD float rm_expf(float x) {
  const float kLog2e = 1.4426950216293335f;
  const float L1 = 0.693115234375f;
  const float L2 = 3.194618329871446e-05f;
  if (x != x) return x;
  if (x > 88.5f) return rm_bits_to_float(0x7f800000u);
  if (x < -104.0f) return 0.0f;
  float k = rm_floorf(x * kLog2e + 0.5f);
  float r = x - k * L1;
  r = r - k * L2;
  /* e^r = sum_{n<=9} r^n/n!, |r| <= 0.347 */
  float p = 2.7557319223985893e-06f;
  p = p * r + 2.4801587301587302e-05f;
  p = p * r + 1.9841269841269841e-04f;
  p = p * r + 1.3888888888888889e-03f;
  p = p * r + 8.3333333333333333e-03f;
  p = p * r + 4.1666666666666664e-02f;
  p = p * r + 1.6666666666666667e-01f;
  p = p * r + 0.5f;
  p = p * r + 1.0f;
  p = p * r + 1.0f;
  int ki = (int)k;
  /* scale by 2^k in at most two exact power-of-two steps */
  if (ki > 127) { p = p * rm_bits_to_float(0x7f000000u); ki -= 127; }
  if (ki < -126) { p = p * rm_bits_to_float(0x00800000u); ki += 126; }
  return p * rm_bits_to_float((uint32_t)(ki + 127) << 23);
}

/* x^16 by four squarings (the a-trous normal weight uses pow(x, 16)). */
RM_HD float rm_pow16f(float x) {
  float x2 = x * x;
  float x4 = x2 * x2;
  float x8 = x4 * x4;
  return x8 * x8;
}

#ifdef __cplusplus
}
#endif

#endif /* RM_DETMATH_H */
