/*
 * st_math.h - the elementary functions of the FLIP step (exp, sin, cos), defined from the mathematics so that the
 * CUDA kernels and any host restatement compute bit-identical results.
 *
 * The reference evaluates these in WGSL, whose exp/sin/cos accuracy is left to the implementation (exp within
 * 3 + 2|x| ULP). These versions stay within 2 ULP of the correctly rounded value on the ranges the step uses; the
 * tests check them against the C library.
 *
 * Method: Cody and Waite's argument reduction (W. J. Cody, W. Waite, "Software Manual for the Elementary Functions",
 * 1980): x = k*c + r with the constant c split into a short high part (so k*c_hi is exact) and a low part, then a
 * truncated Taylor series for the reduced argument, evaluated by Horner's rule. Only IEEE single precision add,
 * subtract, multiply and rint are used; compile without contraction (-ffp-contract=off / -fmad=false).
 */
#ifndef ST_MATH_H
#define ST_MATH_H

#include <math.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define ST_HD __host__ __device__ __forceinline__
#else
#define ST_HD static inline
#endif

/* ln 2 = LN2_HI + LN2_LO; LN2_HI = 22713 / 32768 has 15 significant bits, so k * LN2_HI is exact for |k| < 256 */
#define ST_LN2_HI 0.693145751953125f
#define ST_LN2_LO 1.42860682030941723212e-6f
#define ST_LOG2E 1.44269504088896340736f
/* pi / 2 = PIO2_HI + PIO2_LO; PIO2_HI = 6433 / 4096 (13 significant bits), k * PIO2_HI exact for |k| < 2048 */
#define ST_PIO2_HI 1.570556640625f
#define ST_PIO2_LO 2.39686197355588503521e-4f
#define ST_2OPI 0.636619772367581343076f

ST_HD float st_bits_to_float(uint32_t u) {
#if defined(__CUDA_ARCH__)
  return __uint_as_float(u);
#else
  float f;
  memcpy(&f, &u, 4);
  return f;
#endif
}

/* 2^k for integer k in [-149, 127] */
ST_HD float st_exp2i(int k) {
  if (k >= -126) return st_bits_to_float((uint32_t)(k + 127) << 23);
  return st_bits_to_float(1u << (k + 149));
}

/* e^x */
ST_HD float st_expf(float x) {
  if (x != x) return x;
  if (x > 88.72283f) return st_bits_to_float(0x7f800000u);
  if (x < -103.97209f) return 0.0f;
  const float kf = rintf(x * ST_LOG2E);
  const float r = (x - kf * ST_LN2_HI) - kf * ST_LN2_LO;          /* |r| <= ln2/2 (plus rounding) */
  /* e^r = 1 + r + r^2/2 + ... + r^8/8!: the first term left out is below 2^-29 relative */
  float p = 2.48015873015873015873e-5f;                            /* 1/8! */
  p = 1.98412698412698412698e-4f + r * p;                          /* 1/7! */
  p = 1.38888888888888888889e-3f + r * p;                          /* 1/6! */
  p = 8.33333333333333333333e-3f + r * p;                          /* 1/5! */
  p = 4.16666666666666666667e-2f + r * p;                          /* 1/4! */
  p = 1.66666666666666666667e-1f + r * p;                          /* 1/3! */
  p = 0.5f + r * p;
  p = 1.0f + r * p;
  p = 1.0f + r * p;
  int k = (int)kf;
  /* scale in two steps so neither factor leaves the normal range */
  if (k > 127) { p = p * 2.0f; k -= 1; }
  if (k < -126) { p = p * st_exp2i(-64); k += 64; }
  return p * st_exp2i(k);
}

/* sin and cos of the reduced argument r, |r| <= pi/4: Taylor series to r^13 and r^14 */
ST_HD float st_sin_poly(float r) {
  const float r2 = r * r;
  float p = 1.60590438368216145994e-10f;                           /* 1/13! */
  p = -2.50521083854417187751e-8f + r2 * p;                        /* -1/11! */
  p = 2.75573192239858906526e-6f + r2 * p;                         /* 1/9! */
  p = -1.98412698412698412698e-4f + r2 * p;                        /* -1/7! */
  p = 8.33333333333333333333e-3f + r2 * p;                         /* 1/5! */
  p = -1.66666666666666666667e-1f + r2 * p;                        /* -1/3! */
  return r + r * (r2 * p);
}
ST_HD float st_cos_poly(float r) {
  const float r2 = r * r;
  float p = -1.14707455977297247139e-11f;                          /* -1/14! */
  p = 2.08767569878680989792e-9f + r2 * p;                         /* 1/12! */
  p = -2.75573192239858906526e-7f + r2 * p;                        /* -1/10! */
  p = 2.48015873015873015873e-5f + r2 * p;                         /* 1/8! */
  p = -1.38888888888888888889e-3f + r2 * p;                        /* -1/6! */
  p = 4.16666666666666666667e-2f + r2 * p;                         /* 1/4! */
  p = -0.5f + r2 * p;
  return 1.0f + r2 * p;
}
/* sin x and cos x for |x| < 2048 * pi/2 (the step only uses angles in [0, 2 pi)) */
ST_HD void st_sincosf(float x, float* s, float* c) {
  const float kf = rintf(x * ST_2OPI);
  const float r = (x - kf * ST_PIO2_HI) - kf * ST_PIO2_LO;
  const float sr = st_sin_poly(r), cr = st_cos_poly(r);
  const int q = ((int)kf) & 3;
  if (q == 0) { *s = sr; *c = cr; }
  else if (q == 1) { *s = cr; *c = -sr; }
  else if (q == 2) { *s = -sr; *c = -cr; }
  else { *s = -cr; *c = sr; }
}

#endif
