// Single-precision complex helpers whose rounding follows numpy's complex64
// loops operation by operation (explicit round-to-nearest intrinsics, so no
// contraction into FMAs): the host restatements of the retrieval front-end
// are numpy programs, and these keep the device results within a few ulp.
#pragma once

#include <cuda_runtime.h>

namespace odt {

// |z| with one rounding (the double sum of squares is exact enough)
__device__ __forceinline__ float cabs_f(float2 v) { return (float)sqrt((double)v.x * v.x + (double)v.y * v.y); }

// y / x: Smith's division with the reciprocal of the scale, as numpy
__device__ __forceinline__ float2 cdiv_np(float2 y, float2 x) {
  const float br = x.x, bi = x.y;
  float re, im;
  if (fabsf(br) >= fabsf(bi)) {
    if (br == 0.f && bi == 0.f) {
      re = y.x / fabsf(br);
      im = y.y / fabsf(br);
    } else {
      const float rat = bi / br, scl = 1.0f / __fadd_rn(br, __fmul_rn(bi, rat));
      re = __fmul_rn(__fadd_rn(y.x, __fmul_rn(y.y, rat)), scl);
      im = __fmul_rn(__fsub_rn(y.y, __fmul_rn(y.x, rat)), scl);
    }
  } else {
    const float rat = br / bi, scl = 1.0f / __fadd_rn(bi, __fmul_rn(br, rat));
    re = __fmul_rn(__fadd_rn(__fmul_rn(y.x, rat), y.y), scl);
    im = __fmul_rn(__fsub_rn(__fmul_rn(y.y, rat), y.x), scl);
  }
  return make_float2(re, im);
}

// a * b, the textbook product
__device__ __forceinline__ float2 cmul_np(float2 a, float2 b) {
  return make_float2(__fsub_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)),
                     __fadd_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
}

// exp(1i * angle(z))
__device__ __forceinline__ float2 unit_phasor(float2 z) {
  float s, c;
  sincosf(atan2f(z.y, z.x), &s, &c);
  return make_float2(c, s);
}

// exp(z)
__device__ __forceinline__ float2 cexp_f(float2 z) {
  float s, c;
  sincosf(z.y, &s, &c);
  const float m = expf(z.x);
  return make_float2(__fmul_rn(m, c), __fmul_rn(m, s));
}

}  // namespace odt
