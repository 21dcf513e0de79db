// 16-bit block floating-point storage of complex fields (the reduced-
// precision storage mode of the Born loop).
//
// A block of 8 complex values shares one power-of-two exponent e (int8, kept
// in a separate byte array, one byte per block); each value is stored as two
// int16 mantissas (re, im), value = m * 2^(e - 15).  e is the smallest
// integer with max |re|, |im| over the block < 2^e, so every mantissa fits
// in [-32767, 32767]: 15 bits of precision relative to the block's largest
// component, against 11 for fp16 and 8 for bf16, which is what keeps the
// Born series within 1e-4 of the FP64 result when its spectral array and
// Field_n are stored this way in every iteration.  A block of zeros gets the
// exponent -100 (any value decodes to zero).
//
// Blocks are groups of 8 consecutive threads' values (lanes 8j .. 8j+7 of a
// warp), which the callers arrange to be 8 consecutive elements of a row (T)
// or a fixed grouping of work items (Field_n in the fused xy-pass); the block
// maximum is a 3-step butterfly of warp shuffles inside the group.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace odt {

constexpr int kB16MinExp = -100;
constexpr int kB16MaxExp = 127;

#if defined(__CUDA_ARCH__)
// 2^(e - 15) and 2^(15 - e), exact powers of two for e in [-100, 127]
__device__ __forceinline__ float b16_scale(int e) { return __int_as_float((e - 15 + 127) << 23); }
__device__ __forceinline__ float b16_inv_scale(int e) { return __int_as_float((15 - e + 127) << 23); }

__device__ __forceinline__ float2 b16_decode(short2 m, int e) {
  const float s = b16_scale(e);
  return make_float2((float)m.x * s, (float)m.y * s);
}

// Block exponent of the 8-lane group this lane belongs to (all 8 lanes of the
// group must be active; `mask` = the active lanes of the warp).
__device__ __forceinline__ int b16_group_exponent(float2 v, unsigned mask) {
  float M = fmaxf(fabsf(v.x), fabsf(v.y));
  M = fmaxf(M, __shfl_xor_sync(mask, M, 1));
  M = fmaxf(M, __shfl_xor_sync(mask, M, 2));
  M = fmaxf(M, __shfl_xor_sync(mask, M, 4));
  const int eb = (__float_as_int(M) >> 23) & 0xff;   // M in [2^(eb-127), 2^(eb-126))
  return max(kB16MinExp, min(kB16MaxExp, eb - 126));
}

__device__ __forceinline__ short b16_sat(float x) {
  return (short)max(-32767, min(32767, __float2int_rn(x)));
}

__device__ __forceinline__ short2 b16_encode(float2 v, int e) {
  const float is = b16_inv_scale(e);
  return make_short2(b16_sat(v.x * is), b16_sat(v.y * is));
}
#endif

}  // namespace odt
