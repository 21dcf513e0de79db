// Tile-FFT kernels of the CBS solver: __global__ wrappers around the bodies
// in tile_bodies.cuh (fused x-pass, z-pass with the Green's multiply, line
// and column FFTs).
//
// This file is compiled once per (kernel kind, radix class) pair
// (-DODT_KIND=0..3 -DODT_CLS=0..3, see the Makefile) so the heavily unrolled
// radix code builds in parallel; cbs_kernels.cu dispatches.
#include "tile_bodies.cuh"

#ifndef ODT_KIND
#error "compile with -DODT_KIND=<0..3> -DODT_CLS=<0..3>"
#endif

namespace odt {

namespace {

__device__ __forceinline__ Thr thr() { return Thr{(int)threadIdx.x, (int)blockDim.x}; }

// launch bound of the tile kernels: 256 threads (128-register budget), 128
// for radix class 3 (butterflies of up to 31 points held in registers); the
// launches use 128 threads in every class
template <int CLS>
constexpr int kMaxThreads = CLS == 3 ? 128 : 256;

template <int CLS, int MODE>
__global__ void __launch_bounds__(kMaxThreads<CLS>, 2)
born_x_kernel(BornArgs a, int jj, FftPlan plan, const float2* __restrict__ twg, int W) {
  extern __shared__ __align__(16) unsigned char smraw[];
  born_x_body<CLS, MODE>(a, jj, plan, twg, W, smraw, blockIdx.x, thr());
}

template <int CLS>
__global__ void __launch_bounds__(kMaxThreads<CLS>, 2)
born_z_kernel(BornArgs a, int jj, FftPlan plan, const float2* __restrict__ twg, int lgW) {
  extern __shared__ __align__(16) unsigned char smraw[];
  born_z_body<CLS>(a, jj, plan, twg, lgW, smraw, blockIdx.x, thr());
}

template <int CLS, bool INV>
__global__ void __launch_bounds__(kMaxThreads<CLS>, 2)
fft_lines_kernel(const float2* in, float2* out, long long nlines, int in_shift, int out_shift,
                 float scale, FftPlan plan, const float2* __restrict__ twg, int W) {
  extern __shared__ __align__(16) unsigned char smraw[];
  fft_lines_body<CLS, INV>(in, out, nlines, in_shift, out_shift, scale, plan, twg, W, smraw,
                           blockIdx.x, thr());
}

template <int CLS, bool INV, bool SHIFT>
__global__ void __launch_bounds__(kMaxThreads<CLS>, 2)
fft_cols_kernel(const float2* in, float2* out, long long n0, int in_shift, int out_shift,
                float scale, FftPlan plan, const float2* __restrict__ twg, int lgW) {
  extern __shared__ __align__(16) unsigned char smraw[];
  fft_cols_body<CLS, INV, SHIFT>(in, out, n0, in_shift, out_shift, scale, plan, twg, lgW, smraw,
                                 blockIdx.x, thr());
}

template <typename K>
cudaError_t set_smem(K kernel, size_t bytes) {
  return raise_smem_limit(reinterpret_cast<const void*>(kernel), bytes);
}

}  // namespace

#if ODT_KIND == 0
template <>
cudaError_t born_x_launch<ODT_CLS>(const BornArgs& a, int mode, int jj, const DevFft& f,
                                    unsigned blocks, size_t sm, cudaStream_t s) {
  cudaError_t err;
  switch (mode) {
    case kBornFirst:
      if ((err = set_smem(born_x_kernel<ODT_CLS, kBornFirst>, sm)) != cudaSuccess) return err;
      born_x_kernel<ODT_CLS, kBornFirst><<<blocks, f.nthr, sm, s>>>(a, jj, f.plan, f.tw, f.W);
      break;
    case kBornMid:
      if ((err = set_smem(born_x_kernel<ODT_CLS, kBornMid>, sm)) != cudaSuccess) return err;
      born_x_kernel<ODT_CLS, kBornMid><<<blocks, f.nthr, sm, s>>>(a, jj, f.plan, f.tw, f.W);
      break;
    default:
      if ((err = set_smem(born_x_kernel<ODT_CLS, kBornLast>, sm)) != cudaSuccess) return err;
      born_x_kernel<ODT_CLS, kBornLast><<<blocks, f.nthr, sm, s>>>(a, jj, f.plan, f.tw, f.W);
      break;
  }
  return cudaGetLastError();
}
#elif ODT_KIND == 1
template <>
cudaError_t born_z_launch<ODT_CLS>(const BornArgs& a, int jj, const DevFft& f, unsigned blocks,
                                    size_t sm, cudaStream_t s) {
  cudaError_t err = set_smem(born_z_kernel<ODT_CLS>, sm);
  if (err != cudaSuccess) return err;
  born_z_kernel<ODT_CLS><<<blocks, f.nthr, sm, s>>>(a, jj, f.plan, f.tw, f.lgW);
  return cudaGetLastError();
}
#elif ODT_KIND == 2
template <>
cudaError_t lines_launch<ODT_CLS>(const float2* in, float2* out, long long nlines, int is, int os,
                                   float sc, bool inv, const DevFft& f, unsigned blocks, size_t sm,
                                   cudaStream_t s) {
  cudaError_t err;
  if (inv) {
    if ((err = set_smem(fft_lines_kernel<ODT_CLS, true>, sm)) != cudaSuccess) return err;
    fft_lines_kernel<ODT_CLS, true><<<blocks, f.nthr, sm, s>>>(in, out, nlines, is, os, sc,
                                                                f.plan, f.tw, f.W);
  } else {
    if ((err = set_smem(fft_lines_kernel<ODT_CLS, false>, sm)) != cudaSuccess) return err;
    fft_lines_kernel<ODT_CLS, false><<<blocks, f.nthr, sm, s>>>(in, out, nlines, is, os, sc,
                                                                 f.plan, f.tw, f.W);
  }
  return cudaGetLastError();
}
#else
template <>
cudaError_t cols_launch<ODT_CLS>(const float2* in, float2* out, long long n0, long long n2, int is,
                                  int os, float sc, bool inv, bool shift, const DevFft& f,
                                  unsigned blocks, size_t sm, cudaStream_t s) {
  (void)n2;
  cudaError_t err;
#define ODT_COLS(I, S)                                                                       \
  if ((err = set_smem(fft_cols_kernel<ODT_CLS, I, S>, sm)) != cudaSuccess) return err;       \
  fft_cols_kernel<ODT_CLS, I, S><<<blocks, f.nthr, sm, s>>>(in, out, n0, is, os, sc, f.plan,  \
                                                            f.tw, f.lgW);
  if (inv) {
    if (shift) { ODT_COLS(true, true) } else { ODT_COLS(true, false) }
  } else {
    if (shift) { ODT_COLS(false, true) } else { ODT_COLS(false, false) }
  }
#undef ODT_COLS
  return cudaGetLastError();
}
#endif

}  // namespace odt
