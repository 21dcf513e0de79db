// Per-call device scratch of the stateless entry points (odt_rytov,
// odt_bpm_solve, the retrieval front-end): stream-ordered allocations that
// are released, in stream order, when the call returns; FFT plans of the
// generic tile kernels whose twiddle tables live in that scratch; and the
// centred 2D FFT built on them.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "cbs_kernels.cuh"
#include "fft_plan.h"

namespace odt {

struct Scratch {
  std::vector<void*> ptrs;
  cudaStream_t s = nullptr;
  ~Scratch() {
    for (void* p : ptrs) cudaFreeAsync(p, s);
  }
  template <typename T>
  T* get(size_t n) {
    void* p = nullptr;
    if (cudaMallocAsync(&p, n * sizeof(T) + 16, s) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
};

// plan of length n for the line / column kernels (16 pencils per CTA up to
// length 512, 8 up to 1280, else 4 so that the tiles fit shared memory;
// 128 threads)
inline bool scratch_fft(Scratch& B, int n, DevFft* f, std::string* why) {
  if (!make_plan(n, &f->plan, why, kLargeFirst)) {
    if (why->empty()) *why = "length " + std::to_string(n) + " has a prime factor > 31";
    return false;
  }
  f->lgW = n <= 512 ? 4 : (n <= 1280 ? 3 : 2);
  f->W = 1 << f->lgW;
  f->nthr = 128;
  std::vector<float2> tw = make_twiddles(n);
  float2* d = B.get<float2>(n);
  if (!d || cudaMemcpyAsync(d, tw.data(), n * sizeof(float2), cudaMemcpyHostToDevice, B.s) != cudaSuccess) {
    *why = "twiddle upload failed";
    return false;
  }
  f->tw = d;
  return true;
}

// centred 2D FFT (fftshift(fft2(ifftshift(.))), or the inverse) of every
// [n1, n2] plane of x, in place
inline cudaError_t fftc2(float2* x, int n1, int n2, long long nsl, bool inv, const DevFft& f1, const DevFft& f2,
                         cudaStream_t s) {
  cudaError_t e = launch_fft_lines(x, x, (long long)n2 * nsl, n1 / 2, n1 / 2, 1.f, inv, f1, s);
  if (e != cudaSuccess) return e;
  return launch_fft_cols(x, x, n1, nsl, n2 / 2, n2 / 2, inv ? 1.0f / ((float)n1 * (float)n2) : 1.f, inv, f2, s);
}

}  // namespace odt
