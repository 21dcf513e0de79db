// Per-call device scratch of the stateless entry points (odt_rytov,
// odt_bpm_solve): stream-ordered allocations that are released, in stream
// order, when the call returns; and FFT plans of the generic tile kernels
// whose twiddle tables live in that scratch.
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
// length 512, else 8; 128 threads)
inline bool scratch_fft(Scratch& B, int n, DevFft* f, std::string* why) {
  if (!make_plan(n, &f->plan, why, kLargeFirst)) {
    if (why->empty()) *why = "length " + std::to_string(n) + " has a prime factor > 31";
    return false;
  }
  f->lgW = n <= 512 ? 4 : 3;
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

}  // namespace odt
