// Centred 2D FFTs of any length for the stateless entry points.  A length
// whose prime factors are all <= 31 uses the radix tiles directly; any other
// length uses Bluestein's algorithm (the chirp-z transform): with
// w_j = exp(-1i pi j^2 / n),
//   X_k = w_k sum_j (x_j w_j) conj(w_(k-j)),
// a linear convolution evaluated with radix-tile FFTs of a 5-smooth length
// m >= 2n - 1 (conj(w) and its transform precomputed; the inverse DFT uses
// the conjugate chirps).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "scratch.cuh"

namespace odt {

struct AnyFft {
  int n = 0;
  bool direct = true;
  DevFft f{};                      // length n (direct) or m (Bluestein)
  int m = 0;
  const float2* chirp = nullptr;   // [n] exp(-1i pi j^2 / n)
  const float2* bhat_f = nullptr;  // [m] FFT_m(conj(w) wrapped) / m, forward DFT
  const float2* bhat_i = nullptr;  // [m] FFT_m(w wrapped) / m, inverse DFT
};

// Plan for length n on B's stream (tables in B's scratch).
bool scratch_fft_any(Scratch& B, int n, AnyFft* f, std::string* why);

// Smallest 5-smooth m >= 2 n - 1 (the convolution length of Bluestein's
// algorithm for length n).
int bluestein_length(int n);

// Fills the tables of a Bluestein plan of length n whose length-m transforms
// run through `inner`: chirp [n] and bhat [2 m] (forward, then inverse), on
// stream s.
cudaError_t bluestein_tables(int n, int m, const DevFft& inner, float2* chirp, float2* bhat, cudaStream_t s);

// DFT of length n = f.n (not direct) along the middle axis of x [n0, n, n2]
// in place, with index shift sh on input and output (0: plain transform;
// n / 2: centred) and the result multiplied by scale; one kernel, no work
// array (bs_fused.cu).
cudaError_t bluestein_axis(float2* x, int n0, long long n2, bool inv, int sh, float scale, const AnyFft& f,
                           cudaStream_t s);

// fftshift(fft2(ifftshift(x))) (or the normalised inverse) of every [N1, N2]
// plane of x [N1, N2, nsl], in place.  With both lengths direct this is
// fftc2; otherwise each axis is transformed on its own (the Bluestein axes
// by bluestein_axis, without work buffers).
cudaError_t fftc2_any(float2* x, int N1, int N2, long long nsl, bool inv, const AnyFft& f1,
                      const AnyFft& f2, cudaStream_t s);

}  // namespace odt
