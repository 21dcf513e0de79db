// Bluestein (chirp-z) transforms for lengths with a prime factor > 31; the
// algorithm and layout are described in fft_any.cuh.
#include "fft_any.cuh"

#include <cmath>
#include <vector>

namespace odt {
namespace {

constexpr int kThreads = 256;

int grid_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  if (b > 148LL * 16) b = 148LL * 16;
  return (int)(b < 1 ? 1 : b);
}


__global__ void bs_scale(float2* __restrict__ x, long long n, float s) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    x[i] = make_float2(x[i].x * s, x[i].y * s);
}

bool five_smooth(int m) {
  for (int p : {2, 3, 5})
    while (m % p == 0) m /= p;
  return m == 1;
}

// centred transform of one axis: the cyclic shift by n / 2 on both sides,
// 1 / n on the inverse
cudaError_t bluestein(float2* x, int n0, int n, long long n2, bool inv, const AnyFft& f, cudaStream_t s) {
  return bluestein_axis(x, n0, n2, inv, n / 2, inv ? 1.0f / (float)n : 1.0f, f, s);
}

}  // namespace

int bluestein_length(int n) {
  int m = 2 * n - 1;
  while (!five_smooth(m)) ++m;
  return m;
}

cudaError_t bluestein_tables(int n, int m, const DevFft& inner, float2* dw, float2* db, cudaStream_t s) {
  std::vector<float2> w(n), b(2 * (size_t)m, make_float2(0.f, 0.f));
  const double pi = 3.14159265358979323846;
  for (int j = 0; j < n; ++j) {
    const long long r = ((long long)j * j) % (2LL * n);   // j^2 mod 2n keeps the angle exact
    const double ang = pi * (double)r / (double)n;
    w[j] = make_float2((float)std::cos(ang), (float)-std::sin(ang));
    const float2 cw = make_float2(w[j].x, -w[j].y);
    b[j] = cw;                 // forward: conj(w), wrapped
    b[m + j] = w[j];           // inverse: w, wrapped
    if (j > 0) {
      b[m - j] = cw;
      b[2 * (size_t)m - j] = w[j];
    }
  }
  cudaError_t e;
  if ((e = cudaMemcpyAsync(dw, w.data(), n * sizeof(float2), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(db, b.data(), 2 * (size_t)m * sizeof(float2), cudaMemcpyHostToDevice, s)) !=
          cudaSuccess ||
      (e = launch_fft_lines(db, db, 2, 0, 0, 1.f, false, inner, s)) != cudaSuccess)
    return e;
  bs_scale<<<grid_for(2LL * m), kThreads, 0, s>>>(db, 2LL * m, 1.0f / (float)m);
  // (copies from pageable host memory have read their source when they return)
  return cudaGetLastError();
}

bool scratch_fft_any(Scratch& B, int n, AnyFft* f, std::string* why) {
  f->n = n;
  FftPlan probe{};
  std::string w2;
  if (make_plan(n, &probe, &w2, kLargeFirst)) {
    f->direct = true;
    return scratch_fft(B, n, &f->f, why);
  }
  f->direct = false;
  const int m = bluestein_length(n);
  f->m = m;
  if (!scratch_fft(B, m, &f->f, why)) return false;
  float2* dw = B.get<float2>(n);
  float2* db = B.get<float2>(2 * (size_t)m);
  if (!dw || !db) {
    *why = "device allocation failed";
    return false;
  }
  const cudaError_t e = bluestein_tables(n, m, f->f, dw, db, B.s);
  if (e != cudaSuccess) {
    *why = std::string("Bluestein tables: ") + cudaGetErrorString(e);
    return false;
  }
  f->chirp = dw;
  f->bhat_f = db;
  f->bhat_i = db + m;
  return true;
}

cudaError_t fftc2_any(float2* x, int N1, int N2, long long nsl, bool inv, const AnyFft& f1,
                      const AnyFft& f2, cudaStream_t s) {
  if (f1.direct && f2.direct) return fftc2(x, N1, N2, nsl, inv, f1.f, f2.f, s);
  cudaError_t e;
  if (f1.direct)
    e = launch_fft_lines(x, x, (long long)N2 * nsl, N1 / 2, N1 / 2, inv ? 1.0f / (float)N1 : 1.f, inv, f1.f, s);
  else
    e = bluestein(x, 1, N1, (long long)N2 * nsl, inv, f1, s);
  if (e != cudaSuccess) return e;
  if (f2.direct)
    return launch_fft_cols(x, x, N1, nsl, N2 / 2, N2 / 2, inv ? 1.0f / (float)N2 : 1.f, inv, f2.f, s);
  return bluestein(x, N1, N2, nsl, inv, f2, s);
}

}  // namespace odt
