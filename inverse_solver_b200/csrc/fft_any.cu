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

__device__ __forceinline__ float2 cmul_c(float2 a, float2 b, int conj_b) {
  const float by = conj_b ? -b.y : b.y;
  return make_float2(a.x * b.x - a.y * by, a.x * by + a.y * b.x);
}

// lines [n, nl] -> tmp [m, nl]: tmp[j, L] = x[(j + sh) mod n, L] w_j (j < n), else 0
__global__ void bs_gather_lines(const float2* __restrict__ x, int n, int m, long long nl, int sh,
                                const float2* __restrict__ w, int conj, float2* __restrict__ tmp) {
  const long long total = (long long)m * nl;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long L = i / m;
    const int j = (int)(i - L * m);
    float2 v = make_float2(0.f, 0.f);
    if (j < n) {
      int q = j + sh;
      if (q >= n) q -= n;
      v = cmul_c(x[q + (long long)n * L], w[j], conj);
    }
    tmp[i] = v;
  }
}

// x[(k + sh) mod n, L] = tmp[k, L] w_k scale
__global__ void bs_scatter_lines(const float2* __restrict__ tmp, int n, int m, long long nl, int sh,
                                 const float2* __restrict__ w, int conj, float scale, float2* __restrict__ x) {
  const long long total = (long long)n * nl;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long L = i / n;
    const int k = (int)(i - L * n);
    int q = k + sh;
    if (q >= n) q -= n;
    const float2 v = cmul_c(tmp[k + (long long)m * L], w[k], conj);
    x[q + (long long)n * L] = make_float2(v.x * scale, v.y * scale);
  }
}

// columns [n0, n, n2] -> tmp [n0, m, n2]
__global__ void bs_gather_cols(const float2* __restrict__ x, int n0, int n, int m, long long n2, int sh,
                               const float2* __restrict__ w, int conj, float2* __restrict__ tmp) {
  const long long total = (long long)n0 * m * n2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long t = i / n0;
    const int r = (int)(i - t * n0);
    const long long l = t / m;
    const int j = (int)(t - l * m);
    float2 v = make_float2(0.f, 0.f);
    if (j < n) {
      int q = j + sh;
      if (q >= n) q -= n;
      v = cmul_c(x[r + (long long)n0 * (q + (long long)n * l)], w[j], conj);
    }
    tmp[i] = v;
  }
}

__global__ void bs_scatter_cols(const float2* __restrict__ tmp, int n0, int n, int m, long long n2, int sh,
                                const float2* __restrict__ w, int conj, float scale, float2* __restrict__ x) {
  const long long total = (long long)n0 * n * n2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long t = i / n0;
    const int r = (int)(i - t * n0);
    const long long l = t / n;
    const int k = (int)(t - l * n);
    int q = k + sh;
    if (q >= n) q -= n;
    const float2 v = cmul_c(tmp[r + (long long)n0 * (k + (long long)m * l)], w[k], conj);
    x[r + (long long)n0 * (q + (long long)n * l)] = make_float2(v.x * scale, v.y * scale);
  }
}

// tmp[.., j, ..] *= bh[j], j the index along the transformed axis (stride `inner`)
__global__ void bs_mul(float2* __restrict__ tmp, long long total, long long inner, int m,
                       const float2* __restrict__ bh) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
    tmp[i] = cmul_c(tmp[i], bh[(i / inner) % m], 0);
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

cudaError_t bluestein(Scratch& B, float2* x, int n0, int n, long long n2, bool inv, const AnyFft& f,
                      cudaStream_t s) {
  float2* tmp = B.get<float2>((long long)n0 * f.m * n2);
  if (!tmp) return cudaErrorMemoryAllocation;
  return bluestein_axis(x, n0, n2, inv, n / 2, inv ? 1.0f / (float)n : 1.0f, f, tmp, s);
}

}  // namespace

int bluestein_length(int n) {
  int m = 2 * n - 1;
  while (!five_smooth(m)) ++m;
  return m;
}

cudaError_t bluestein_axis(float2* x, int n0, long long n2, bool inv, int sh, float scale, const AnyFft& f,
                           float2* tmp, cudaStream_t s) {
  const int n = f.n, m = f.m;
  const bool lines = n0 == 1;
  const long long total = (long long)n0 * m * n2;
  const int cj = inv ? 1 : 0;
  cudaError_t e;
  if (lines) bs_gather_lines<<<grid_for(total), kThreads, 0, s>>>(x, n, m, n2, sh, f.chirp, cj, tmp);
  else bs_gather_cols<<<grid_for(total), kThreads, 0, s>>>(x, n0, n, m, n2, sh, f.chirp, cj, tmp);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = lines ? launch_fft_lines(tmp, tmp, n2, 0, 0, 1.f, false, f.f, s)
                 : launch_fft_cols(tmp, tmp, n0, n2, 0, 0, 1.f, false, f.f, s)) != cudaSuccess)
    return e;
  bs_mul<<<grid_for(total), kThreads, 0, s>>>(tmp, total, n0, m, inv ? f.bhat_i : f.bhat_f);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = lines ? launch_fft_lines(tmp, tmp, n2, 0, 0, 1.f, true, f.f, s)
                 : launch_fft_cols(tmp, tmp, n0, n2, 0, 0, 1.f, true, f.f, s)) != cudaSuccess)
    return e;
  const long long nout = (long long)n0 * n * n2;
  if (lines) bs_scatter_lines<<<grid_for(nout), kThreads, 0, s>>>(tmp, n, m, n2, sh, f.chirp, cj, scale, x);
  else bs_scatter_cols<<<grid_for(nout), kThreads, 0, s>>>(tmp, n0, n, m, n2, sh, f.chirp, cj, scale, x);
  return cudaGetLastError();
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

cudaError_t fftc2_any(Scratch& B, float2* x, int N1, int N2, long long nsl, bool inv, const AnyFft& f1,
                      const AnyFft& f2, cudaStream_t s) {
  if (f1.direct && f2.direct) return fftc2(x, N1, N2, nsl, inv, f1.f, f2.f, s);
  cudaError_t e;
  if (f1.direct)
    e = launch_fft_lines(x, x, (long long)N2 * nsl, N1 / 2, N1 / 2, inv ? 1.0f / (float)N1 : 1.f, inv, f1.f, s);
  else
    e = bluestein(B, x, 1, N1, (long long)N2 * nsl, inv, f1, s);
  if (e != cudaSuccess) return e;
  if (f2.direct)
    return launch_fft_cols(x, x, N1, nsl, N2 / 2, N2 / 2, inv ? 1.0f / (float)N2 : 1.f, inv, f2.f, s);
  return bluestein(B, x, N1, N2, nsl, inv, f2, s);
}

}  // namespace odt
