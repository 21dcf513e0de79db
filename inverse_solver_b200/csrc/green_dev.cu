// The plane part of truncated_green_plus (sub_code/truncated_green_plus.m
// :67-110) on the GPU.  For every z the band-limited radial profile [n_r, nz]
// of the xy-truncated Green's function (or refocusing kernel) is
// interpolated onto the oversized grid [S1, S2] (bin_search_nearest's maps,
// computed by the host); the reference then applies a centred inverse 2D
// FFT of size S1 x S2, crops to the output size o0 x o1 and applies a centred
// forward 2D FFT, and afterwards the same along z (inverse of size nz, crop
// to o2, forward).  Each of these chains is one fixed linear map: with
// C_n the centred DFT matrix of size n (fftshift(fft(ifftshift(.)))),
//   M1 = C_o0 * rows(r0 .. r0+o0-1 of C_S1^-1)      [o0 x S1]
//   M2 = C_o1 * rows(r1 .. r1+o1-1 of C_S2^-1)      [o1 x S2]
//   Mz = C_o2 * rows(z0 .. z0+o2-1 of C_nz^-1)      [o2 x nz]
// (built by the host in double), the output is
//   out(:, :, k) = sum_z Mz(k, z) * M1 * G_z * M2^T,
// three single-precision complex GEMMs (two batched over z).  Unlike the
// FFT route this takes the oversized grid's lengths as they come out of the
// reference's formula (ceil(1.556 n + 10), often prime).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <string>

#include "../../include/odt.h"
#include "cbs_kernels.cuh"
#include "scratch.cuh"

namespace odt {
const char* set_last_error(const std::string& msg);  // odt_api.cu
// tcgen05 (TF32 split) complex GEMM, tc_gemm.cu
cudaError_t tc_cgemm(int M, int N, int K, const float2* A, int lda, long long sA, const float2* B, int ldb,
                     long long sB, bool transB, float2* C, int ldc, long long sC, int batch, float* work,
                     long long work_floats, int* fault, cudaStream_t s);
long long tc_cgemm_work(int M, int N, int K, bool batchedA, bool batchedB, int batch);
}

using namespace odt;

namespace {

constexpr int kThreads = 256;

int grid_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  if (b > 148LL * 16) b = 148LL * 16;
  return (int)(b < 1 ? 1 : b);
}

// out[p + S z] = (g[near1[p]-1, z] w[p] + g[near2[p]-1, z] (1 - w[p])) * scale
__global__ void radial_interp_kernel(const float2* __restrict__ g, int n_r, const int* __restrict__ near1,
                                     const int* __restrict__ near2, const float* __restrict__ w, long long S,
                                     int nz, float scale, float2* __restrict__ out) {
  const long long total = S * nz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long z = i / S, p = i - z * S;
    const float b = w[p];
    const float2 a1 = g[(near1[p] - 1) + (long long)n_r * z];
    const float2 a2 = g[(near2[p] - 1) + (long long)n_r * z];
    const float c = 1.f - b;
    out[i] = make_float2((a1.x * b + a2.x * c) * scale, (a1.y * b + a2.y * c) * scale);
  }
}

// Batched complex GEMM, column-major: C_b[M x N] = A_b[M x K] * op(B_b)
// with op(B) = B [K x N] (ldb) or, transB, B^T with B stored [N x K] (ldb).
// 64 x 64 C tile per CTA, K in slices of 16 through shared memory, each of
// the 256 threads accumulating a 4 x 4 block in single precision.
constexpr int kTM = 64, kTN = 64, kTK = 16;

__global__ void __launch_bounds__(256) cgemm_kernel(int M, int N, int K, const float2* __restrict__ A, int lda,
                                                    long long sA, const float2* __restrict__ B, int ldb,
                                                    long long sB, int transB, float2* __restrict__ C, int ldc,
                                                    long long sC) {
  __shared__ float2 As[kTK][kTM + 1];
  __shared__ float2 Bs[kTK][kTN + 1];
  const int bz = blockIdx.z;
  A += sA * bz;
  B += sB * bz;
  C += sC * bz;
  const int m0 = blockIdx.x * kTM, n0 = blockIdx.y * kTN;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;   // 16 x 16 threads, 4 x 4 outputs each
  float2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_float2(0.f, 0.f);
  for (int k0 = 0; k0 < K; k0 += kTK) {
    for (int e = threadIdx.x; e < kTK * kTM; e += 256) {   // A tile: rows m0.., columns k0..
      const int m = e % kTM, k = e / kTM;
      const int gm = m0 + m, gk = k0 + k;
      As[k][m] = (gm < M && gk < K) ? A[gm + (long long)lda * gk] : make_float2(0.f, 0.f);
    }
    for (int e = threadIdx.x; e < kTK * kTN; e += 256) {   // B tile: (k, n)
      int k, n;
      if (transB) {
        n = e % kTN;
        k = e / kTN;
      } else {
        k = e % kTK;
        n = e / kTK;
      }
      const int gk = k0 + k, gn = n0 + n;
      float2 v = make_float2(0.f, 0.f);
      if (gk < K && gn < N) v = transB ? B[gn + (long long)ldb * gk] : B[gk + (long long)ldb * gn];
      Bs[k][n] = v;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kTK; ++k) {
      float2 a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[k][tx + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[k][ty + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          acc[i][j].x += a[i].x * b[j].x - a[i].y * b[j].y;
          acc[i][j].y += a[i].x * b[j].y + a[i].y * b[j].x;
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gm = m0 + tx + 16 * i, gn = n0 + ty + 16 * j;
      if (gm < M && gn < N) C[gm + (long long)ldc * gn] = acc[i][j];
    }
}

cudaError_t cgemm(int M, int N, int K, const float2* A, int lda, long long sA, const float2* B, int ldb,
                  long long sB, bool transB, float2* C, int ldc, long long sC, int batch, cudaStream_t s) {
  const dim3 grid((M + kTM - 1) / kTM, (N + kTN - 1) / kTN, batch);
  cgemm_kernel<<<grid, 256, 0, s>>>(M, N, K, A, lda, sA, B, ldb, sB, transB ? 1 : 0, C, ldc, sC);
  return cudaGetLastError();
}

odt_status gfail(odt_status st, const std::string& m) {
  set_last_error(m);
  return st;
}

#define G_CHECK(call)                                                                      \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) {                                                               \
      cudaGetLastError();                                                                  \
      return gfail(ODT_ERR_CUDA, std::string("odt_green_planes: ") + cudaGetErrorString(e_)); \
    }                                                                                      \
  } while (0)

// ------------------------------------------------------------------ Hankel
// The cropped order-0 Hankel transform pair (discrete_hankel_croped_fourier.m
// :19-47, as truncated_green_plus.m:33-66 uses it) with the single-precision
// rounding of the reference's besselj matrices and scalings: c (zeros of J_0)
// and C rounded to float, I = |J_1(c)|, s = sqrt(2/C) / I, K = (2 pi / C) I,
// F[i, j] = (s_i s_j) J_0((c_i / C) c_j).

__global__ void hankel_scalars_kernel(const double* __restrict__ roots, int n, float* __restrict__ c,
                                      float* __restrict__ I, float* __restrict__ sc, float* __restrict__ K) {
  const float C = (float)roots[n];
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const float cj = (float)roots[j];
    const float ij = fabsf((float)j1((double)cj));
    c[j] = cj;
    I[j] = ij;
    sc[j] = __fdiv_rn(__fsqrt_rn(__fdiv_rn(2.0f, C)), ij);
    K[j] = __fmul_rn(__fdiv_rn(6.28318548202514648f, C), ij);   // float(2 pi) / C * I
  }
}

// F [pos, n] column-major
__global__ void hankel_matrix_kernel(const float* __restrict__ c, const float* __restrict__ sc, float C, int pos,
                                     long long n, float* __restrict__ F) {
  const long long total = (long long)pos * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % pos);
    const long long j = e / pos;
    const float arg = __fmul_rn(__fdiv_rn(c[i], C), c[j]);
    F[e] = __fmul_rn(__fmul_rn(sc[i], sc[j]), (float)j0((double)arg));
  }
}

// A[j, z] = values[j, z] / I_j
__global__ void hankel_div_rows_kernel(const float2* __restrict__ v, const float* __restrict__ d, long long n,
                                       int nz, float2* __restrict__ out) {
  const long long total = n * nz;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const float q = d[e % n];
    out[e] = make_float2(__fdiv_rn(v[e].x, q), __fdiv_rn(v[e].y, q));
  }
}

// Partial products of out[m, nn] = sum_k f(m, k) * B[k, nn] over one k-chunk
// per blockIdx.z, double accumulation: f(m, k) = F[m + ldf k] (F [M, K]) or,
// transF, F[k + ldf m] (F [K, M]); B complex [K, N] (ldb).  Tiles of 32 x 32
// outputs, 256 threads with 2 x 2 outputs each, k in slices of 32.
__global__ void __launch_bounds__(256) rc_gemm_part_kernel(int M, int N, int K, int kchunk,
                                                           const float* __restrict__ F, int ldf, int transF,
                                                           const float2* __restrict__ B, int ldb,
                                                           double2* __restrict__ part) {
  __shared__ float Fs[32][33];     // [k][m]
  __shared__ float2 Bs[32][33];    // [k][n]
  const int m0 = blockIdx.x * 32, n0 = blockIdx.y * 32;
  const int k_lo = blockIdx.z * kchunk, k_hi = min(K, k_lo + kchunk);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double2 acc[2][2];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) acc[a][b] = make_double2(0.0, 0.0);
  for (int k0 = k_lo; k0 < k_hi; k0 += 32) {
    for (int e = threadIdx.x; e < 32 * 32; e += 256) {
      const int r = e & 31, q = e >> 5;   // F: (m = r, k = q) or (k = r, m = q) so loads run along memory
      int m, k;
      if (transF) { k = r; m = q; } else { m = r; k = q; }
      const int gm = m0 + m, gk = k0 + k;
      float v = 0.f;
      if (gm < M && gk < k_hi) v = transF ? F[gk + (long long)ldf * gm] : F[gm + (long long)ldf * gk];
      Fs[k][m] = v;
      const int bk = r, bn = q;           // B: (k = r, n = q)
      const int gbk = k0 + bk, gbn = n0 + bn;
      Bs[bk][bn] = (gbk < k_hi && gbn < N) ? B[gbk + (long long)ldb * gbn] : make_float2(0.f, 0.f);
    }
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < 32; ++k) {
      const double f0 = Fs[k][tx], f1 = Fs[k][tx + 16];
      const float2 b0 = Bs[k][ty], b1 = Bs[k][ty + 16];
      acc[0][0].x += f0 * b0.x; acc[0][0].y += f0 * b0.y;
      acc[0][1].x += f0 * b1.x; acc[0][1].y += f0 * b1.y;
      acc[1][0].x += f1 * b0.x; acc[1][0].y += f1 * b0.y;
      acc[1][1].x += f1 * b1.x; acc[1][1].y += f1 * b1.y;
    }
    __syncthreads();
  }
  double2* P = part + (long long)blockIdx.z * M * N;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const int gm = m0 + tx + 16 * a, gn = n0 + ty + 16 * b;
      if (gm < M && gn < N) P[gm + (long long)M * gn] = acc[a][b];
    }
}

// out[m, n] = round(sum over the chunks, in order) -- then times post[m] if given
__global__ void rc_gemm_reduce_kernel(const double2* __restrict__ part, int nchunk, long long MN, int M,
                                      const float* __restrict__ post, float2* __restrict__ out) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < MN;
       e += (long long)gridDim.x * blockDim.x) {
    double x = 0.0, y = 0.0;
    for (int c = 0; c < nchunk; ++c) {
      x += part[c * MN + e].x;
      y += part[c * MN + e].y;
    }
    float2 r = make_float2((float)x, (float)y);
    if (post) {
      const float q = post[e % M];
      r = make_float2(__fmul_rn(r.x, q), __fmul_rn(r.y, q));
    }
    out[e] = r;
  }
}

// V2[i, z] = ((T[i, z] * K_i) * band_i) / K_i, as forward(), the band window
// and backward() round it
__global__ void hankel_band_kernel(const float2* __restrict__ T, const float* __restrict__ K,
                                   const float* __restrict__ band, int pos, int nz, float2* __restrict__ out) {
  const long long total = (long long)pos * nz;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % pos);
    const float k = K[i], b = band[i];
    float2 v = make_float2(__fmul_rn(T[e].x, k), __fmul_rn(T[e].y, k));
    v = make_float2(__fmul_rn(v.x, b), __fmul_rn(v.y, b));
    out[e] = make_float2(__fdiv_rn(v.x, k), __fdiv_rn(v.y, k));
  }
}

}  // namespace

extern "C" odt_status odt_hankel_filter(const odt_hankel_args* a) {
  if (!a || !a->roots || !a->values || !a->band || !a->out)
    return gfail(ODT_ERR_INVALID_ARGUMENT, "odt_hankel_filter: NULL argument");
  const int n = a->n, pos = a->pos, nz = a->nz;
  if (n < 1 || pos < 1 || pos > n || nz < 1 || nz > 65535 || (long long)pos * n > (1LL << 31))
    return gfail(ODT_ERR_INVALID_ARGUMENT, "odt_hankel_filter: bad sizes");
  if (a->device >= 0) G_CHECK(cudaSetDevice(a->device));
  cudaStream_t s = nullptr;
  G_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  odt_status st = ODT_OK;
  {
    Scratch B;
    B.s = s;
    const int kchunk = 1024;
    const int nsplit = (n + kchunk - 1) / kchunk;
    const long long pn = (long long)pos * nz, nn = (long long)n * nz;
    double* roots = B.get<double>((size_t)n + 1);
    float* c = B.get<float>(n);
    float* I = B.get<float>(n);
    float* sc = B.get<float>(n);
    float* K = B.get<float>(n);
    float* band = B.get<float>(pos);
    float* F = B.get<float>((size_t)pos * n);
    float2* V = B.get<float2>(nn);
    float2* A = B.get<float2>(nn);
    float2* T = B.get<float2>(pn);
    float2* V2 = B.get<float2>(pn);
    double2* part = B.get<double2>((size_t)(nsplit > 1 ? nsplit : 1) * (size_t)(nn > pn ? nn : pn));
    if (!roots || !c || !I || !sc || !K || !band || !F || !V || !A || !T || !V2 || !part) {
      st = gfail(ODT_ERR_OUT_OF_MEMORY, "odt_hankel_filter: device allocation failed");
    } else {
      auto run = [&]() -> cudaError_t {
        const cudaMemcpyKind h2d = cudaMemcpyHostToDevice;
        cudaError_t e;
        if ((e = cudaMemcpyAsync(roots, a->roots, ((size_t)n + 1) * sizeof(double), h2d, s)) ||
            (e = cudaMemcpyAsync(band, a->band, (size_t)pos * sizeof(float), h2d, s)) ||
            (e = cudaMemcpyAsync(V, a->values, (size_t)nn * sizeof(float2), h2d, s)))
          return e;
        const float C = (float)a->roots[n];
        hankel_scalars_kernel<<<grid_for(n), kThreads, 0, s>>>(roots, n, c, I, sc, K);
        hankel_matrix_kernel<<<grid_for((long long)pos * n), kThreads, 0, s>>>(c, sc, C, pos, n, F);
        hankel_div_rows_kernel<<<grid_for(nn), kThreads, 0, s>>>(V, I, n, nz, A);
        if ((e = cudaGetLastError())) return e;
        // T = F A   [pos, nz], k = n split into chunks
        rc_gemm_part_kernel<<<dim3((pos + 31) / 32, (nz + 31) / 32, nsplit), 256, 0, s>>>(
            pos, nz, n, kchunk, F, pos, 0, A, n, part);
        rc_gemm_reduce_kernel<<<grid_for(pn), kThreads, 0, s>>>(part, nsplit, pn, pos, nullptr, T);
        hankel_band_kernel<<<grid_for(pn), kThreads, 0, s>>>(T, K, band, pos, nz, V2);
        // out = (F^T V2) .* I   [n, nz], k = pos in one chunk
        rc_gemm_part_kernel<<<dim3((n + 31) / 32, (nz + 31) / 32, 1), 256, 0, s>>>(
            n, nz, pos, pos, F, pos, 1, V2, pos, part);
        rc_gemm_reduce_kernel<<<grid_for(nn), kThreads, 0, s>>>(part, 1, nn, n, I, A);
        if ((e = cudaGetLastError())) return e;
        if ((e = cudaMemcpyAsync(a->out, A, (size_t)nn * sizeof(float2), cudaMemcpyDeviceToHost, s))) return e;
        return cudaStreamSynchronize(s);
      };
      const cudaError_t e = run();
      if (e != cudaSuccess) {
        cudaGetLastError();
        st = gfail(ODT_ERR_CUDA, std::string("odt_hankel_filter: ") + cudaGetErrorString(e));
      }
    }
  }
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  return st;
}

extern "C" odt_status odt_green_planes(const odt_green_args* a) {
  if (!a || !a->radial || !a->near1 || !a->near2 || !a->w || !a->m1 || !a->m2 || !a->mz || !a->out)
    return gfail(ODT_ERR_INVALID_ARGUMENT, "odt_green_planes: NULL argument");
  const int S1 = a->creation[0], S2 = a->creation[1], nz = a->creation[2], nr = a->n_r;
  const int o0 = a->out_size[0], o1 = a->out_size[1], o2 = a->out_size[2];
  if (S1 < 1 || S2 < 1 || nz < 1 || nr < 1 || o0 < 1 || o1 < 1 || o2 < 1 || o0 > S1 || o1 > S2 || o2 > nz ||
      (long long)nz > 65535)
    return gfail(ODT_ERR_INVALID_ARGUMENT, "odt_green_planes: bad sizes");
  if (a->device >= 0) G_CHECK(cudaSetDevice(a->device));
  cudaStream_t s = nullptr;
  G_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  odt_status st = ODT_OK;
  {
    Scratch B;
    B.s = s;
    const long long S = (long long)S1 * S2, o01 = (long long)o0 * o1;
    float2* g = B.get<float2>((size_t)nr * nz);
    int* n1 = B.get<int>(S);
    int* n2 = B.get<int>(S);
    float* w = B.get<float>(S);
    float2* m1 = B.get<float2>((size_t)o0 * S1);
    float2* m2 = B.get<float2>((size_t)o1 * S2);
    float2* mz = B.get<float2>((size_t)o2 * nz);
    float2* G = B.get<float2>(S * nz);
    float2* T = B.get<float2>((size_t)o0 * S2 * nz);
    float2* Z = B.get<float2>(o01 * nz);
    float2* D = B.get<float2>(o01 * o2);
    int* fault = B.get<int>(1);
    if (!g || !n1 || !n2 || !w || !m1 || !m2 || !mz || !G || !T || !Z || !D || !fault) {
      st = gfail(ODT_ERR_OUT_OF_MEMORY, "odt_green_planes: device allocation failed");
    } else {
      auto run = [&]() -> cudaError_t {
        const cudaMemcpyKind h2d = cudaMemcpyHostToDevice;
        cudaError_t e;
        if ((e = cudaMemcpyAsync(g, a->radial, (size_t)nr * nz * sizeof(float2), h2d, s)) ||
            (e = cudaMemcpyAsync(n1, a->near1, S * sizeof(int), h2d, s)) ||
            (e = cudaMemcpyAsync(n2, a->near2, S * sizeof(int), h2d, s)) ||
            (e = cudaMemcpyAsync(w, a->w, S * sizeof(float), h2d, s)) ||
            (e = cudaMemcpyAsync(m1, a->m1, (size_t)o0 * S1 * sizeof(float2), h2d, s)) ||
            (e = cudaMemcpyAsync(m2, a->m2, (size_t)o1 * S2 * sizeof(float2), h2d, s)) ||
            (e = cudaMemcpyAsync(mz, a->mz, (size_t)o2 * nz * sizeof(float2), h2d, s)))
          return e;
        radial_interp_kernel<<<grid_for(S * nz), kThreads, 0, s>>>(g, nr, n1, n2, w, S, nz, a->scale, G);
        if ((e = cudaGetLastError())) return e;
        // T_z = M1 G_z ; Z_z = T_z M2^T ; D = Z Mz^T (Z viewed as [o0 o1, nz]):
        // on the tensor cores (TF32 split, FP32 accuracy) unless
        // ODT_GREEN_GEMM=simt selects the FP32 SIMT kernel
        const char* gm = std::getenv("ODT_GREEN_GEMM");
        const bool simt = gm && std::string(gm) == "simt";
        if ((e = cudaMemsetAsync(fault, 0, sizeof(int), s))) return e;
        // one operand workspace for the three tensor-core GEMMs
        float* work = nullptr;
        long long work_n = 0;
        if (!simt) {
          work_n = std::max(std::max(tc_cgemm_work(o0, S2, S1, false, true, nz),
                                     tc_cgemm_work(o0, o1, S2, true, false, nz)),
                            tc_cgemm_work((int)o01, o2, nz, false, false, 1));
          work = B.get<float>((size_t)work_n);
          if (!work) return cudaErrorMemoryAllocation;
        }
        auto gemm = [&](int M, int N, int K, const float2* A, int lda, long long sA, const float2* Bm, int ldb,
                        long long sB, bool tB, float2* C, int ldc, long long sC, int nb) {
          return simt ? cgemm(M, N, K, A, lda, sA, Bm, ldb, sB, tB, C, ldc, sC, nb, s)
                      : tc_cgemm(M, N, K, A, lda, sA, Bm, ldb, sB, tB, C, ldc, sC, nb, work, work_n, fault, s);
        };
        if ((e = gemm(o0, S2, S1, m1, o0, 0, G, S1, S, false, T, o0, (long long)o0 * S2, nz)) ||
            (e = gemm(o0, o1, S2, T, o0, (long long)o0 * S2, m2, o1, 0, true, Z, o0, o01, nz)) ||
            (e = gemm((int)o01, o2, nz, Z, (int)o01, 0, mz, o2, 0, true, D, (int)o01, 0, 1)))
          return e;
        if ((e = cudaMemcpyAsync(a->out, D, o01 * o2 * sizeof(float2), cudaMemcpyDeviceToHost, s))) return e;
        int f = 0;
        if ((e = cudaMemcpyAsync(&f, fault, sizeof(int), cudaMemcpyDeviceToHost, s))) return e;
        if ((e = cudaStreamSynchronize(s))) return e;
        return f ? cudaErrorLaunchTimeout : cudaSuccess;
      };
      const cudaError_t e = run();
      if (e != cudaSuccess) {
        cudaGetLastError();
        st = gfail(ODT_ERR_CUDA, std::string("odt_green_planes: ") + cudaGetErrorString(e));
      }
    }
  }  // scratch released (stream ordered) before the stream goes
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  return st;
}
