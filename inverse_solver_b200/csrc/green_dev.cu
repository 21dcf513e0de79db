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

#include <string>

#include "../../include/odt.h"
#include "cbs_kernels.cuh"
#include "scratch.cuh"

namespace odt {
const char* set_last_error(const std::string& msg);  // odt_api.cu
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

}  // namespace

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
    if (!g || !n1 || !n2 || !w || !m1 || !m2 || !mz || !G || !T || !Z || !D) {
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
        // T_z = M1 G_z ; Z_z = T_z M2^T ; D = Z Mz^T (Z viewed as [o0 o1, nz])
        if ((e = cgemm(o0, S2, S1, m1, o0, 0, G, S1, S, false, T, o0, (long long)o0 * S2, nz, s)) ||
            (e = cgemm(o0, o1, S2, T, o0, (long long)o0 * S2, m2, o1, 0, true, Z, o0, o01, nz, s)) ||
            (e = cgemm((int)o01, o2, nz, Z, (int)o01, 0, mz, o2, 0, true, D, (int)o01, 0, 1, s)))
          return e;
        if ((e = cudaMemcpyAsync(a->out, D, o01 * o2 * sizeof(float2), cudaMemcpyDeviceToHost, s))) return e;
        return cudaStreamSynchronize(s);
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
