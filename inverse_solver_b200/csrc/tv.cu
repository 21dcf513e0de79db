// Isotropic-TV proximal operator by dual FISTA (TV_FISTA_inner_v2.m:1-53),
// two fused stencil kernels per inner iteration:
//   tv_z : z = project(in - lambda * TV_L(R))                       (:38, :99-113)
//   tv_p : P' = project_TV(R + c * TV_L^T(z)) ; R' = P' + beta (P' - P)  (:38-47)
// and a final tv_out : out = project(in - lambda * TV_L(P)) (:51).  The FISTA
// scalars t_n, c = 1/(12 lambda), beta = (t_n - 1)/t_{n+1} are computed in
// double on the host.  Arrays are float (or complex64 when the imaginary
// part is bounded, Vimag_max > 0), periodic in all three axes, column-major.
// Bytes per voxel and inner iteration (real): tv_z reads in + R1..R3 (16 B,
// neighbours from L1/L2) and writes z (4 B); tv_p reads z, R1..R3, P1..P3 and
// writes P1..P3, R1..R3 (52 B).
#include <cmath>
#include <string>
#include <vector>

#include "../../include/odt.h"

namespace odt {
const char* set_last_error(const std::string& msg);
}

namespace {

constexpr int kThreads = 256;

struct Geo {
  int nx, ny, nz;
  long long n;
};

__device__ __forceinline__ long long at(const Geo& g, int x, int y, int z) {
  return x + (long long)g.nx * (y + (long long)g.ny * z);
}

// value traits: float (real path) or float2 (complex path)
__device__ __forceinline__ float sub(float a, float b) { return a - b; }
__device__ __forceinline__ float2 sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float add(float a, float b) { return a + b; }
__device__ __forceinline__ float2 add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float scl(float s, float a) { return s * a; }
__device__ __forceinline__ float2 scl(float s, float2 a) { return make_float2(s * a.x, s * a.y); }
__device__ __forceinline__ float abs2(float a) { return a * a; }
__device__ __forceinline__ float abs2(float2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ float divs(float a, float d) { return a / d; }
__device__ __forceinline__ float2 divs(float2 a, float d) { return make_float2(a.x / d, a.y / d); }

struct Proj {
  double vmin, vmax, vimag_max;
  int non_neg, dirichlet;
};

// project_non_neg (:57-75); comparisons against the double bounds are exact
__device__ __forceinline__ float project(float v, const Proj& p) {
  if (p.non_neg) {
    if ((double)v < p.vmin) v = (float)p.vmin;
    if ((double)v > p.vmax) v = (float)p.vmax;
  }
  return v;
}
__device__ __forceinline__ float2 project(float2 v, const Proj& p) {
  if (p.non_neg) {
    if ((double)v.x < p.vmin) v.x = (float)p.vmin;
    if ((double)v.x > p.vmax) v.x = (float)p.vmax;
  }
  if (v.y < 0.f) v.y = 0.f;
  if (p.vimag_max > 0 && (double)v.y > p.vimag_max) v.y = (float)p.vimag_max;
  return v;
}

template <typename T>
__device__ __forceinline__ T zero() { return T(); }
template <>
__device__ __forceinline__ float2 zero<float2>() { return make_float2(0.f, 0.f); }

__device__ __forceinline__ bool on_face(const Geo& g, int x, int y, int z) {
  return x == 0 || y == 0 || z == 0 || x == g.nx - 1 || y == g.ny - 1 || z == g.nz - 1;
}

// in - lambda * TV_L(R) at (x, y, z), then project
template <typename T>
__device__ __forceinline__ T z_at(const Geo& g, const T* in, const T* R1, const T* R2, const T* R3,
                                  float lam, const Proj& p, int x, int y, int z) {
  const long long i = at(g, x, y, z);
  const int xm = x == 0 ? g.nx - 1 : x - 1;
  const int ym = y == 0 ? g.ny - 1 : y - 1;
  const int zm = z == 0 ? g.nz - 1 : z - 1;
  T L = add(R1[i], R2[i]);
  L = add(L, R3[i]);
  L = sub(L, R1[at(g, xm, y, z)]);
  L = sub(L, R2[at(g, x, ym, z)]);
  L = sub(L, R3[at(g, x, y, zm)]);
  T v = project(sub(in[i], scl(lam, L)), p);
  if (p.dirichlet && on_face(g, x, y, z)) v = zero<T>();
  return v;
}

template <typename T>
__global__ void tv_z_kernel(Geo g, const T* in, const T* R1, const T* R2, const T* R3, T* zout,
                            float lam, Proj p) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < g.n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % g.nx);
    const long long t = i / g.nx;
    const int y = (int)(t % g.ny);
    const int z = (int)(t / g.ny);
    zout[i] = z_at(g, in, R1, R2, R3, lam, p, x, y, z);
  }
}

template <typename T>
__global__ void tv_p_kernel(Geo g, const T* zin, T* R1, T* R2, T* R3, T* P1, T* P2, T* P3,
                            float c, float beta) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < g.n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % g.nx);
    const long long t = i / g.nx;
    const int y = (int)(t % g.ny);
    const int z = (int)(t / g.ny);
    const T zc = zin[i];
    const T q1 = sub(zc, zin[at(g, x == g.nx - 1 ? 0 : x + 1, y, z)]);  // TV_L_trans
    const T q2 = sub(zc, zin[at(g, x, y == g.ny - 1 ? 0 : y + 1, z)]);
    const T q3 = sub(zc, zin[at(g, x, y, z == g.nz - 1 ? 0 : z + 1)]);
    T n1 = add(R1[i], scl(c, q1));
    T n2 = add(R2[i], scl(c, q2));
    T n3 = add(R3[i], scl(c, q3));
    const float A = sqrtf(fmaxf((abs2(n1) + abs2(n2)) + abs2(n3), 1.f));  // project_TV
    n1 = divs(n1, A);
    n2 = divs(n2, A);
    n3 = divs(n3, A);
    R1[i] = add(n1, scl(beta, sub(n1, P1[i])));
    R2[i] = add(n2, scl(beta, sub(n2, P2[i])));
    R3[i] = add(n3, scl(beta, sub(n3, P3[i])));
    P1[i] = n1;
    P2[i] = n2;
    P3[i] = n3;
  }
}

template <typename T>
__global__ void tv_out_kernel(Geo g, const T* in, const T* P1, const T* P2, const T* P3, T* out,
                              float lam, Proj p) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < g.n;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % g.nx);
    const long long t = i / g.nx;
    const int y = (int)(t % g.ny);
    const int z = (int)(t / g.ny);
    out[i] = z_at(g, in, P1, P2, P3, lam, p, x, y, z);
  }
}

int grid_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  if (b > 148LL * 32) b = 148LL * 32;
  return (int)(b < 1 ? 1 : b);
}

odt_status fail(odt_status st, const std::string& m) {
  odt::set_last_error(m);
  return st;
}

template <typename T>
cudaError_t run_tv(const odt_tv_args& a, const T* in_d, T* out_d, cudaStream_t s) {
  Geo g{a.size[0], a.size[1], a.size[2], 0};
  g.n = (long long)g.nx * g.ny * g.nz;
  const size_t bytes = sizeof(T) * (size_t)g.n;
  T* buf = nullptr;
  cudaError_t e = cudaMallocAsync((void**)&buf, 7 * bytes, s);
  if (e != cudaSuccess) return e;
  T* z = buf;
  T* R[3] = {buf + g.n, buf + 2 * g.n, buf + 3 * g.n};
  T* P[3] = {buf + 4 * g.n, buf + 5 * g.n, buf + 6 * g.n};
  e = cudaMemsetAsync(buf + g.n, 0, 6 * bytes, s);  // R = P = 0 (:23-28)
  const Proj p{a.vmin, a.vmax, a.vimag_max, a.non_neg, a.dirichlet};
  const float lam = (float)a.lambda;
  const int dividend = (a.size[2] > 1) ? 12 : 8;
  const float c = (float)(1.0 / (dividend * a.lambda));
  double t_np = 1.0;
  const int grid = grid_for(g.n);
  for (int mm = 0; mm < a.inner_itt && e == cudaSuccess; ++mm) {
    const double t_n = t_np;
    t_np = (1.0 + std::sqrt(1.0 + 4.0 * t_n * t_n)) / 2.0;
    const float beta = (float)((t_n - 1.0) / t_np);
    tv_z_kernel<T><<<grid, kThreads, 0, s>>>(g, in_d, R[0], R[1], R[2], z, lam, p);
    tv_p_kernel<T><<<grid, kThreads, 0, s>>>(g, z, R[0], R[1], R[2], P[0], P[1], P[2], c, beta);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    tv_out_kernel<T><<<grid, kThreads, 0, s>>>(g, in_d, P[0], P[1], P[2], out_d, lam, p);
    e = cudaGetLastError();
  }
  cudaError_t e2 = cudaFreeAsync(buf, s);
  return e != cudaSuccess ? e : e2;
}

}  // namespace

extern "C" odt_status odt_tv_prox(const odt_tv_args* a) {
  if (!a || !a->in || !a->out) return fail(ODT_ERR_INVALID_ARGUMENT, "odt_tv_prox: NULL argument");
  if (a->size[0] < 1 || a->size[1] < 1 || a->size[2] < 1 || a->inner_itt < 0 || !(a->lambda > 0))
    return fail(ODT_ERR_INVALID_ARGUMENT, "odt_tv_prox: bad size, inner_itt or lambda");
  if (a->memory != ODT_MEM_HOST && a->memory != ODT_MEM_DEVICE)
    return fail(ODT_ERR_INVALID_ARGUMENT, "odt_tv_prox: bad memory flag");
  if (!a->is_complex && a->vimag_max > 0)
    return fail(ODT_ERR_INVALID_ARGUMENT,
                "odt_tv_prox: Vimag_max > 0 needs the complex path (is_complex = 1)");
  const size_t n = (size_t)a->size[0] * a->size[1] * a->size[2];
  const size_t esz = a->is_complex ? sizeof(float2) : sizeof(float);
  cudaStream_t s = a->memory == ODT_MEM_DEVICE ? (cudaStream_t)a->stream : (cudaStream_t)0;
  cudaError_t e = cudaSuccess;
  void* din = const_cast<void*>(a->in);
  void* dout = a->out;
  void* tmp = nullptr;
  if (a->memory == ODT_MEM_HOST) {
    e = cudaMallocAsync(&tmp, 2 * n * esz, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(tmp, a->in, n * esz, cudaMemcpyHostToDevice, s);
    din = tmp;
    dout = static_cast<char*>(tmp) + n * esz;
  }
  if (e == cudaSuccess)
    e = a->is_complex ? run_tv<float2>(*a, (const float2*)din, (float2*)dout, s)
                      : run_tv<float>(*a, (const float*)din, (float*)dout, s);
  if (a->memory == ODT_MEM_HOST) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(a->out, dout, n * esz, cudaMemcpyDeviceToHost, s);
    if (tmp) cudaFreeAsync(tmp, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? ODT_ERR_OUT_OF_MEMORY : ODT_ERR_CUDA,
                std::string("odt_tv_prox: ") + cudaGetErrorString(e));
  }
  odt::set_last_error("");
  return ODT_OK;
}
