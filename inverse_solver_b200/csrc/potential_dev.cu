// Device-resident pieces of BACKWARD_SOLVER_MULTI's outer loop:
//
//   * the scattering potential built on the GPU from an RI array already in
//     device memory (FORWARD_SOLVER_CONVERGENT_BORN.m:199-279: condition_RI's
//     eps_imag = 1.01 max|RI2potential(RI)|, create_boundary_RI's zero-potential
//     padding and the RI2potential / potential2RI round trips, init's
//     V - i eps_imag), for the forward solve or for the adjoint solve
//     (conj(flip(RI, 3)), BACKWARD_SOLVER_MULTI.m:48);
//   * the FISTA element-wise steps around the TV prox
//     (BACKWARD_SOLVER_MULTI.m:150-160): the prox input u - grad / alpha and
//     the momentum update u = s + c (s - x), x = s, RI = n_bg sqrt(u + 1).
//
// The host path evaluates the same formulas with numpy's complex64
// arithmetic; the device values agree with it to a few units in the last
// place (the order and contraction of the single-precision operations is
// not numpy's), which the tests bound.
#include <cuda_runtime.h>

#include <cmath>

#include "cbs_kernels.cuh"

namespace odt {
namespace {

constexpr int kThreads = 256;

int grid_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  if (b > 148LL * 16) b = 148LL * 16;
  return (int)(b < 1 ? 1 : b);
}

struct Conv {   // RI2potential / potential2RI constants (sub_code/RI2potential.m, potential2RI.m)
  float k2;     // (2 pi n_bg / lambda)^2
  float nb2;    // n_bg^2
  float nb;     // n_bg
  int cplx;     // complex RI: the host divides by the real scalars as complex
                // numbers, i.e. multiplies by their rounded reciprocals
};

// products and sums rounded one by one (no contraction), as the host's
// single-precision arithmetic does them
__device__ __forceinline__ float2 csq(float2 a) {
  const float p = __fmul_rn(a.x, a.y);
  return make_float2(__fsub_rn(__fmul_rn(a.x, a.x), __fmul_rn(a.y, a.y)), __fadd_rn(p, p));
}

__device__ __forceinline__ float2 cdiv_real(float2 a, float d, int cplx) {
  if (cplx) {
    const float r = __fdiv_rn(1.f, d);
    return make_float2(__fmul_rn(a.x, r), __fmul_rn(a.y, r));
  }
  return make_float2(__fdiv_rn(a.x, d), __fdiv_rn(a.y, d));
}

// k^2 (RI^2 / n_bg^2 - 1)
__device__ __forceinline__ float2 ri2pot(float2 ri, const Conv& c) {
  const float2 q = cdiv_real(csq(ri), c.nb2, c.cplx);
  return make_float2(__fmul_rn(c.k2, __fsub_rn(q.x, 1.f)), __fmul_rn(c.k2, q.y));
}

// principal square root, in double (then rounded): |z| by hypot, the larger
// component from sqrt((|z| + |x|) / 2), the other by division
__device__ __forceinline__ float2 csqrt_f(float2 z) {
  const double x = z.x, y = z.y;
  if (x == 0.0 && y == 0.0) return make_float2(0.f, z.y);
  const double t = sqrt(0.5 * (hypot(x, y) + fabs(x)));
  if (x >= 0.0) return make_float2((float)t, (float)(y / (2.0 * t)));
  return make_float2((float)(fabs(y) / (2.0 * t)), (float)copysign(t, y));
}

// n_bg sqrt(1 + pot / k^2)
__device__ __forceinline__ float2 pot2ri(float2 pot, const Conv& c) {
  const float2 q = cdiv_real(pot, c.k2, c.cplx);
  const float2 s = csqrt_f(make_float2(__fadd_rn(1.f, q.x), q.y));
  return make_float2(__fmul_rn(c.nb, s.x), __fmul_rn(c.nb, s.y));
}

__device__ __forceinline__ float2 load_ri(const void* ri, int is_complex, long long i) {
  return is_complex ? reinterpret_cast<const float2*>(ri)[i]
                    : make_float2(reinterpret_cast<const float*>(ri)[i], 0.f);
}

// max over the RI grid of |RI2potential(RI)|, as the bits of a non-negative
// float (ordered like the values)
__global__ void pot_absmax_kernel(const void* __restrict__ ri, int is_complex, long long n, Conv c,
                                  unsigned int* __restrict__ out) {
  float m = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 v = ri2pot(load_ri(ri, is_complex, i), c);
    const float a = (float)sqrt((double)v.x * v.x + (double)v.y * v.y);
    m = fmaxf(m, a);
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

// V on the padded grid [px, py, pz]: inside the ROI window (offset r0, size
// rs) the RI value (adjoint: conj(RI(x, y, rz-1-z))), zero potential outside;
// then potential2RI -> RI2potential -> potential2RI -> RI2potential, - i eps
__global__ void build_potential_kernel(const void* __restrict__ ri, int is_complex, int adjoint, int px, int py,
                                       int pz, int3 r0, int3 rs, Conv c, float eps, float2* __restrict__ V) {
  const long long n = (long long)px * py * pz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % px);
    const long long t = i / px;
    const int y = (int)(t % py), z = (int)(t / py);
    const int xr = x - r0.x, yr = y - r0.y, zr = z - r0.z;
    float2 v0 = make_float2(0.f, 0.f);
    if ((unsigned)xr < (unsigned)rs.x && (unsigned)yr < (unsigned)rs.y && (unsigned)zr < (unsigned)rs.z) {
      const int zs = adjoint ? rs.z - 1 - zr : zr;
      float2 r = load_ri(ri, is_complex, xr + (long long)rs.x * (yr + (long long)rs.y * zs));
      if (adjoint) r.y = -r.y;
      v0 = ri2pot(r, c);
    }
    const float2 v = ri2pot(pot2ri(ri2pot(pot2ri(v0, c), c), c), c);
    V[i] = make_float2(v.x, __fsub_rn(v.y, eps));
  }
}

// prox input: u - step * grad, complex or its real part
__global__ void fista_prox_input_kernel(const float2* __restrict__ u, const float2* __restrict__ grad, float step,
                                        int complex_out, void* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 a = u[i], g = grad[i];
    const float2 v = make_float2(a.x - step * g.x, a.y - step * g.y);
    if (complex_out) reinterpret_cast<float2*>(out)[i] = v;
    else reinterpret_cast<float*>(out)[i] = v.x;
  }
}

// u = s + coef (s - x); x = s; RI = n_bg sqrt(u + 1)
__global__ void fista_update_kernel(const void* __restrict__ s, int s_complex, float coef, float nb,
                                    float2* __restrict__ u, float2* __restrict__ x, float2* __restrict__ ri, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 sv = load_ri(s, s_complex, i);
    const float2 xv = x[i];
    const float2 uv = make_float2(sv.x + coef * (sv.x - xv.x), sv.y + coef * (sv.y - xv.y));
    u[i] = uv;
    x[i] = sv;
    const float2 r = csqrt_f(make_float2(uv.x + 1.f, uv.y));
    ri[i] = make_float2(nb * r.x, nb * r.y);
  }
}

Conv make_conv(double wavelength, double ri_bg, int cplx) {
  const double k = 2.0 * M_PI * ri_bg * (1.0 / wavelength);
  return Conv{(float)(k * k), (float)(ri_bg * ri_bg), (float)ri_bg, cplx};
}

}  // namespace

cudaError_t launch_potential_absmax(const void* ri, int is_complex, long long n, double wavelength, double ri_bg,
                                    unsigned int* d_out, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(d_out, 0, sizeof(unsigned int), s);
  if (e != cudaSuccess) return e;
  pot_absmax_kernel<<<grid_for(n), kThreads, 0, s>>>(ri, is_complex, n, make_conv(wavelength, ri_bg, is_complex),
                                                      d_out);
  return cudaGetLastError();
}

cudaError_t launch_build_potential(const void* ri, int is_complex, int adjoint, const int sim[3], const int roi0[3],
                                   const int ri_size[3], double wavelength, double ri_bg, float eps, float2* V,
                                   cudaStream_t s) {
  const long long n = (long long)sim[0] * sim[1] * sim[2];
  build_potential_kernel<<<grid_for(n), kThreads, 0, s>>>(
      ri, is_complex, adjoint, sim[0], sim[1], sim[2], make_int3(roi0[0], roi0[1], roi0[2]),
      make_int3(ri_size[0], ri_size[1], ri_size[2]), make_conv(wavelength, ri_bg, is_complex), eps, V);
  return cudaGetLastError();
}

cudaError_t launch_fista_prox_input(const float2* u, const float2* grad, float step, int complex_out, void* out,
                                    long long n, cudaStream_t s) {
  fista_prox_input_kernel<<<grid_for(n), kThreads, 0, s>>>(u, grad, step, complex_out, out, n);
  return cudaGetLastError();
}

cudaError_t launch_fista_update(const void* sv, int s_complex, float coef, float nb, float2* u, float2* x, float2* ri,
                                long long n, cudaStream_t s) {
  fista_update_kernel<<<grid_for(n), kThreads, 0, s>>>(sv, s_complex, coef, nb, u, x, ri, n);
  return cudaGetLastError();
}

}  // namespace odt
