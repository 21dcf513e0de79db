// Rytov reconstruction with Ewald-sphere mapping (BACKWARD_SOLVER_RYTOV.m:22-127)
// and the overlap counts of BACKWARD_SOLVER_RYTOV_precompute.m:87-137 /
// OVERLAP_COUNTER.m:19-23, on the GPU.
//
//   1. spectrum of each background field (centred fft2) and its peak
//      (MATLAB max of a complex array: largest abs, then largest angle, then
//      the first in column-major order)                           (:61-70)
//   2. per-illumination k0 (double, host)                          (:72-74)
//   3. Rytov field log|sp/bg| + i*phase, centred fft2 (res1*res2), shifted by
//      the peak offset, NA-filtered, times kz/1i                   (:80-89)
//   4. Ewald scatter, one launch per illumination in order: each pixel's
//      voxel index is computed with the reference's single-precision
//      arithmetic (no contraction), so Count is bit-exact; within one
//      illumination no two pixels share a voxel, so the adds need no atomics
//      and ORytov accumulates in the reference's order             (:90-104)
//   5. ORytov ./ Count / prod(res), centred ifftn, potential2RI     (:107-109)
//   6. optional non-negativity iterations                         (:111-125)
// MATLAB's dimension 1 is "y" and dimension 2 "x" here, as in the reference.
#include <cmath>
#include <string>
#include <vector>

#include "../../include/odt.h"
#include "cbs_kernels.cuh"
#include "fft_plan.h"
#include "scratch.cuh"

namespace odt {
const char* set_last_error(const std::string& msg);
}

namespace {

using namespace odt;

constexpr int kThreads = 256;

int grid_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  if (b > 148LL * 32) b = 148LL * 32;
  return (int)(b < 1 ? 1 : b);
}

// ---- peak of |F| per illumination (one block per illumination)
struct Peak {
  float a, g;  // abs, angle
  int idx;     // column-major index
};

__device__ __forceinline__ bool better(const Peak& p, const Peak& q) {  // p beats q
  if (p.a != q.a) return p.a > q.a;
  if (p.g != q.g) return p.g > q.g;
  return p.idx < q.idx;
}

__global__ void peak_kernel(const float2* F, int n12, int* peak) {
  const float2* f = F + (long long)blockIdx.x * n12;
  Peak best{-1.f, -10.f, 0x7fffffff};
  for (int i = threadIdx.x; i < n12; i += blockDim.x) {
    const float2 v = f[i];
    Peak c{hypotf(v.x, v.y), atan2f(v.y, v.x), i};
    if (better(c, best)) best = c;
  }
  __shared__ Peak red[1024];
  red[threadIdx.x] = best;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s && better(red[threadIdx.x + s], red[threadIdx.x]))
      red[threadIdx.x] = red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) peak[blockIdx.x] = red[0].idx;
}

// ---- Rytov field log|sp/bg| + i*phase
__global__ void rytov_field_kernel(const float2* bg, const float2* sp, const float* phase,
                                   float2* out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float2 b = bg[i], s = sp[i];
    // complex division sp/bg, then abs
    const float den = b.x * b.x + b.y * b.y;
    const float qr = (s.x * b.x + s.y * b.y) / den;
    const float qi = (s.y * b.x - s.x * b.y) / den;
    out[i] = make_float2(logf(hypotf(qr, qi)), phase ? phase[i] : 0.f);
  }
}

struct Angle {
  float k0x, k0y, k0z;  // single(k0_x), single(k0_y), single(k0_z)
  int sy, sx;           // circshift of the spectrum (rows, cols)
};

struct EwaldGeo {
  int n1, n2, n3;
  float res1f, res2f, res3f;                 // single(fourier res)
  float h1, h2, h3;                          // single(floor(n/2))
  double lo1, lo2, lo3, hi1, hi2, hi3;       // res * (-floor(n/2)), res * (floor(n/2) - 1)
  float scale;                               // single(res_x * res_y) (image-space)
};

// single-precision index of one axis: round(K / res + floor(n/2) + 1), no contraction
__device__ __forceinline__ int ewald_index(float K, float resf, float half) {
  float t = __fdiv_rn(K, resf);
  t = __fadd_rn(t, half);
  t = __fadd_rn(t, 1.0f);
  return (int)roundf(t);  // half away from zero, as MATLAB round
}

__global__ void scatter_kernel(EwaldGeo g, Angle an, const float2* Us, const float* coor1,
                               const float* coor2, const float* k3, const unsigned char* na,
                               float2* O, float* C, int* kzmap, int count_one) {
  const int n12 = g.n1 * g.n2;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n12; p += gridDim.x * blockDim.x) {
    const int i1 = p % g.n1, i2 = p / g.n1;
    if (!na[p]) continue;
    const float kz = k3[p];
    if (!(kz > 0.f)) continue;
    const float Kx = __fsub_rn(coor2[i2], an.k0x);
    const float Ky = __fsub_rn(coor1[i1], an.k0y);
    const float Kz = __fsub_rn(kz, an.k0z);
    if (!((double)Kx > g.lo2 && (double)Ky > g.lo1 && (double)Kz > g.lo3 && (double)Kx < g.hi2 &&
          (double)Ky < g.hi1 && (double)Kz < g.hi3))
      continue;
    // spectrum value after circshift by (sy, sx): Us(i1 - sy, i2 - sx)
    int j1 = i1 - an.sy, j2 = i2 - an.sx;
    j1 %= g.n1;
    if (j1 < 0) j1 += g.n1;
    j2 %= g.n2;
    if (j2 < 0) j2 += g.n2;
    const float2 u0 = Us[j1 + (long long)g.n1 * j2];
    const float2 u = make_float2(__fmul_rn(u0.x, g.scale), __fmul_rn(u0.y, g.scale));
    const float2 up = make_float2(__fmul_rn(kz, u.y), -__fmul_rn(kz, u.x));  // (kz/1i) * u
    const int iKx = ewald_index(Kx, g.res2f, g.h2);
    const int iKy = ewald_index(Ky, g.res1f, g.h1);
    const int iKz = ewald_index(Kz, g.res3f, g.h3);
    const long long lin = (long long)(iKy - 1) + (long long)g.n1 * ((iKx - 1) + (long long)g.n2 * (iKz - 1));
    const float2 o = O[lin];
    O[lin] = make_float2(__fadd_rn(o.x, up.x), __fadd_rn(o.y, up.y));
    const bool nz = up.x != 0.f || up.y != 0.f;
    C[lin] = __fadd_rn(C[lin], (count_one || nz) ? 1.f : 0.f);
    kzmap[(iKy - 1) + g.n1 * (iKx - 1)] = (int)lin;
  }
}

__global__ void normalize_kernel(float2* O, const float* C, long long n, float prod_res) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float c = C[i];
    if (c > 0.f) {
      const float2 o = O[i];
      O[i] = make_float2(__fdiv_rn(__fdiv_rn(o.x, c), prod_res), __fdiv_rn(__fdiv_rn(o.y, c), prod_res));
    }
  }
}

__global__ void overlap_field_kernel(const int* kzmap, const float* C, float* ov, int n1, int n2,
                                     int sy, int sx) {
  const int n12 = n1 * n2;
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n12; p += gridDim.x * blockDim.x) {
    const int i1 = p % n1, i2 = p / n1;
    int j1 = (i1 - sy) % n1, j2 = (i2 - sx) % n2;
    if (j1 < 0) j1 += n1;
    if (j2 < 0) j2 += n2;
    const int m = kzmap[j1 + n1 * j2];
    ov[p] = m >= 0 ? C[m] : 0.f;
  }
}

__global__ void fill_int_kernel(int* p, long long n, int v) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    p[i] = v;
}

// principal complex square root
__device__ __forceinline__ float2 csqrtf_(float2 z) {
  const float r = hypotf(z.x, z.y);
  if (r == 0.f) return make_float2(0.f, 0.f);
  if (z.x >= 0.f) {
    const float t = sqrtf(0.5f * (r + z.x));
    return make_float2(t, z.y / (2.f * t));
  }
  const float t = sqrtf(0.5f * (r - z.x));
  return make_float2(fabsf(z.y) / (2.f * t), copysignf(t, z.y));
}

// RI = n_m * sqrt(1 + (rec * 4pi) / k^2)      (potential2RI.m:1-5)
__global__ void potential2ri_kernel(const float2* rec, float2* ri, long long n, float four_pi,
                                    float k2, float nm) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float2 p = make_float2(rec[i].x * four_pi, rec[i].y * four_pi);
    const float2 a = make_float2(1.f + p.x / k2, p.y / k2);
    const float2 s = csqrtf_(a);
    ri[i] = make_float2(nm * s.x, nm * s.y);
  }
}

// non-negativity: real part clipped at 0
__global__ void clip_real_kernel(float2* x, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    if (x[i].x < 0.f) x[i].x = 0.f;
}

// On = Emask .* On .* (abs(O) == 0) + O
__global__ void nn_merge_kernel(float2* On, const float2* O, const unsigned char* emask, int n12,
                                long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float2 o = O[i];
    const bool keep = emask[i % n12] && o.x == 0.f && o.y == 0.f;
    const float2 v = keep ? On[i] : make_float2(0.f, 0.f);
    On[i] = make_float2(v.x + o.x, v.y + o.y);
  }
}

odt_status fail(odt_status st, const std::string& m) {
  odt::set_last_error(m);
  return st;
}

#define RY_CHECK(call)                                                              \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      cudaGetLastError();                                                           \
      return fail(ODT_ERR_CUDA, std::string("odt_rytov: ") + cudaGetErrorString(e_)); \
    }                                                                               \
  } while (0)

}  // namespace

extern "C" odt_status odt_rytov(const odt_rytov_args* a) {
  if (!a || !a->bg || !a->coor1 || !a->coor2 || !a->k3 || !a->na_circle)
    return fail(ODT_ERR_INVALID_ARGUMENT, "odt_rytov: NULL argument");
  const int n1 = a->size[0], n2 = a->size[1], n3 = a->size[2], nill = a->n_ill;
  if (n1 < 1 || n2 < 1 || n3 < 1 || nill < 1)
    return fail(ODT_ERR_INVALID_ARGUMENT, "odt_rytov: bad sizes");
  if (a->memory != ODT_MEM_HOST && a->memory != ODT_MEM_DEVICE)
    return fail(ODT_ERR_INVALID_ARGUMENT, "odt_rytov: bad memory flag");
  const bool dev = a->memory == ODT_MEM_DEVICE;
  cudaStream_t s = dev ? (cudaStream_t)a->stream : (cudaStream_t)0;
  Scratch B;
  B.s = s;
  const long long n12 = (long long)n1 * n2, n3d = n12 * n3, nf = n12 * nill;
  const cudaMemcpyKind kin = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const cudaMemcpyKind kout = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  // inputs on the device
  float2* bg = B.get<float2>(nf);
  float2* sp = B.get<float2>(nf);
  float* ph = a->phase ? B.get<float>(nf) : nullptr;
  float* coor1 = B.get<float>(n1);
  float* coor2 = B.get<float>(n2);
  float* k3 = B.get<float>(n12);
  unsigned char* na = B.get<unsigned char>(n12);
  float2* spec = B.get<float2>(nf);
  int* peak = B.get<int>(nill);
  float2* O = B.get<float2>(n3d);
  float* C = B.get<float>(n3d);
  int* kzmap = B.get<int>(n12 * nill);
  if (!bg || !sp || (a->phase && !ph) || !coor1 || !coor2 || !k3 || !na || !spec || !peak || !O ||
      !C || !kzmap)
    return fail(ODT_ERR_OUT_OF_MEMORY, "odt_rytov: device allocation failed");
  RY_CHECK(cudaMemcpyAsync(bg, a->bg, nf * sizeof(float2), kin, s));
  RY_CHECK(cudaMemcpyAsync(sp, a->sp ? a->sp : a->bg, nf * sizeof(float2), kin, s));
  if (ph) RY_CHECK(cudaMemcpyAsync(ph, a->phase, nf * sizeof(float), kin, s));
  RY_CHECK(cudaMemcpyAsync(coor1, a->coor1, n1 * sizeof(float), kin, s));
  RY_CHECK(cudaMemcpyAsync(coor2, a->coor2, n2 * sizeof(float), kin, s));
  RY_CHECK(cudaMemcpyAsync(k3, a->k3, n12 * sizeof(float), kin, s));
  RY_CHECK(cudaMemcpyAsync(na, a->na_circle, n12, kin, s));
  RY_CHECK(cudaMemsetAsync(O, 0, n3d * sizeof(float2), s));
  RY_CHECK(cudaMemsetAsync(C, 0, n3d * sizeof(float), s));
  fill_int_kernel<<<grid_for(n12 * nill), kThreads, 0, s>>>(kzmap, n12 * nill, -1);
  DevFft f1{}, f2{}, f3{};
  std::string why;
  if (!scratch_fft(B, n1, &f1, &why) || !scratch_fft(B, n2, &f2, &why) || !scratch_fft(B, n3, &f3, &why))
    return fail(ODT_ERR_UNSUPPORTED, "odt_rytov: " + why);
  auto fftc2 = [&](float2* x, long long nsl, bool inv) -> cudaError_t {
    cudaError_t e = launch_fft_lines(x, x, (long long)n2 * nsl, n1 / 2, n1 / 2, 1.f, inv, f1, s);
    if (e != cudaSuccess) return e;
    return launch_fft_cols(x, x, n1, nsl, n2 / 2, n2 / 2, inv ? 1.0f / ((float)n1 * n2) : 1.f, inv,
                           f2, s);
  };
  auto fftc3 = [&](float2* x, bool inv) -> cudaError_t {
    cudaError_t e = fftc2(x, n3, inv);
    if (e != cudaSuccess) return e;
    return launch_fft_cols(x, x, n12, 1, n3 / 2, n3 / 2, inv ? 1.0f / (float)n3 : 1.f, inv, f3, s);
  };
  // 1. peaks of the background spectra
  RY_CHECK(cudaMemcpyAsync(spec, bg, nf * sizeof(float2), cudaMemcpyDeviceToDevice, s));
  RY_CHECK(fftc2(spec, nill, false));
  peak_kernel<<<nill, 1024, 0, s>>>(spec, (int)n12, peak);
  RY_CHECK(cudaGetLastError());
  std::vector<int> pk(nill);
  RY_CHECK(cudaMemcpyAsync(pk.data(), peak, nill * sizeof(int), cudaMemcpyDeviceToHost, s));
  RY_CHECK(cudaStreamSynchronize(s));
  // 2. k0 per illumination, in double as the reference (:72-74)
  const int mj0 = pk[0] % n1, mi0 = pk[0] / n1;
  std::vector<Angle> ang(nill);
  for (int k = 0; k < nill; ++k) {
    const double fdy = (double)(pk[k] % n1 - mj0), fdx = (double)(pk[k] / n1 - mi0);
    const double k0x = a->fourier_res[1] * fdx, k0y = a->fourier_res[0] * fdy;
    const double arg = a->k0_nm * a->k0_nm - k0x * k0x - k0y * k0y;
    const double k0z = arg > 0 ? std::sqrt(arg) : 0.0;
    ang[k] = Angle{(float)k0x, (float)k0y, (float)k0z, (int)std::lround(k0y / a->fourier_res[0]),
                   (int)std::lround(k0x / a->fourier_res[1])};
    if (a->shifts) {
      a->shifts[2 * k] = ang[k].sy;
      a->shifts[2 * k + 1] = ang[k].sx;
    }
  }
  // 3. Rytov spectra
  rytov_field_kernel<<<grid_for(nf), kThreads, 0, s>>>(bg, sp, ph, spec, nf);
  RY_CHECK(cudaGetLastError());
  RY_CHECK(fftc2(spec, nill, false));
  // 4. Ewald scatter, in illumination order
  EwaldGeo g{};
  g.n1 = n1;
  g.n2 = n2;
  g.n3 = n3;
  g.res1f = (float)a->fourier_res[0];
  g.res2f = (float)a->fourier_res[1];
  g.res3f = (float)a->fourier_res[2];
  g.h1 = (float)(n1 / 2);
  g.h2 = (float)(n2 / 2);
  g.h3 = (float)(n3 / 2);
  g.lo1 = a->fourier_res[0] * (-(double)(n1 / 2));
  g.lo2 = a->fourier_res[1] * (-(double)(n2 / 2));
  g.lo3 = a->fourier_res[2] * (-(double)(n3 / 2));
  g.hi1 = a->fourier_res[0] * ((double)(n1 / 2) - 1);
  g.hi2 = a->fourier_res[1] * ((double)(n2 / 2) - 1);
  g.hi3 = a->fourier_res[2] * ((double)(n3 / 2) - 1);
  g.scale = (float)(a->resolution[0] * a->resolution[1]);
  for (int k = 0; k < nill; ++k) {
    scatter_kernel<<<grid_for(n12), kThreads, 0, s>>>(g, ang[k], spec + (long long)k * n12, coor1,
                                                      coor2, k3, na, O, C, kzmap + (long long)k * n12,
                                                      a->count_one);
    RY_CHECK(cudaGetLastError());
  }
  // overlap field (:129-135) uses the counts before normalisation
  if (a->overlap_field) {
    float* ov = B.get<float>(nf);
    if (!ov) return fail(ODT_ERR_OUT_OF_MEMORY, "odt_rytov: device allocation failed");
    for (int k = 0; k < nill; ++k)
      overlap_field_kernel<<<grid_for(n12), kThreads, 0, s>>>(kzmap + (long long)k * n12, C,
                                                              ov + (long long)k * n12, n1, n2,
                                                              ang[k].sy, ang[k].sx);
    RY_CHECK(cudaGetLastError());
    RY_CHECK(cudaMemcpyAsync(a->overlap_field, ov, nf * sizeof(float), kout, s));
  }
  // 5. normalisation, reconstruction
  const float prod_res = (float)(a->resolution[0] * a->resolution[1] * a->resolution[2]);
  normalize_kernel<<<grid_for(n3d), kThreads, 0, s>>>(O, C, n3d, prod_res);
  RY_CHECK(cudaGetLastError());
  if (a->count) RY_CHECK(cudaMemcpyAsync(a->count, C, n3d * sizeof(float), kout, s));
  if (a->ORytov) RY_CHECK(cudaMemcpyAsync(a->ORytov, O, n3d * sizeof(float2), kout, s));
  if (a->RI) {
    float2* rec = B.get<float2>(n3d);
    if (!rec) return fail(ODT_ERR_OUT_OF_MEMORY, "odt_rytov: device allocation failed");
    RY_CHECK(cudaMemcpyAsync(rec, O, n3d * sizeof(float2), cudaMemcpyDeviceToDevice, s));
    RY_CHECK(fftc3(rec, true));
    if (a->non_negativity_iteration > 0) {
      unsigned char* emask = B.get<unsigned char>(n12);
      float2* On = B.get<float2>(n3d);
      if (!emask || !On) return fail(ODT_ERR_OUT_OF_MEMORY, "odt_rytov: device allocation failed");
      RY_CHECK(cudaMemcpyAsync(emask, a->emask, n12, kin, s));
      for (int it = 0; it < a->non_negativity_iteration; ++it) {
        clip_real_kernel<<<grid_for(n3d), kThreads, 0, s>>>(rec, n3d);
        RY_CHECK(cudaMemcpyAsync(On, rec, n3d * sizeof(float2), cudaMemcpyDeviceToDevice, s));
        RY_CHECK(fftc3(On, false));
        nn_merge_kernel<<<grid_for(n3d), kThreads, 0, s>>>(On, O, emask, (int)n12, n3d);
        RY_CHECK(cudaMemcpyAsync(rec, On, n3d * sizeof(float2), cudaMemcpyDeviceToDevice, s));
        RY_CHECK(fftc3(rec, true));
      }
      clip_real_kernel<<<grid_for(n3d), kThreads, 0, s>>>(rec, n3d);
    }
    const double k = 2.0 * M_PI * a->ri_bg / a->wavelength;
    potential2ri_kernel<<<grid_for(n3d), kThreads, 0, s>>>(rec, rec, n3d, (float)(4.0 * M_PI),
                                                           (float)(k * k), (float)a->ri_bg);
    RY_CHECK(cudaGetLastError());
    RY_CHECK(cudaMemcpyAsync(a->RI, rec, n3d * sizeof(float2), kout, s));
  }
  RY_CHECK(cudaStreamSynchronize(s));
  odt::set_last_error("");
  return ODT_OK;
}
