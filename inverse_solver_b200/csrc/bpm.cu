// Beam-propagation forward solver (FORWARD_SOLVER_BPM.m:44-117) on the
// generic tile FFTs.  All illuminations of a call march through the RI grid
// together, one z-slice per step:
//
//   field = fftshift(fft2(ifftshift(in))) .* pre       (refocus to the first
//   field = fftshift(ifft2(ifftshift(field)))           slice, :93-95)
//   field = fft2(field)
//   for each slice z:                                    (:97-109)
//     field = ifft2(field .* refocus_kernel)            (free-space step)
//     field = field .* exp(field_multiplier(:,:,z) / cos_theta(peak))
//     field = fft2(field)
//     fields_3D(:,:,z) = ifft2(field .* filter_out)      (return_3D only)
//   field = ifft2(field)                                 (refocus back to the
//   trans = fftshift(ifft2(ifftshift(                      focal plane, :110-114)
//             fftshift(fft2(ifftshift(field))) .* post)))
//
// The cosine correction takes cos_theta at the peak of each illumination's
// centred spectrum (:59-63: the first maximum of |.| in column-major order).
#include <cuda_runtime.h>

#include <cmath>
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

// x[i] *= k[i % plane]
__global__ void cmul_plane_kernel(float2* __restrict__ x, const float2* __restrict__ k, long long plane,
                                  long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = cmul(x[i], k[i % plane]);
}

// out[i] = x[i] * f[i % plane]
__global__ void fmul_plane_kernel(const float2* __restrict__ x, const float* __restrict__ f, float2* __restrict__ out,
                                  long long plane, long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = cscale(x[i], f[i % plane]);
}

// x[p, b] *= exp(fm[p] * inv_cos[b])   (inv_cos NULL: exp(fm[p]))
__global__ void phase_kernel(float2* __restrict__ x, const float2* __restrict__ fm, const float* __restrict__ inv_cos,
                             long long plane, long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long p = i % plane;
    float2 e = fm[p];
    if (inv_cos) e = cscale(e, inv_cos[i / plane]);
    float sn, cs;
    sincosf(e.y, &sn, &cs);
    const float m = expf(e.x);
    x[i] = cmul(x[i], make_float2(m * cs, m * sn));
  }
}

// out3d[p + plane * (z + nz * b)] = t[p + plane * b]
__global__ void scatter_slice_kernel(const float2* __restrict__ t, float2* __restrict__ out3d, int z, int nz,
                                     long long plane, long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long b = i / plane, p = i - b * plane;
    out3d[p + plane * (z + (long long)nz * b)] = t[i];
  }
}

// one CTA per illumination: inv_cos[b] = 1 / cos_theta(first argmax |spec|)
__global__ void peak_inv_cos_kernel(const float2* __restrict__ spec, const float* __restrict__ cos_theta, int plane,
                                    float* __restrict__ inv_cos) {
  __shared__ float sv[32];
  __shared__ int si[32];
  const float2* x = spec + (long long)blockIdx.x * plane;
  float best = -1.f;
  int bi = 0;
  for (int p = threadIdx.x; p < plane; p += blockDim.x) {
    const float2 v = x[p];
    const float a = (float)sqrt((double)v.x * v.x + (double)v.y * v.y);
    if (a > best) {  // strictly greater: a thread keeps its first maximum
      best = a;
      bi = p;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const float ob = __shfl_xor_sync(0xffffffffu, best, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (ob > best || (ob == best && oi < bi)) {
      best = ob;
      bi = oi;
    }
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    sv[w] = best;
    si[w] = bi;
  }
  __syncthreads();
  if (w == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    best = l < nw ? sv[l] : -1.f;
    bi = l < nw ? si[l] : 0;
    for (int o = 16; o > 0; o >>= 1) {
      const float ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (l == 0) inv_cos[blockIdx.x] = 1.f / cos_theta[bi];
  }
}

odt_status bpm_fail(odt_status st, const std::string& m) {
  set_last_error(m);
  return st;
}

bool is_dev(const void* p) {
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

#define BPM_CHECK(call)                                                                   \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) {                                                              \
      cudaGetLastError();                                                                 \
      return bpm_fail(ODT_ERR_CUDA, std::string("odt_bpm_solve: ") + cudaGetErrorString(e_)); \
    }                                                                                     \
  } while (0)

}  // namespace

extern "C" odt_status odt_bpm_solve(const odt_bpm_args* a) {
  if (!a || !a->field_multiplier || !a->refocus_kernel || !a->pre || !a->post || !a->fields_in || !a->trans)
    return bpm_fail(ODT_ERR_INVALID_ARGUMENT, "odt_bpm_solve: NULL argument");
  const int n1 = a->size[0], n2 = a->size[1], nz = a->size[2], nill = a->n_ill;
  if (n1 < 1 || n2 < 1 || nz < 1 || nill < 1) return bpm_fail(ODT_ERR_INVALID_ARGUMENT, "odt_bpm_solve: bad sizes");
  if (a->field3d && !a->filter_out)
    return bpm_fail(ODT_ERR_INVALID_ARGUMENT, "odt_bpm_solve: field3d needs filter_out");
  if (a->memory != ODT_MEM_HOST && a->memory != ODT_MEM_DEVICE)
    return bpm_fail(ODT_ERR_INVALID_ARGUMENT, "odt_bpm_solve: bad memory flag");
  const bool dev = a->memory == ODT_MEM_DEVICE;
  if (dev) {
    for (const void* p : {(const void*)a->field_multiplier, (const void*)a->refocus_kernel, (const void*)a->pre,
                          (const void*)a->post, (const void*)a->fields_in, (const void*)a->trans})
      if (!is_dev(p)) return bpm_fail(ODT_ERR_INVALID_ARGUMENT, "odt_bpm_solve: ODT_MEM_DEVICE with a host pointer");
    if ((a->field3d && !is_dev(a->field3d)) || (a->filter_out && !is_dev(a->filter_out)) ||
        (a->cos_theta && !is_dev(a->cos_theta)))
      return bpm_fail(ODT_ERR_INVALID_ARGUMENT, "odt_bpm_solve: ODT_MEM_DEVICE with a host pointer");
  }
  cudaStream_t s = dev ? (cudaStream_t)a->stream : (cudaStream_t)0;
  Scratch B;
  B.s = s;
  const long long plane = (long long)n1 * n2, nf = plane * nill, n3 = plane * nz;
  const cudaMemcpyKind kin = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  float2* fld = B.get<float2>(nf);
  float2* tmp = a->field3d ? B.get<float2>(nf) : nullptr;
  float* inv_cos = a->cos_theta ? B.get<float>(nill) : nullptr;
  const float2* fm = reinterpret_cast<const float2*>(a->field_multiplier);
  const float2* rk = reinterpret_cast<const float2*>(a->refocus_kernel);
  const float2* pre = reinterpret_cast<const float2*>(a->pre);
  const float2* post = reinterpret_cast<const float2*>(a->post);
  const float* filt = a->filter_out;
  const float* cth = a->cos_theta;
  float2* out3d = reinterpret_cast<float2*>(a->field3d);
  if (!fld || (a->field3d && !tmp) || (a->cos_theta && !inv_cos))
    return bpm_fail(ODT_ERR_OUT_OF_MEMORY, "odt_bpm_solve: device allocation failed");
  if (!dev) {  // tables and the 3D output on the device
    float2* d_fm = B.get<float2>(n3);
    float2* d_t = B.get<float2>(3 * plane);
    float* d_f = B.get<float>(2 * plane);
    if (!d_fm || !d_t || !d_f) return bpm_fail(ODT_ERR_OUT_OF_MEMORY, "odt_bpm_solve: device allocation failed");
    BPM_CHECK(cudaMemcpyAsync(d_fm, fm, n3 * sizeof(float2), kin, s));
    BPM_CHECK(cudaMemcpyAsync(d_t, rk, plane * sizeof(float2), kin, s));
    BPM_CHECK(cudaMemcpyAsync(d_t + plane, pre, plane * sizeof(float2), kin, s));
    BPM_CHECK(cudaMemcpyAsync(d_t + 2 * plane, post, plane * sizeof(float2), kin, s));
    if (filt) BPM_CHECK(cudaMemcpyAsync(d_f, filt, plane * sizeof(float), kin, s));
    if (cth) BPM_CHECK(cudaMemcpyAsync(d_f + plane, cth, plane * sizeof(float), kin, s));
    fm = d_fm;
    rk = d_t;
    pre = d_t + plane;
    post = d_t + 2 * plane;
    filt = filt ? d_f : nullptr;
    cth = cth ? d_f + plane : nullptr;
    if (a->field3d) {
      out3d = B.get<float2>(n3 * nill);
      if (!out3d) return bpm_fail(ODT_ERR_OUT_OF_MEMORY, "odt_bpm_solve: device allocation failed");
    }
  }
  BPM_CHECK(cudaMemcpyAsync(fld, a->fields_in, nf * sizeof(float2), kin, s));
  DevFft f1{}, f2{};
  std::string why;
  if (!scratch_fft(B, n1, &f1, &why) || !scratch_fft(B, n2, &f2, &why))
    return bpm_fail(ODT_ERR_UNSUPPORTED, "odt_bpm_solve: " + why);
  const float inv_n = 1.0f / ((float)n1 * (float)n2);
  // 2D FFT of every plane of x; centred: fftshift(fft2(ifftshift(.)))
  auto fft2 = [&](float2* x, bool inv, bool centred) -> cudaError_t {
    const int s1 = centred ? n1 / 2 : 0, s2 = centred ? n2 / 2 : 0;
    cudaError_t e = launch_fft_lines(x, x, (long long)n2 * nill, s1, s1, 1.f, inv, f1, s);
    if (e != cudaSuccess) return e;
    return launch_fft_cols(x, x, n1, nill, s2, s2, inv ? inv_n : 1.f, inv, f2, s);
  };
  const int g = grid_for(nf);
  BPM_CHECK(fft2(fld, false, true));
  if (cth) {
    peak_inv_cos_kernel<<<nill, 256, 0, s>>>(fld, cth, (int)plane, inv_cos);
    BPM_CHECK(cudaGetLastError());
  }
  cmul_plane_kernel<<<g, kThreads, 0, s>>>(fld, pre, plane, nf);
  BPM_CHECK(fft2(fld, true, true));
  BPM_CHECK(fft2(fld, false, false));
  for (int z = 0; z < nz; ++z) {
    cmul_plane_kernel<<<g, kThreads, 0, s>>>(fld, rk, plane, nf);
    BPM_CHECK(fft2(fld, true, false));
    phase_kernel<<<g, kThreads, 0, s>>>(fld, fm + plane * z, inv_cos, plane, nf);
    BPM_CHECK(fft2(fld, false, false));
    if (out3d) {
      fmul_plane_kernel<<<g, kThreads, 0, s>>>(fld, filt, tmp, plane, nf);
      BPM_CHECK(fft2(tmp, true, false));
      scatter_slice_kernel<<<g, kThreads, 0, s>>>(tmp, out3d, z, nz, plane, nf);
    }
  }
  BPM_CHECK(fft2(fld, true, false));
  BPM_CHECK(fft2(fld, false, true));
  cmul_plane_kernel<<<g, kThreads, 0, s>>>(fld, post, plane, nf);
  BPM_CHECK(fft2(fld, true, true));
  const cudaMemcpyKind kout = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  BPM_CHECK(cudaMemcpyAsync(a->trans, fld, nf * sizeof(float2), kout, s));
  if (a->field3d && !dev) BPM_CHECK(cudaMemcpyAsync(a->field3d, out3d, n3 * nill * sizeof(float2), kout, s));
  if (!dev) BPM_CHECK(cudaStreamSynchronize(s));
  return ODT_OK;
}
