// Field retrieval from off-axis holograms, the transform-heavy part of
// get_fields (FIELD_EXPERIMENTAL_RETRIEVAL.m:110-178) on the GPU:
//
//   F = fftshift(fft2(ifftshift(hologram)))            background and sample
//   sideband peak = first max of |F_bg(:,:,1)| outside the deleted bands
//   F = fftshift(fftshift(circshift(F, 1 - peak)))    sideband to the centre
//   crop or zero-pad to the output side (resolution matching), .* NA_circle
//   per image: the maximum of |F_bg| and its four neighbours (the data of
//     peak_subpixel_positioner)
//   field = fftshift(ifft2(ifftshift(F)))(3:end-2, 3:end-2)
//
// the per-pixel steps after them (:179-201: normalisation, the phase and
// amplitude of sp / bg, and the recombination with the ramp-free phase), and
// the centred 2D refocus of refocus (:392-394).  Phase unwrapping has its
// own kernels; the per-image scalar steps (sub-pixel positions, the border
// plane fit of PhiShiftMS) are the host mirror's.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "../../include/odt.h"
#include "cbs_kernels.cuh"
#include "np_complex.cuh"
#include "fft_any.cuh"
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


__global__ void to_complex_kernel(const float* __restrict__ a, float2* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = make_float2(a[i], 0.f);
}

// first (column-major) maximum of |F| over the search window of plane 0:
// rows < r_end and columns in [c_lo, c_hi) (0-based), as (value, index)
__global__ void sideband_kernel(const float2* __restrict__ F, int n1, int n2, int r_end, int c_lo, int c_hi,
                                int* __restrict__ peak) {
  __shared__ float sv[32];
  __shared__ int si[32];
  float best = -1.f;
  int bi = 0x7fffffff;
  const long long total = (long long)n1 * n2;
  for (long long i = threadIdx.x; i < total; i += blockDim.x) {
    const int r = (int)(i % n1), c = (int)(i / n1);
    if (r >= r_end || c < c_lo || c >= c_hi) continue;
    const float a = cabs_f(F[i]);
    if (a > best) {
      best = a;
      bi = (int)i;
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
    bi = l < nw ? si[l] : 0x7fffffff;
    for (int o = 16; o > 0; o >>= 1) {
      const float ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (l == 0) {
      peak[0] = bi % n1 + 1;   // 1-based, as find returns
      peak[1] = bi / n1 + 1;
    }
  }
}

// out[m1, m2, k] = F[(m1 + d - N/2 + s1) mod N, (m2 + d - N/2 + s2) mod N, k] * na[m1, m2]
// for source rows / columns m + d inside [0, N) (crop: d >= 0; pad: d < 0), else 0
__global__ void centre_crop_kernel(const float2* __restrict__ F, int N, int M, int d, const int* __restrict__ peak,
                                   const unsigned char* __restrict__ na, int nimg, float2* __restrict__ out) {
  const int s1 = peak[0] - 1, s2 = peak[1] - 1;
  const long long plane = (long long)M * M, total = plane * nimg;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long k = i / plane, p = i - k * plane;
    const int m1 = (int)(p % M), m2 = (int)(p / M);
    const int k1 = m1 + d, k2 = m2 + d;
    float2 v = make_float2(0.f, 0.f);
    if (na[p] && (unsigned)k1 < (unsigned)N && (unsigned)k2 < (unsigned)N) {
      int r = (k1 - N / 2 + s1) % N, c = (k2 - N / 2 + s2) % N;
      if (r < 0) r += N;
      if (c < 0) c += N;
      v = F[r + (long long)N * (c + (long long)N * k)];
    }
    out[i] = v;
  }
}

// one CTA per image: i1, i2 (1-based) of the first max of |F| and |F| there
// and at (i1-1, i2), (i1+1, i2), (i1, i2-1), (i1, i2+1) (0 outside the image)
__global__ void peak_kernel(const float2* __restrict__ F, int M, float* __restrict__ out) {
  __shared__ float sv[32];
  __shared__ int si[32];
  const float2* x = F + (long long)blockIdx.x * M * M;
  float best = -1.f;
  int bi = 0x7fffffff;
  for (int p = threadIdx.x; p < M * M; p += blockDim.x) {
    const float a = cabs_f(x[p]);
    if (a > best) {
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
    bi = l < nw ? si[l] : 0x7fffffff;
    for (int o = 16; o > 0; o >>= 1) {
      const float ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (l == 0) {
      const int i1 = bi % M, i2 = bi / M;
      auto at = [&](int a, int b) { return (a >= 0 && a < M && b >= 0 && b < M) ? cabs_f(x[a + M * b]) : 0.f; };
      float* o = out + 7LL * blockIdx.x;
      o[0] = (float)(i1 + 1);
      o[1] = (float)(i2 + 1);
      o[2] = best;
      o[3] = at(i1 - 1, i2);
      o[4] = at(i1 + 1, i2);
      o[5] = at(i1, i2 - 1);
      o[6] = at(i1, i2 + 1);
    }
  }
}

// x[i] *= k[i % plane]
__global__ void cmul_plane_kernel(float2* __restrict__ x, const float2* __restrict__ k, long long plane,
                                  long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = cmul(x[i], k[i % plane]);
}

odt_status hfail(odt_status st, const std::string& m) {
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


}  // namespace

extern "C" odt_status odt_hologram_fields(const odt_hologram_args* a) {
  if (!a || !a->bg || !a->sp || !a->na_circle || !a->bg_field || !a->sp_field || !a->peaks || !a->sideband)
    return hfail(ODT_ERR_INVALID_ARGUMENT, "odt_hologram_fields: NULL argument");
  const int N = a->size[0], nimg = a->size[2], M = a->out_size;
  if (N < 8 || a->size[1] != N || nimg < 1 || M < 5 || !(a->cutout_portion > 0.0 && a->cutout_portion < 1.0))
    return hfail(ODT_ERR_INVALID_ARGUMENT, "odt_hologram_fields: bad sizes or cutout_portion");
  if (a->memory != ODT_MEM_HOST && a->memory != ODT_MEM_DEVICE)
    return hfail(ODT_ERR_INVALID_ARGUMENT, "odt_hologram_fields: bad memory flag");
  const bool dev = a->memory == ODT_MEM_DEVICE;
  if (dev && (!is_dev(a->bg) || !is_dev(a->sp) || !is_dev(a->na_circle) || !is_dev(a->bg_field) ||
              !is_dev(a->sp_field) || !is_dev(a->peaks)))
    return hfail(ODT_ERR_INVALID_ARGUMENT, "odt_hologram_fields: ODT_MEM_DEVICE with a host pointer");
  cudaStream_t s = dev ? (cudaStream_t)a->stream : (cudaStream_t)0;
  Scratch B;
  B.s = s;
  const long long nin = (long long)N * N * nimg, nmid = (long long)M * M * nimg;
  const long long nout = (long long)(M - 4) * (M - 4) * nimg;
  float* hb = dev ? nullptr : B.get<float>(nin);
  float* hs = dev ? nullptr : B.get<float>(nin);
  float2* Fb = B.get<float2>(nin);
  float2* Fs = B.get<float2>(nin);
  float2* Gb = B.get<float2>(nmid);
  float2* Gs = B.get<float2>(nmid);
  unsigned char* na = dev ? nullptr : B.get<unsigned char>((size_t)M * M);
  float2* ob = dev ? nullptr : B.get<float2>(nout);
  float2* os = dev ? nullptr : B.get<float2>(nout);
  float* pk = dev ? nullptr : B.get<float>(7 * (size_t)nimg);
  int* sb = B.get<int>(2);
  if (!Fb || !Fs || !Gb || !Gs || !sb || (!dev && (!hb || !hs || !na || !ob || !os || !pk)))
    return hfail(ODT_ERR_OUT_OF_MEMORY, "odt_hologram_fields: device allocation failed");
  AnyFft fN{}, fM{};
  std::string why;
  if (!scratch_fft_any(B, N, &fN, &why) || !scratch_fft_any(B, M, &fM, &why))
    return hfail(ODT_ERR_UNSUPPORTED, "odt_hologram_fields: " + why);
  auto run = [&]() -> cudaError_t {
    cudaError_t e;
    const float* db = a->bg;
    const float* ds = a->sp;
    const unsigned char* dna = a->na_circle;
    if (!dev) {
      if ((e = cudaMemcpyAsync(hb, a->bg, nin * sizeof(float), cudaMemcpyHostToDevice, s)) ||
          (e = cudaMemcpyAsync(hs, a->sp, nin * sizeof(float), cudaMemcpyHostToDevice, s)) ||
          (e = cudaMemcpyAsync(na, a->na_circle, (size_t)M * M, cudaMemcpyHostToDevice, s)))
        return e;
      db = hb;
      ds = hs;
      dna = na;
    }
    to_complex_kernel<<<grid_for(nin), kThreads, 0, s>>>(db, Fb, nin);
    to_complex_kernel<<<grid_for(nin), kThreads, 0, s>>>(ds, Fs, nin);
    if ((e = cudaGetLastError()) || (e = fftc2_any(Fb, N, N, nimg, false, fN, fN, s)) ||
        (e = fftc2_any(Fs, N, N, nimg, false, fN, fN, s)))
      return e;
    // deleted bands (1-based): rows round(N cp):N; columns round(N cp):N, or
    // 1:round(N (1 - cp)) with other_corner
    const int r_end = (int)std::floor(N * a->cutout_portion + 0.5) - 1;
    int c_lo = 0, c_hi = r_end;
    if (a->other_corner) {
      c_lo = (int)std::floor(N * (1.0 - a->cutout_portion) + 0.5);
      c_hi = N;
    }
    sideband_kernel<<<1, 1024, 0, s>>>(Fb, N, N, r_end, c_lo, c_hi, sb);
    const int d = a->crop;   // source offset: crop (>= 0) or minus the padding
    centre_crop_kernel<<<grid_for(nmid), kThreads, 0, s>>>(Fb, N, M, d, sb, dna, nimg, Gb);
    centre_crop_kernel<<<grid_for(nmid), kThreads, 0, s>>>(Fs, N, M, d, sb, dna, nimg, Gs);
    peak_kernel<<<nimg, 256, 0, s>>>(Gb, M, dev ? a->peaks : pk);
    if ((e = cudaGetLastError()) || (e = fftc2_any(Gb, M, M, nimg, true, fM, fM, s)) ||
        (e = fftc2_any(Gs, M, M, nimg, true, fM, fM, s)))
      return e;
    float2* outb = dev ? reinterpret_cast<float2*>(a->bg_field) : ob;
    float2* outs = dev ? reinterpret_cast<float2*>(a->sp_field) : os;
    if ((e = launch_crop2d(Gb, outb, M - 4, M - 4, M, M, 2, 2, nimg, s)) ||
        (e = launch_crop2d(Gs, outs, M - 4, M - 4, M, M, 2, 2, nimg, s)))
      return e;
    if ((e = cudaMemcpyAsync(a->sideband, sb, 2 * sizeof(int), cudaMemcpyDeviceToHost, s))) return e;
    if (!dev) {
      if ((e = cudaMemcpyAsync(a->bg_field, ob, nout * sizeof(float2), cudaMemcpyDeviceToHost, s)) ||
          (e = cudaMemcpyAsync(a->sp_field, os, nout * sizeof(float2), cudaMemcpyDeviceToHost, s)) ||
          (e = cudaMemcpyAsync(a->peaks, pk, 7 * (size_t)nimg * sizeof(float), cudaMemcpyDeviceToHost, s)))
        return e;
    }
    return cudaStreamSynchronize(s);
  };
  const cudaError_t e = run();
  if (e != cudaSuccess) {
    cudaGetLastError();
    return hfail(ODT_ERR_CUDA, std::string("odt_hologram_fields: ") + cudaGetErrorString(e));
  }
  return ODT_OK;
}

namespace {
// The arithmetic below follows numpy's complex64 loops (np_complex.cuh):
// x / r (r real) is x * (1 / r) per component (r is promoted to r + 0i),
// r * x (r real) is r * x per component.
// one CTA per image: amean = sum |bg| / plane (summed in double); bg and sp
// divided by amean (conjugated if asked); phase = angle(sp / bg) and
// amp = |sp / bg|
__global__ void __launch_bounds__(1024) norm_phase_kernel(float2* __restrict__ bg, float2* __restrict__ sp,
                                                          long long plane, int conj, float* __restrict__ phase,
                                                          float* __restrict__ amp) {
  __shared__ double red[32];
  __shared__ float amean;
  float2* b = bg + plane * blockIdx.x;
  float2* q = sp + plane * blockIdx.x;
  double s = 0.0;
  for (long long i = threadIdx.x; i < plane; i += blockDim.x) s += (double)cabs_f(b[i]);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < (blockDim.x + 31) / 32 ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) amean = (float)t / (float)plane;
  }
  __syncthreads();
  const float r = 1.0f / amean;
  float* ph = phase + plane * blockIdx.x;
  float* am = amp + plane * blockIdx.x;
  for (long long i = threadIdx.x; i < plane; i += blockDim.x) {
    float2 x = make_float2(__fmul_rn(b[i].x, r), __fmul_rn(b[i].y, r));
    float2 y = make_float2(__fmul_rn(q[i].x, r), __fmul_rn(q[i].y, r));
    if (conj) {
      x.y = -x.y;
      y.y = -y.y;
    }
    b[i] = x;
    q[i] = y;
    const float2 z = cdiv_np(y, x);
    ph[i] = atan2f(z.y, z.x);
    am[i] = cabs_f(z);
  }
}

// sp = (amp * bg) * exp(1i g), g = ((phase - c0) - c1 x) - c2 y with x, y
// the 1-based column / row of the [n1, n2] plane (coef [3, n]: height, x
// and y slopes per image)
__global__ void combine_kernel(const float2* __restrict__ bg, const float* __restrict__ amp,
                               const float* __restrict__ phase, const float* __restrict__ coef, int n1, int n2,
                               long long total, float2* __restrict__ sp) {
  const long long plane = (long long)n1 * n2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long k = i / plane, p = i - k * plane;
    const float y = (float)(p % n1 + 1), x = (float)(p / n1 + 1);
    const float* c = coef + 3 * k;
    const float g = __fsub_rn(__fsub_rn(__fsub_rn(phase[i], c[0]), __fmul_rn(c[1], x)), __fmul_rn(c[2], y));
    float sn, cs;
    sincosf(g, &sn, &cs);
    const float2 b = bg[i];
    const float tr = __fmul_rn(amp[i], b.x), ti = __fmul_rn(amp[i], b.y);
    sp[i] = make_float2(__fsub_rn(__fmul_rn(tr, cs), __fmul_rn(ti, sn)), __fadd_rn(__fmul_rn(tr, sn), __fmul_rn(ti, cs)));
  }
}
}  // namespace

extern "C" odt_status odt_hologram_phase(const odt_hologram_phase_args* a) {
  if (!a || !a->bg || !a->sp || !a->phase || !a->amp)
    return hfail(ODT_ERR_INVALID_ARGUMENT, "odt_hologram_phase: NULL argument");
  if (a->size[0] < 1 || a->size[1] < 1 || a->size[2] < 1)
    return hfail(ODT_ERR_INVALID_ARGUMENT, "odt_hologram_phase: bad sizes");
  for (const void* p : {(const void*)a->bg, (const void*)a->sp, (const void*)a->phase, (const void*)a->amp})
    if (!is_dev(p)) return hfail(ODT_ERR_INVALID_ARGUMENT, "odt_hologram_phase: arrays must be device pointers");
  const long long plane = (long long)a->size[0] * a->size[1];
  norm_phase_kernel<<<a->size[2], 1024, 0, (cudaStream_t)a->stream>>>(
      reinterpret_cast<float2*>(a->bg), reinterpret_cast<float2*>(a->sp), plane, a->conjugate, a->phase, a->amp);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return hfail(ODT_ERR_CUDA, std::string("odt_hologram_phase: ") + cudaGetErrorString(e));
  return ODT_OK;
}

extern "C" odt_status odt_hologram_combine(const odt_hologram_combine_args* a) {
  if (!a || !a->bg || !a->amp || !a->phase || !a->coef || !a->sp)
    return hfail(ODT_ERR_INVALID_ARGUMENT, "odt_hologram_combine: NULL argument");
  if (a->size[0] < 1 || a->size[1] < 1 || a->size[2] < 1)
    return hfail(ODT_ERR_INVALID_ARGUMENT, "odt_hologram_combine: bad sizes");
  for (const void* p : {(const void*)a->bg, (const void*)a->amp, (const void*)a->phase, (const void*)a->coef,
                        (const void*)a->sp})
    if (!is_dev(p)) return hfail(ODT_ERR_INVALID_ARGUMENT, "odt_hologram_combine: arrays must be device pointers");
  const long long total = (long long)a->size[0] * a->size[1] * a->size[2];
  combine_kernel<<<grid_for(total), kThreads, 0, (cudaStream_t)a->stream>>>(
      reinterpret_cast<const float2*>(a->bg), a->amp, a->phase, a->coef, a->size[0], a->size[1], total,
      reinterpret_cast<float2*>(a->sp));
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return hfail(ODT_ERR_CUDA, std::string("odt_hologram_combine: ") + cudaGetErrorString(e));
  return ODT_OK;
}

extern "C" odt_status odt_refocus_2d(const odt_refocus_args* a) {
  if (!a || !a->field || !a->kernel) return hfail(ODT_ERR_INVALID_ARGUMENT, "odt_refocus_2d: NULL argument");
  const int n1 = a->size[0], n2 = a->size[1], n = a->size[2];
  if (n1 < 1 || n2 < 1 || n < 1) return hfail(ODT_ERR_INVALID_ARGUMENT, "odt_refocus_2d: bad sizes");
  cudaStream_t s = (cudaStream_t)0;
  Scratch B;
  B.s = s;
  const long long plane = (long long)n1 * n2, tot = plane * n;
  float2* x = B.get<float2>(tot);
  float2* k = B.get<float2>(plane);
  if (!x || !k) return hfail(ODT_ERR_OUT_OF_MEMORY, "odt_refocus_2d: device allocation failed");
  AnyFft f1{}, f2{};
  std::string why;
  if (!scratch_fft_any(B, n1, &f1, &why) || !scratch_fft_any(B, n2, &f2, &why))
    return hfail(ODT_ERR_UNSUPPORTED, "odt_refocus_2d: " + why);
  auto run = [&]() -> cudaError_t {
    cudaError_t e;
    if ((e = cudaMemcpyAsync(x, a->field, tot * sizeof(float2), cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(k, a->kernel, plane * sizeof(float2), cudaMemcpyHostToDevice, s)) ||
        (e = fftc2_any(x, n1, n2, n, false, f1, f2, s)))
      return e;
    cmul_plane_kernel<<<grid_for(tot), kThreads, 0, s>>>(x, k, plane, tot);
    if ((e = cudaGetLastError()) || (e = fftc2_any(x, n1, n2, n, true, f1, f2, s)) ||
        (e = cudaMemcpyAsync(a->out, x, tot * sizeof(float2), cudaMemcpyDeviceToHost, s)))
      return e;
    return cudaStreamSynchronize(s);
  };
  const cudaError_t e = run();
  if (e != cudaSuccess) {
    cudaGetLastError();
    return hfail(ODT_ERR_CUDA, std::string("odt_refocus_2d: ") + cudaGetErrorString(e));
  }
  return ODT_OK;
}
