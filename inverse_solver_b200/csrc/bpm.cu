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
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <string>

#include "../../include/odt.h"
#include "cbs_kernels.cuh"
#include "scratch.cuh"

namespace odt {
const char* set_last_error(const std::string& msg);  // odt_api.cu
}

using namespace odt;
namespace cg = cooperative_groups;

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

// ---- fused march for 128 x 128 planes
// A cluster of two CTAs per illumination keeps the 128 x 128 plane in shared
// memory for the whole march over z: CTA r holds rows y = 64 r .. 64 r + 63
// (row pitch 129 complex, so column accesses are free of bank conflicts) and
// reads the other half of each column through distributed shared memory.
// Each 128-point transform is done by one warp with the line in registers,
// lane l holding elements l + 32 r (r = 0..3):
//   forward : 4-point DFT over r, twiddles W128^(l k1), then a 32-point
//             decimation-in-frequency DFT across lanes (shuffles); element
//             k1 + 4 brev5(l) of the result ends in lane l, register k1,
//             i.e. at position l + 32 k1 of the line ("permuted" order);
//   inverse : the same steps undone in reverse order (decimation in time
//             across lanes with conjugate twiddles, conjugate twiddles, inverse
//             4-point DFT): permuted input, natural output, unnormalised.
// The spectrum stays in permuted order between slices, so every transform
// reads and writes its line in place.  Per slice (z):
//   x-pass: inverse x-FFT, * (1/N) exp(field_multiplier(:,:,z) * inv_cos),
//           forward x-FFT (one register pass per row, rows of this CTA);
//   y-pass: forward y-FFT, then (except after the last slice)
//           * refocus_kernel and inverse y-FFT of the next slice's
//           ifft2(field .* refocus_kernel) (one register pass per column,
//           columns 64 r .. 64 r + 63 for CTA r).
constexpr int kM = 128;           // plane side
constexpr int kMP = 129;          // shared-memory row pitch (complex)
constexpr int kMH = kM / 2;       // rows per CTA
constexpr int kMarchThreads = 512;

__device__ __forceinline__ int march_perm(int p) {  // position -> frequency
  return (p >> 5) + 4 * (int)(__brev((unsigned)(p & 31)) >> 27);
}

__device__ __forceinline__ float2 shfl_c(float2 v, int m) {
  return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

// per-lane twiddles: w[s] = W_{2h}^(l mod h) for h = 16 >> s, b[k-1] = W128^(l k)
struct MarchTw {
  float2 w[5];
  float2 b[3];
};

__device__ __forceinline__ void march_tw(MarchTw& t, const float2* tw, int l) {
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    const int h = 16 >> s;
    t.w[s] = tw[(l & (h - 1)) * (64 / h)];
  }
#pragma unroll
  for (int k = 1; k < 4; ++k) t.b[k - 1] = tw[l * k];
}

// natural -> permuted, W = exp(-2 pi i / 128)
__device__ __forceinline__ void wfft128_fwd(float2 (&v)[4], const MarchTw& t, int l) {
  const float2 a0 = cadd(v[0], v[2]), a1 = csub(v[0], v[2]);
  const float2 a2 = cadd(v[1], v[3]), a3 = csub(v[1], v[3]);
  const float2 ma3 = make_float2(a3.y, -a3.x);  // -i * a3
  v[0] = cadd(a0, a2);
  v[1] = cmul(cadd(a1, ma3), t.b[0]);
  v[2] = cmul(csub(a0, a2), t.b[1]);
  v[3] = cmul(csub(a1, ma3), t.b[2]);
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    const int h = 16 >> s;
    const bool up = (l & h) == 0;  // upper lane: x_j + x_{j+h}; lower: (x_j - x_{j+h}) W
    const float sg = up ? 1.f : -1.f;
    const float2 w = up ? make_float2(1.f, 0.f) : t.w[s];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float2 p = shfl_c(v[k], h);
      v[k] = cmul(make_float2(fmaf(sg, v[k].x, p.x), fmaf(sg, v[k].y, p.y)), w);
    }
  }
}

// permuted -> natural, unnormalised inverse (W = exp(+2 pi i / 128))
__device__ __forceinline__ void wfft128_inv(float2 (&v)[4], const MarchTw& t, int l) {
#pragma unroll
  for (int s = 4; s >= 0; --s) {
    const int h = 16 >> s;
    const bool up = (l & h) == 0;
    // upper lane: top + bot conj(W); lower lane: top - bot conj(W), i.e.
    // v * ca + partner * cb with (ca, cb) = (1, conj W) or (-conj W, 1)
    const float2 cw = cconj(t.w[s]);
    const float2 ca = up ? make_float2(1.f, 0.f) : make_float2(-cw.x, -cw.y);
    const float2 cb = up ? cw : make_float2(1.f, 0.f);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float2 p = shfl_c(v[k], h);
      const float2 x = v[k];
      v[k] = make_float2(fmaf(x.x, ca.x, fmaf(-x.y, ca.y, fmaf(p.x, cb.x, -p.y * cb.y))),
                         fmaf(x.x, ca.y, fmaf(x.y, ca.x, fmaf(p.x, cb.y, p.y * cb.x))));
    }
  }
  const float2 b1 = cmul(v[1], cconj(t.b[0]));
  const float2 b2 = cmul(v[2], cconj(t.b[1]));
  const float2 b3 = cmul(v[3], cconj(t.b[2]));
  const float2 a0 = cadd(v[0], b2), a1 = csub(v[0], b2);
  const float2 a2 = cadd(b1, b3), a3 = csub(b1, b3);
  const float2 ia3 = make_float2(-a3.y, a3.x);  // i * a3
  v[0] = cadd(a0, a2);
  v[1] = cadd(a1, ia3);
  v[2] = csub(a0, a2);
  v[3] = csub(a1, ia3);
}

// fld [128 * 128, nill]: spectrum of every illumination (natural order)
// before the first slice's refocus multiply; on return the spectrum after
// the last slice's fft2.  Grid: 2 CTAs (one cluster) per illumination.
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kMarchThreads, 1)
bpm_march128_kernel(float2* __restrict__ fld, const float2* __restrict__ rk, const float2* __restrict__ fm,
                    const float* __restrict__ inv_cos, const float2* __restrict__ twg, int nz, float inv_n) {
  extern __shared__ float2 march_sm[];
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  float2* S = march_sm;                       // rows 64 rank .. 64 rank + 63
  float2* tw = march_sm + kMH * kMP;
  float2* const S0 = cluster.map_shared_rank(S, 0);
  float2* const S1 = cluster.map_shared_rank(S, 1);
  const int tid = threadIdx.x, l = tid & 31, w = tid >> 5;
  constexpr int nw = kMarchThreads / 32;
  const int ill = blockIdx.x >> 1;
  float2* F = fld + (long long)ill * kM * kM;
  const float ic = inv_cos ? inv_cos[ill] : 1.f;
  for (int i = tid; i < kM; i += kMarchThreads) tw[i] = twg[i];
  for (int i = tid; i < kMH * kM; i += kMarchThreads) {
    const int px = i & (kM - 1), jy = i >> 7;
    S[px + kMP * jy] = F[march_perm(px) + kM * march_perm(kMH * rank + jy)];
  }
  __syncthreads();
  MarchTw t;
  march_tw(t, tw, l);
  cluster.sync();
  // column px, element y = l + 32 r: rows 0..63 live in CTA 0, 64..127 in CTA 1
  const int ylo = l;  // row inside the owning CTA for r = 0, 2 (r = 1, 3: + 32)
  // the first slice's refocus multiply and inverse y-FFT
  for (int px = kMH * rank + w; px < kMH * rank + kMH; px += nw) {
    const int kx = march_perm(px);
    float2 v[4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
      v[r] = cmul((r < 2 ? S0 : S1)[px + kMP * (ylo + 32 * (r & 1))], rk[kx + kM * march_perm(l + 32 * r)]);
    wfft128_inv(v, t, l);
#pragma unroll
    for (int r = 0; r < 4; ++r) (r < 2 ? S0 : S1)[px + kMP * (ylo + 32 * (r & 1))] = v[r];
  }
  cluster.sync();
  for (int z = 0; z < nz; ++z) {
    const float2* fz = fm + (long long)z * kM * kM;
    for (int jy = w; jy < kMH; jy += nw) {
      const int py = kMH * rank + jy;
      float2 v[4], e4[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        v[r] = S[(l + 32 * r) + kMP * jy];
        e4[r] = fz[(l + 32 * r) + kM * py];  // issued before the transform hides its latency
      }
      wfft128_inv(v, t, l);
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        float2 e = e4[r];
        if (inv_cos) e = cscale(e, ic);
        float sn, cs;
        sincosf(e.y, &sn, &cs);
        const float m = expf(e.x);
        v[r] = cmul(cscale(v[r], inv_n), make_float2(m * cs, m * sn));
      }
      wfft128_fwd(v, t, l);
#pragma unroll
      for (int r = 0; r < 4; ++r) S[(l + 32 * r) + kMP * jy] = v[r];
    }
    cluster.sync();
    const bool more = z + 1 < nz;
    for (int px = kMH * rank + w; px < kMH * rank + kMH; px += nw) {
      const int kx = march_perm(px);
      float2 v[4], k4[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        v[r] = (r < 2 ? S0 : S1)[px + kMP * (ylo + 32 * (r & 1))];
        k4[r] = more ? rk[kx + kM * march_perm(l + 32 * r)] : make_float2(0.f, 0.f);
      }
      wfft128_fwd(v, t, l);
      if (more) {
#pragma unroll
        for (int r = 0; r < 4; ++r) v[r] = cmul(v[r], k4[r]);
        wfft128_inv(v, t, l);
#pragma unroll
        for (int r = 0; r < 4; ++r) (r < 2 ? S0 : S1)[px + kMP * (ylo + 32 * (r & 1))] = v[r];
      } else {
#pragma unroll
        for (int r = 0; r < 4; ++r) F[kx + kM * march_perm(l + 32 * r)] = v[r];
      }
    }
    cluster.sync();  // also keeps this CTA's rows alive until the partner is done
  }
}

constexpr size_t kMarchSmem = sizeof(float2) * (kMH * kMP + kM);

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
  // fused march (shared-memory resident planes) for 128 x 128 fields without
  // the 3D output; ODT_KERNELS=generic keeps the per-slice launches
  const char* kenv = std::getenv("ODT_KERNELS");
  const bool generic = kenv && std::string(kenv) == "generic";
  if (n1 == kM && n2 == kM && !out3d && !generic && nz > 0) {
    BPM_CHECK(cudaFuncSetAttribute(bpm_march128_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)kMarchSmem));
    bpm_march128_kernel<<<2 * nill, kMarchThreads, kMarchSmem, s>>>(fld, rk, fm, inv_cos, f1.tw, nz, inv_n);
    BPM_CHECK(cudaGetLastError());
  } else {
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
