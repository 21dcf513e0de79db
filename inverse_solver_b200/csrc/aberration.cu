// Aberration correction and dirty-field rejection of the field retrieval
// front-end on the GPU.
//
// odt_aberration_pattern, FIELD_EXPERIMENTAL_RETRIEVAL.m:216-352
// (get_aberration_pattern), with the fields [N, N, n]:
//   fE  = fftshift(fft2(ifftshift(output ./ input)))
//   P_k = circshift(exp(1i angle(fE_k .* conj(fE_1))) .* fMask, round(k0s_k)) .* NA
//   phase matching in the order of |k0s| (seq): S = P_seq1, then for each
//     next image b = angle(sum(S .* conj(P_seqi) .* (|S|>0 & |P_seqi|>0))),
//     P_seqi *= exp(1i b), S += P_seqi;  P2 = sum_k P_k (index order)
//   defocus: cc(d) = |sum(exp(rk d) .* exp(-1i angle(P2)) .* NA)|, d* the
//     first maximum; approx = d* rk - d* rk(centre)
//   psf = ifft2c(P2 .* exp(1i approx)) cut to the box of half-width N / dist
//     (dist = 2 |mode(diff(round(k0s(2,:))))|); P3 = fft2c(psf) .* exp(1i approx)
//   pattern = P3 .* exp(-1i angle(P3(centre))) .* NA
//   fields_f = ifft2c(fft2c(fields) .* exp(-1i angle(pattern)))
// The image order, the integer shifts and the box come from k0s on the host
// (single precision, as the reference computes them).  The pixel sums run
// in double with a fixed order; the sum over images in single, in index
// order.  A complex value times a real mask scales both parts (MATLAB's
// real-times-complex product), which fixes the signed zeros that angle()
// sees outside the NA circle.
//
// odt_fft2c: the centred 2D FFT of a stack (the transforms of
// correct_aberration's resolution matching, :356-370).
//
// odt_field_quality, remove_dirty_fields (:399-452) up to its decision: the
// phase (unwrapped with the Goldstein kernels) and amplitude of sp ./ bg,
// per image the standard deviation of |grad(amp_k - amp_1)|^2 and the count
// of phase values above 1.5 max(phase_1) or below 1.5 min(phase_1).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <string>
#include <vector>

#include "../../include/odt.h"
#include "cbs_kernels.cuh"
#include "fft_any.cuh"
#include "np_complex.cuh"
#include "scratch.cuh"

namespace odt {
const char* set_last_error(const std::string& msg);  // odt_api.cu
}

using namespace odt;

namespace {

constexpr int kThreads = 256;
constexpr int kRedBlocks = 148 * 4;   // partial sums per pixel reduction

int grid_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  if (b > 148LL * 16) b = 148LL * 16;
  return (int)(b < 1 ? 1 : b);
}

odt_status afail(odt_status st, const std::string& m) {
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

// x * m for a real m (both parts scaled)
__device__ __forceinline__ float2 rscale(float2 x, float m) { return make_float2(__fmul_rn(x.x, m), __fmul_rn(x.y, m)); }

// block-wide sum of a double2 into red[0] (blockDim.x == kThreads)
__device__ __forceinline__ double2 block_sum(double2 v, double2* red) {
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < kThreads / 32 ? red[threadIdx.x] : make_double2(0.0, 0.0);
    for (int o = 16; o > 0; o >>= 1) {
      v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
      v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
  }
  return v;   // valid in thread 0
}

__global__ void ratio_kernel(const float2* __restrict__ in, const float2* __restrict__ out, long long n,
                             float2* __restrict__ q) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    q[i] = cdiv_np(out[i], in[i]);
}

// P[r, c, k] = NA[r, c] * (fmask[src] * exp(1i angle(F[src, k] conj(F[src, 0])))),
// src = ((r - s1_k) mod N1, (c - s2_k) mod N2)
__global__ void stitch_kernel(const float2* __restrict__ F, int N1, int N2, long long total,
                              const int* __restrict__ shift, const unsigned char* __restrict__ fmask,
                              const unsigned char* __restrict__ na, float2* __restrict__ P) {
  const long long plane = (long long)N1 * N2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long k = i / plane, p = i - k * plane;
    const int r = (int)(p % N1), c = (int)(p / N1);
    int sr = (r - shift[2 * k]) % N1, sc = (c - shift[2 * k + 1]) % N2;
    if (sr < 0) sr += N1;
    if (sc < 0) sc += N2;
    const long long q = sr + (long long)N1 * sc;
    const float2 a = F[q + plane * k], b = F[q];
    const float2 fdp = rscale(unit_phasor(cmul_np(a, make_float2(b.x, -b.y))), fmask[q] ? 1.f : 0.f);
    P[i] = rscale(fdp, na[p] ? 1.f : 0.f);
  }
}

// one phase-matching step: (rotate P_prev by exp(1i b[it-1]) when it > 1),
// S += P_prev (S = P_prev when it == 1), partial sums of
// S .* conj(P_cur) over the pixels where both are non-zero
__global__ void __launch_bounds__(kThreads) match_kernel(float2* __restrict__ P, float2* __restrict__ S,
                                                          long long plane, int kprev, int kcur, int it,
                                                          const float* __restrict__ b, double2* __restrict__ part) {
  __shared__ double2 red[kThreads / 32];
  float2 rot = make_float2(1.f, 0.f);
  if (it > 1) sincosf(b[it - 1], &rot.y, &rot.x);
  float2* pp = P + plane * kprev;
  const float2* pc = P + plane * kcur;
  double2 acc = make_double2(0.0, 0.0);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane;
       i += (long long)gridDim.x * blockDim.x) {
    float2 x = pp[i];
    if (it > 1) {
      x = cmul_np(x, rot);
      pp[i] = x;
    }
    float2 s = it == 1 ? x : make_float2(__fadd_rn(S[i].x, x.x), __fadd_rn(S[i].y, x.y));
    S[i] = s;
    const float2 y = pc[i];
    if ((s.x != 0.f || s.y != 0.f) && (y.x != 0.f || y.y != 0.f)) {
      const float2 t = cmul_np(s, make_float2(y.x, -y.y));
      acc.x += t.x;
      acc.y += t.y;
    }
  }
  const double2 v = block_sum(acc, red);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

// b[it] = angle of the (single-precision) sum of the partials, in a fixed order
__global__ void __launch_bounds__(kThreads) match_reduce_kernel(const double2* __restrict__ part, int nparts, int it,
                                                                 float* __restrict__ b) {
  __shared__ double2 red[kThreads / 32];
  double2 acc = make_double2(0.0, 0.0);
  for (int i = threadIdx.x; i < nparts; i += kThreads) {
    acc.x += part[i].x;
    acc.y += part[i].y;
  }
  const double2 v = block_sum(acc, red);
  if (threadIdx.x == 0) b[it] = atan2f((float)v.y, (float)v.x);
}

// rotate the last image of the order (klast, by b[n-1]; n > 1) and
// P2 = sum_k P_k in index order
__global__ void pupil_sum_kernel(float2* __restrict__ P, long long plane, int n, int klast,
                                 const float* __restrict__ b, float2* __restrict__ P2) {
  float2 rot = make_float2(1.f, 0.f);
  if (n > 1) sincosf(b[n - 1], &rot.y, &rot.x);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane;
       i += (long long)gridDim.x * blockDim.x) {
    if (n > 1) P[i + plane * klast] = cmul_np(P[i + plane * klast], rot);
    float2 acc = P[i];
    for (int k = 1; k < n; ++k) {
      const float2 x = P[i + plane * k];
      acc = make_float2(__fadd_rn(acc.x, x.x), __fadd_rn(acc.y, x.y));
    }
    P2[i] = acc;
  }
}

// partial sums over the pixels of exp(rk d) .* exp(-1i angle(P2)) .* NA, one
// distance per blockIdx.y
__global__ void __launch_bounds__(kThreads) defocus_kernel(const float2* __restrict__ P2,
                                                            const float2* __restrict__ rk,
                                                            const unsigned char* __restrict__ na, long long plane,
                                                            const float* __restrict__ dist,
                                                            double2* __restrict__ part) {
  __shared__ double2 red[kThreads / 32];
  const float d = dist[blockIdx.y];
  double2 acc = make_double2(0.0, 0.0);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane;
       i += (long long)gridDim.x * blockDim.x) {
    const float2 e = cexp_f(make_float2(__fmul_rn(rk[i].x, d), __fmul_rn(rk[i].y, d)));
    const float2 u = unit_phasor(P2[i]);
    const float2 t = rscale(cmul_np(e, make_float2(u.x, -u.y)), na[i] ? 1.f : 0.f);
    acc.x += t.x;
    acc.y += t.y;
  }
  const double2 v = block_sum(acc, red);
  if (threadIdx.x == 0) part[blockIdx.y * (long long)gridDim.x + blockIdx.x] = v;
}

// X .*= exp(1i approx), approx = rk d - rk(centre) d
__global__ void approx_kernel(float2* __restrict__ X, const float2* __restrict__ rk, long long plane,
                              long long centre, float d) {
  const float2 rc = make_float2(__fmul_rn(rk[centre].x, d), __fmul_rn(rk[centre].y, d));
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane;
       i += (long long)gridDim.x * blockDim.x) {
    const float2 a = make_float2(__fsub_rn(__fmul_rn(rk[i].x, d), rc.x), __fsub_rn(__fmul_rn(rk[i].y, d), rc.y));
    X[i] = cmul_np(X[i], cexp_f(make_float2(-a.y, a.x)));   // 1i approx = (-approx.y, approx.x)
  }
}

// X .*= lpf, the box rows [r0, r1] x columns [c0, c1] (0-based, inclusive)
__global__ void box_kernel(float2* __restrict__ X, int N1, long long plane, int r0, int r1, int c0, int c1) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i % N1), c = (int)(i / N1);
    X[i] = rscale(X[i], (r >= r0 && r <= r1 && c >= c0 && c <= c1) ? 1.f : 0.f);
  }
}

// pattern = P3 .* exp(-1i angle(P3(centre))) .* NA; filt = exp(-1i angle(pattern))
__global__ void pattern_kernel(const float2* __restrict__ P3, long long plane, long long centre,
                               const unsigned char* __restrict__ na, float2* __restrict__ pattern,
                               float2* __restrict__ filt) {
  const float2 u = unit_phasor(P3[centre]);
  const float2 ph = make_float2(u.x, -u.y);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < plane;
       i += (long long)gridDim.x * blockDim.x) {
    const float2 p = rscale(cmul_np(P3[i], ph), na[i] ? 1.f : 0.f);
    pattern[i] = p;
    const float2 v = unit_phasor(p);
    filt[i] = make_float2(v.x, -v.y);
  }
}

// x[i] = x[i] * k[i % plane]
__global__ void cmul_plane_np_kernel(float2* __restrict__ x, const float2* __restrict__ k, long long plane,
                                     long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = cmul_np(x[i], k[i % plane]);
}

// phase = angle(sp ./ bg), amp = |sp ./ bg|
__global__ void ratio_phase_kernel(const float2* __restrict__ bg, const float2* __restrict__ sp, long long n,
                                   float* __restrict__ phase, float* __restrict__ amp) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float2 z = cdiv_np(sp[i], bg[i]);
    phase[i] = atan2f(z.y, z.x);
    amp[i] = cabs_f(z);
  }
}

// lim = (fl(max(phase_1) * 1.5), fl(min(phase_1) * 1.5)), one CTA
__global__ void __launch_bounds__(kThreads) phase_limits_kernel(const float* __restrict__ ph, long long plane,
                                                                 float* __restrict__ lim) {
  __shared__ float smax[kThreads / 32], smin[kThreads / 32];
  float mx = -INFINITY, mn = INFINITY;
  for (long long i = threadIdx.x; i < plane; i += kThreads) {
    mx = fmaxf(mx, ph[i]);
    mn = fminf(mn, ph[i]);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
  }
  if ((threadIdx.x & 31) == 0) {
    smax[threadIdx.x >> 5] = mx;
    smin[threadIdx.x >> 5] = mn;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kThreads / 32; ++w) {
      mx = fmaxf(mx, smax[w]);
      mn = fminf(mn, smin[w]);
    }
    lim[0] = __fmul_rn(mx, 1.5f);
    lim[1] = __fmul_rn(mn, 1.5f);
  }
}

// g = XX^2 + YY^2 of [XX, YY] = gradient(amp_k - amp_1) at pixel (r, c)
// (central differences inside, one-sided at the edges; XX along columns)
__device__ __forceinline__ float grad_energy(const float* __restrict__ a, const float* __restrict__ a1, int N1,
                                             int N2, int r, int c) {
  auto f = [&](int rr, int cc) {
    const long long q = rr + (long long)N1 * cc;
    return __fsub_rn(a[q], a1[q]);
  };
  float gx, gy;
  if (N2 == 1) gx = 0.f;
  else if (c == 0) gx = __fsub_rn(f(r, 1), f(r, 0));
  else if (c == N2 - 1) gx = __fsub_rn(f(r, N2 - 1), f(r, N2 - 2));
  else gx = __fsub_rn(f(r, c + 1), f(r, c - 1)) / 2.f;
  if (N1 == 1) gy = 0.f;
  else if (r == 0) gy = __fsub_rn(f(1, c), f(0, c));
  else if (r == N1 - 1) gy = __fsub_rn(f(N1 - 1, c), f(N1 - 2, c));
  else gy = __fsub_rn(f(r + 1, c), f(r - 1, c)) / 2.f;
  return __fadd_rn(__fmul_rn(gx, gx), __fmul_rn(gy, gy));
}

// one CTA per image: std of the gradient energy (two passes, double) and the
// count of phase values outside (lim[1], lim[0])
__global__ void __launch_bounds__(kThreads) quality_kernel(const float* __restrict__ phase,
                                                            const float* __restrict__ amp, int N1, int N2,
                                                            const float* __restrict__ lim, float* __restrict__ sd,
                                                            long long* __restrict__ count) {
  __shared__ double2 red[kThreads / 32];
  __shared__ double mean;
  const long long plane = (long long)N1 * N2;
  const float* a = amp + plane * blockIdx.x;
  const float* ph = phase + plane * blockIdx.x;
  const float hi = lim[0], lo = lim[1];
  double2 acc = make_double2(0.0, 0.0);
  for (long long i = threadIdx.x; i < plane; i += kThreads) {
    acc.x += grad_energy(a, amp, N1, N2, (int)(i % N1), (int)(i / N1));
    acc.y += (ph[i] > hi ? 1.0 : 0.0) + (ph[i] < lo ? 1.0 : 0.0);
  }
  double2 v = block_sum(acc, red);
  if (threadIdx.x == 0) {
    mean = v.x / (double)plane;
    count[blockIdx.x] = (long long)v.y;
  }
  __syncthreads();
  double ss = 0.0;
  for (long long i = threadIdx.x; i < plane; i += kThreads) {
    const double dlt = grad_energy(a, amp, N1, N2, (int)(i % N1), (int)(i / N1)) - mean;
    ss += dlt * dlt;
  }
  __syncthreads();
  v = block_sum(make_double2(ss, 0.0), red);
  if (threadIdx.x == 0) sd[blockIdx.x] = plane > 1 ? (float)sqrt(v.x / (double)(plane - 1)) : 0.f;
}

#define A_CHECK(call)       \
  do {                      \
    cudaError_t e_ = (call); \
    if (e_ != cudaSuccess) return e_; \
  } while (0)

}  // namespace

extern "C" odt_status odt_aberration_pattern(const odt_aberration_args* a) {
  if (!a || !a->input_field || !a->output_field || !a->k0s || !a->pupil_mask || !a->na_circle ||
      !a->refocusing_kernel || !a->dist_list || !a->pattern || !a->input_out || !a->output_out)
    return afail(ODT_ERR_INVALID_ARGUMENT, "odt_aberration_pattern: NULL argument");
  const int N1 = a->size[0], N2 = a->size[1], n = a->size[2], nd = a->n_dist;
  if (N1 < 2 || N2 < 2 || n < 2 || nd < 1 || nd > 65535)
    return afail(ODT_ERR_INVALID_ARGUMENT,
                 "odt_aberration_pattern: bad sizes (at least 2 x 2 pixels, 2 fields and 1 distance)");
  if (a->memory != ODT_MEM_HOST && a->memory != ODT_MEM_DEVICE)
    return afail(ODT_ERR_INVALID_ARGUMENT, "odt_aberration_pattern: bad memory flag");
  const bool dev = a->memory == ODT_MEM_DEVICE;
  if (dev && (!is_dev(a->input_field) || !is_dev(a->output_field) || !is_dev(a->pattern) ||
              !is_dev(a->input_out) || !is_dev(a->output_out)))
    return afail(ODT_ERR_INVALID_ARGUMENT, "odt_aberration_pattern: ODT_MEM_DEVICE with a host pointer");

  // ---- host side: image order, integer shifts, low-pass box (single precision)
  const float* k0 = a->k0s;
  std::vector<int> seq(n), shift(2 * n);
  std::vector<float> mag(n);
  for (int k = 0; k < n; ++k) {
    mag[k] = std::sqrt(k0[2 * k] * k0[2 * k] + k0[2 * k + 1] * k0[2 * k + 1]);
    shift[2 * k] = (int)std::round(k0[2 * k]);
    shift[2 * k + 1] = (int)std::round(k0[2 * k + 1]);
    seq[k] = k;
  }
  std::stable_sort(seq.begin(), seq.end(), [&](int x, int y) { return mag[x] < mag[y]; });
  // mode of diff(round(k0s(2, :))): the most frequent, the smallest on ties
  std::map<float, int> freq;
  for (int k = 1; k < n; ++k) ++freq[std::round(k0[2 * k + 1]) - std::round(k0[2 * k - 1])];
  float mode = 0.f;
  int best = 0;
  for (const auto& kv : freq)
    if (kv.second > best) {
      best = kv.second;
      mode = kv.first;
    }
  const float dist = std::fabs(mode) * 2.f;
  if (!(dist > 0.f))
    return afail(ODT_ERR_INVALID_ARGUMENT,
                 "odt_aberration_pattern: the most frequent step of round(k0s(2,:)) is 0 (no low-pass box)");
  const int cr = N1 / 2, cc = N2 / 2;   // floor(N/2 + 1), 0-based
  const int r0 = cr - (int)std::floor((float)N1 / dist), r1 = cr + (int)std::ceil((float)N1 / dist);
  const int c0 = cc - (int)std::floor((float)N2 / dist), c1 = cc + (int)std::ceil((float)N2 / dist);
  if (r0 < 0 || c0 < 0 || r1 > N1 - 1 || c1 > N2 - 1)
    return afail(ODT_ERR_INVALID_ARGUMENT, "odt_aberration_pattern: the low-pass box leaves the image");
  std::vector<float> dl(nd);
  for (int i = 0; i < nd; ++i) dl[i] = (float)a->dist_list[i];

  cudaStream_t s = dev ? (cudaStream_t)a->stream : (cudaStream_t)0;
  Scratch B;
  B.s = s;
  const long long plane = (long long)N1 * N2, tot = plane * n;
  float2* fin = dev ? nullptr : B.get<float2>(tot);
  float2* fout = dev ? nullptr : B.get<float2>(tot);
  float2* Q = B.get<float2>(tot);
  float2* P = B.get<float2>(tot);
  float2* S = B.get<float2>(plane);
  float2* P2 = B.get<float2>(plane);
  float2* pat = dev ? nullptr : B.get<float2>(plane);
  float2* filt = B.get<float2>(plane);
  float2* rk = B.get<float2>(plane);
  unsigned char* fm = B.get<unsigned char>(plane);
  unsigned char* na = B.get<unsigned char>(plane);
  int* dsh = B.get<int>(2 * n);
  float* bv = B.get<float>(n);
  float* ddl = B.get<float>(nd);
  double2* part = B.get<double2>((size_t)kRedBlocks * nd);
  if (!Q || !P || !S || !P2 || !filt || !rk || !fm || !na || !dsh || !bv || !ddl || !part ||
      (!dev && (!fin || !fout || !pat)))
    return afail(ODT_ERR_OUT_OF_MEMORY, "odt_aberration_pattern: device allocation failed");
  AnyFft f1{}, f2{};
  std::string why;
  if (!scratch_fft_any(B, N1, &f1, &why) || !scratch_fft_any(B, N2, &f2, &why))
    return afail(ODT_ERR_UNSUPPORTED, "odt_aberration_pattern: " + why);
  int chosen = 0;
  auto run = [&]() -> cudaError_t {
    const cudaMemcpyKind h2d = cudaMemcpyHostToDevice;
    A_CHECK(cudaMemcpyAsync(rk, a->refocusing_kernel, plane * sizeof(float2), h2d, s));
    A_CHECK(cudaMemcpyAsync(fm, a->pupil_mask, plane, h2d, s));
    A_CHECK(cudaMemcpyAsync(na, a->na_circle, plane, h2d, s));
    A_CHECK(cudaMemcpyAsync(dsh, shift.data(), 2 * n * sizeof(int), h2d, s));
    A_CHECK(cudaMemcpyAsync(ddl, dl.data(), nd * sizeof(float), h2d, s));
    const float2* in = reinterpret_cast<const float2*>(a->input_field);
    const float2* out = reinterpret_cast<const float2*>(a->output_field);
    if (!dev) {
      A_CHECK(cudaMemcpyAsync(fin, in, tot * sizeof(float2), h2d, s));
      A_CHECK(cudaMemcpyAsync(fout, out, tot * sizeof(float2), h2d, s));
      in = fin;
      out = fout;
    }
    // stitched pupil
    ratio_kernel<<<grid_for(tot), kThreads, 0, s>>>(in, out, tot, Q);
    A_CHECK(cudaGetLastError());
    A_CHECK(fftc2_any(Q, N1, N2, n, false, f1, f2, s));
    stitch_kernel<<<grid_for(tot), kThreads, 0, s>>>(Q, N1, N2, tot, dsh, fm, na, P);
    A_CHECK(cudaGetLastError());
    for (int it = 1; it < n; ++it) {
      match_kernel<<<kRedBlocks, kThreads, 0, s>>>(P, S, plane, seq[it - 1], seq[it], it, bv, part);
      match_reduce_kernel<<<1, kThreads, 0, s>>>(part, kRedBlocks, it, bv);
    }
    pupil_sum_kernel<<<grid_for(plane), kThreads, 0, s>>>(P, plane, n, seq[n - 1], bv, P2);
    // defocus search
    defocus_kernel<<<dim3(kRedBlocks, nd), kThreads, 0, s>>>(P2, rk, na, plane, ddl, part);
    A_CHECK(cudaGetLastError());
    std::vector<double2> hp((size_t)kRedBlocks * nd);
    A_CHECK(cudaMemcpyAsync(hp.data(), part, hp.size() * sizeof(double2), cudaMemcpyDeviceToHost, s));
    A_CHECK(cudaStreamSynchronize(s));
    float cbest = -1.f;
    for (int j = 0; j < nd; ++j) {
      double re = 0.0, im = 0.0;
      for (int i = 0; i < kRedBlocks; ++i) {
        re += hp[(size_t)j * kRedBlocks + i].x;
        im += hp[(size_t)j * kRedBlocks + i].y;
      }
      const float fr = (float)re, fi = (float)im;
      const float c = (float)std::sqrt((double)fr * fr + (double)fi * fi);
      if (c > cbest) {
        cbest = c;
        chosen = j;
      }
    }
    const float d = dl[chosen];
    const long long centre = cr + (long long)N1 * cc;
    // low-passed pupil and the pattern
    approx_kernel<<<grid_for(plane), kThreads, 0, s>>>(P2, rk, plane, centre, d);
    A_CHECK(cudaGetLastError());
    A_CHECK(fftc2_any(P2, N1, N2, 1, true, f1, f2, s));
    box_kernel<<<grid_for(plane), kThreads, 0, s>>>(P2, N1, plane, r0, r1, c0, c1);
    A_CHECK(cudaGetLastError());
    A_CHECK(fftc2_any(P2, N1, N2, 1, false, f1, f2, s));
    approx_kernel<<<grid_for(plane), kThreads, 0, s>>>(P2, rk, plane, centre, d);
    float2* dpat = dev ? reinterpret_cast<float2*>(a->pattern) : pat;
    pattern_kernel<<<grid_for(plane), kThreads, 0, s>>>(P2, plane, centre, na, dpat, filt);
    A_CHECK(cudaGetLastError());
    // corrected fields
    float2* oi = dev ? reinterpret_cast<float2*>(a->input_out) : fin;
    float2* oo = dev ? reinterpret_cast<float2*>(a->output_out) : fout;
    if (dev) {
      A_CHECK(cudaMemcpyAsync(oi, in, tot * sizeof(float2), cudaMemcpyDeviceToDevice, s));
      A_CHECK(cudaMemcpyAsync(oo, out, tot * sizeof(float2), cudaMemcpyDeviceToDevice, s));
    }
    for (float2* x : {oi, oo}) {
      A_CHECK(fftc2_any(x, N1, N2, n, false, f1, f2, s));
      cmul_plane_np_kernel<<<grid_for(tot), kThreads, 0, s>>>(x, filt, plane, tot);
      A_CHECK(cudaGetLastError());
      A_CHECK(fftc2_any(x, N1, N2, n, true, f1, f2, s));
    }
    if (!dev) {
      const cudaMemcpyKind d2h = cudaMemcpyDeviceToHost;
      A_CHECK(cudaMemcpyAsync(a->pattern, pat, plane * sizeof(float2), d2h, s));
      A_CHECK(cudaMemcpyAsync(a->input_out, fin, tot * sizeof(float2), d2h, s));
      A_CHECK(cudaMemcpyAsync(a->output_out, fout, tot * sizeof(float2), d2h, s));
    }
    return cudaStreamSynchronize(s);
  };
  const cudaError_t e = run();
  if (e != cudaSuccess) {
    cudaGetLastError();
    return afail(ODT_ERR_CUDA, std::string("odt_aberration_pattern: ") + cudaGetErrorString(e));
  }
  if (a->chosen) *a->chosen = chosen;
  return ODT_OK;
}

extern "C" odt_status odt_fft2c(const odt_fft2c_args* a) {
  if (!a || !a->data) return afail(ODT_ERR_INVALID_ARGUMENT, "odt_fft2c: NULL argument");
  const int N1 = a->size[0], N2 = a->size[1], n = a->size[2];
  if (N1 < 1 || N2 < 1 || n < 1) return afail(ODT_ERR_INVALID_ARGUMENT, "odt_fft2c: bad sizes");
  if (a->memory != ODT_MEM_HOST && a->memory != ODT_MEM_DEVICE)
    return afail(ODT_ERR_INVALID_ARGUMENT, "odt_fft2c: bad memory flag");
  const bool dev = a->memory == ODT_MEM_DEVICE;
  if (dev && !is_dev(a->data)) return afail(ODT_ERR_INVALID_ARGUMENT, "odt_fft2c: ODT_MEM_DEVICE with a host pointer");
  cudaStream_t s = dev ? (cudaStream_t)a->stream : (cudaStream_t)0;
  Scratch B;
  B.s = s;
  const long long tot = (long long)N1 * N2 * n;
  float2* x = dev ? reinterpret_cast<float2*>(a->data) : B.get<float2>(tot);
  if (!x) return afail(ODT_ERR_OUT_OF_MEMORY, "odt_fft2c: device allocation failed");
  AnyFft f1{}, f2{};
  std::string why;
  if (!scratch_fft_any(B, N1, &f1, &why) || !scratch_fft_any(B, N2, &f2, &why))
    return afail(ODT_ERR_UNSUPPORTED, "odt_fft2c: " + why);
  auto run = [&]() -> cudaError_t {
    if (!dev) A_CHECK(cudaMemcpyAsync(x, a->data, tot * sizeof(float2), cudaMemcpyHostToDevice, s));
    A_CHECK(fftc2_any(x, N1, N2, n, a->inverse != 0, f1, f2, s));
    if (!dev) A_CHECK(cudaMemcpyAsync(a->data, x, tot * sizeof(float2), cudaMemcpyDeviceToHost, s));
    return cudaStreamSynchronize(s);
  };
  const cudaError_t e = run();
  if (e != cudaSuccess) {
    cudaGetLastError();
    return afail(ODT_ERR_CUDA, std::string("odt_fft2c: ") + cudaGetErrorString(e));
  }
  return ODT_OK;
}

extern "C" odt_status odt_field_quality(const odt_field_quality_args* a) {
  if (!a || !a->bg || !a->sp || !a->gradient_std || !a->outside_count)
    return afail(ODT_ERR_INVALID_ARGUMENT, "odt_field_quality: NULL argument");
  const int N1 = a->size[0], N2 = a->size[1], n = a->size[2];
  if (N1 < 2 || N2 < 2 || n < 1) return afail(ODT_ERR_INVALID_ARGUMENT, "odt_field_quality: bad sizes");
  if (a->memory != ODT_MEM_HOST && a->memory != ODT_MEM_DEVICE)
    return afail(ODT_ERR_INVALID_ARGUMENT, "odt_field_quality: bad memory flag");
  const bool dev = a->memory == ODT_MEM_DEVICE;
  if (dev && (!is_dev(a->bg) || !is_dev(a->sp)))
    return afail(ODT_ERR_INVALID_ARGUMENT, "odt_field_quality: ODT_MEM_DEVICE with a host pointer");
  cudaStream_t s = dev ? (cudaStream_t)a->stream : (cudaStream_t)0;
  const long long plane = (long long)N1 * N2, tot = plane * n;
  odt_status st = ODT_OK;
  {
    Scratch B;
    B.s = s;
    float2* hb = dev ? nullptr : B.get<float2>(tot);
    float2* hs = dev ? nullptr : B.get<float2>(tot);
    float* ph = B.get<float>(tot);
    float* uw = B.get<float>(tot);
    float* amp = B.get<float>(tot);
    float* lim = B.get<float>(2);
    float* sd = B.get<float>(n);
    long long* cnt = B.get<long long>(n);
    if (!ph || !uw || !amp || !lim || !sd || !cnt || (!dev && (!hb || !hs)))
      return afail(ODT_ERR_OUT_OF_MEMORY, "odt_field_quality: device allocation failed");
    const float2* bg = reinterpret_cast<const float2*>(a->bg);
    const float2* sp = reinterpret_cast<const float2*>(a->sp);
    cudaError_t e = cudaSuccess;
    if (!dev) {
      if ((e = cudaMemcpyAsync(hb, bg, tot * sizeof(float2), cudaMemcpyHostToDevice, s)) == cudaSuccess)
        e = cudaMemcpyAsync(hs, sp, tot * sizeof(float2), cudaMemcpyHostToDevice, s);
      bg = hb;
      sp = hs;
    }
    if (e == cudaSuccess) {
      ratio_phase_kernel<<<grid_for(tot), kThreads, 0, s>>>(bg, sp, tot, ph, amp);
      e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
      cudaGetLastError();
      return afail(ODT_ERR_CUDA, std::string("odt_field_quality: ") + cudaGetErrorString(e));
    }
    odt_unwrap_args u{};
    u.size[0] = N1;
    u.size[1] = N2;
    u.size[2] = n;
    u.phase_in = ph;
    u.phase_out = uw;
    u.memory = ODT_MEM_DEVICE;
    u.stream = s;
    st = odt_unwrap_goldstein(&u);
    if (st == ODT_OK) {
      phase_limits_kernel<<<1, kThreads, 0, s>>>(uw, plane, lim);
      quality_kernel<<<n, kThreads, 0, s>>>(uw, amp, N1, N2, lim, sd, cnt);
      if ((e = cudaGetLastError()) == cudaSuccess &&
          (e = cudaMemcpyAsync(a->gradient_std, sd, n * sizeof(float), cudaMemcpyDeviceToHost, s)) ==
              cudaSuccess &&
          (e = cudaMemcpyAsync(a->outside_count, cnt, n * sizeof(long long), cudaMemcpyDeviceToHost, s)) ==
              cudaSuccess)
        e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) {
        cudaGetLastError();
        st = afail(ODT_ERR_CUDA, std::string("odt_field_quality: ") + cudaGetErrorString(e));
      }
    }
  }
  return st;
}
