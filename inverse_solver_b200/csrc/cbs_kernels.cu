// CUDA kernels of the convergent-Born-series solver (sm_100a).
//
// Born iteration jj (FORWARD_SOLVER_CONVERGENT_BORN.m:577-643), for all
// illuminations of a batch at once, is three kinds of launch:
//   born_x(jj)  : [inverse x-FFT of iteration jj-1 -> CBS update of jj-1]
//                 -> source term of jj -> forward x-FFT
//   fft_cols    : y-FFT (forward), in place
//   born_z(jj)  : forward z-FFT -> Green's multiply (evaluated on the fly,
//                 1/N folded in) -> inverse z-FFT, in place
//   fft_cols    : y-FFT (inverse), in place
// so each iteration streams the spectral array T through HBM four times and
// Field_n, Field, V once (the update and the next source term are fused into
// the x-pass).  The two interleaved half-series of the reference (:634-642,
// the `temp` bookkeeping of jj = 2, 3) are handled without an extra buffer:
// after jj = 2 the Field array keeps Field_n(1) and the jj = 3 update forms
// Field = (Field_n(1) + Field_n(2)) + Field_n(3), Field_n = Field_n(3) +
// Field_n(1), which is the reference's order of additions.
#include <cstdio>

#include "cbs_kernels.cuh"
#include "tile_launch.cuh"

namespace odt {

namespace {

constexpr int kThreads = 256;  // elementwise kernels

// ------------------------------------------------------ elementwise stages
__global__ void mul_plane_kernel(const float2* in, float2* out, float2* keep, const float* filt,
                                 long long plane, long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const float2 v = cscale(in[i], filt[i % plane]);
    out[i] = v;
    if (keep) keep[i] = v;
  }
}

__global__ void pad2d_kernel(const float2* in, float2* out, int n0, int n1, int m0, int m1,
                             int o0, int o1, long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int X = (int)(i % m0);
    const long long t = i / m0;
    const int Y = (int)(t % m1);
    const long long b = t / m1;
    const int x = X - o0, y = Y - o1;
    float2 v = make_float2(0.f, 0.f);
    if ((unsigned)x < (unsigned)n0 && (unsigned)y < (unsigned)n1)
      v = in[x + (long long)n0 * (y + (long long)n1 * b)];
    out[i] = v;
  }
}

__global__ void crop2d_kernel(const float2* in, float2* out, int n0, int n1, int m0, int m1,
                              int o0, int o1, long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % n0);
    const long long t = i / n0;
    const int y = (int)(t % n1);
    const long long b = t / n1;
    out[i] = in[(x + o0) + (long long)m0 * ((y + o1) + (long long)m1 * b)];
  }
}

__global__ void refocus_expand_kernel(const float2* sk, const float2* ref, float2* conv, int c0,
                                      int c1, int rz, long long total) {
  const long long plane = (long long)c0 * c1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long p = i % plane;
    const long long t = i / plane;
    const long long z = t % rz;
    const long long b = t / rz;
    conv[i] = cmul(sk[p + plane * b], ref[p + plane * z]);
  }
}

__global__ void crop_volume_kernel(const float2* conv, float2* einc, int c0, int c1, int rx,
                                   int ry, int rz, int o0, int o1, long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int x = (int)(i % rx);
    long long t = i / rx;
    const int y = (int)(t % ry);
    t /= ry;  // = z + rz * b
    einc[i] = conv[(x + o0) + (long long)c0 * ((y + o1) + (long long)c1 * t)];
  }
}

__global__ void emitter_kernel(BornArgs a, float2* conv, int c0, int c1, int o0, int o1,
                               float dV, long long total) {
  const long long est = (long long)a.rx * a.ry * a.rz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int X = (int)(i % c0);
    long long t = i / c0;
    const int Y = (int)(t % c1);
    t /= c1;
    const int z = (int)(t % a.rz);
    const long long b = t / a.rz;
    const int x = X - o0, y = Y - o1;
    float2 v = make_float2(0.f, 0.f);
    if ((unsigned)x < (unsigned)a.rx && (unsigned)y < (unsigned)a.ry) {
      const float2 f = a.Fout[b * est + x + (long long)a.rx * (y + (long long)a.ry * z)];
      const float2 V = a.V[(x + a.rx0) + (long long)a.px * ((y + a.ry0) + (long long)a.py * (z + a.rz0))];
      const float2 pot = make_float2(V.x, V.y + a.eps);
      v = cscale(cmul(f, pot), dV);
    }
    conv[i] = v;
  }
}

__global__ void zreduce_kernel(const float2* conv, const float2* Kt, const float2* Kr, float2* tk,
                               float2* rk, int c0, int c1, int rz, long long total) {
  const long long plane = (long long)c0 * c1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long p = i % plane;
    const long long b = i / plane;
    float2 st = make_float2(0.f, 0.f), sr = make_float2(0.f, 0.f);
    const float2* e = conv + b * plane * rz + p;
    for (int z = 0; z < rz; ++z) {
      const float2 v = e[plane * z];
      if (Kt) st = cadd(st, cmul(v, Kt[p + plane * z]));
      if (Kr) sr = cadd(sr, cmul(v, Kr[p + plane * z]));
    }
    if (tk) tk[i] = st;
    if (rk) rk[i] = sr;
  }
}

__global__ void combine_kernel(const float2* x, const float2* add, const float* filt, float2* out,
                               long long plane, long long total) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    float2 v = x[i];
    if (add) v = cadd(v, add[i]);
    out[i] = cscale(v, filt[i % plane]);
  }
}

__global__ void count_nonfinite_kernel(const float2* x, long long n, unsigned int* count) {
  unsigned int local = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float2 v = x[i];
    if (!isfinite(v.x) || !isfinite(v.y)) ++local;
  }
  if (local) atomicAdd(count, local);
}

__global__ void residual_kernel(const float2* trans, const float2* meas, float2* adj_in,
                                long long n, double* err) {
  double local = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float2 d = csub(trans[i], meas[i]);
    local += (double)d.x * d.x + (double)d.y * d.y;
    adj_in[i] = cconj(d);
  }
  __shared__ double red[kThreads / 32];
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = local;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) atomicAdd(err, v);
  }
}

__global__ void grad_accumulate_kernel(const float2* E, const float2* A, float2* acc, int rx,
                                       int ry, int rz, int nb) {
  const long long n = (long long)rx * ry * rz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const long long plane = (long long)rx * ry;
    const long long z = i / plane;
    const long long iflip = i + (rz - 1 - 2 * z) * plane;  // (x, y, rz-1-z)
    float2 s = acc[i];
    for (int b = 0; b < nb; ++b) {
      const float2 e = E[i + b * n];
      const float2 a = A[iflip + b * n];
      s = cadd(s, cmul(cconj(e), cconj(a)));
    }
    acc[i] = s;
  }
}

__global__ void grad_finalize_kernel(const float2* acc, float2* grad, long long n, float n_ill) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const float2 m = make_float2(acc[i].x / n_ill, acc[i].y / n_ill);
    grad[i] = make_float2(m.y, -m.x);  // -(1i * m)
  }
}

int grid_for(long long total) {
  long long g = (total + kThreads - 1) / kThreads;
  const long long cap = 148LL * 16;  // enough resident blocks; grid-stride beyond
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace

size_t fft_smem_bytes(int n, int W, int kind) {
  switch (kind) {
    case kKindLines:
      return align16(sizeof(float2) * (size_t)n) + 2 * sizeof(float2) * (size_t)W * smem_line_ld(n);
    case kKindBornX: return born_x_smem(n, W);
    case kKindBornZ: return col_smem(n, W, sizeof(float) * W);
    default: return col_smem(n, W, 0);
  }
}

// radix classes 0-3 (radices <= 8, <= 15, <= 19, <= 31) each have device kernels
#define ODT_CLS_DISPATCH(cls, F, ...)                 \
  switch (cls) {                                      \
    case 0: return F<0>(__VA_ARGS__);                 \
    case 1: return F<1>(__VA_ARGS__);                 \
    case 2: return F<2>(__VA_ARGS__);                 \
    default: return F<3>(__VA_ARGS__);                \
  }

cudaError_t launch_born_x(const BornArgs& a, int mode, int jj, const DevFft& fx, cudaStream_t s) {
  const int nty = (a.py + fx.W - 1) / fx.W;
  const unsigned blocks = (unsigned)((long long)nty * a.pz * a.nbatch);
  const size_t sm = fft_smem_bytes(fx.plan.n, fx.W, kKindBornX);
  ODT_CLS_DISPATCH(fx.plan.rclass, born_x_launch, a, mode, jj, fx, blocks, sm, s)
}

cudaError_t launch_born_z(const BornArgs& a, int jj, const DevFft& fz, cudaStream_t s) {
  const long long n0 = (long long)a.px * a.py;
  const long long ntile = (n0 + fz.W - 1) / fz.W;
  const unsigned blocks = (unsigned)(ntile * a.nbatch);
  const size_t sm = fft_smem_bytes(fz.plan.n, fz.W, kKindBornZ);
  ODT_CLS_DISPATCH(fz.plan.rclass, born_z_launch, a, jj, fz, blocks, sm, s)
}

cudaError_t launch_fft_lines(const float2* in, float2* out, long long nlines, int in_shift,
                             int out_shift, float scale, bool inverse, const DevFft& f,
                             cudaStream_t s) {
  const unsigned blocks = (unsigned)((nlines + f.W - 1) / f.W);
  const size_t sm = fft_smem_bytes(f.plan.n, f.W, kKindLines);
  ODT_CLS_DISPATCH(f.plan.rclass, lines_launch, in, out, nlines, in_shift, out_shift, scale,
                   inverse, f, blocks, sm, s)
}

cudaError_t launch_fft_cols(const float2* in, float2* out, long long n0, long long n2,
                            int in_shift, int out_shift, float scale, bool inverse,
                            const DevFft& f, cudaStream_t s) {
  const long long ntile = (n0 + f.W - 1) / f.W;
  const unsigned blocks = (unsigned)(ntile * n2);
  const size_t sm = fft_smem_bytes(f.plan.n, f.W, kKindCols);
  const bool sh = in_shift != 0 || out_shift != 0 || scale != 1.0f;
  ODT_CLS_DISPATCH(f.plan.rclass, cols_launch, in, out, n0, n2, in_shift, out_shift, scale,
                   inverse, sh, f, blocks, sm, s)
}

cudaError_t launch_mul_plane(const float2* in, float2* out, float2* keep, const float* filt,
                             long long plane, long long total, cudaStream_t s) {
  mul_plane_kernel<<<grid_for(total), kThreads, 0, s>>>(in, out, keep, filt, plane, total);
  return cudaGetLastError();
}

cudaError_t launch_pad2d(const float2* in, float2* out, int n0, int n1, int m0, int m1, int o0,
                         int o1, long long nb, cudaStream_t s) {
  const long long total = (long long)m0 * m1 * nb;
  pad2d_kernel<<<grid_for(total), kThreads, 0, s>>>(in, out, n0, n1, m0, m1, o0, o1, total);
  return cudaGetLastError();
}

cudaError_t launch_crop2d(const float2* in, float2* out, int n0, int n1, int m0, int m1, int o0,
                          int o1, long long nb, cudaStream_t s) {
  const long long total = (long long)n0 * n1 * nb;
  crop2d_kernel<<<grid_for(total), kThreads, 0, s>>>(in, out, n0, n1, m0, m1, o0, o1, total);
  return cudaGetLastError();
}

cudaError_t launch_refocus_expand(const float2* sk, const float2* refocus, float2* conv, int c0,
                                  int c1, int rz, long long nb, cudaStream_t s) {
  const long long total = (long long)c0 * c1 * rz * nb;
  refocus_expand_kernel<<<grid_for(total), kThreads, 0, s>>>(sk, refocus, conv, c0, c1, rz, total);
  return cudaGetLastError();
}

cudaError_t launch_crop_volume(const float2* conv, float2* einc, int c0, int c1, int rx, int ry,
                               int rz, int o0, int o1, long long nb, cudaStream_t s) {
  const long long total = (long long)rx * ry * rz * nb;
  crop_volume_kernel<<<grid_for(total), kThreads, 0, s>>>(conv, einc, c0, c1, rx, ry, rz, o0, o1,
                                                         total);
  return cudaGetLastError();
}

cudaError_t launch_emitter(const BornArgs& a, float2* conv, int c0, int c1, int o0, int o1,
                           float dV, cudaStream_t s) {
  const long long total = (long long)c0 * c1 * a.rz * a.nbatch;
  emitter_kernel<<<grid_for(total), kThreads, 0, s>>>(a, conv, c0, c1, o0, o1, dV, total);
  return cudaGetLastError();
}

cudaError_t launch_zreduce(const float2* conv, const float2* Kt, const float2* Kr, float2* tk,
                           float2* rk, int c0, int c1, int rz, long long nb, cudaStream_t s) {
  const long long total = (long long)c0 * c1 * nb;
  zreduce_kernel<<<grid_for(total), kThreads, 0, s>>>(conv, Kt, Kr, tk, rk, c0, c1, rz, total);
  return cudaGetLastError();
}

cudaError_t launch_combine(const float2* x, const float2* add, const float* filt, float2* out,
                           long long plane, long long total, cudaStream_t s) {
  combine_kernel<<<grid_for(total), kThreads, 0, s>>>(x, add, filt, out, plane, total);
  return cudaGetLastError();
}

cudaError_t launch_residual(const float2* trans, const float2* meas, float2* adj_in, long long n,
                            double* err, cudaStream_t s) {
  residual_kernel<<<grid_for(n), kThreads, 0, s>>>(trans, meas, adj_in, n, err);
  return cudaGetLastError();
}

cudaError_t launch_grad_accumulate(const float2* E, const float2* A, float2* acc, int rx, int ry,
                                   int rz, int nb, cudaStream_t s) {
  const long long n = (long long)rx * ry * rz;
  grad_accumulate_kernel<<<grid_for(n), kThreads, 0, s>>>(E, A, acc, rx, ry, rz, nb);
  return cudaGetLastError();
}

cudaError_t launch_grad_finalize(const float2* acc, float2* grad, long long n, float n_ill,
                                 cudaStream_t s) {
  grad_finalize_kernel<<<grid_for(n), kThreads, 0, s>>>(acc, grad, n, n_ill);
  return cudaGetLastError();
}

cudaError_t launch_count_nonfinite(const float2* x, long long n, unsigned int* count,
                                   cudaStream_t s) {
  count_nonfinite_kernel<<<grid_for(n), kThreads, 0, s>>>(x, n, count);
  return cudaGetLastError();
}

}  // namespace odt
