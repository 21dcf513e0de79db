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

namespace odt {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ int wrap_neg(int i, int n) { return i == 0 ? 0 : n - i; }

// Run all passes of `plan` on the tile in `a` (scratch `b`); returns the
// buffer that holds the result.  Ends with a __syncthreads().
template <int CLS, bool INV>
__device__ float2* tile_fft(float2* a, float2* b, const FftPlan& plan, int lgW, int ld,
                            const float2* tw) {
  int ns = 1;
  for (int p = 0; p < plan.npass; ++p) {
    const int R = plan.radix[p];
    run_pass<CLS, INV>(R, a, b, plan.n, ns, lgW, ld, tw, threadIdx.x, blockDim.x);
    __syncthreads();
    ns *= R;
    float2* t = a;
    a = b;
    b = t;
  }
  return a;
}

// Shared memory: twiddles (n, padded to even), then two n x ld tiles.
struct Smem {
  float2* tw;
  float2* a;
  float2* b;
};

__device__ __forceinline__ Smem carve(float2* base, int n, int ld) {
  Smem s;
  s.tw = base;
  s.a = base + ((n + 1) & ~1);
  s.b = s.a + (size_t)n * ld;
  return s;
}

__device__ __forceinline__ void load_twiddles(float2* dst, const float2* src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

__device__ __forceinline__ float2 ramp_at(const BornArgs& a, int x, int y, int z) {
  return cmul(cmul(a.ramp[0][x], a.ramp[1][y]), a.ramp[2][z]);
}

// ------------------------------------------------------------------ born_x
template <int CLS, int MODE>
__global__ void __launch_bounds__(kThreads)
born_x_kernel(BornArgs a, int jj, FftPlan plan, const float2* __restrict__ twg, int lgW) {
  extern __shared__ float2 smem[];
  const int n = plan.n;  // == px
  const int W = 1 << lgW;
  const int ld = W + 1;
  Smem s = carve(smem, n, ld);
  load_twiddles(s.tw, twg, n);
  const long long nlines = (long long)a.py * a.pz * a.nbatch;
  const long long L0 = (long long)blockIdx.x * W;
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  const int tot = n << lgW;

  float2* cur = s.a;
  if (MODE != kBornFirst) {
    const float2* src = a.T + L0 * n;
    for (int g = tid; g < tot; g += nthr) {
      const int line = g / n;
      const int i = g - line * n;
      s.a[i * ld + line] = (L0 + line < nlines) ? src[g] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    cur = tile_fft<CLS, true>(s.a, s.b, plan, lgW, ld, s.tw);
  } else {
    __syncthreads();
  }

  const int e = jj - 1;  // iteration whose update is completed here
  const float2 c = make_float2(0.f, a.c_im);
  const long long est = (long long)a.rx * a.ry * a.rz;
  for (int g = tid; g < tot; g += nthr) {
    const int line = g / n;
    const int x = g - line * n;
    const long long L = L0 + line;
    if (L >= nlines) {
      cur[x * ld + line] = make_float2(0.f, 0.f);
      continue;
    }
    const int y = (int)(L % a.py);
    const long long t = L / a.py;
    const int z = (int)(t % a.pz);
    const int b = (int)(t / a.pz);
    const long long gi = L * n + x;                     // batched index
    const long long vi = x + (long long)n * (y + (long long)a.py * z);
    const float2 v = a.V[vi];
    const float2 r0 = a.acyclic ? ramp_at(a, x, y, z) : make_float2(1.f, 0.f);
    const bool in_roi = (unsigned)(x - a.rx0) < (unsigned)a.rx &&
                        (unsigned)(y - a.ry0) < (unsigned)a.ry &&
                        (unsigned)(z - a.rz0) < (unsigned)a.rz;
    long long ri = 0;
    if (in_roi)
      ri = (long long)b * est + (x - a.rx0) +
           (long long)a.rx * ((y - a.ry0) + (long long)a.ry * (z - a.rz0));
    float2 fn_new = make_float2(0.f, 0.f);
    float2 ftot = make_float2(0.f, 0.f);
    if (MODE != kBornFirst && e >= 1) {
      // PSI = ifftn(...) .* conj(phase_ramp_e); phase_ramp_e = conj(r0) for odd e
      float2 P = cur[x * ld + line];
      if (a.acyclic) P = cmul(P, (e & 1) ? r0 : cconj(r0));
      const float m = (a.mask[0][x] * a.mask[1][y]) * a.mask[2][z];
      const float2 vP = cmul(v, P);
      if (e <= 2) {
        fn_new = cscale(vP, m);                        // (0 + V.*PSI) .* mask
        if (MODE == kBornMid) {
          a.Fn[gi] = fn_new;
          if (e == 1) a.F[gi] = fn_new;                // Field = 0 + Field_n
          // e == 2: Field keeps Field_n(1) until the e == 3 update
        } else {
          ftot = (e == 1) ? fn_new : cadd(a.F[gi], fn_new);
        }
      } else {
        const float2 fo = a.Fn[gi];
        const float2 psi = cmul(cmul(c, fo), v);
        const float2 fn = cscale(cadd(csub(fo, psi), vP), m);
        const float2 fp = a.F[gi];
        if (e == 3) {
          ftot = cadd(cadd(fp, fo), fn);
          fn_new = cadd(fn, fp);
        } else {
          ftot = cadd(fp, fn);
          fn_new = fn;
        }
        if (MODE == kBornMid) {
          a.F[gi] = ftot;
          a.Fn[gi] = fn_new;
        }
      }
    }
    if (MODE == kBornLast) {
      if (in_roi) a.Fout[ri] = cadd(ftot, a.Einc[ri]);
      continue;
    }
    // source term of iteration jj
    float2 psi = make_float2(0.f, 0.f);
    if (jj <= 2) {
      if (in_roi) {
        const float2 sv = cmul(make_float2(v.x, v.y + a.eps), a.Einc[ri]);
        psi = cscale(cmul(c, sv), 0.5f);
      }
    } else {
      psi = cmul(cmul(c, fn_new), v);
    }
    if (a.acyclic) psi = cmul(psi, (jj & 1) ? cconj(r0) : r0);
    cur[x * ld + line] = psi;
  }
  if (MODE == kBornLast) return;
  __syncthreads();
  float2* other = (cur == s.a) ? s.b : s.a;
  float2* res = tile_fft<CLS, false>(cur, other, plan, lgW, ld, s.tw);
  float2* dst = a.T + L0 * n;
  for (int g = tid; g < tot; g += nthr) {
    const int line = g / n;
    const int i = g - line * n;
    if (L0 + line < nlines) dst[g] = res[i * ld + line];
  }
}

// ------------------------------------------------------------------ born_z
template <int CLS>
__global__ void __launch_bounds__(kThreads)
born_z_kernel(BornArgs a, int jj, FftPlan plan, const float2* __restrict__ twg, int lgW) {
  extern __shared__ float2 smem[];
  const int n = plan.n;  // == pz
  const int W = 1 << lgW;
  const int ld = W + 1;
  Smem s = carve(smem, n, ld);
  load_twiddles(s.tw, twg, n);
  const long long n0 = (long long)a.px * a.py;
  const long long ntile = (n0 + W - 1) >> lgW;
  const long long b = blockIdx.x / ntile;
  const long long i00 = (blockIdx.x - b * ntile) << lgW;
  float2* base = a.T + b * a.nvox;
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  const int tot = n << lgW;
  for (int g = tid; g < tot; g += nthr) {
    const int c = g & (W - 1);
    const int j = g >> lgW;
    const long long i0 = i00 + c;
    s.a[j * ld + c] = (i0 < n0) ? base[i0 + n0 * j] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* cur = tile_fft<CLS, false>(s.a, s.b, plan, lgW, ld, s.tw);
  const bool flip = a.acyclic && (jj & 1);
  for (int g = tid; g < tot; g += nthr) {
    const int c = g & (W - 1);
    const int kz = g >> lgW;
    const long long i0 = i00 + c;
    if (i0 >= n0) continue;
    const int kx = (int)(i0 % a.px);
    const int ky = (int)(i0 / a.px);
    const int ix = flip ? wrap_neg(kx, a.px) : kx;
    const int iy = flip ? wrap_neg(ky, a.py) : ky;
    const int iz = flip ? wrap_neg(kz, a.pz) : kz;
    float q = (a.kq2[0][ix] + a.kq2[1][iy]) + a.kq2[2][iz];
    q = a.g_scale * q - a.g_off;
    const float den = q * q + a.eps * a.eps;
    const float2 G = make_float2(q / den, a.eps / den);  // 1 / (q - i eps)
    cur[kz * ld + c] = cscale(cmul(G, cur[kz * ld + c]), a.inv_n);
  }
  __syncthreads();
  float2* other = (cur == s.a) ? s.b : s.a;
  float2* res = tile_fft<CLS, true>(cur, other, plan, lgW, ld, s.tw);
  for (int g = tid; g < tot; g += nthr) {
    const int c = g & (W - 1);
    const int j = g >> lgW;
    const long long i0 = i00 + c;
    if (i0 < n0) base[i0 + n0 * j] = res[j * ld + c];
  }
}

// --------------------------------------------------------- generic FFTs
template <int CLS, bool INV>
__global__ void __launch_bounds__(kThreads)
fft_lines_kernel(const float2* in, float2* out, long long nlines, int in_shift, int out_shift,
                 float scale, FftPlan plan, const float2* __restrict__ twg, int lgW) {
  extern __shared__ float2 smem[];
  const int n = plan.n;
  const int W = 1 << lgW;
  const int ld = W + 1;
  Smem s = carve(smem, n, ld);
  load_twiddles(s.tw, twg, n);
  const long long L0 = (long long)blockIdx.x * W;
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  const int tot = n << lgW;
  const float2* src = in + L0 * n;
  for (int g = tid; g < tot; g += nthr) {
    const int line = g / n;
    const int i = g - line * n;
    int k = i - in_shift;  // element i of the line lands at tile row (i - shift) mod n
    if (k < 0) k += n;
    s.a[k * ld + line] = (L0 + line < nlines) ? src[g] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* res = tile_fft<CLS, INV>(s.a, s.b, plan, lgW, ld, s.tw);
  float2* dst = out + L0 * n;
  for (int g = tid; g < tot; g += nthr) {
    const int line = g / n;
    const int i = g - line * n;
    int k = i - out_shift;  // output index i holds spectrum element (i - shift) mod n
    if (k < 0) k += n;
    if (L0 + line < nlines) dst[g] = cscale(res[k * ld + line], scale);
  }
}

template <int CLS, bool INV>
__global__ void __launch_bounds__(kThreads)
fft_cols_kernel(const float2* in, float2* out, long long n0, long long n2, int in_shift,
                int out_shift, float scale, FftPlan plan, const float2* __restrict__ twg,
                int lgW) {
  extern __shared__ float2 smem[];
  const int n = plan.n;
  const int W = 1 << lgW;
  const int ld = W + 1;
  Smem s = carve(smem, n, ld);
  load_twiddles(s.tw, twg, n);
  const long long ntile = (n0 + W - 1) >> lgW;
  const long long o = blockIdx.x / ntile;
  const long long i00 = (blockIdx.x - o * ntile) << lgW;
  const long long slab = n0 * n;
  const float2* src = in + o * slab;
  float2* dst = out + o * slab;
  const int tid = threadIdx.x;
  const int nthr = blockDim.x;
  const int tot = n << lgW;
  for (int g = tid; g < tot; g += nthr) {
    const int c = g & (W - 1);
    const int j = g >> lgW;  // source row
    const long long i0 = i00 + c;
    int k = j - in_shift;
    if (k < 0) k += n;
    s.a[k * ld + c] = (i0 < n0) ? src[i0 + n0 * j] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* res = tile_fft<CLS, INV>(s.a, s.b, plan, lgW, ld, s.tw);
  for (int g = tid; g < tot; g += nthr) {
    const int c = g & (W - 1);
    const int j = g >> lgW;  // destination row
    const long long i0 = i00 + c;
    int k = j - out_shift;
    if (k < 0) k += n;
    if (i0 < n0) dst[i0 + n0 * j] = cscale(res[k * ld + c], scale);
  }
}

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

int grid_for(long long total) {
  long long g = (total + kThreads - 1) / kThreads;
  const long long cap = 148LL * 16;  // enough resident blocks; grid-stride beyond
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

template <typename K>
cudaError_t set_smem(K kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace

int pick_lgW(int n) { return n <= 512 ? 4 : 3; }

size_t fft_smem_bytes(int n, int lgW) {
  const int ld = (1 << lgW) + 1;
  return sizeof(float2) * (((size_t)n + 1) / 2 * 2 + 2 * (size_t)n * ld);
}

template <int CLS, int MODE>
cudaError_t born_x_cls(const BornArgs& a, int jj, const DevFft& fx, unsigned blocks, size_t sm,
                       cudaStream_t s) {
  cudaError_t err = set_smem(born_x_kernel<CLS, MODE>, sm);
  if (err != cudaSuccess) return err;
  born_x_kernel<CLS, MODE><<<blocks, kThreads, sm, s>>>(a, jj, fx.plan, fx.tw, fx.lgW);
  return cudaGetLastError();
}

template <int MODE>
cudaError_t born_x_mode(const BornArgs& a, int jj, const DevFft& fx, unsigned blocks, size_t sm,
                        cudaStream_t s) {
  switch (fx.plan.rclass) {
    case 0: return born_x_cls<0, MODE>(a, jj, fx, blocks, sm, s);
    case 1: return born_x_cls<1, MODE>(a, jj, fx, blocks, sm, s);
    case 2: return born_x_cls<2, MODE>(a, jj, fx, blocks, sm, s);
    default: return born_x_cls<3, MODE>(a, jj, fx, blocks, sm, s);
  }
}

cudaError_t launch_born_x(const BornArgs& a, int mode, int jj, const DevFft& fx, cudaStream_t s) {
  const long long nlines = (long long)a.py * a.pz * a.nbatch;
  const unsigned blocks = (unsigned)((nlines + (1 << fx.lgW) - 1) >> fx.lgW);
  const size_t sm = fft_smem_bytes(fx.plan.n, fx.lgW);
  switch (mode) {
    case kBornFirst: return born_x_mode<kBornFirst>(a, jj, fx, blocks, sm, s);
    case kBornMid: return born_x_mode<kBornMid>(a, jj, fx, blocks, sm, s);
    default: return born_x_mode<kBornLast>(a, jj, fx, blocks, sm, s);
  }
}

template <int CLS>
cudaError_t born_z_cls(const BornArgs& a, int jj, const DevFft& fz, unsigned blocks, size_t sm,
                       cudaStream_t s) {
  cudaError_t err = set_smem(born_z_kernel<CLS>, sm);
  if (err != cudaSuccess) return err;
  born_z_kernel<CLS><<<blocks, kThreads, sm, s>>>(a, jj, fz.plan, fz.tw, fz.lgW);
  return cudaGetLastError();
}

cudaError_t launch_born_z(const BornArgs& a, int jj, const DevFft& fz, cudaStream_t s) {
  const long long n0 = (long long)a.px * a.py;
  const long long ntile = (n0 + (1 << fz.lgW) - 1) >> fz.lgW;
  const unsigned blocks = (unsigned)(ntile * a.nbatch);
  const size_t sm = fft_smem_bytes(fz.plan.n, fz.lgW);
  switch (fz.plan.rclass) {
    case 0: return born_z_cls<0>(a, jj, fz, blocks, sm, s);
    case 1: return born_z_cls<1>(a, jj, fz, blocks, sm, s);
    case 2: return born_z_cls<2>(a, jj, fz, blocks, sm, s);
    default: return born_z_cls<3>(a, jj, fz, blocks, sm, s);
  }
}

template <int CLS, bool INV>
cudaError_t lines_cls(const float2* in, float2* out, long long nlines, int is, int os, float sc,
                      const DevFft& f, unsigned blocks, size_t sm, cudaStream_t s) {
  cudaError_t err = set_smem(fft_lines_kernel<CLS, INV>, sm);
  if (err != cudaSuccess) return err;
  fft_lines_kernel<CLS, INV><<<blocks, kThreads, sm, s>>>(in, out, nlines, is, os, sc, f.plan, f.tw,
                                                           f.lgW);
  return cudaGetLastError();
}

cudaError_t launch_fft_lines(const float2* in, float2* out, long long nlines, int in_shift,
                             int out_shift, float scale, bool inverse, const DevFft& f,
                             cudaStream_t s) {
  const unsigned blocks = (unsigned)((nlines + (1 << f.lgW) - 1) >> f.lgW);
  const size_t sm = fft_smem_bytes(f.plan.n, f.lgW);
#define ODT_L(C, I) return lines_cls<C, I>(in, out, nlines, in_shift, out_shift, scale, f, blocks, sm, s)
  if (inverse) {
    switch (f.plan.rclass) { case 0: ODT_L(0, true); case 1: ODT_L(1, true); case 2: ODT_L(2, true); default: ODT_L(3, true); }
  } else {
    switch (f.plan.rclass) { case 0: ODT_L(0, false); case 1: ODT_L(1, false); case 2: ODT_L(2, false); default: ODT_L(3, false); }
  }
#undef ODT_L
}

template <int CLS, bool INV>
cudaError_t cols_cls(const float2* in, float2* out, long long n0, long long n2, int is, int os,
                     float sc, const DevFft& f, unsigned blocks, size_t sm, cudaStream_t s) {
  cudaError_t err = set_smem(fft_cols_kernel<CLS, INV>, sm);
  if (err != cudaSuccess) return err;
  fft_cols_kernel<CLS, INV><<<blocks, kThreads, sm, s>>>(in, out, n0, n2, is, os, sc, f.plan, f.tw,
                                                          f.lgW);
  return cudaGetLastError();
}

cudaError_t launch_fft_cols(const float2* in, float2* out, long long n0, long long n2,
                            int in_shift, int out_shift, float scale, bool inverse,
                            const DevFft& f, cudaStream_t s) {
  const long long ntile = (n0 + (1 << f.lgW) - 1) >> f.lgW;
  const unsigned blocks = (unsigned)(ntile * n2);
  const size_t sm = fft_smem_bytes(f.plan.n, f.lgW);
#define ODT_C(C, I) return cols_cls<C, I>(in, out, n0, n2, in_shift, out_shift, scale, f, blocks, sm, s)
  if (inverse) {
    switch (f.plan.rclass) { case 0: ODT_C(0, true); case 1: ODT_C(1, true); case 2: ODT_C(2, true); default: ODT_C(3, true); }
  } else {
    switch (f.plan.rclass) { case 0: ODT_C(0, false); case 1: ODT_C(1, false); case 2: ODT_C(2, false); default: ODT_C(3, false); }
  }
#undef ODT_C
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

cudaError_t launch_count_nonfinite(const float2* x, long long n, unsigned int* count,
                                   cudaStream_t s) {
  count_nonfinite_kernel<<<grid_for(n), kThreads, 0, s>>>(x, n, count);
  return cudaGetLastError();
}

}  // namespace odt
