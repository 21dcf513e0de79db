// Fused field input and output stages of the CBS forward solve.
//
// Input (FORWARD_SOLVER_CONVERGENT_BORN.m:543-554): the padded field spectrum
// sk (conv plane cx x cy per illumination) is refocused to every z of the RI
// grid (sk .* refocus(:,:,z)), brought back to space by a centred inverse 2D
// FFT and cropped to the rx x ry window at (ox, oy) -> E_inc.  The unfused
// path materialises the cx x cy x rz volume three times (expand, line FFT,
// column FFT) and crops it in a fourth pass; here
//   refocus_lines: product formed while the tile is staged, inverse x-FFT,
//                  only the rx kept columns stored (mid buffer rx x cy per
//                  (z, b));
//   refocus_cols : inverse y-FFT of those columns, only the ry kept rows
//                  stored, straight into E_inc.
//
// Output (:445-511): the emitter volume (Field(ROI) .* (V + i eps) dV placed
// at (ox, oy) of the conv plane, zero elsewhere) goes through a centred
// forward 2D FFT and is reduced over z against the transmission / reflection
// kernels.  Here
//   emit_lines      : emitter formed while the tile is staged, forward x-FFT
//                     of the ry lines that are not identically zero (the
//                     others transform to zero), all cx outputs stored (mid
//                     buffer cx x ry);
//   emit_cols_reduce: forward y-FFT of each column (rows outside the window
//                     are zero), multiplied by the kernels and summed over a
//                     chunk of z-planes in shared memory, in z order;
//   reduce_parts    : the chunks' partial sums added in chunk order.
//
// Traffic for the 256^2 conv plane, 128^3 RI grid: about 4 GB per stage for
// 49 illuminations, against about 18 GB for the unfused chain.
//
// The transforms are the same tile FFTs (plans, twiddles, pass order) as the
// unfused path; only the z-sum is regrouped (by chunks of 16 planes).
//
// Every kernel stages its whole input tile in shared memory first (all of a
// thread's global loads of the tile issued back to back) and runs the tile
// FFT from there: a first FFT pass reading global memory itself would wait on
// a few loads per butterfly.  Tiles are 8 lines / columns wide (about 38 KB
// of shared memory, five CTAs per SM).
//
// Compiled once per radix class (-DODT_CLS=0..3, see the Makefile); the
// class-independent dispatchers are compiled with class 0.
#include "tile_bodies.cuh"

#ifndef ODT_CLS
#error "compile with -DODT_CLS=<0..3>"
#endif

namespace odt {

namespace {

constexpr int kIoW = 8;      // lines / columns per tile
constexpr int kIoLgW = 3;
constexpr int kIoThreads = 128;
constexpr int kPf = 16;      // register prefetch of the reduce kernel (elements per thread)

__device__ __forceinline__ Thr thr() { return Thr{(int)threadIdx.x, (int)blockDim.x}; }

ODT_HD int rot_n(int row, int shift, int n) {  // (row + shift) mod n
  const int r = row + shift;
  return r >= n ? r - n : r;
}
ODT_HD int unrot_n(int X, int shift, int n) {  // the row r with rot_n(r, shift, n) == X
  const int r = X - shift;
  return r < 0 ? r + n : r;
}

// Transforms of the power-of-two lengths 128, 256 and 512 run with the plan
// fixed at compile time (radices 8, 8, 2 / 8, 8, 4 / 8, 8, 8: the run-time
// planner's order for these lengths), so the pass loop's strides, radix
// switch and index arithmetic fold to constants; NF = 0 keeps the run-time
// plan for every other length.
template <int N>
struct Pow2Plan {
  static constexpr int P = 3;
  __host__ __device__ static constexpr int rad(int i) { return i < 2 ? 8 : (N == 128 ? 2 : (N == 256 ? 4 : 8)); }
};

template <int N, bool INV, int I, int NS, class Map, class G1, class G2, class S>
__device__ __forceinline__ void pow2_passes(const Thr& th, const Map& m, const float2* tw, const G1& src,
                                            const G2& dst, S cur, S oth) {
  constexpr int P = Pow2Plan<N>::P;
  constexpr int R = INV ? Pow2Plan<N>::rad(P - 1 - I) : Pow2Plan<N>::rad(I);
  if constexpr (I == 0) tile_pass<R, INV>(th, m, N, NS, tw, src, cur);
  else if constexpr (I == P - 1) tile_pass<R, INV>(th, m, N, NS, tw, oth, dst);
  else tile_pass<R, INV>(th, m, N, NS, tw, oth, cur);
  __syncthreads();
  if constexpr (I + 1 < P) pow2_passes<N, INV, I + 1, NS * R>(th, m, tw, src, dst, oth, cur);
}

// the tile FFT of the fused kernels: fixed plan for NF != 0, else run-time plan
template <int CLS, int NF, bool INV, class Map, class S, class G1, class G2>
__device__ __forceinline__ void io_fft(const Thr& th, const FftPlan& plan, const Map& m, const float2* tw,
                                       const G1& src, const G2& dst, S cur, S oth) {
  if constexpr (NF != 0) pow2_passes<NF, INV, 0, 1>(th, m, tw, src, dst, cur, oth);
  else tile_fft_io<CLS, INV>(th, plan, m, tw, src, dst, cur, oth);
}

// stores x = X - lo in [0, len) of line c at out[c * len + x]; X = (row + n/2) % n
struct CropLineDst {
  float2* out;
  int nl, n, shift, lo, len;
  ODT_HD void store(int row, int c, float2 v) const {
    if (c >= nl) return;
    const int x = rot_n(row, shift, n) - lo;
    if ((unsigned)x < (unsigned)len) out[(long long)c * len + x] = v;
  }
};

// column store of rows y = Y - lo in [0, len) at out[y * rs + c], scaled
struct CropColDst {
  float2* out;
  int ncol, n, shift, lo, len, rs;
  float scale;
  ODT_HD void store(int row, int c, float2 v) const {
    if (c >= ncol) return;
    const int y = rot_n(row, shift, n) - lo;
    if ((unsigned)y < (unsigned)len) out[(long long)y * rs + c] = cscale(v, scale);
  }
};

// accumulates v .* K(kx0 + c, ky, z) into acc[ky * W + c] (ky = (row + n/2) % n)
struct ReduceDst {
  float2* accT;
  float2* accR;
  const float2* Kt;  // kernels at (kx0, 0, z); element (c, ky) at [c + cx * ky]
  const float2* Kr;
  int ncol, n, shift, cx;
  ODT_HD void store(int row, int c, float2 v) const {
    if (c >= ncol) return;
    const int ky = rot_n(row, shift, n);
    const long long p = (long long)cx * ky + c;
    const int a = ky * kIoW + c;
    if (accT) accT[a] = cadd(accT[a], cmul(v, Kt[p]));
    if (accR) accR[a] = cadd(accR[a], cmul(v, Kr[p]));
  }
};

size_t lines_smem(int n) {
  return align16(sizeof(float2) * (size_t)n) + 2 * sizeof(float2) * (size_t)kIoW * smem_line_ld(n) +
         2 * sizeof(long long) * (size_t)kIoW;
}

size_t cols_smem(int n, int nacc) {
  return align16(sizeof(float2) * (size_t)n) + 2 * sizeof(float2) * (size_t)n * (kIoW + 1) +
         (size_t)nacc * sizeof(float2) * n * kIoW;
}

template <int CLS, int NF>
__global__ void __launch_bounds__(kIoThreads)
refocus_lines_kernel(const float2* __restrict__ sk, const float2* __restrict__ ref, float2* __restrict__ mid,
                     IoGeom g, FftPlan plan, const float2* __restrict__ twg) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const Thr th = thr();
  const int n = NF ? NF : plan.n;  // == cx
  const int ld = smem_line_ld(n);
  float2* tw = reinterpret_cast<float2*>(smraw);
  float2* bufA = reinterpret_cast<float2*>(smraw + align16(sizeof(float2) * n));
  float2* bufB = bufA + (size_t)kIoW * ld;
  long long* off = reinterpret_cast<long long*>(bufB + (size_t)kIoW * ld);
  load_twiddles(th, tw, twg, n);
  // line L = b + nbp * (Y + cy * z): the illuminations of one (Y, z) are
  // neighbours, so a refocus line is read from DRAM about once
  const long long nlines = g.nbp * g.cy * g.rz;
  const long long L0 = (long long)blockIdx.x * kIoW;
  const int nl = (int)lmin(kIoW, nlines - L0);
  if (th.tid < kIoW) {
    const long long L = L0 + (th.tid < nl ? th.tid : nl - 1);
    const long long b = L % g.nbp, t = L / g.nbp;
    const long long Y = t % g.cy, z = t / g.cy;
    off[th.tid] = (long long)g.cx * (Y + g.cy * b);
    off[kIoW + th.tid] = (long long)g.cx * (Y + g.cy * z);
  }
  __syncthreads();
  const SmemLine S{bufA, ld};
  // conv line (Y, z, b) = sk(:, Y, b) .* refocus(:, Y, z); element X goes to
  // row (X - n/2) mod n (the ifftshift of the centred transform)
  for (int X = th.tid; X < n; X += th.nthr) {
    float2 a[kIoW], r[kIoW];
#pragma unroll
    for (int c = 0; c < kIoW; ++c) {
      if (c < nl) {
        a[c] = sk[off[c] + X];
        r[c] = ref[off[kIoW + c] + X];
      }
    }
    const int row = unrot_n(X, n / 2, n);
#pragma unroll
    for (int c = 0; c < kIoW; ++c) S.store(row, c, c < nl ? cmul(a[c], r[c]) : make_float2(0.f, 0.f));
  }
  __syncthreads();
  const CropLineDst dst{mid + L0 * g.rx, nl, n, n / 2, g.ox, g.rx};
  io_fft<CLS, NF, true>(th, plan, LineMap{kIoW}, tw, S, dst, SmemLine{bufB, ld}, S);
}

template <int CLS, int NF>
__global__ void __launch_bounds__(kIoThreads)
refocus_cols_kernel(const float2* __restrict__ mid, float2* __restrict__ einc, IoGeom g, float scale,
                    FftPlan plan, const float2* __restrict__ twg) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const Thr th = thr();
  const int n = NF ? NF : plan.n;  // == cy
  float2* tw = reinterpret_cast<float2*>(smraw);
  float2* bufA = reinterpret_cast<float2*>(smraw + align16(sizeof(float2) * n));
  float2* bufB = bufA + (size_t)n * (kIoW + 1);
  load_twiddles(th, tw, twg, n);
  const int ntx = (g.rx + kIoW - 1) >> kIoLgW;
  const long long o = blockIdx.x / ntx;  // b + nbp * z
  const int x0 = (int)(blockIdx.x - o * ntx) << kIoLgW;
  const long long b = o % g.nbp, z = o / g.nbp;
  const int ncol = min(kIoW, g.rx - x0);
  // mid: element (x, Y) of (z, b) at rx * (b + nbp * (Y + cy * z)) + x
  const float2* src = mid + g.rx * (b + g.nbp * g.cy * z) + x0;
  const long long rs = g.rx * g.nbp;
  const SmemCol S{bufA, kIoW + 1};
  const int total = n << kIoLgW;
  for (int i0 = th.tid; i0 < total; i0 += 8 * th.nthr) {
    float2 v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int i = i0 + u * th.nthr;
      const int c = i & (kIoW - 1), Y = i >> kIoLgW;
      v[u] = (i < total && c < ncol) ? src[Y * rs + c] : make_float2(0.f, 0.f);
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int i = i0 + u * th.nthr;
      if (i < total) S.store(unrot_n(i >> kIoLgW, n / 2, n), i & (kIoW - 1), v[u]);
    }
  }
  __syncthreads();
  const CropColDst dst{einc + x0 + (long long)g.rx * g.ry * (z + g.rz * b), ncol, n, n / 2, g.oy, g.ry, g.rx,
                       scale};
  io_fft<CLS, NF, true>(th, plan, ColMap{kIoLgW}, tw, S, dst, SmemCol{bufB, kIoW + 1}, S);
}

template <int CLS, int NF>
__global__ void __launch_bounds__(kIoThreads)
emit_lines_kernel(const BornArgs a, float2* __restrict__ mid, IoGeom g, float dV, FftPlan plan,
                  const float2* __restrict__ twg) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const Thr th = thr();
  const int n = NF ? NF : plan.n;  // == cx
  const int ld = smem_line_ld(n);
  float2* tw = reinterpret_cast<float2*>(smraw);
  float2* bufA = reinterpret_cast<float2*>(smraw + align16(sizeof(float2) * n));
  float2* bufB = bufA + (size_t)kIoW * ld;
  long long* off = reinterpret_cast<long long*>(bufB + (size_t)kIoW * ld);
  load_twiddles(th, tw, twg, n);
  // line L = b + nbp * (yr + ry * z): neighbouring illuminations share V
  const long long nlines = g.nbp * g.ry * g.rz;
  const long long L0 = (long long)blockIdx.x * kIoW;
  const int nl = (int)lmin(kIoW, nlines - L0);
  const long long est = (long long)a.rx * a.ry * a.rz;
  if (th.tid < kIoW) {
    const long long L = L0 + (th.tid < nl ? th.tid : nl - 1);
    const long long b = L % g.nbp, t = L / g.nbp;
    const long long y = t % g.ry, z = t / g.ry;
    off[th.tid] = b * est + (long long)a.rx * (y + (long long)a.ry * z);
    off[kIoW + th.tid] = a.rx0 + (long long)a.px * ((y + a.ry0) + (long long)a.py * (z + a.rz0));
  }
  __syncthreads();
  const SmemLine S{bufA, ld};
  // emitter line (yr, z, b): Field(x) .* (V(x) + i eps) * dV at X = x + ox,
  // zero elsewhere; element X goes to row (X - n/2) mod n
  for (int X = th.tid; X < n; X += th.nthr) {
    const int x = X - g.ox;
    const bool in = (unsigned)x < (unsigned)a.rx;
    float2 f[kIoW], v[kIoW];
#pragma unroll
    for (int c = 0; c < kIoW; ++c) {
      if (in && c < nl) {
        f[c] = a.Fout[off[c] + x];
        v[c] = a.V[off[kIoW + c] + x];
      }
    }
    const int row = unrot_n(X, n / 2, n);
#pragma unroll
    for (int c = 0; c < kIoW; ++c)
      S.store(row, c, (in && c < nl) ? cscale(cmul(f[c], make_float2(v[c].x, v[c].y + a.eps)), dV)
                                     : make_float2(0.f, 0.f));
  }
  __syncthreads();
  const GlobalShift dst{nullptr, mid + L0 * n, 1, n, nl, n, n / 2, 1.f};
  io_fft<CLS, NF, false>(th, plan, LineMap{kIoW}, tw, S, dst, SmemLine{bufB, ld}, S);
}

// CTA -> (b fastest, then 8 kx columns, then a chunk of zs z-planes): the CTAs
// resident together sweep z over the same kernel columns (L2 hits).  With
// one chunk the sums go straight to tk / rk, else to part[chunk][t|r][...].
// The window's rows of the next plane are loaded into registers while the
// current plane is transformed (ry * 8 <= kPf * threads).
template <int CLS, int NF>
__global__ void __launch_bounds__(kIoThreads)
emit_cols_reduce_kernel(const float2* __restrict__ mid, const float2* __restrict__ Kt,
                        const float2* __restrict__ Kr, float2* __restrict__ tk, float2* __restrict__ rk,
                        float2* __restrict__ part, IoGeom g, int zs, FftPlan plan,
                        const float2* __restrict__ twg) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const Thr th = thr();
  const int n = NF ? NF : plan.n;  // == cy
  float2* tw = reinterpret_cast<float2*>(smraw);
  float2* bufA = reinterpret_cast<float2*>(smraw + align16(sizeof(float2) * n));
  float2* bufB = bufA + (size_t)n * (kIoW + 1);
  float2* acc = bufB + (size_t)n * (kIoW + 1);
  float2* accT = Kt ? acc : nullptr;
  float2* accR = Kr ? acc + (Kt ? (size_t)n * kIoW : 0) : nullptr;
  load_twiddles(th, tw, twg, n);
  const int nacc = (Kt ? 1 : 0) + (Kr ? 1 : 0);
  for (int i = th.tid; i < nacc * n * kIoW; i += th.nthr) acc[i] = make_float2(0.f, 0.f);
  const int ntx = (g.cx + kIoW - 1) >> kIoLgW;
  const long long b = blockIdx.x % g.nbp;
  const long long r = blockIdx.x / g.nbp;
  const int x0 = (int)(r % ntx) << kIoLgW;
  const int chunk = (int)(r / ntx);
  const int z0 = chunk * zs, z1 = min(g.rz, z0 + zs);
  const int ncol = min(kIoW, g.cx - x0);
  const long long plane = (long long)g.cx * g.cy;
  const long long rs = g.cx * g.nbp;
  const int nwin = g.ry << kIoLgW;
  // mid: element (kx, yr) of (z, b) at cx * (b + nbp * (yr + ry * z)) + kx
  const float2* base = mid + g.cx * b + x0;
  const long long zstride = g.cx * g.nbp * (long long)g.ry;
  float2 pf[kPf];
  if (z0 < z1) {
    const float2* src = base + zstride * z0;
#pragma unroll
    for (int u = 0; u < kPf; ++u) {
      const int i = th.tid + u * kIoThreads;
      const int c = i & (kIoW - 1);
      pf[u] = (i < nwin && c < ncol) ? src[(i >> kIoLgW) * rs + c] : make_float2(0.f, 0.f);
    }
  }
  const SmemCol S{bufA, kIoW + 1};
  for (int z = z0; z < z1; ++z) {
    // rows outside the window are zero; window row yr sits at Y = yr + oy,
    // i.e. at row (Y - n/2) mod n
    for (int i = th.tid; i < n * kIoW; i += th.nthr) {
      const int Y = rot_n(i >> kIoLgW, n / 2, n);
      if ((unsigned)(Y - g.oy) >= (unsigned)g.ry) S.store(i >> kIoLgW, i & (kIoW - 1), make_float2(0.f, 0.f));
    }
#pragma unroll
    for (int u = 0; u < kPf; ++u) {
      const int i = th.tid + u * kIoThreads;
      if (i < nwin) S.store(unrot_n((i >> kIoLgW) + g.oy, n / 2, n), i & (kIoW - 1), pf[u]);
    }
    __syncthreads();
    if (z + 1 < z1) {  // next plane's window, in flight during this transform
      const float2* src = base + zstride * (z + 1);
#pragma unroll
      for (int u = 0; u < kPf; ++u) {
        const int i = th.tid + u * kIoThreads;
        const int c = i & (kIoW - 1);
        pf[u] = (i < nwin && c < ncol) ? src[(i >> kIoLgW) * rs + c] : make_float2(0.f, 0.f);
      }
    }
    const ReduceDst dst{accT, accR, Kt ? Kt + plane * z + x0 : nullptr, Kr ? Kr + plane * z + x0 : nullptr, ncol,
                        n, n / 2, g.cx};
    io_fft<CLS, NF, false>(th, plan, ColMap{kIoLgW}, tw, S, dst, SmemCol{bufB, kIoW + 1}, S);
  }
  __syncthreads();
  const long long tot = plane * g.nbp;
  float2* outT = part ? part + (long long)chunk * nacc * tot : tk;
  float2* outR = part ? part + ((long long)chunk * nacc + (Kt ? 1 : 0)) * tot : rk;
  for (int i = th.tid; i < n * kIoW; i += th.nthr) {
    const int c = i & (kIoW - 1), ky = i >> kIoLgW;
    if (c >= ncol) continue;
    const long long p = x0 + c + (long long)g.cx * ky + plane * b;
    if (Kt) outT[p] = accT[i];
    if (Kr) outR[p] = accR[i];
  }
}

// NF for a transform length: the fixed-plan lengths (class-0 units only), else 0
#define ODT_NF_DISPATCH(n, ...)                                          \
  if (ODT_CLS == 0 && (n) == 256) {                                      \
    constexpr int NF = ODT_CLS == 0 ? 256 : 0;                           \
    __VA_ARGS__;                                                         \
  } else if (ODT_CLS == 0 && (n) == 128) {                               \
    constexpr int NF = ODT_CLS == 0 ? 128 : 0;                           \
    __VA_ARGS__;                                                         \
  } else if (ODT_CLS == 0 && (n) == 512) {                               \
    constexpr int NF = ODT_CLS == 0 ? 512 : 0;                           \
    __VA_ARGS__;                                                         \
  } else {                                                               \
    constexpr int NF = 0;                                                \
    __VA_ARGS__;                                                         \
  }

template <typename K>
cudaError_t raise_smem(K kernel, size_t bytes) {
  return raise_smem_limit(reinterpret_cast<const void*>(kernel), bytes);
}

}  // namespace

template <>
cudaError_t io_in_launch<ODT_CLS>(const float2* sk, const float2* refocus, float2* mid, float2* einc,
                                  const IoGeom& g, const DevFft& fx, const DevFft& fy, cudaStream_t s) {
  cudaError_t e;
  {
    const size_t sm = lines_smem(fx.plan.n);
    const long long nlines = g.nbp * g.cy * g.rz;
    const unsigned blocks = (unsigned)((nlines + kIoW - 1) / kIoW);
    ODT_NF_DISPATCH(fx.plan.n, {
      if ((e = raise_smem(refocus_lines_kernel<ODT_CLS, NF>, sm)) != cudaSuccess) return e;
      refocus_lines_kernel<ODT_CLS, NF><<<blocks, kIoThreads, sm, s>>>(sk, refocus, mid, g, fx.plan, fx.tw);
    })
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  {
    const size_t sm = cols_smem(fy.plan.n, 0);
    const long long ntx = (g.rx + kIoW - 1) / kIoW;
    const unsigned blocks = (unsigned)(ntx * g.nbp * g.rz);
    const float scale = 1.0f / ((float)g.cx * (float)g.cy);
    ODT_NF_DISPATCH(fy.plan.n, {
      if ((e = raise_smem(refocus_cols_kernel<ODT_CLS, NF>, sm)) != cudaSuccess) return e;
      refocus_cols_kernel<ODT_CLS, NF><<<blocks, kIoThreads, sm, s>>>(mid, einc, g, scale, fy.plan, fy.tw);
    })
  }
  return cudaGetLastError();
}

template <>
cudaError_t io_out_lines_launch<ODT_CLS>(const BornArgs& a, float2* mid, const IoGeom& g, float dV,
                                         const DevFft& fx, cudaStream_t s) {
  const size_t sm = lines_smem(fx.plan.n);
  const long long nlines = g.nbp * g.ry * g.rz;
  const unsigned blocks = (unsigned)((nlines + kIoW - 1) / kIoW);
  cudaError_t e;
  ODT_NF_DISPATCH(fx.plan.n, {
    if ((e = raise_smem(emit_lines_kernel<ODT_CLS, NF>, sm)) != cudaSuccess) return e;
    emit_lines_kernel<ODT_CLS, NF><<<blocks, kIoThreads, sm, s>>>(a, mid, g, dV, fx.plan, fx.tw);
  })
  return cudaGetLastError();
}

template <>
cudaError_t io_out_cols_launch<ODT_CLS>(const float2* mid, const float2* Kt, const float2* Kr, float2* tk,
                                        float2* rk, float2* part, int zs, const IoGeom& g, const DevFft& fy,
                                        cudaStream_t s) {
  const int nacc = (Kt ? 1 : 0) + (Kr ? 1 : 0);
  const size_t sm = cols_smem(fy.plan.n, nacc);
  const long long ntx = (g.cx + kIoW - 1) / kIoW;
  const long long nchunk = (g.rz + zs - 1) / zs;
  const unsigned blocks = (unsigned)(ntx * g.nbp * nchunk);
  cudaError_t e;
  ODT_NF_DISPATCH(fy.plan.n, {
    if ((e = raise_smem(emit_cols_reduce_kernel<ODT_CLS, NF>, sm)) != cudaSuccess) return e;
    emit_cols_reduce_kernel<ODT_CLS, NF><<<blocks, kIoThreads, sm, s>>>(mid, Kt, Kr, tk, rk, part, g, zs,
                                                                        fy.plan, fy.tw);
  })
  return cudaGetLastError();
}

#if ODT_CLS == 0
// class dispatch and the chunk reduction (compiled once)
namespace {
// tk[i] = sum over chunks k (in order) of part[k][t][i]; rk likewise
__global__ void reduce_parts_kernel(const float2* __restrict__ part, float2* __restrict__ tk,
                                    float2* __restrict__ rk, int nchunk, long long tot) {
  const int nacc = (tk ? 1 : 0) + (rk ? 1 : 0);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot;
       i += (long long)gridDim.x * blockDim.x) {
    for (int a = 0; a < nacc; ++a) {
      float2 sum = part[a * tot + i];
      for (int k = 1; k < nchunk; ++k) sum = cadd(sum, part[((long long)k * nacc + a) * tot + i]);
      float2* out = (a == 0 && tk) ? tk : rk;
      out[i] = sum;
    }
  }
}
}  // namespace

bool io_fused_fits(const IoGeom& g, const DevFft& fx, const DevFft& fy, int nacc, int max_smem) {
  const size_t m = (size_t)max_smem;
  return (g.ry << kIoLgW) <= kPf * kIoThreads && g.rx <= fx.plan.n && g.ry <= fy.plan.n &&
         lines_smem(fx.plan.n) <= m && cols_smem(fy.plan.n, nacc) <= m;
}

cudaError_t launch_refocus_in(const float2* sk, const float2* refocus, float2* mid, float2* einc,
                              const IoGeom& g, const DevFft& fx, const DevFft& fy, cudaStream_t s) {
  // both kernels of the pair are instantiated for the larger radix class
  // (a class-K kernel holds the butterflies of every class <= K)
  switch (fx.plan.rclass > fy.plan.rclass ? fx.plan.rclass : fy.plan.rclass) {
    case 0: return io_in_launch<0>(sk, refocus, mid, einc, g, fx, fy, s);
    case 1: return io_in_launch<1>(sk, refocus, mid, einc, g, fx, fy, s);
    case 2: return io_in_launch<2>(sk, refocus, mid, einc, g, fx, fy, s);
    default: return io_in_launch<3>(sk, refocus, mid, einc, g, fx, fy, s);
  }
}

cudaError_t launch_project_out(const BornArgs& a, float2* mid, long long cap, const float2* Kt, const float2* Kr,
                               float2* tk, float2* rk, const IoGeom& g, float dV, const DevFft& fx,
                               const DevFft& fy, cudaStream_t s) {
  cudaError_t e;
  switch (fx.plan.rclass) {
    case 0: e = io_out_lines_launch<0>(a, mid, g, dV, fx, s); break;
    case 1: e = io_out_lines_launch<1>(a, mid, g, dV, fx, s); break;
    case 2: e = io_out_lines_launch<2>(a, mid, g, dV, fx, s); break;
    default: e = io_out_lines_launch<3>(a, mid, g, dV, fx, s); break;
  }
  if (e != cudaSuccess) return e;
  // z in chunks of 16 planes (partial sums after the mid buffer) where the
  // work buffer has room, else one chunk
  const int nacc = (Kt ? 1 : 0) + (Kr ? 1 : 0);
  const long long tot = (long long)g.cx * g.cy * g.nbp;
  const long long midn = (long long)g.cx * g.ry * g.rz * g.nbp;
  int zs = 16;
  int nchunk = (g.rz + zs - 1) / zs;
  if (nchunk < 2 || midn + (long long)nchunk * nacc * tot > cap) {
    zs = g.rz;
    nchunk = 1;
  }
  float2* part = nchunk > 1 ? mid + midn : nullptr;
  switch (fy.plan.rclass) {
    case 0: e = io_out_cols_launch<0>(mid, Kt, Kr, tk, rk, part, zs, g, fy, s); break;
    case 1: e = io_out_cols_launch<1>(mid, Kt, Kr, tk, rk, part, zs, g, fy, s); break;
    case 2: e = io_out_cols_launch<2>(mid, Kt, Kr, tk, rk, part, zs, g, fy, s); break;
    default: e = io_out_cols_launch<3>(mid, Kt, Kr, tk, rk, part, zs, g, fy, s); break;
  }
  if (e != cudaSuccess || !part) return e;
  long long blocks = (tot + 255) / 256;
  if (blocks > 148LL * 16) blocks = 148LL * 16;
  reduce_parts_kernel<<<(unsigned)blocks, 256, 0, s>>>(part, tk, rk, nchunk, tot);
  return cudaGetLastError();
}
#endif

}  // namespace odt
