// Bluestein transforms of one axis in one kernel.  A DFT of length n (with a
// prime factor above 31) is the linear convolution
//   X_k = w_k sum_j (x_j w_j) conj(w_(k-j)),   w_j = exp(-i pi j^2 / n),
// evaluated with FFTs of a 5-smooth length m >= 2n - 1 (fft_any.cuh).  Here
// a tile of pencils goes through the whole chain in shared memory: the first
// FFT pass reads the n input values of each pencil from global memory,
// multiplied by the chirp and zero-padded to m; the middle of the chain
// multiplies by the precomputed spectrum of the convolution kernel; the last
// inverse pass multiplies by the chirp and writes the n outputs back.  So an
// axis transform reads and writes each element once, as a radix-tile FFT
// does, instead of going through a 2m-element work array five times.
//
// The pass sequence is the z-pass's (tile_bodies.cuh, born_z_body): forward
// passes f[0] .. f[P-2], the last forward and first inverse pass fused with
// the pointwise multiply, inverse passes f[P-2] .. f[0].  m is 5-smooth, but
// its plan may combine factors into radices 15, 25 or 27, so the kernels are
// instantiated per radix class as the other tile kernels are.
#include <cuda_runtime.h>

#include "fft_any.cuh"
#include "tile_bodies.cuh"

namespace odt {

cudaError_t raise_smem_limit(const void* kernel, size_t bytes);   // smem_attr.cu

namespace {

ODT_HD float2 cmul_by(float2 a, float2 b, int conj_b) {
  const float by = conj_b ? -b.y : b.y;
  return make_float2(a.x * b.x - a.y * by, a.x * by + a.y * b.x);
}

// element (row, c) of the padded pencil: row < n reads x at the cyclic shift
// (row + sh) mod n times the chirp (conjugated for the inverse), rows n .. m-1
// are zero; pencils c >= ncol read as zero
struct BsIn {
  const float2* x;
  int rs, cs, ncol, n, sh;
  const float2* chirp;
  int conj;
  ODT_HD float2 load(int row, int c) const {
    if (c >= ncol || row >= n) return make_float2(0.f, 0.f);
    int q = row + sh;
    if (q >= n) q -= n;
    return cmul_by(x[q * rs + c * cs], chirp[row], conj);
  }
  ODT_HD void store(int, int, float2) const {}
};

// output k < n goes to (k + sh) mod n, times the chirp and the scale; rows
// n .. m-1 and pencils c >= ncol are dropped
struct BsOut {
  float2* x;
  int rs, cs, ncol, n, sh;
  const float2* chirp;
  int conj;
  float scale;
  ODT_HD float2 load(int, int) const { return make_float2(0.f, 0.f); }
  ODT_HD void store(int row, int c, float2 v) const {
    if (c >= ncol || row >= n) return;
    int q = row + sh;
    if (q >= n) q -= n;
    x[q * rs + c * cs] = cscale(cmul_by(v, chirp[row], conj), scale);
  }
};

// the spectrum of the convolution kernel at frequency row j + r nb
struct BsMul {
  const float2* bh;
  template <int R>
  ODT_HD void apply(int, int j, int nb, float2* v) const {
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = cmul(v[r], bh[j + r * nb]);
  }
};

template <int CLS, class Map, class S>
__device__ void bs_chain(const FftPlan& plan, const float2* tw, const Map& mp, const BsIn& src, const BsOut& dst,
                         const BsMul& op, S cur, S oth, const Thr& th) {
  const int m = plan.n;
  const int P = plan.npass;
  int ns = 1;
  for (int p = 0; p + 1 < P; ++p) {   // forward passes f[0] .. f[P-2]
    const int R = plan.radix[p];
    if (p == 0) tile_pass_any<CLS, false>(th, R, mp, m, ns, tw, src, cur);
    else tile_pass_any<CLS, false>(th, R, mp, m, ns, tw, oth, cur);
    __syncthreads();
    ns *= R;
    const S t2 = cur;
    cur = oth;
    oth = t2;
  }
  const int RL = plan.radix[P - 1];
  if (P == 1) {
    tile_mid_any<CLS, false, kMidBoth>(th, RL, mp, m, tw, src, dst, op);
    return;
  }
  tile_mid_any<CLS, false, kMidBoth>(th, RL, mp, m, tw, oth, cur, op);
  __syncthreads();
  {
    const S t2 = cur;
    cur = oth;
    oth = t2;
  }
  ns = RL;
  for (int i = P - 2; i >= 0; --i) {   // inverse passes f[P-2] .. f[0]; the last writes x
    const int R = plan.radix[i];
    if (i == 0) tile_pass_any<CLS, true>(th, R, mp, m, ns, tw, oth, dst);
    else tile_pass_any<CLS, true>(th, R, mp, m, ns, tw, oth, cur);
    __syncthreads();
    ns *= R;
    const S t2 = cur;
    cur = oth;
    oth = t2;
  }
}

// launch bound: 256 threads (class 3: 128, butterflies of up to 31 points in
// registers); the launches use the plan's 128 threads
template <int CLS>
constexpr int kBsMaxThreads = CLS == 3 ? 128 : 256;

// pencils contiguous in memory: line L of x [n, nlines] at x + L n
template <int CLS>
__global__ void __launch_bounds__(kBsMaxThreads<CLS>, 2)
    bs_lines_kernel(float2* x, long long nlines, int n, int sh, float scale, int inv, const float2* chirp,
                    const float2* bh, FftPlan plan, const float2* __restrict__ twg, int W) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const Thr th{(int)threadIdx.x, (int)blockDim.x};
  const int m = plan.n;
  const int ld = smem_line_ld(m);
  float2* tw = reinterpret_cast<float2*>(smraw);
  float2* bufA = reinterpret_cast<float2*>(smraw + align16(sizeof(float2) * m));
  float2* bufB = bufA + (size_t)W * ld;
  load_twiddles(th, tw, twg, m);
  __syncthreads();
  const long long L0 = (long long)blockIdx.x * W;
  const int nl = (int)lmin(W, nlines - L0);
  const BsIn src{x + L0 * n, 1, n, nl, n, sh, chirp, inv};
  const BsOut dst{x + L0 * n, 1, n, nl, n, sh, chirp, inv, scale};
  bs_chain<CLS>(plan, tw, LineMap{W}, src, dst, BsMul{bh}, SmemLine{bufA, ld}, SmemLine{bufB, ld}, th);
}

// pencils along the middle axis of x [n0, n, n2]: 2^lgW adjacent columns per
// tile, element (row, c) at row n0 + c
template <int CLS>
__global__ void __launch_bounds__(kBsMaxThreads<CLS>, 2)
    bs_cols_kernel(float2* x, long long n0, int n, int sh, float scale, int inv, const float2* chirp,
                   const float2* bh, FftPlan plan, const float2* __restrict__ twg, int lgW) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const Thr th{(int)threadIdx.x, (int)blockDim.x};
  const int m = plan.n;
  const int W = 1 << lgW;
  float2* tw = reinterpret_cast<float2*>(smraw);
  float2* bufA = reinterpret_cast<float2*>(smraw + align16(sizeof(float2) * m));
  float2* bufB = bufA + (size_t)m * (W + 1);
  load_twiddles(th, tw, twg, m);
  __syncthreads();
  const long long ntile = (n0 + W - 1) >> lgW;
  const long long o = blockIdx.x / ntile;
  const long long i00 = (blockIdx.x - o * ntile) << lgW;
  const int ncol = (int)lmin(W, n0 - i00);
  const long long off = o * n0 * n + i00;
  const BsIn src{x + off, (int)n0, 1, ncol, n, sh, chirp, inv};
  const BsOut dst{x + off, (int)n0, 1, ncol, n, sh, chirp, inv, scale};
  bs_chain<CLS>(plan, tw, ColMap{lgW}, src, dst, BsMul{bh}, SmemCol{bufA, W + 1}, SmemCol{bufB, W + 1}, th);
}

}  // namespace

namespace {

// pencils per tile: at most 8 (the padded length m is about twice the
// transform's, so 16 pencils of two stages would hold a third of an SM's
// shared memory and leave 3 CTAs per SM)
constexpr int kBsLgW = 3;

template <int CLS>
cudaError_t bs_launch(float2* x, int n0, long long n2, int cj, int sh, float scale, const AnyFft& f,
                      const float2* bh, int max_smem, cudaStream_t s) {
  const int n = f.n, m = f.m;
  const DevFft& g = f.f;
  const int lgW = g.lgW < kBsLgW ? g.lgW : kBsLgW;
  const int W = 1 << lgW;
  cudaError_t e;
  if (n0 == 1) {   // contiguous lines
    const size_t sm = align16(sizeof(float2) * m) + 2 * sizeof(float2) * (size_t)W * smem_line_ld(m);
    if (sm > (size_t)max_smem) return cudaErrorInvalidConfiguration;
    if ((e = raise_smem_limit(reinterpret_cast<const void*>(bs_lines_kernel<CLS>), sm)) != cudaSuccess) return e;
    const long long blocks = (n2 + W - 1) / W;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    bs_lines_kernel<CLS><<<(unsigned)blocks, g.nthr, sm, s>>>(x, n2, n, sh, scale, cj, f.chirp, bh, g.plan, g.tw,
                                                               W);
  } else {
    const size_t sm = align16(sizeof(float2) * m) + 2 * sizeof(float2) * (size_t)m * (W + 1);
    if (sm > (size_t)max_smem) return cudaErrorInvalidConfiguration;
    if ((e = raise_smem_limit(reinterpret_cast<const void*>(bs_cols_kernel<CLS>), sm)) != cudaSuccess) return e;
    const long long blocks = ((long long)(n0 + W - 1) / W) * n2;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    bs_cols_kernel<CLS><<<(unsigned)blocks, g.nthr, sm, s>>>(x, n0, n, sh, scale, cj, f.chirp, bh, g.plan, g.tw,
                                                              lgW);
  }
  return cudaGetLastError();
}

}  // namespace

cudaError_t bluestein_axis(float2* x, int n0, long long n2, bool inv, int sh, float scale, const AnyFft& f,
                           cudaStream_t s) {
  const DevFft& g = f.f;
  if (f.direct || g.plan.n != f.m || g.plan.npass < 1 || g.nthr > 128 || f.n < 1 || n0 < 1 || n2 < 1)
    return cudaErrorInvalidValue;
  const int cj = inv ? 1 : 0;
  const float2* bh = inv ? f.bhat_i : f.bhat_f;
  int dev = 0, max_smem = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if ((e = cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess)
    return e;
  switch (g.plan.rclass) {
    case 0: return bs_launch<0>(x, n0, n2, cj, sh, scale, f, bh, max_smem, s);
    case 1: return bs_launch<1>(x, n0, n2, cj, sh, scale, f, bh, max_smem, s);
    case 2: return bs_launch<2>(x, n0, n2, cj, sh, scale, f, bh, max_smem, s);
    default: return bs_launch<3>(x, n0, n2, cj, sh, scale, f, bh, max_smem, s);
  }
}

}  // namespace odt
