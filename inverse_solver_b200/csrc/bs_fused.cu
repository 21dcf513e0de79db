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

#include <map>
#include <mutex>
#include <set>
#include <tuple>

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

// pencil-major shared memory with one pad element every 2^sh rows
// (s[c * ld + row + (row >> sh)]; sh = 31: no pad).  Which spacing keeps the
// strided accesses of a plan's passes off shared banks depends on its radices
// (bs_line_shift picks it); the pencil pitch ld is = 8 (mod 16) elements.
struct BsLine {
  float2* s;
  int ld, sh;
  ODT_HD int at(int row, int c) const { return c * ld + row + (row >> sh); }
  ODT_HD float2 load(int row, int c) const { return s[at(row, c)]; }
  ODT_HD void store(int row, int c, float2 v) const { s[at(row, c)] = v; }
};

ODT_HD int bs_line_ld(int m, int sh) {
  const int p = m + (sh < 31 ? (m >> sh) : 0) + 1;
  return p + ((8 - (p & 15)) & 15);
}

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
                    const float2* bh, FftPlan plan, const float2* __restrict__ twg, int W, int pad_sh) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const Thr th{(int)threadIdx.x, (int)blockDim.x};
  const int m = plan.n;
  const int ld = bs_line_ld(m, pad_sh);
  float2* tw = reinterpret_cast<float2*>(smraw);
  float2* bufA = reinterpret_cast<float2*>(smraw + align16(sizeof(float2) * m));
  float2* bufB = bufA + (size_t)W * ld;
  load_twiddles(th, tw, twg, m);
  __syncthreads();
  const long long L0 = (long long)blockIdx.x * W;
  const int nl = (int)lmin(W, nlines - L0);
  const BsIn src{x + L0 * n, 1, n, nl, n, sh, chirp, inv};
  const BsOut dst{x + L0 * n, 1, n, nl, n, sh, chirp, inv, scale};
  bs_chain<CLS>(plan, tw, LineMap{W}, src, dst, BsMul{bh}, BsLine{bufA, ld, pad_sh}, BsLine{bufB, ld, pad_sh}, th);
}

// pencils along the middle axis of x [n0, n, n2]: 2^lgW adjacent columns per
// tile, element (row, c) at row n0 + c
template <int CLS>
__global__ void __launch_bounds__(kBsMaxThreads<CLS>, 2)
    bs_cols_kernel(float2* x, long long n0, int n, int sh, float scale, int inv, const float2* chirp,
                   const float2* bh, FftPlan plan, const float2* __restrict__ twg, int lgW, int pitch) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const Thr th{(int)threadIdx.x, (int)blockDim.x};
  const int m = plan.n;
  const int W = 1 << lgW;
  float2* tw = reinterpret_cast<float2*>(smraw);
  float2* bufA = reinterpret_cast<float2*>(smraw + align16(sizeof(float2) * m));
  float2* bufB = bufA + (size_t)m * pitch;
  load_twiddles(th, tw, twg, m);
  __syncthreads();
  const long long ntile = (n0 + W - 1) >> lgW;
  const long long o = blockIdx.x / ntile;
  const long long i00 = (blockIdx.x - o * ntile) << lgW;
  const int ncol = (int)lmin(W, n0 - i00);
  const long long off = o * n0 * n + i00;
  const BsIn src{x + off, (int)n0, 1, ncol, n, sh, chirp, inv};
  const BsOut dst{x + off, (int)n0, 1, ncol, n, sh, chirp, inv, scale};
  bs_chain<CLS>(plan, tw, ColMap{lgW}, src, dst, BsMul{bh}, SmemCol{bufA, pitch}, SmemCol{bufB, pitch}, th);
}

}  // namespace

namespace {

// pencils per tile: at most 8 (the padded length m is about twice the
// transform's, so 16 pencils of two stages would hold a third of an SM's
// shared memory and leave 3 CTAs per SM)
constexpr int kBsLgW = 3;

// Shared-memory wavefronts of one warp-wide 8-byte access: the most
// distinct 4-byte words any of the 32 banks must serve (2 when conflict-free).
int warp_wavefronts(const int* elem, int nact) {
  std::set<int> words[32];
  for (int t = 0; t < nact; ++t)
    for (int h = 0; h < 2; ++h) words[(2 * elem[t] + h) & 31].insert(2 * elem[t] + h);
  int w = 0;
  for (const auto& b : words) w = b.size() > (size_t)w ? (int)b.size() : w;
  return w;
}

// Wavefronts of the shared-memory accesses of bs_chain on lines (LineMap,
// pencil pitch and pad of BsLine with shift sh) for plan p, W pencils and
// nthr threads: loads and stores of every pass that touches shared memory.
long long line_chain_wavefronts(const FftPlan& p, int W, int nthr, int sh) {
  const int m = p.n, P = p.npass, ld = bs_line_ld(m, sh);
  auto at = [&](int row, int c) { return c * ld + row + (sh < 31 ? (row >> sh) : 0); };
  long long wf = 0;
  int el[32];
  // one pass: for each warp of each round, the R loads (unless it reads
  // global memory) and the R stores (unless it writes global memory)
  auto pass = [&](int R, int ns, bool loads, bool stores, bool mid) {
    const int nb = m / R, total = W * nb;
    for (int base = 0; base < total; base += nthr)
      for (int w0 = 0; w0 < nthr; w0 += 32) {
        int cs[32], js[32], na = 0;
        for (int l = 0; l < 32 && base + w0 + l < total; ++l) {
          const int idx = base + w0 + l;
          cs[na] = idx / nb;
          js[na++] = idx % nb;
        }
        if (!na) continue;
        for (int r = 0; r < R; ++r) {
          if (loads) {
            for (int t = 0; t < na; ++t) el[t] = at(js[t] + r * nb, cs[t]);
            wf += warp_wavefronts(el, na);
          }
          if (stores) {
            for (int t = 0; t < na; ++t) {
              const int k = mid ? 0 : js[t] % ns;
              const int d = mid ? js[t] * R : (js[t] - k) * R + k;
              el[t] = at(d + r * (mid ? 1 : ns), cs[t]);
            }
            wf += warp_wavefronts(el, na);
          }
        }
      }
  };
  int ns = 1;
  for (int q = 0; q + 1 < P; ++q) {
    pass(p.radix[q], ns, q > 0, true, false);
    ns *= p.radix[q];
  }
  if (P > 1) pass(p.radix[P - 1], 0, true, true, true);
  ns = p.radix[P - 1];
  for (int q = P - 2; q >= 0; --q) {
    pass(p.radix[q], ns, true, q > 0, false);
    ns *= p.radix[q];
  }
  return wf;
}

// The pad spacing (every 8 or 16 rows, or none) with the fewest shared-memory
// wavefronts for this plan on W-pencil line tiles; computed once per plan.
int bs_line_shift(const FftPlan& p, int W, int nthr) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int, long long>, int> cache;
  long long rk = 0;
  for (int q = 0; q < p.npass; ++q) rk = rk * 64 + p.radix[q];
  const auto key = std::make_tuple(p.n, W, nthr, rk);
  std::lock_guard<std::mutex> lock(mu);
  const auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  int best = 3;
  long long bw = -1;
  for (int sh : {3, 4, 31}) {
    const long long w = line_chain_wavefronts(p, W, nthr, sh);
    if (bw < 0 || w < bw) {
      bw = w;
      best = sh;
    }
  }
  cache[key] = best;
  return best;
}

template <int CLS>
cudaError_t bs_launch(float2* x, int n0, long long n2, int cj, int sh, float scale, const AnyFft& f,
                      const float2* bh, int max_smem, cudaStream_t s) {
  const int n = f.n, m = f.m;
  const DevFft& g = f.f;
  const int lgW = g.lgW < kBsLgW ? g.lgW : kBsLgW;
  const int W = 1 << lgW;
  cudaError_t e;
  if (n0 == 1) {   // contiguous lines
    const int pad_sh = bs_line_shift(g.plan, W, g.nthr);
    const size_t sm = align16(sizeof(float2) * m) + 2 * sizeof(float2) * (size_t)W * bs_line_ld(m, pad_sh);
    if (sm > (size_t)max_smem) return cudaErrorInvalidConfiguration;
    if ((e = raise_smem_limit(reinterpret_cast<const void*>(bs_lines_kernel<CLS>), sm)) != cudaSuccess) return e;
    const long long blocks = (n2 + W - 1) / W;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    bs_lines_kernel<CLS><<<(unsigned)blocks, g.nthr, sm, s>>>(x, n2, n, sh, scale, cj, f.chirp, bh, g.plan, g.tw,
                                                               W, pad_sh);
  } else {
    // row pitch W + 1 elements (a wider pitch that would remove more bank
    // conflicts at W = 8 costs shared memory: 4 CTAs per SM instead of 6 at
    // m = 256, slower)
    const int pitch = W + 1;
    const size_t sm = align16(sizeof(float2) * m) + 2 * sizeof(float2) * (size_t)m * pitch;
    if (sm > (size_t)max_smem) return cudaErrorInvalidConfiguration;
    if ((e = raise_smem_limit(reinterpret_cast<const void*>(bs_cols_kernel<CLS>), sm)) != cudaSuccess) return e;
    const long long blocks = ((long long)(n0 + W - 1) / W) * n2;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    bs_cols_kernel<CLS><<<(unsigned)blocks, g.nthr, sm, s>>>(x, n0, n, sh, scale, cj, f.chirp, bh, g.plan, g.tw,
                                                              lgW, pitch);
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
