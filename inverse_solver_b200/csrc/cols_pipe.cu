// Pipelined column passes of the Born iteration for lengths n = 8 * R2 (R2
// odd): the y-FFTs (forward / inverse, in place on T) and the z-pass
// (forward z-FFT, Green's multiply G(k -/+ dk/4) / N, inverse z-FFT;
// FORWARD_SOLVER_CONVERGENT_BORN.m:606-615) -- the same transforms as
// fft_cols_body / born_z_body, restructured like the pipelined x-pass:
//
//   * persistent CTAs (as many per SM as shared memory and registers allow:
//     three for the y-FFTs, five for the z-pass at n <= 152) walk tiles of
//     16 adjacent columns;
//   * a tile (16 columns x n rows, each row a 128-byte segment at a stride of
//     px or px*py elements) arrives in shared memory through one tiled TMA
//     copy (cp.async.bulk.tensor, 3D map for y, 4D for z) on an mbarrier,
//     while the CTA computes the previous tile from the other stage;
//   * y-FFTs: radix-R2 pass in place in the landing buffer (one butterfly
//     per thread held in registers across a barrier), then radix-8 with
//     twiddles straight to global memory;
//   * z-pass: with z = R2 n1 + n2 and kz = k1 + 8 k2, an 8-point DFT over n1
//     with twiddles, then per (column, k1) the R2-point DFT, the Green's
//     multiply at kz and the inverse R2-point DFT in registers, then the
//     inverse 8-point DFT to global memory; every step writes the rows it
//     read, so the landing buffer is the only buffer.
//
// Layout in shared memory: [row][column], 16 columns = 128 bytes per row; the
// column index is the fastest thread index, so every access of a half-warp
// covers one row: conflict-free.  Columns past the grid edge arrive as zeros
// (TMA out-of-bounds fill) and are not stored.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <string>

#include "b16.cuh"
#include "cbs_kernels.cuh"
#include "fft_core.cuh"
#include "tma.cuh"

namespace odt {
namespace {

constexpr int kW = 16;               // columns per tile
constexpr int kR1 = 8;
constexpr int kThreads = kW * kR1;   // y-FFTs: one radix-R2 butterfly per thread
// z-pass: 160 threads, so its steps A and C (16 R2 radix-8 items) take two
// rounds for R2 <= 19 instead of three; step B uses the first 128
constexpr int kThreadsZ = 160;
template <int KIND>
__host__ __device__ constexpr int threads_of() { return KIND >= 2 ? kThreadsZ : kThreads; }

constexpr size_t a16(size_t b) { return (b + 15) & ~(size_t)15; }
constexpr size_t a1k(size_t b) { return (b + 1023) & ~(size_t)1023; }

// Tiled TMA copies need 128-byte aligned shared-memory destinations; the tile
// buffers start on 1024-byte boundaries (the dynamic window itself is
// 1024-byte aligned, checked at run time).
template <int N>
struct ColSmem {
  static constexpr size_t kTw = 64;                                  // after 3 mbarriers
  static constexpr size_t kKz = kTw + a16(sizeof(float2) * N);       // kq2 along z (born_z)
  static constexpr size_t kGxy = kKz + a16(sizeof(float) * N);
  static constexpr size_t kTile = sizeof(float2) * N * kW;           // 1024 * R2 bytes
  static constexpr size_t kS0 = a1k(kGxy + a16(sizeof(float) * kW));
  static constexpr size_t kS1 = kS0 + kTile;
  static constexpr size_t kB = kS1 + kTile;
  static constexpr size_t kTotalY = kB;                             // both kinds: two stages only
  static constexpr size_t kTotalZ = kB;
  // z-pass on 16-bit block floating-point storage: two landing stages of
  // int16 (re, im) pairs, one complex64 work tile, the tile's exponents
  static constexpr size_t kTile16 = sizeof(short2) * N * kW;
  static constexpr size_t kS1_16 = kS0 + kTile16;
  static constexpr size_t kW16 = a1k(kS1_16 + kTile16);
  static constexpr size_t kEx16 = kW16 + kTile;
  static constexpr size_t kExStage = a16(2 * N);                  // one stage of [row][2] exponents
  static constexpr size_t kTotalZ16 = kEx16 + 2 * kExStage;
};

#if defined(__CUDA_ARCH__)
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            int c3, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
      : "memory");
}
// Reciprocal to within the hardware approximation (PTX rcp.approx.ftz.f32,
// at most 1 ulp from the rounded quotient); its argument here is
// q^2 + eps^2 >= eps^2, far from zero, subnormals and infinity.
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
#endif

// KIND 0: forward y-FFT, 1: inverse y-FFT, 2: z-pass with Green's multiply,
// 3: the z-pass on 16-bit block floating-point storage (a.T16 / a.Te: the
// tile lands as int16 pairs, is decoded into a complex64 work tile and the
// result is encoded again with one exponent per 8 columns of a row).
// Tile t -> (x-tile fastest, then the outer index o): y-pass o = z + pz*b
// (3D map {px, py, pz*nb}), z-pass o = y + py*b (4D map {px, py, pz, nb}).
template <int R2, int KIND>
__global__ void __launch_bounds__(threads_of<KIND>(), KIND >= 2 ? (R2 <= 19 ? 5 : 4) : 3)
    cols_pipe_kernel(const __grid_constant__ CUtensorMap map, const BornArgs a, const int jj,
                     const float2* __restrict__ twg, const int nxt, const int ntiles,
                     int* __restrict__ fault) {
#if defined(__CUDA_ARCH__)
  constexpr int N = kR1 * R2;
  constexpr bool kZ = KIND >= 2;
  constexpr bool k16 = KIND == 3;
  constexpr int kT = threads_of<KIND>();
  // y-columns longer than a TMA box dimension (256) arrive as two halves
  constexpr bool kSplitY = !kZ && N > 256;
  static_assert(!kSplitY || (N % 2 == 0 && N / 2 <= 256 && ((N / 2) * kW * sizeof(float2)) % 128 == 0),
                "split y-tile halves must fit a box and stay 128-byte aligned");
  static_assert(!kZ || N <= 256, "z-tiles are one box");
  constexpr bool kInvFirst = KIND == 1;  // direction of the first transform
  using L = ColSmem<N>;
  extern __shared__ __align__(128) unsigned char sm[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm);
  float2* tw = reinterpret_cast<float2*>(sm + L::kTw);
  float* kz = reinterpret_cast<float*>(sm + L::kKz);
  float* gxy = reinterpret_cast<float*>(sm + L::kGxy);
  float2* const s0 = reinterpret_cast<float2*>(sm + L::kS0);
  float2* const s1 = reinterpret_cast<float2*>(sm + (k16 ? L::kS1_16 : L::kS1));
  float2* const w16 = reinterpret_cast<float2*>(sm + L::kW16);     // k16: work tile
  signed char* const ex16 = reinterpret_cast<signed char*>(sm + L::kEx16);  // k16: [row][2]
  const int tid = threadIdx.x;
  const bool flip = kZ && a.acyclic && (jj & 1);
  if ((smem_addr(s0) & 127u) != 0u || (smem_addr(s1) & 127u) != 0u) {  // never issue a misaligned copy
    if (tid == 0) atomicCAS(fault, 0, kFaultAlign);
    return;
  }

  for (int i = tid; i < N; i += kT) {
    tw[i] = twg[i];
    if (kZ) kz[i] = a.kq2[2][flip ? (i == 0 ? 0 : N - i) : i];
  }
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_fence_init();
  }
  __syncthreads();
  int tile = blockIdx.x;
  if (tile >= ntiles) return;
  const long long rstride = kZ ? (long long)a.px * a.py : a.px;   // element stride between rows
  constexpr uint32_t kBytes = (uint32_t)((k16 ? sizeof(short2) : sizeof(float2)) * N * kW);
  auto issue = [&](int t, int stage) {
    const int xt = t % nxt, o = t / nxt;
    mbar_arrive_expect_tx(&bar[stage], kBytes);
    float2* dst = stage ? s1 : s0;
    if (k16) tma_load_4d(dst, &map, kW * xt, o % a.py, 0, o / a.py, &bar[stage]);
    else if (kZ) tma_load_4d(dst, &map, 2 * kW * xt, o % a.py, 0, o / a.py, &bar[stage]);
    else if (kSplitY) {
      tma_load_3d(dst, &map, 2 * kW * xt, 0, o, &bar[stage]);
      tma_load_3d(dst + (N / 2) * kW, &map, 2 * kW * xt, N / 2, o, &bar[stage]);
    } else {
      tma_load_3d(dst, &map, 2 * kW * xt, 0, o, &bar[stage]);
    }
  };
  if (tid == 0) issue(tile, 0);
  uint32_t ph0 = 0, ph1 = 0;
  const int c = tid & (kW - 1), jr = tid >> 4;   // column, butterfly of the radix-R2 passes

  for (int it = 0; tile < ntiles; ++it, tile += gridDim.x) {
    const int s = it & 1;
    const int next = tile + gridDim.x;
    if (tid == 0 && next < ntiles) {
      fence_proxy_async();
      issue(next, s ^ 1);
    }
    const int xt = tile % nxt, o = tile / nxt;
    const int x0 = kW * xt;
    const int ncol = min(kW, a.px - x0);
    if (kZ && tid < kW) {
      int y = o % a.py;
      int kx = min(x0 + tid, a.px - 1);
      if (a.perm_xy) {   // position R k1 + k2 holds spectral index k1 + 8 k2
        const int rx = a.px >> 3, ry = a.py >> 3;
        kx = kx / rx + 8 * (kx % rx);
        y = y / ry + 8 * (y % ry);
      }
      const int ix = flip ? (kx == 0 ? 0 : a.px - kx) : kx;
      const int iy = flip ? (y == 0 ? 0 : a.py - y) : y;
      gxy[tid] = a.kq2[0][ix] + a.kq2[1][iy];
    }
    // k16: the two exponents per row of a tile (blocks x0 .. x0+7 and
    // x0+8 .. x0+15), loaded one tile ahead into registers and stored to the
    // next stage's exponent buffer after this tile's last step
    constexpr int kExPer = (2 * N + kT - 1) / kT;
    signed char exn[k16 ? kExPer : 1];
    auto ex_load = [&](int t, signed char* dst_regs, signed char* dst_smem) {
      const int txt = t % nxt, to = t / nxt;
      const int tx0 = kW * txt, y = to % a.py, b = to / a.py;
      const long long e0 = ((long long)b * a.nvox + (long long)y * a.px + tx0) >> 3;
      const long long es = ((long long)a.px * a.py) >> 3;
#pragma unroll
      for (int q = 0; q < kExPer; ++q) {
        const int i = tid + q * kT;
        const int row = i >> 1, h = i & 1;
        signed char e = 0;
        if (i < 2 * N && (h == 0 || tx0 + 8 < a.px)) e = a.Te[e0 + row * es + h];
        if (dst_smem) {
          if (i < 2 * N) dst_smem[i] = e;
        } else {
          dst_regs[q] = e;
        }
      }
    };
    if constexpr (k16) {
      if (it == 0) ex_load(tile, nullptr, ex16);   // the first tile's, exposed once
      if (next < ntiles) ex_load(next, exn, nullptr);
    }
    signed char* const exs = ex16 + s * L::kExStage;   // this tile's exponents
    const bool ok = mbar_wait(&bar[s], s ? ph1 : ph0, a.wait_limit);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {  // give up; let the copies in flight land first
        atomicCAS(fault, 0, kFaultTimeout);
        mbar_wait(&bar[s], s ? ph1 : ph0);
        if (next < ntiles) mbar_wait(&bar[s ^ 1], s ? ph0 : ph1);
      }
      return;
    }
    if (s) ph1 ^= 1; else ph0 ^= 1;
    float2* S = s ? s1 : s0;
    // global address of (row, column) of this tile
    long long gbase;
    if (kZ) {
      const int y = o % a.py, b = o / a.py;
      gbase = (long long)b * a.nvox + (long long)y * a.px + x0;
    } else {
      gbase = (long long)o * a.px * a.py + x0;
    }
    if constexpr (kZ) {
      // z-pass with z = R2 n1 + n2, kz = k1 + 8 k2 (k1 < 8, k2 < R2), every
      // step in place on the landing buffer:
      //   A  8-point DFT over n1 at rows R2 n1 + n2, times W_N^(n2 k1)
      //   B  R2-point DFT over n2 at rows R2 k1 + n2 (kz = k1 + 8 k2), Green's
      //      multiply, inverse R2-point DFT, times conj W_N^(n2 k1)
      //   C  inverse 8-point DFT over k1 -> rows R2 n1 + n2 of T
      float2* const Wt = k16 ? w16 : S;   // the tile the steps work on
      for (int idx = tid; idx < kW * R2; idx += kT) {
        const int n2 = idx >> 4;  // column c is idx & 15 == tid & 15
        float2 v[kR1];
        if constexpr (k16) {
          const short2* S16 = reinterpret_cast<const short2*>(S);
#pragma unroll
          for (int r = 0; r < kR1; ++r) {
            const int row = R2 * r + n2;
            v[r] = b16_decode(S16[row * kW + c], exs[2 * row + (c >> 3)]);
          }
        } else {
#pragma unroll
          for (int r = 0; r < kR1; ++r) v[r] = S[(R2 * r + n2) * kW + c];
        }
        Butterfly<kR1, false>::run(v, tw, N);
#pragma unroll
        for (int r = 1; r < kR1; ++r) v[r] = cmul(v[r], tw[r * n2]);
#pragma unroll
        for (int r = 0; r < kR1; ++r) Wt[(R2 * r + n2) * kW + c] = v[r];
      }
      __syncthreads();
      if (tid < kW * kR1) {   // step B: (column, k1) items on the first 128 threads
        const int k1 = jr;   // tid >> 4
        float2 v[R2];
#pragma unroll
        for (int r = 0; r < R2; ++r) v[r] = Wt[(R2 * k1 + r) * kW + c];
        Butterfly<R2, false>::run(v, tw, N);
        const float qxy = gxy[c];
#pragma unroll
        for (int r = 0; r < R2; ++r) {
          float q = qxy + kz[k1 + kR1 * r];
          q = a.g_scale * q - a.g_off;
          const float rden = rcp_approx(q * q + a.eps * a.eps) * a.inv_n;
          const float2 G = make_float2(q * rden, a.eps * rden);  // (1 / (q - i eps)) / N
          v[r] = cmul(G, v[r]);
        }
        Butterfly<R2, true>::run(v, tw, N);
#pragma unroll
        for (int r = 1; r < R2; ++r) v[r] = cmul(v[r], cconj(tw[r * k1]));
#pragma unroll
        for (int r = 0; r < R2; ++r) Wt[(R2 * k1 + r) * kW + c] = v[r];
      }
      __syncthreads();
      for (int idx = tid; idx < kW * R2; idx += kT) {
        const int n2 = idx >> 4;
        float2 v[kR1];
#pragma unroll
        for (int r = 0; r < kR1; ++r) v[r] = Wt[(R2 * r + n2) * kW + c];
        Butterfly<kR1, true>::run(v, tw, N);
        if constexpr (k16) {   // lanes 8j .. 8j+7 hold columns 8h .. 8h+7 of the same rows
          const unsigned mask = __activemask();
          short2* out = a.T16 + gbase + c;
#pragma unroll
          for (int r = 0; r < kR1; ++r) {
            const int ex = b16_group_exponent(v[r], mask);
            const long long off = (long long)(R2 * r + n2) * rstride;
            if (c < ncol) {
              out[off] = b16_encode(v[r], ex);
              if ((c & 7) == 0) a.Te[(gbase + c + off) >> 3] = (signed char)ex;
            }
          }
        } else if (c < ncol) {
          float2* out = a.T + gbase + c;
#pragma unroll
          for (int r = 0; r < kR1; ++r) out[(R2 * r + n2) * rstride] = v[r];
        }
      }
      if constexpr (k16) {
        if (next < ntiles) {
          signed char* nx = ex16 + (s ^ 1) * L::kExStage;
#pragma unroll
          for (int q = 0; q < kExPer; ++q) {
            const int i = tid + q * kT;
            if (i < 2 * N) nx[i] = exn[q];
          }
        }
      }
      // the next iteration's copy refills the stage just read
      __syncthreads();
    } else {
      // ---- radix-R2 pass (ns = 1), in place: rows jr + 8r -> rows jr*R2 + r
      {
        float2 v[R2];
#pragma unroll
        for (int r = 0; r < R2; ++r) v[r] = S[(jr + kR1 * r) * kW + c];
        Butterfly<R2, kInvFirst>::run(v, tw, N);
        __syncthreads();
#pragma unroll
        for (int r = 0; r < R2; ++r) S[(jr * R2 + r) * kW + c] = v[r];
      }
      __syncthreads();
      // ---- radix-8 pass (ns = R2): rows j + R2 r, twiddles tw[r j], to global
      for (int idx = tid; idx < kW * R2; idx += kThreads) {
        const int j = idx >> 4;  // c is idx & 15 == tid & 15
        float2 v[kR1];
#pragma unroll
        for (int r = 0; r < kR1; ++r) v[r] = S[(j + R2 * r) * kW + c];
#pragma unroll
        for (int r = 1; r < kR1; ++r) {
          float2 w = tw[r * j];
          if (kInvFirst) w.y = -w.y;
          v[r] = cmul(v[r], w);
        }
        Butterfly<kR1, kInvFirst>::run(v, tw, N);
        if (c < ncol) {
          float2* out = a.T + gbase + c;
#pragma unroll
          for (int r = 0; r < kR1; ++r) out[(j + R2 * r) * rstride] = v[r];
        }
      }
      // the next iteration's copy refills the stage just read
      __syncthreads();
    }
  }
#endif
}

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// T viewed as float32 pairs: dims (inner first) {2*px, py, pz*nb} (y-pass) or
// {2*px, py, pz, nb} (z-pass); box 32 floats = 16 complex columns.  With
// 16-bit storage (b16) the map covers T16 viewed as 32-bit (re, im) int16
// pairs: dims {px, py, pz, nb}, box 16 columns (64 bytes).
bool make_map(const BornArgs& a, bool zpass, CUtensorMap* m, bool b16 = false) {
  auto enc = encoder();
  if (!enc) return false;
  const cuuint64_t px2 = 2ull * a.px;
  const cuuint64_t rowb = (cuuint64_t)a.px * sizeof(float2);
  const cuuint64_t planeb = rowb * a.py;
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r;
  if (b16) {
    const cuuint64_t rowb16 = (cuuint64_t)a.px * sizeof(short2);
    const cuuint64_t dims[4] = {(cuuint64_t)a.px, (cuuint64_t)a.py, (cuuint64_t)a.pz, (cuuint64_t)a.nbatch};
    const cuuint64_t strides[3] = {rowb16, rowb16 * a.py, rowb16 * a.py * a.pz};
    const cuuint32_t box[4] = {kW, 1, (cuuint32_t)a.pz, 1};
    r = enc(m, CU_TENSOR_MAP_DATA_TYPE_INT32, 4, a.T16, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  } else if (!zpass) {
    const cuuint64_t dims[3] = {px2, (cuuint64_t)a.py, (cuuint64_t)a.pz * a.nbatch};
    const cuuint64_t strides[2] = {rowb, planeb};
    // a box dimension holds at most 256 elements: longer columns (280) land
    // as two boxes of py / 2 rows on the same mbarrier
    const cuuint32_t rows = a.py > 256 ? (cuuint32_t)(a.py / 2) : (cuuint32_t)a.py;
    const cuuint32_t box[3] = {2 * kW, rows, 1};
    r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, a.T, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  } else {
    const cuuint64_t dims[4] = {px2, (cuuint64_t)a.py, (cuuint64_t)a.pz, (cuuint64_t)a.nbatch};
    const cuuint64_t strides[3] = {rowb, planeb, planeb * a.pz};
    const cuuint32_t box[4] = {2 * kW, 1, (cuuint32_t)a.pz, 1};
    r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.T, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  }
  return r == CUDA_SUCCESS;
}

template <int R2, int KIND>
cudaError_t launch_kind(const BornArgs& a, int jj, const DevFft& f, int* fault, cudaStream_t s) {
  using L = ColSmem<kR1 * R2>;
  constexpr size_t smem = KIND == 3 ? L::kTotalZ16 : KIND == 2 ? L::kTotalZ : L::kTotalY;
  static DeviceFlags configured;   // attribute raised once per device
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (!configured.test(dev)) {
    e = cudaFuncSetAttribute(cols_pipe_kernel<R2, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e != cudaSuccess) return e;
    configured.set(dev);
  }
  CUtensorMap map;
  if (!make_map(a, KIND >= 2, &map, KIND == 3)) return cudaErrorInvalidValue;
  int nsm = 0;
  e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  const int nxt = (a.px + kW - 1) / kW;
  const long long nout = KIND >= 2 ? (long long)a.py * a.nbatch : (long long)a.pz * a.nbatch;
  const long long ntiles = nout * nxt;
  int per_sm = 0;   // resident CTAs per SM (shared memory and registers allowing)
  constexpr int nthr = threads_of<KIND>();
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cols_pipe_kernel<R2, KIND>, nthr, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const long long cap = (long long)per_sm * nsm;
  const int grid = (int)(ntiles < cap ? ntiles : cap);
  cols_pipe_kernel<R2, KIND><<<grid, nthr, smem, s>>>(map, a, jj, f.tw, nxt, (int)ntiles, fault);
  return cudaGetLastError();
}

template <int KIND>
cudaError_t dispatch(const BornArgs& a, int jj, const DevFft& f, int* fault, cudaStream_t s) {
  switch (f.plan.n / kR1) {
    case 11: return launch_kind<11, KIND>(a, jj, f, fault, s);
    case 12:   // z-pass only (96 = 8 x 12, the fused passes' even length)
      if constexpr (KIND >= 2) return launch_kind<12, KIND>(a, jj, f, fault, s);
      return cudaErrorNotSupported;
    case 13: case 14: case 16: case 17: case 18: case 20:
      // z-pass only (104 - 160-point columns behind the fused xy-pass)
      if constexpr (KIND >= 2) {
        switch (f.plan.n / kR1) {
          case 13: return launch_kind<13, KIND>(a, jj, f, fault, s);
          case 14: return launch_kind<14, KIND>(a, jj, f, fault, s);
          case 16: return launch_kind<16, KIND>(a, jj, f, fault, s);
          case 17: return launch_kind<17, KIND>(a, jj, f, fault, s);
          case 18: return launch_kind<18, KIND>(a, jj, f, fault, s);
          default: return launch_kind<20, KIND>(a, jj, f, fault, s);
        }
      }
      return cudaErrorNotSupported;
    case 15: return launch_kind<15, KIND>(a, jj, f, fault, s);
    case 19: return launch_kind<19, KIND>(a, jj, f, fault, s);
    case 25: return launch_kind<25, KIND>(a, jj, f, fault, s);
    case 27: return launch_kind<27, KIND>(a, jj, f, fault, s);
    case 35:   // y-FFTs only (280 = 8 x 35 x-y planes)
      if constexpr (KIND < 2) return launch_kind<35, KIND>(a, jj, f, fault, s);
      return cudaErrorNotSupported;
    default: return cudaErrorNotSupported;
  }
}

}  // namespace

bool cols_pipe_supported(const BornArgs& a, const DevFft& f, bool zpass) {
  const int n = f.plan.n;
  if (n != (zpass ? a.pz : a.py) || n % kR1 != 0) return false;
  const int r2 = n / kR1;
  const bool zonly = r2 == 12 || r2 == 13 || r2 == 14 || r2 == 16 || r2 == 17 || r2 == 18 || r2 == 20;
  if (r2 != 11 && r2 != 15 && r2 != 19 && r2 != 25 && r2 != 27 && !(zpass && zonly) && !(!zpass && r2 == 35))
    return false;
  if (a.px % 2 != 0 || !encoder()) return false;   // row strides must be multiples of 16 bytes
  const long long nout = zpass ? (long long)a.py * a.nbatch : (long long)a.pz * a.nbatch;
  return nout * ((a.px + kW - 1) / kW) < (1LL << 31);
}

cudaError_t launch_fft_y_pipe(const BornArgs& a, bool inverse, const DevFft& fy, int* fault,
                              cudaStream_t s) {
  return inverse ? dispatch<1>(a, 0, fy, fault, s) : dispatch<0>(a, 0, fy, fault, s);
}

cudaError_t launch_born_z_pipe(const BornArgs& a, int jj, const DevFft& fz, int* fault, cudaStream_t s) {
  if (a.storage) {
    if (a.px % 8 != 0) return cudaErrorInvalidValue;   // 8-column exponent blocks, 16-byte rows
    return dispatch<3>(a, jj, fz, fault, s);
  }
  return dispatch<2>(a, jj, fz, fault, s);
}

}  // namespace odt
