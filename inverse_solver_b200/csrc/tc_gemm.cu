// Complex single-precision GEMM on the 5th-generation tensor cores
// (tcgen05, kind::tf32) for the plane part of the Green's function set-up
// (green_dev.cu: the three chains of centred DFT maps of
// truncated_green_plus.m:67-110).
//
// FP32 accuracy from TF32 operands: every operand is split into two TF32
// parts x = h + m (h = tf32(x), m = tf32(x - h), round to nearest; 22
// significant bits) and the accumulator takes m*h + h*m + h*h, smallest
// first (the dropped m*m and the split's remainder are near 2^-22 of each
// product).  A three-part split (h, m, l = tf32(x - h - m)) with six products
// is kept as a build option (ODT_TC_PARTS=3); it measured no more accurate
// (8.3e-7 against 8.1e-7 - 8.6e-7 rel-L2 on the Green's function planes)
// once the K sums are taken in FP32 registers (below).
//
// The complex product C = A B is one real GEMM of twice the size with the
// interleaved complex layout kept on the A side:
//   A'[m][2k + c]      = (Re, Im)(A(m, k))[c]                     (M x 2K)
//   B'^T[2n + j][2k + c] = [[Re B, -Im B], [Im B, Re B]](k, n)[j][c] (2N x 2K)
//   C'[m][2n + j]      = (Re, Im)(C(m, n))[j]
// Both operands are K-major (rows of 2K reals), written by a conversion
// kernel together with their TF32 split, zero-padded to whole tiles, into a
// workspace the caller provides (tc_cgemm_work floats).
//
// The tensor cores' own accumulation over K is not IEEE-rounded FP32: over
// the Green's function GEMMs (K up to 2 x 409 reals) it left 2.1e-6 rel-L2
// against the host build, with two-part and with three-part operands alike,
// where the FP32 SIMT GEMM leaves 5.6e-7.  So every 32-wide K block is
// accumulated afresh in tensor memory and the blocks are added in FP32
// registers: 8.1e-7 - 8.6e-7.
//
// Kernel: one CTA of 160 threads per 128 x 128 tile of C' (and batch
// entry).  Warp 4 (one thread) issues the tiled copies (cp.async.bulk.tensor,
// 128-byte swizzle, 128 rows x 32 reals per operand part and stage, two
// stages) and the MMAs (M = 128, N = 128, K = 8 per instruction, 12 per K
// block) into one of two 128 x 128 FP32 accumulators in tensor memory;
// tcgen05.commit hands a stage back once its MMAs have read it and tells the
// epilogue that the accumulator is complete.  Warps 0-3 (rows 32 w ..
// 32 w + 31, the tensor-memory lanes their warp may read) add each block's
// accumulator into registers with tcgen05.ld and hand it back; at the end
// they store the complex values into the column-major output.  Every wait is
// bounded and a timeout leaves a fault code (no copy or MMA is in flight
// when the CTA frees its tensor memory and exits).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <string>

#include "tma.cuh"

namespace odt {
namespace {

constexpr int kTM = 128, kTN = 128, kTK = 32;   // tile of C' and K block (reals)
constexpr int kEpiWarps = 4;                    // warps reading the accumulator (32 rows each)
constexpr int kThreads = 32 * (kEpiWarps + 1);  // + one warp issuing copies and MMAs
constexpr int kTmemCols = 2 * kTN;              // two FP32 accumulators of 128 columns
constexpr uint32_t kOpBytes = kTM * kTK * 4;    // one operand tile: 16 KB
#ifndef ODT_TC_PARTS
#define ODT_TC_PARTS 2
#endif
constexpr int kParts = ODT_TC_PARTS;            // TF32 parts per operand (2 or 3)
static_assert(kParts == 2 || kParts == 3, "two or three TF32 parts");
constexpr uint32_t kStageBytes = 2 * kParts * kOpBytes;  // the parts of A, then of B
constexpr size_t kSmem = 1024 + 2 * (size_t)kStageBytes + 1024;   // barriers, 2 stages, alignment slack

// instruction descriptor: D FP32, A and B TF32, both K-major, N = 128, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTN >> 3) << 17) |
                            ((uint32_t)(kTM >> 4) << 24);

#if defined(__CUDA_ARCH__)
// shared-memory matrix descriptor of a K-major operand tile with the 128-byte
// swizzle: 8-row groups 1024 bytes apart (stride byte offset), leading byte
// offset 1 (unused for this layout), version 1, layout type 2
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;
  d |= (uint64_t)(1024u >> 4) << 32;
  d |= (uint64_t)1u << 46;
  d |= (uint64_t)2u << 61;
  return d;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int c0, int c1, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_addr(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate)
      : "memory");
}

// arrives on `bar` once every MMA this thread issued so far has completed
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 32 consecutive FP32 columns of this thread's lane
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// the TF32 parts of x into out[i], out[total + i] (, out[2 total + i])
__device__ __forceinline__ void split3(float x, float* out, long long i, long long total) {
  const float h = to_tf32(x);
  const float r = x - h;   // exact
  const float m = to_tf32(r);
  out[i] = h;
  out[total + i] = m;
  if (kParts == 3) out[2 * total + i] = to_tf32(r - m);
}
#endif

// A (column-major complex, element (m, k) at A[m + lda k + sA b]) -> hi / lo
// of A' [batch][Mp][Kp] (K-major reals, zero padding)
__global__ void tc_split_a(const float2* __restrict__ A, int M, int K, int lda, long long sA, int Mp, int Kp,
                           long long total, float* __restrict__ out) {
#if defined(__CUDA_ARCH__)
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int kk = (int)(i % Kp);
    const long long t = i / Kp;
    const int m = (int)(t % Mp);
    const long long b = t / Mp;
    const int k = kk >> 1;
    float x = 0.f;
    if (m < M && k < K) {
      const float2 v = A[sA * b + m + (long long)lda * k];
      x = (kk & 1) ? v.y : v.x;
    }
    split3(x, out, i, total);
  }
#endif
}

// B (complex, op(B)(k, n) = transB ? B[n + ldb k] : B[k + ldb n], batch
// stride sB) -> hi / lo of B'^T [batch][Np][Kp]: row 2n (real part of the
// output) = (Re, -Im), row 2n + 1 (imaginary part) = (Im, Re) over k
__global__ void tc_split_b(const float2* __restrict__ B, int N, int K, int ldb, long long sB, int transB, int Np,
                           int Kp, long long total, float* __restrict__ out) {
#if defined(__CUDA_ARCH__)
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int kk = (int)(i % Kp);
    const long long t = i / Kp;
    const int j = (int)(t % Np);
    const long long b = t / Np;
    const int n = j >> 1, k = kk >> 1;
    float x = 0.f;
    if (n < N && k < K) {
      const float2 v = transB ? B[sB * b + n + (long long)ldb * k] : B[sB * b + k + (long long)ldb * n];
      const int jc = j & 1, kc = kk & 1;
      x = jc == 0 ? (kc == 0 ? v.x : -v.y) : (kc == 0 ? v.y : v.x);
    }
    split3(x, out, i, total);
  }
#endif
}

struct TcMaps {
  CUtensorMap a[kParts], b[kParts];   // h, m, l
};

__global__ void __launch_bounds__(kThreads, 1)
    tc_cgemm_kernel(const __grid_constant__ TcMaps maps, int M, int N2, int nkb, int Mp, int Np, int batchA,
                    int batchB, float2* __restrict__ C, int ldc, long long sC, int* __restrict__ fault) {
#if defined(__CUDA_ARCH__)
  extern __shared__ __align__(1024) unsigned char smt[];
  // [0, 72): full[2], empty[2], accf[2], acce[2], done; [96, 100): tensor-memory base
  uint64_t* full = reinterpret_cast<uint64_t*>(smt);
  uint64_t* empty = full + 2;
  uint64_t* accf = full + 4;   // accumulator t holds a finished K block
  uint64_t* acce = full + 6;   // accumulator t has been read by the 4 epilogue warps
  uint64_t* done = full + 8;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(smt + 96);
  unsigned char* tiles = smt + 1024;
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  if ((smem_addr(tiles) & 1023u) != 0u) {   // the swizzle atoms need 1024-byte alignment
    if (tid == 0) atomicCAS(fault, 0, kFaultAlign);
    return;
  }
  const int b = blockIdx.z;
  const int m0 = blockIdx.x * kTM, j0 = blockIdx.y * kTN;
  const int rowA = (batchA > 1 ? b : 0) * Mp + m0;
  const int rowB = (batchB > 1 ? b : 0) * Np + j0;
  if (tid == 0) {
    for (int i = 0; i < 6; ++i) mbar_init(&full[i], 1);
    mbar_init(&acce[0], kEpiWarps);
    mbar_init(&acce[1], kEpiWarps);
    mbar_init(done, 1);
    mbar_fence_init();
  }
  if (w == 0) {   // tensor memory: two accumulators of 128 x 128 FP32
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;

  bool ok = true;
  if (w == kEpiWarps) {
    // ---- producer / MMA issuer (one thread)
    if (lane == 0) {
      auto stage = [&](int st, int q) { return tiles + (size_t)st * kStageBytes + (size_t)q * kOpBytes; };
      auto issue = [&](int kb) {
        const int st = kb & 1;
        mbar_arrive_expect_tx(&full[st], kStageBytes);
#pragma unroll
        for (int q = 0; q < kParts; ++q) {
          tma_load_2d(stage(st, q), &maps.a[q], kTK * kb, rowA, &full[st]);
          tma_load_2d(stage(st, kParts + q), &maps.b[q], kTK * kb, rowB, &full[st]);
        }
      };
      int landed = 0, issued = 1;   // K blocks whose copies were waited for / issued
      issue(0);
      for (int kb = 0; kb < nkb && ok; ++kb) {
        const int st = kb & 1, t = kb & 1;
        if (kb + 1 < nkb) {
          // stage (kb + 1) & 1 held block kb - 1: its MMAs must have read it
          if (kb >= 1) ok = mbar_wait(&empty[(kb + 1) & 1], (uint32_t)((kb - 1) >> 1) & 1u);
          if (!ok) break;
          issue(kb + 1);
          issued = kb + 2;
        }
        ok = mbar_wait(&full[st], (uint32_t)(kb >> 1) & 1u);
        if (!ok) break;
        landed = kb + 1;
        // accumulator t held block kb - 2: the epilogue warps must have read it
        if (kb >= 2) ok = mbar_wait(&acce[t], (uint32_t)((kb - 2) >> 1) & 1u);
        if (!ok) break;
        tc_fence_after();
        const uint32_t acc = tmem + (uint32_t)(t * kTN);
        const uint32_t a_h = smem_addr(stage(st, 0)), a_m = smem_addr(stage(st, 1));
        const uint32_t b_h = smem_addr(stage(st, kParts)), b_m = smem_addr(stage(st, kParts + 1));
#pragma unroll
        for (int ks = 0; ks < kTK / 8; ++ks) {   // 8 TF32 = 32 bytes of K per MMA
          const uint32_t o = 32u * ks;
          if constexpr (kParts == 3) {   // l h + h l + m m + m h + h m + h h
            const uint32_t a_l = smem_addr(stage(st, 2)), b_l = smem_addr(stage(st, 5));
            umma_tf32(acc, sw128_desc(a_l + o), sw128_desc(b_h + o), ks > 0 ? 1u : 0u);
            umma_tf32(acc, sw128_desc(a_h + o), sw128_desc(b_l + o), 1u);
            umma_tf32(acc, sw128_desc(a_m + o), sw128_desc(b_m + o), 1u);
            umma_tf32(acc, sw128_desc(a_m + o), sw128_desc(b_h + o), 1u);
          } else {                       // m h + h m + h h (m is the second, last part)
            umma_tf32(acc, sw128_desc(a_m + o), sw128_desc(b_h + o), ks > 0 ? 1u : 0u);
          }
          umma_tf32(acc, sw128_desc(a_h + o), sw128_desc(b_m + o), 1u);
          umma_tf32(acc, sw128_desc(a_h + o), sw128_desc(b_h + o), 1u);
        }
        umma_commit(&empty[st]);
        umma_commit(&accf[t]);
      }
      umma_commit(done);   // every MMA issued above
      if (!ok) {
        atomicCAS(fault, 0, kFaultTimeout);
        // the copies issued but not waited for (blocks landed .. issued - 1, in
        // different stages) must land before the CTA exits
        for (int kb = landed; kb < issued; ++kb) mbar_wait(&full[kb & 1], (uint32_t)(kb >> 1) & 1u);
      }
    }
    __syncwarp();
  } else {
    // ---- epilogue warps: row m0 + 32 w + lane; each K block's accumulator is
    // added into FP32 registers (IEEE rounding) and handed back
    float sum[kTN];
#pragma unroll
    for (int i = 0; i < kTN; ++i) sum[i] = 0.f;
    const uint32_t lane_off = (uint32_t)(32 * w) << 16;
    for (int kb = 0; kb < nkb; ++kb) {
      const int t = kb & 1;
      const bool got = __all_sync(0xffffffffu, mbar_wait(&accf[t], (uint32_t)(kb >> 1) & 1u));
      if (!got) {
        ok = false;
        break;
      }
      tc_fence_after();
#pragma unroll
      for (int c0 = 0; c0 < kTN; c0 += 32) {
        float v[32];
        tmem_ld32(tmem + lane_off + (uint32_t)(t * kTN + c0), v);
#pragma unroll
        for (int i = 0; i < 32; ++i) sum[c0 + i] += v[i];
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acce[t]);
    }
    if (ok) {
      const int m = m0 + 32 * w + lane;
      if (m < M) {
#pragma unroll
        for (int q = 0; q < kTN / 2; ++q) {
          const int j = j0 + 2 * q;
          if (j < N2) C[sC * b + m + (long long)ldc * (j >> 1)] = make_float2(sum[2 * q], sum[2 * q + 1]);
        }
      }
    } else if (lane == 0) {
      atomicCAS(fault, 0, kFaultTimeout);
    }
  }
  // no MMA may still be writing tensor memory when it is freed
  mbar_wait(done, 0u);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (w == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
#endif
}

PFN_cuTensorMapEncodeTiled_v12000 tc_encoder() {
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

// [rows][Kp] FP32, box 32 x 128 with the 128-byte swizzle
bool tc_map(CUtensorMap* m, const float* base, long long rows, int Kp) {
  auto enc = tc_encoder();
  if (!enc) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)Kp * sizeof(float)};
  const cuuint32_t box[2] = {(cuuint32_t)kTK, (cuuint32_t)kTM};
  const cuuint32_t estr[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int grid_for(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148LL * 16) b = 148LL * 16;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

// C_b[M x N] = A_b[M x K] * op(B_b), complex, column-major, as green_dev.cu's
// SIMT cgemm (op(B) = B [K x N] with ldb, or transB: B stored [N x K]); a
// batch stride of 0 shares the operand across the batch.  *fault (device
// int) receives a timeout / alignment code.
// Floats of operand workspace tc_cgemm needs for these sizes (the TF32 parts
// of both operands, padded to whole tiles).
long long tc_cgemm_work(int M, int N, int K, bool batchedA, bool batchedB, int batch) {
  const long long Mp = (M + kTM - 1) / kTM * kTM;
  const long long Np = (2LL * N + kTN - 1) / kTN * kTN;
  const long long Kp = (2LL * K + kTK - 1) / kTK * kTK;
  return kParts * ((batchedA ? batch : 1) * Mp * Kp + (batchedB ? batch : 1) * Np * Kp);
}

cudaError_t tc_cgemm(int M, int N, int K, const float2* A, int lda, long long sA, const float2* B, int ldb,
                     long long sB, bool transB, float2* C, int ldc, long long sC, int batch, float* work,
                     long long work_floats, int* fault, cudaStream_t s) {
  if (M < 1 || N < 1 || K < 1 || batch < 1 || batch > 65535 || !work) return cudaErrorInvalidValue;
  const int Mp = (M + kTM - 1) / kTM * kTM;
  const int Np = (2 * N + kTN - 1) / kTN * kTN;
  const int Kp = (2 * K + kTK - 1) / kTK * kTK;
  const int bA = sA ? batch : 1, bB = sB ? batch : 1;
  const long long na = (long long)bA * Mp * Kp, nb = (long long)bB * Np * Kp;
  if ((long long)bA * Mp > (1LL << 31) || (long long)bB * Np > (1LL << 31)) return cudaErrorInvalidValue;
  if (work_floats < kParts * (na + nb)) return cudaErrorInvalidValue;
  float *pa = work, *pb = work + kParts * na;   // the parts of each operand, one after the other
  tc_split_a<<<grid_for(na), 256, 0, s>>>(A, M, K, lda, sA, Mp, Kp, na, pa);
  tc_split_b<<<grid_for(nb), 256, 0, s>>>(B, N, K, ldb, sB, transB ? 1 : 0, Np, Kp, nb, pb);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  TcMaps maps;
  for (int q = 0; q < kParts; ++q) {
    if (!tc_map(&maps.a[q], pa + q * na, (long long)bA * Mp, Kp) ||
        !tc_map(&maps.b[q], pb + q * nb, (long long)bB * Np, Kp))
      return cudaErrorInvalidValue;
  }
  static DeviceFlags configured;
  int dev = 0;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
  if (!configured.test(dev)) {
    e = cudaFuncSetAttribute(tc_cgemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem);
    if (e != cudaSuccess) return e;
    configured.set(dev);
  }
  const dim3 grid(Mp / kTM, Np / kTN, batch);
  tc_cgemm_kernel<<<grid, kThreads, kSmem, s>>>(maps, M, 2 * N, Kp / kTK, Mp, Np, bA, bB, C, ldc, sC, fault);
  return cudaGetLastError();
}

}  // namespace odt
