// Goldstein branch-cut phase unwrapping (unwrapp2_gpu.m:1-6) on the GPU with
// a host linker.
//
//   1. residues of every 2x2 loop                 (get_residue_cuda.cu:34-66)
//   2. dipole removal, four neighbour directions  (remove_dipoles_cuda.cu:52-146)
//      -- within one direction every positive residue pairs with its own
//      neighbour, and residues never change sign, so a pass over the whole
//      map gives the reference's result whatever the thread order
//   3. ordered compaction of the non-zero residues (find(residue_map) - 1)
//   4. host: residue table, boxes and lookup     (goldstein_branch_cut.m:10-33)
//   5. the 8 nearest residues of each residue    (get_shortest_sort_cuda.cu)
//   6. host: branch linker, one thread per slice  (get_branches_goldstein_compute_v2.cpp)
//   7. rasterise the branches into the step maps (raster_branches_cuda.cu:67-131)
//   8. integrate along dimension 2 on row 1, then down every column
//                                                  (unwrapp_phase_goldstein_cuda.cu:62-115)
// Floating-point work follows the reference kernels' single-precision
// expressions operation by operation, with explicit round-to-nearest
// intrinsics so that no multiply-add is contracted: residues, dipole steps
// and raster positions are bit-exact, and the unwrapped phase is the
// reference's integration evaluated without contraction.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/odt.h"
#include "goldstein.h"
#include "goldstein_search.cuh"

namespace odt {
const char* set_last_error(const std::string& msg);
}

namespace {

using odt::gs::Branch;
using odt::gs::Table;
using odt::gs::TableView;

constexpr float kPi = 3.141592654f;  // the reference kernels' CUDART_PI_F
constexpr int kThreads = 256;
constexpr int kNearest = 8;           // precomputed_shortest_number
constexpr int kChunk = 16 * kThreads; // residues per compaction block

int grid_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  if (b > 148LL * 32) b = 148LL * 32;
  return (int)(b < 1 ? 1 : b);
}

__device__ __forceinline__ float wrap2pi(float a) {  // fmodf(fmodf(a, 2pi) + 2pi, 2pi)
  const float t = 2.0f * kPi;
  return fmodf(__fadd_rn(fmodf(a, t), t), t);
}

__global__ void residue_kernel(const float* __restrict__ ph, float* __restrict__ res, int M1, int M2,
                               long long total) {
  const int N1 = M1 + 1;
  const long long m12 = (long long)M1 * M2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long z = i / m12;
    const int d12 = (int)(i - z * m12);
    const int d2 = d12 / M1, d1 = d12 - d2 * M1;
    const float* p = ph + z * (long long)N1 * (M2 + 1) + (long long)d2 * N1 + d1;
    const float v11 = p[0], v21 = p[1], v12 = p[N1], v22 = p[N1 + 1];
    const float a = wrap2pi(__fadd_rn(__fsub_rn(v11, v12), kPi));
    const float b = wrap2pi(__fadd_rn(__fsub_rn(v21, v22), kPi));
    const float c = wrap2pi(__fadd_rn(__fsub_rn(v11, v21), kPi));
    const float d = wrap2pi(__fadd_rn(__fsub_rn(v12, v22), kPi));
    const float sum = __fsub_rn(__fsub_rn(__fadd_rn(a, d), b), c);
    res[i] = roundf(__fdiv_rn(sum, 2.0f * kPi));
  }
}

// One direction of the dipole pass: 0 = d1-1, 1 = d2-1, 2 = d1+1, 3 = d2+1.
__global__ void dipole_kernel(float* __restrict__ res, int32_t* __restrict__ step1, int M1, int M2,
                              long long total, int dir) {
  const long long m12 = (long long)M1 * M2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    float v = res[i];
    if (!(v > 0.f)) continue;
    const long long z = i / m12;
    const int d12 = (int)(i - z * m12);
    const int d2 = d12 / M1, d1 = d12 - d2 * M1;
    const int p1 = d1 - (dir == 0) + (dir == 2);
    const int p2 = d2 - (dir == 1) + (dir == 3);
    if (p1 < 0 || p2 < 0 || p1 >= M1 || p2 >= M2) continue;
    const long long ip = z * m12 + (long long)p2 * M1 + p1;
    float pv = res[ip];
    if (!(pv < 0.f)) continue;
    const float take = fminf(v, -pv);
    v = roundf(__fsub_rn(v, take));
    pv = roundf(__fadd_rn(pv, take));
    res[i] = v;
    res[ip] = pv;
    if (dir == 1 || dir == 3) {
      const int N1 = M1 + 1, N2 = M2 + 1;
      const long long o = z * (long long)N1 * N2 + (long long)(min(d2, p2) + 1) * N1 + (p1 + 1);
      step1[o] = (int32_t)(dir == 1 ? take : -take);
    }
  }
}

__device__ __forceinline__ int block_sum(int v, int* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) sh[w] = v;
  __syncthreads();
  int t = 0;
  for (int k = 0; k < kThreads / 32; ++k) t += sh[k];
  __syncthreads();
  return t;
}

__global__ void nz_count_kernel(const float* __restrict__ res, long long total, int* __restrict__ cnt) {
  __shared__ int sh[kThreads / 32];
  const long long base = (long long)blockIdx.x * kChunk;
  int c = 0;
  for (int k = 0; k < kChunk / kThreads; ++k) {
    const long long e = base + k * kThreads + threadIdx.x;
    c += (e < total && res[e] != 0.f) ? 1 : 0;
  }
  c = block_sum(c, sh);
  if (threadIdx.x == 0) cnt[blockIdx.x] = c;
}

// Exclusive scan of n counts in one block of 1024 threads; total in *sum.
__global__ void scan_kernel(int* __restrict__ a, int n, long long* __restrict__ sum) {
  __shared__ int s[1024];
  long long carry = 0;
  for (int b = 0; b < n; b += 1024) {
    const int i = b + threadIdx.x;
    const int v = i < n ? a[i] : 0;
    s[threadIdx.x] = v;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
      const int t = threadIdx.x >= off ? s[threadIdx.x - off] : 0;
      __syncthreads();
      s[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < n) a[i] = (int)(carry + s[threadIdx.x] - v);
    carry += s[1023];
    __syncthreads();
  }
  if (threadIdx.x == 0) *sum = carry;
}

// Non-zero residues in index order: idx (0-based) and integer value.
__global__ void nz_scatter_kernel(const float* __restrict__ res, long long total, const int* __restrict__ off,
                                  int32_t* __restrict__ idx, int32_t* __restrict__ val) {
  __shared__ int wsum[kThreads / 32];
  const long long base = (long long)blockIdx.x * kChunk;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int run = off[blockIdx.x];
  for (int k = 0; k < kChunk / kThreads; ++k) {
    const long long e = base + k * kThreads + threadIdx.x;
    const float r = e < total ? res[e] : 0.f;
    const bool f = r != 0.f;
    const unsigned m = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wsum[w] = __popc(m);
    __syncthreads();
    int before = 0, all = 0;
    for (int q = 0; q < kThreads / 32; ++q) {
      before += q < w ? wsum[q] : 0;
      all += wsum[q];
    }
    if (f) {
      const int at = run + before + __popc(m & ((1u << lane) - 1u));
      idx[at] = (int32_t)e;
      val[at] = (int32_t)r;
    }
    run += all;
    __syncthreads();
  }
}

__global__ void nearest_kernel(TableView T, int32_t* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= T.R) return;
  int cur[2 * kNearest];
  odt::gs::nearest<kNearest>(T, i, nullptr, cur);
  for (int k = 0; k < 2 * kNearest; ++k) out[2 * kNearest * (long long)i + k] = cur[k];
}

// Add each branch's charge to the steps it crosses (raster_compute_kernel).
__global__ void raster_kernel(const Branch* __restrict__ br, int nb, int32_t* __restrict__ step1,
                              int32_t* __restrict__ step2, int N1, int N2) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  int x1 = br[b].x1, y1 = br[b].y1, x2 = br[b].x2, y2 = br[b].y2;
  const int z = br[b].z;
  int jump = br[b].jump;
  if (x1 == -1) {  // to the nearest border
    const bool xs = x2 < N1 - x2, ys = y2 < N2 - y2;
    const int dx = xs ? x2 : N1 - x2, dy = ys ? y2 : N2 - y2;
    x1 = dx > dy ? x2 : (xs ? -1 : N1 - 1);
    y1 = dx < dy ? y2 : (ys ? -1 : N2 - 1);
    if (x1 == -1) {
      atomicAdd(&step2[(long long)N2 * z + y2 + 1], jump);
      return;
    }
  }
  if (y1 == y2) return;
  if (y2 > y1) {
    int t = y1; y1 = y2; y2 = t;
    t = x1; x1 = x2; x2 = t;
    jump = -jump;
  }
  const int steps = y1 - y2;
  const long long zo = (long long)N1 * N2 * z;
  for (int i = 0; i < steps; ++i) {
    const int cy = y2 + i + 1;
    const int cx = x2 + (int)__fmul_rn(__fdiv_rn((float)i, (float)steps), (float)(x1 - x2)) + 1;
    atomicAdd(&step1[zo + (long long)N1 * cy + cx], jump);
  }
}

__device__ __forceinline__ float unwrap_step(float last, float cur, int32_t step) {
  const float d = __fsub_rn(wrap2pi(__fadd_rn(__fsub_rn(cur, last), kPi)), kPi);
  return __fsub_rn(__fadd_rn(last, d), __fmul_rn(__fmul_rn((float)step, 2.0f), kPi));
}

__global__ void unwrap_row_kernel(float* __restrict__ ph, const int32_t* __restrict__ step2, int N1, int N2,
                                  int n) {
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= n) return;
  float* p = ph + (long long)z * N1 * N2;
  float last = p[0];
  for (int i = 1; i < N2; ++i) {
    last = unwrap_step(last, p[(long long)i * N1], step2[(long long)z * N2 + i]);
    p[(long long)i * N1] = last;
  }
}

__global__ void unwrap_col_kernel(float* __restrict__ ph, const int32_t* __restrict__ step1, int N1, int N2,
                                  int n) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c >= (long long)N2 * n) return;
  float* p = ph + c * N1;
  const int32_t* s = step1 + c * N1;
  float last = p[0];
  for (int i = 1; i < N1; ++i) {
    last = unwrap_step(last, p[i], s[i]);
    p[i] = last;
  }
}

odt_status fail(odt_status st, const std::string& m) {
  odt::set_last_error(m);
  return st;
}

struct Buffers {
  std::vector<void*> ptrs;
  cudaStream_t s;
  ~Buffers() {
    for (void* p : ptrs) cudaFreeAsync(p, s);
  }
  template <typename T>
  T* get(size_t n) {
    void* p = nullptr;
    if (cudaMallocAsync(&p, (n ? n : 1) * sizeof(T) + 16, s) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return static_cast<T*>(p);
  }
};

#define GS_CHECK(call)                                                                        \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if (e_ != cudaSuccess) {                                                                  \
      cudaGetLastError();                                                                     \
      return fail(ODT_ERR_CUDA, std::string("odt_unwrap_goldstein: ") + cudaGetErrorString(e_)); \
    }                                                                                         \
  } while (0)

}  // namespace

extern "C" odt_status odt_unwrap_goldstein(const odt_unwrap_args* a) {
  if (!a || !a->phase_in || !a->phase_out) return fail(ODT_ERR_INVALID_ARGUMENT, "odt_unwrap_goldstein: NULL phase");
  const int N1 = a->size[0], N2 = a->size[1], n = a->size[2];
  if (N1 < 2 || N2 < 2 || n < 1)
    return fail(ODT_ERR_INVALID_ARGUMENT, "odt_unwrap_goldstein: size must be >= [2, 2, 1]");
  const long long np = (long long)N1 * N2 * n;
  if (np >= (1LL << 31)) return fail(ODT_ERR_INVALID_ARGUMENT, "odt_unwrap_goldstein: more than 2^31 elements");
  if (a->memory != ODT_MEM_HOST && a->memory != ODT_MEM_DEVICE)
    return fail(ODT_ERR_INVALID_ARGUMENT, "odt_unwrap_goldstein: bad memory flag");
  if ((a->table_out || a->nearest_out) && a->residue_cap < 0)
    return fail(ODT_ERR_INVALID_ARGUMENT, "odt_unwrap_goldstein: negative residue_cap");
  if (a->branches_out && a->branch_cap < 0)
    return fail(ODT_ERR_INVALID_ARGUMENT, "odt_unwrap_goldstein: negative branch_cap");
  const bool dev = a->memory == ODT_MEM_DEVICE;
  cudaStream_t s = dev ? (cudaStream_t)a->stream : (cudaStream_t)0;
  const cudaMemcpyKind kin = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const cudaMemcpyKind kout = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  const int M1 = N1 - 1, M2 = N2 - 1;
  const long long nr = (long long)M1 * M2 * n;
  Buffers B;
  B.s = s;
  float* ph = dev ? a->phase_out : B.get<float>(np);
  float* res = B.get<float>(nr);
  int32_t* step1 = B.get<int32_t>(np);
  int32_t* step2 = B.get<int32_t>((size_t)N2 * n);
  const int nchunks = (int)((nr + kChunk - 1) / kChunk);
  int* chunk = B.get<int>(nchunks);
  long long* total = B.get<long long>(1);
  if (!ph || !res || !step1 || !step2 || !chunk || !total)
    return fail(ODT_ERR_OUT_OF_MEMORY, "odt_unwrap_goldstein: device allocation failed");
  if (ph != a->phase_in) GS_CHECK(cudaMemcpyAsync(ph, a->phase_in, np * sizeof(float), kin, s));
  GS_CHECK(cudaMemsetAsync(step1, 0, np * sizeof(int32_t), s));
  GS_CHECK(cudaMemsetAsync(step2, 0, (size_t)N2 * n * sizeof(int32_t), s));
  residue_kernel<<<grid_for(nr), kThreads, 0, s>>>(ph, res, M1, M2, nr);
  for (int dir = 0; dir < 4; ++dir) dipole_kernel<<<grid_for(nr), kThreads, 0, s>>>(res, step1, M1, M2, nr, dir);
  GS_CHECK(cudaGetLastError());
  if (a->residue_out) GS_CHECK(cudaMemcpyAsync(a->residue_out, res, nr * sizeof(float), kout, s));

  // ordered list of the non-zero residues
  nz_count_kernel<<<nchunks, kThreads, 0, s>>>(res, nr, chunk);
  scan_kernel<<<1, 1024, 0, s>>>(chunk, nchunks, total);
  GS_CHECK(cudaGetLastError());
  long long R = 0;
  GS_CHECK(cudaMemcpyAsync(&R, total, sizeof(R), cudaMemcpyDeviceToHost, s));
  GS_CHECK(cudaStreamSynchronize(s));
  if (a->n_residues) *a->n_residues = R;
  std::vector<Branch> branches;
  if (R > 0) {
    int32_t* idx = B.get<int32_t>(R);
    int32_t* val = B.get<int32_t>(R);
    if (!idx || !val) return fail(ODT_ERR_OUT_OF_MEMORY, "odt_unwrap_goldstein: device allocation failed");
    nz_scatter_kernel<<<nchunks, kThreads, 0, s>>>(res, nr, chunk, idx, val);
    GS_CHECK(cudaGetLastError());
    std::vector<int32_t> hidx(R), hval(R);
    GS_CHECK(cudaMemcpyAsync(hidx.data(), idx, R * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    GS_CHECK(cudaMemcpyAsync(hval.data(), val, R * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    GS_CHECK(cudaStreamSynchronize(s));
    Table t;
    odt::gs::build_table(hidx.data(), hval.data(), R, M1, M2, n, &t);

    // 8 nearest residues of every residue
    TableView T = odt::gs::view_of(t);
    int32_t* drows = B.get<int32_t>(t.rows.size());
    int32_t* dlook = B.get<int32_t>(t.lookup.size());
    int32_t* dzs = B.get<int32_t>(n);
    int32_t* dsq = B.get<int32_t>(n);
    int32_t* dnear = B.get<int32_t>((size_t)2 * kNearest * R);
    if (!drows || !dlook || !dzs || !dsq || !dnear)
      return fail(ODT_ERR_OUT_OF_MEMORY, "odt_unwrap_goldstein: device allocation failed");
    GS_CHECK(cudaMemcpyAsync(drows, t.rows.data(), t.rows.size() * 4, cudaMemcpyHostToDevice, s));
    GS_CHECK(cudaMemcpyAsync(dlook, t.lookup.data(), t.lookup.size() * 4, cudaMemcpyHostToDevice, s));
    GS_CHECK(cudaMemcpyAsync(dzs, t.zstart.data(), n * 4, cudaMemcpyHostToDevice, s));
    GS_CHECK(cudaMemcpyAsync(dsq, t.square.data(), n * 4, cudaMemcpyHostToDevice, s));
    TableView D = T;
    D.rows = drows;
    D.lookup = dlook;
    D.zstart = dzs;
    D.square = dsq;
    nearest_kernel<<<(int)((R + 127) / 128), 128, 0, s>>>(D, dnear);
    GS_CHECK(cudaGetLastError());
    std::vector<int32_t> hnear((size_t)2 * kNearest * R);
    GS_CHECK(cudaMemcpyAsync(hnear.data(), dnear, hnear.size() * 4, cudaMemcpyDeviceToHost, s));
    GS_CHECK(cudaStreamSynchronize(s));
    if (a->table_out && a->residue_cap > 0)
      GS_CHECK(cudaMemcpyAsync(a->table_out, t.rows.data(), std::min<long long>(R, a->residue_cap) * 6 * 4,
                               dev ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost, s));
    if (a->nearest_out && a->residue_cap > 0)
      GS_CHECK(cudaMemcpyAsync(a->nearest_out, hnear.data(),
                               std::min<long long>(R, a->residue_cap) * 2 * kNearest * 4,
                               dev ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost, s));

    // branch cuts, then their charges into the step maps
    odt::gs::link_branches(t, hnear.data(), kNearest, a->link_threads, &branches);
    const long long nb = (long long)branches.size();
    if (nb > 0) {
      Branch* dbr = B.get<Branch>(nb);
      if (!dbr) return fail(ODT_ERR_OUT_OF_MEMORY, "odt_unwrap_goldstein: device allocation failed");
      GS_CHECK(cudaMemcpyAsync(dbr, branches.data(), nb * sizeof(Branch), cudaMemcpyHostToDevice, s));
      raster_kernel<<<(int)((nb + kThreads - 1) / kThreads), kThreads, 0, s>>>(dbr, (int)nb, step1, step2, N1, N2);
      GS_CHECK(cudaGetLastError());
    }
    if (a->branches_out && a->branch_cap > 0 && nb > 0)
      GS_CHECK(cudaMemcpyAsync(a->branches_out, branches.data(), std::min<long long>(nb, a->branch_cap) * sizeof(Branch),
                               dev ? cudaMemcpyHostToDevice : cudaMemcpyHostToHost, s));
  }
  if (a->n_branches) *a->n_branches = (long long)branches.size();

  unwrap_row_kernel<<<(n + 127) / 128, 128, 0, s>>>(ph, step2, N1, N2, n);
  unwrap_col_kernel<<<(int)(((long long)N2 * n + 127) / 128), 128, 0, s>>>(ph, step1, N1, N2, n);
  GS_CHECK(cudaGetLastError());
  if (a->step1_out) GS_CHECK(cudaMemcpyAsync(a->step1_out, step1, np * 4, kout, s));
  if (a->step2_out) GS_CHECK(cudaMemcpyAsync(a->step2_out, step2, (size_t)N2 * n * 4, kout, s));
  if (!dev) GS_CHECK(cudaMemcpyAsync(a->phase_out, ph, np * sizeof(float), cudaMemcpyDeviceToHost, s));
  GS_CHECK(cudaStreamSynchronize(s));  // host tables above are freed on return
  return ODT_OK;
}
