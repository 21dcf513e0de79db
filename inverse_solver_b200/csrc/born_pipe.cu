// Pipelined x-pass of the Born iteration for x-lengths n = 8 * R2 (R2 odd:
// 11, 15, 19, 25, 27, and 35 = 5 x 7 as one composite butterfly):
// the same arithmetic as born_x_body in modes Mid (inverse x-FFT, update of
// iteration jj-1, source term of iteration jj, forward x-FFT;
// FORWARD_SOLVER_CONVERGENT_BORN.m:588-605, :616-642; jj >= 2) and Last
// (update of the final iteration, Field(ROI) + incident field, :646-647),
// restructured for the
// B200 memory system:
//
//   * persistent CTAs (two per SM) walk the tiles of 16 x-lines (8 lines and
//     three CTAs per SM for n = 200, 216); a tile of
//     consecutive lines is one contiguous block of T, Field_n and Field, so
//     one thread moves it into shared memory with bulk asynchronous copies
//     (the TMA engine) completing on an mbarrier;
//   * T of the next tile is copied while the current one is computed, and
//     Field_n / Field of the next tile while the current one finishes its
//     last FFT pass, so DRAM latency overlaps the FFT arithmetic instead of
//     stalling it;
//   * the plan is fixed at compile time: inverse radix-R2 pass (in place in
//     the landing buffer: every thread holds its butterfly in registers across
//     a barrier), fused inverse-8 / update / forward-8 pass, forward radix-R2
//     pass written straight to global memory.
//
// Shared-memory layouts: landing buffers are the global layout [line][x]
// (pitch n; with 16 lines and R1 = 8 the radix-R2 passes' accesses are
// conflict-free for any odd R2), the mid pass writes a [line][x + x/8]
// buffer with pitch = 8 (mod 16) (conflict-free stride-8 stores).
#include <cuda_runtime.h>

#include "cbs_kernels.cuh"
#include "fft_core.cuh"
#include "fft_tile.cuh"
#include "tile_launch.cuh"
#include "tma.cuh"

namespace odt {
namespace {

constexpr int kR1 = 8;                 // a tile of W x-lines takes W * 8 threads:
                                       // one radix-R2 butterfly per thread

struct PipeLine {      // per-line constants of a tile
  long long g;         // element offset of x = 0 in T / Field_n / Field
  long long einc;      // Einc / Fout offset of x = 0 (when roi != 0)
  int v;               // element offset of x = 0 in V
  int valid;
  int roi;             // y and z inside the ROI
  float my, mz;
  float2 ry, rz;
};

constexpr size_t a16(size_t b) { return (b + 15) & ~(size_t)15; }

template <int N, int kW>
struct PipeSmem {
  static constexpr int kLdB = (N + N / 8 + 1) + ((8 - ((N + N / 8 + 1) & 15)) & 15);
  static constexpr size_t kBars = 0;                                   // 3 mbarriers
  static constexpr size_t kTw = 64;
  static constexpr size_t kR0 = kTw + a16(sizeof(float2) * N);
  static constexpr size_t kM0 = kR0 + a16(sizeof(float2) * N);
  static constexpr size_t kLines = kM0 + a16(sizeof(float) * N);
  static constexpr size_t kT0 = kLines + a16(sizeof(PipeLine) * kW);
  static constexpr size_t kTile = sizeof(float2) * N * kW;
  static constexpr size_t kT1 = kT0 + kTile;
  static constexpr size_t kFn = kT1 + kTile;
  static constexpr size_t kF = kFn + kTile;
  static constexpr size_t kB = kF + kTile;
  static constexpr size_t kTotal = kB + sizeof(float2) * kLdB * kW;
};

// W = 16 x-lines per tile (two CTAs per SM) where the shared memory allows,
// else 8 (n = 200, 216: three CTAs per SM).  KIND (compile time, so the
// steady-state kernel carries none of the other cases' work):
//   kSteady: jj >= 5 (update of iteration jj-1 >= 4: Field += Field_n,
//            reduced in L2; source V .* Field_n)
//   kEarly:  jj = 2, 3, 4 (first updates, the e = 3 bookkeeping, incident-
//            field source for jj = 2)
//   kFinal:  the final pass (update of the last iteration, Field(ROI) +
//            incident field into Fout, :646-647; no source, no forward FFT)
enum PipeKind { kSteady = 0, kEarly = 1, kFinal = 2 };

template <int R2, int W, int KIND>
__global__ void __launch_bounds__(W * 8, W == 16 ? 2 : 3)
    born_x_pipe_kernel(const BornArgs a, const int jj, const float2* __restrict__ twg, const int ntiles,
                       int* __restrict__ fault) {
#if defined(__CUDA_ARCH__)
  constexpr int N = kR1 * R2;
  constexpr int kW = W;
  constexpr int kThreads = W * kR1;
  using L = PipeSmem<N, W>;
  extern __shared__ __align__(128) unsigned char sm[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + L::kBars);  // [0], [1]: T stages, [2]: Fn/F
  float2* tw = reinterpret_cast<float2*>(sm + L::kTw);
  float2* r0t = reinterpret_cast<float2*>(sm + L::kR0);
  float* m0t = reinterpret_cast<float*>(sm + L::kM0);
  PipeLine* lines = reinterpret_cast<PipeLine*>(sm + L::kLines);
  float2* const sT0 = reinterpret_cast<float2*>(sm + L::kT0);
  float2* const sT1 = reinterpret_cast<float2*>(sm + L::kT1);
  float2* sFn = reinterpret_cast<float2*>(sm + L::kFn);
  float2* sF = reinterpret_cast<float2*>(sm + L::kF);
  float2* sB = reinterpret_cast<float2*>(sm + L::kB);
  const int tid = threadIdx.x;

  for (int i = tid; i < N; i += kThreads) {
    tw[i] = twg[i];
    r0t[i] = a.acyclic ? a.ramp[0][i] : make_float2(1.f, 0.f);
    m0t[i] = a.mask[0][i];
  }
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init(&bar[2], 1);
    mbar_fence_init();
  }
  __syncthreads();
  int tile = blockIdx.x;
  if (tile >= ntiles) return;

  const int nty = (a.py + kW - 1) / kW;
  const long long lineN = N;
  // tile -> (illumination b fastest, then y-tile, then z): concurrent tiles
  // share the V lines, which then come from L2
  auto decode = [&](int t, int& b, int& y0, int& z, int& nl) {
    b = t % a.nbatch;
    const int r = t / a.nbatch;
    const int ty = r % nty;
    z = r / nty;
    y0 = ty * kW;
    nl = min(kW, a.py - y0);
  };
  auto tile_off = [&](int b, int y0, int z) {
    return ((long long)y0 + (long long)a.py * (z + (long long)a.pz * b)) * lineN;
  };
  auto issue_T = [&](int t, int stage) {
    int b, y0, z, nl;
    decode(t, b, y0, z, nl);
    const uint32_t bytes = (uint32_t)(nl * N * sizeof(float2));
    mbar_arrive_expect_tx(&bar[stage], bytes);
    bulk_g2s(stage ? sT1 : sT0, a.T + tile_off(b, y0, z), bytes, &bar[stage]);
  };
  // the steady kind only adds Field_n to Field (red_add2 in L2): no copy of
  // Field into shared memory
  constexpr bool kLoadF = KIND != kSteady;
  auto issue_F = [&](int t) {
    int b, y0, z, nl;
    decode(t, b, y0, z, nl);
    const uint32_t bytes = (uint32_t)(nl * N * sizeof(float2));
    const long long o = tile_off(b, y0, z);
    mbar_arrive_expect_tx(&bar[2], kLoadF ? 2 * bytes : bytes);
    bulk_g2s(sFn, a.Fn + o, bytes, &bar[2]);
    if (kLoadF) bulk_g2s(sF, a.F + o, bytes, &bar[2]);
  };
  if (tid == 0) {
    issue_T(tile, 0);
    issue_F(tile);
  }
  uint32_t phT0 = 0, phT1 = 0, phF = 0;
  const int e = jj - 1;  // iteration whose update completes here (>= 1)
  const long long est = (long long)a.rx * a.ry * a.rz;
  const float2 cc = make_float2(0.f, a.c_im);
  const float2 z2 = make_float2(0.f, 0.f);

  for (int it = 0; tile < ntiles; ++it, tile += gridDim.x) {
    const int s = it & 1;
    const int next = tile + gridDim.x;
    if (tid == 0 && next < ntiles) {
      fence_proxy_async();
      issue_T(next, s ^ 1);
    }
    int b, y0, z, nl;
    decode(tile, b, y0, z, nl);
    // V of this thread's first mid-pass butterfly, loaded now so that its
    // latency hides behind the wait for T and the first FFT pass; each later
    // round's V is loaded before the previous round's arithmetic
    //
    // Mid-pass work items: a half-warp takes two lines x 8 consecutive
    // butterflies, slot s -> line 2 (s/16 / kJB) + (s%16)/8, butterfly
    // 8 (s/16 % kJB) + s%8.  The line pitch N = 8 (mod 16) elements puts the
    // other line 8 banks away, so every shared-memory access of the pass
    // (T, Field_n, Field, the second buffer) hits 16 distinct 8-byte banks
    // per half-warp; slots with j >= R2 idle.  (kW / 2) kJB 16 slots take as
    // many rounds of kThreads as the kW R2 butterflies would.
    constexpr int kJB = (R2 + 7) / 8;
    constexpr int kSlots = (kW / 2) * kJB * 16;
    auto item = [&](int sl, int& c, int& j) {
      const int hw = sl >> 4, l = sl & 15;
      const int pair = hw / kJB;
      c = 2 * pair + (l >> 3);
      j = 8 * (hw - pair * kJB) + (l & 7);
      return j < R2;
    };
    auto v_base = [&](int c, int j) {
      const int yy = c < nl ? y0 + c : y0;
      return (yy + a.py * z) * N + j;
    };
    float2 Vn[kR1];
    {
      int c0, j0;
      if (tid < kSlots && item(tid, c0, j0)) {
        const int vb = v_base(c0, j0);
#pragma unroll
        for (int r = 0; r < kR1; ++r) Vn[r] = a.V[vb + R2 * r];
      }
    }
    // the incident field (iteration 2's source, the final pass's Fout) is
    // prefetched the same way; zero outside the ROI
    constexpr bool kHasE = KIND != kSteady;
    const bool need_e = KIND == kFinal || (KIND == kEarly && jj <= 2);
    auto e_load = [&](int c, int j, float2* En) {
      const int yy = c < nl ? y0 + c : y0;
      const bool roi = need_e && (unsigned)(yy - a.ry0) < (unsigned)a.ry && (unsigned)(z - a.rz0) < (unsigned)a.rz;
      const long long base = (long long)b * est + (long long)(yy - a.ry0) * a.rx +
                             (long long)(z - a.rz0) * a.rx * a.ry - a.rx0;
#pragma unroll
      for (int r = 0; r < kR1; ++r) {
        const int x = j + R2 * r;
        En[r] = roi && (unsigned)(x - a.rx0) < (unsigned)a.rx ? a.Einc[base + x] : z2;
      }
    };
    float2 En[kHasE ? kR1 : 1];
    if constexpr (kHasE) {
      int c0, j0;
      if (tid < kSlots && item(tid, c0, j0)) e_load(c0, j0, En);
    }
    if (tid < kW) {
      PipeLine P;
      P.valid = tid < nl;
      const int yy = P.valid ? y0 + tid : y0;
      P.g = tile_off(b, yy, z);
      P.v = (yy + a.py * z) * N;
      P.roi = (unsigned)(yy - a.ry0) < (unsigned)a.ry && (unsigned)(z - a.rz0) < (unsigned)a.rz;
      P.einc = (long long)b * est + (long long)(yy - a.ry0) * a.rx +
               (long long)(z - a.rz0) * a.rx * a.ry - a.rx0;
      P.my = a.mask[1][yy];
      P.mz = a.mask[2][z];
      P.ry = a.ramp[1][yy];
      P.rz = a.ramp[2][z];
      lines[tid] = P;
    }
    bool ok = mbar_wait(&bar[s], s ? phT1 : phT0, a.wait_limit);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {  // give up; let this CTA's copies in flight land first
        atomicCAS(fault, 0, kFaultTimeout);
        mbar_wait(&bar[s], s ? phT1 : phT0);
        if (next < ntiles) mbar_wait(&bar[s ^ 1], s ? phT0 : phT1);
        mbar_wait(&bar[2], phF);
      }
      return;
    }
    if (s) phT1 ^= 1; else phT0 ^= 1;
    float2* T0 = s ? sT1 : sT0;
    // ---- inverse radix-R2 pass (ns = 1), in place
    {
      const int c = tid >> 3, j = tid & 7;
      float2 v[R2];
#pragma unroll
      for (int r = 0; r < R2; ++r) v[r] = T0[c * N + j + kR1 * r];
      Butterfly<R2, true>::run(v, tw, N);
      __syncthreads();
#pragma unroll
      for (int r = 0; r < R2; ++r) T0[c * N + j * R2 + r] = v[r];
    }
    ok = mbar_wait(&bar[2], phF, a.wait_limit);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        atomicCAS(fault, 0, kFaultTimeout);
        mbar_wait(&bar[2], phF);
        if (next < ntiles) mbar_wait(&bar[s ^ 1], s ? phT0 : phT1);
      }
      return;
    }
    phF ^= 1;
    // ---- inverse radix-8 (ns = R2) -> update + source -> forward radix-8
    for (int sl = tid; sl < kSlots; sl += kThreads) {
      int c, j;
      const bool live = item(sl, c, j);
      float2 Vv[kR1];
#pragma unroll
      for (int r = 0; r < kR1; ++r) Vv[r] = Vn[r];
      float2 Ev[kHasE ? kR1 : 1];
      if constexpr (kHasE) {
#pragma unroll
        for (int r = 0; r < kR1; ++r) Ev[r] = En[r];
      }
      {
        int cn, jn;
        if (sl + kThreads < kSlots && item(sl + kThreads, cn, jn)) {
          const int vb = v_base(cn, jn);
#pragma unroll
          for (int r = 0; r < kR1; ++r) Vn[r] = a.V[vb + R2 * r];
          if constexpr (kHasE) e_load(cn, jn, En);
        }
      }
      if (!live) continue;
      const PipeLine& Ln = lines[c];
      float2 v[kR1];
#pragma unroll
      for (int r = 0; r < kR1; ++r) v[r] = T0[c * N + j + R2 * r];
#pragma unroll
      for (int r = 1; r < kR1; ++r) {
        float2 w = tw[r * j];
        w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
      Butterfly<kR1, true>::run(v, tw, N);
#pragma unroll
      for (int r = 0; r < kR1; ++r) {
        const int x = j + R2 * r;
        const float2 V = Vv[r];
        const float2 r0 = a.acyclic ? cmul(cmul(r0t[x], Ln.ry), Ln.rz) : make_float2(1.f, 0.f);
        const bool in_roi = KIND != kSteady && Ln.roi && (unsigned)(x - a.rx0) < (unsigned)a.rx;
        float2 Ei = z2;
        if constexpr (kHasE) Ei = Ev[r];
        float2 P = v[r];
        if (a.acyclic) P = cmul(P, (e & 1) ? r0 : cconj(r0));
        const float m = (m0t[x] * Ln.my) * Ln.mz;
        const float2 vP = cmul(V, P);
        float2 ftot, fn_new;
        if (KIND != kSteady && e <= 2) {   // Field_n = (0 + V.*PSI) .* mask
          fn_new = cscale(vP, m);
          // Field = 0 + Field_n after iteration 1; after iteration 2 Field
          // keeps Field_n(1) until the e == 3 update
          ftot = e == 1 ? fn_new : cadd(sF[c * N + x], fn_new);
          if (KIND != kFinal && Ln.valid) {
            a.Fn[Ln.g + x] = fn_new;
            if (e == 1) a.F[Ln.g + x] = fn_new;
          }
        } else if (KIND == kSteady) {   // e >= 4: Field += Field_n (the same IEEE add, done in L2)
          const float2 fo = sFn[c * N + x];
          const float2 psi = cmul(cmul(cc, fo), V);
          const float2 fn = cscale(cadd(csub(fo, psi), vP), m);
          fn_new = fn;
          ftot = z2;   // not used by this kind
          if (Ln.valid) {
            red_add2(a.F + Ln.g + x, fn);
            a.Fn[Ln.g + x] = fn_new;
          }
        } else {
          const float2 fo = sFn[c * N + x];
          const float2 fp = sF[c * N + x];
          const float2 psi = cmul(cmul(cc, fo), V);
          const float2 fn = cscale(cadd(csub(fo, psi), vP), m);
          if (e == 3) {  // Field = (Field_n1 + Field_n2) + Field_n3; Field_n = Field_n3 + Field_n1
            ftot = cadd(cadd(fp, fo), fn);
            fn_new = cadd(fn, fp);
          } else {
            ftot = cadd(fp, fn);
            fn_new = fn;
          }
          if (KIND != kFinal && Ln.valid) {
            a.F[Ln.g + x] = ftot;
            a.Fn[Ln.g + x] = fn_new;
          }
        }
        if (KIND == kFinal) {
          if (Ln.valid && in_roi) a.Fout[Ln.einc + x] = cadd(ftot, Ei);
          continue;
        }
        float2 src;
        if (KIND == kEarly && jj <= 2) {  // (1i/eps) .* ((V(ROI) + 1i*eps) .* E_inc) / 2 inside the ROI
          src = in_roi ? cscale(cmul(cc, cmul(make_float2(V.x, V.y + a.eps), Ei)), 0.5f) : z2;
        } else {        // (1i/eps) .* Field_n .* V
          src = cmul(cmul(cc, fn_new), V);
        }
        if (a.acyclic) src = cmul(src, (jj & 1) ? cconj(r0) : r0);
        v[r] = Ln.valid ? src : z2;
      }
      if (KIND == kFinal) continue;
      Butterfly<kR1, false>::run(v, tw, N);
#pragma unroll
      for (int r = 0; r < kR1; ++r) {
        const int row = j * kR1 + r;
        sB[c * L::kLdB + row + (row >> 3)] = v[r];
      }
    }
    __syncthreads();
    if (tid == 0 && next < ntiles) {
      fence_proxy_async();
      issue_F(next);
    }
    if (KIND == kFinal) continue;   // nothing to transform back: Fout is written
    // ---- forward radix-R2 pass (ns = 8) -> T
    {
      const int c = tid >> 3, j = tid & 7;
      float2 v[R2];
#pragma unroll
      for (int r = 0; r < R2; ++r) {
        const int row = j + kR1 * r;
        v[r] = sB[c * L::kLdB + row + (row >> 3)];
      }
#pragma unroll
      for (int r = 1; r < R2; ++r) v[r] = cmul(v[r], tw[r * j]);
      Butterfly<R2, false>::run(v, tw, N);
      if (c < nl) {
        float2* out = a.T + tile_off(b, y0 + c, z);
#pragma unroll
        for (int r = 0; r < R2; ++r) out[j + kR1 * r] = v[r];
      }
    }
    __syncthreads();
  }
#endif
}

constexpr size_t kSmemCap = 113 * 1024;   // two CTAs per SM

template <int R2>
constexpr int tile_lines() {
#if defined(ODT_X_LINES)  // build-time override of the tile height (8 or 16) for measurements
  return ODT_X_LINES;
#else
  return PipeSmem<kR1 * R2, 16>::kTotal <= kSmemCap ? 16 : 8;
#endif
}

template <int R2, int KIND>
cudaError_t launch_r2(const BornArgs& a, int jj, const DevFft& fx, int* fault, cudaStream_t s) {
  constexpr int W = tile_lines<R2>();
  using L = PipeSmem<kR1 * R2, W>;
  static DeviceFlags configured;   // attribute raised once per device
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (!configured.test(dev)) {
    e = cudaFuncSetAttribute(born_x_pipe_kernel<R2, W, KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)L::kTotal);
    if (e != cudaSuccess) return e;
    configured.set(dev);
  }
  int nsm = 0;
  e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  int per_sm = 0;   // resident CTAs per SM (2 or 3; 2 for the 280-point lines)
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, born_x_pipe_kernel<R2, W, KIND>, W * kR1, L::kTotal);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorLaunchOutOfResources;
  const int nty = (a.py + W - 1) / W;
  const long long ntiles = (long long)nty * a.pz * a.nbatch;
  const int grid = (int)(ntiles < (long long)per_sm * nsm ? ntiles : (long long)per_sm * nsm);
  born_x_pipe_kernel<R2, W, KIND><<<grid, W * kR1, L::kTotal, s>>>(a, jj, fx.tw, (int)ntiles, fault);
  return cudaGetLastError();
}

int lines_of(int r2) {
  switch (r2) {
    case 11: return tile_lines<11>();
    case 15: return tile_lines<15>();
    case 19: return tile_lines<19>();
    case 25: return tile_lines<25>();
    case 27: return tile_lines<27>();
    case 35: return tile_lines<35>();
    default: return 0;
  }
}

}  // namespace

bool born_x_pipe_supported(const BornArgs& a, const DevFft& fx) {
  if (fx.plan.n != a.px || a.px % kR1 != 0) return false;
  const int r2 = a.px / kR1;
  const int W = lines_of(r2);
  if (W == 0) return false;
  const long long ntiles = (long long)((a.py + W - 1) / W) * a.pz * a.nbatch;
  return ntiles < (1LL << 31);
}

cudaError_t launch_born_x_pipe(const BornArgs& a, int mode, int jj, const DevFft& fx, int* fault,
                               cudaStream_t s) {
  if (jj < 2 || (mode != kBornMid && mode != kBornLast)) return cudaErrorInvalidValue;
  const int kind = mode == kBornLast ? kFinal : (jj <= 4 ? kEarly : kSteady);
  switch (a.px / kR1) {
#define ODT_PIPE_CASE(R)                                                     \
  case R:                                                                    \
    return kind == kFinal   ? launch_r2<R, kFinal>(a, jj, fx, fault, s)      \
           : kind == kEarly ? launch_r2<R, kEarly>(a, jj, fx, fault, s)      \
                            : launch_r2<R, kSteady>(a, jj, fx, fault, s);
    ODT_PIPE_CASE(11)
    ODT_PIPE_CASE(15)
    ODT_PIPE_CASE(19)
    ODT_PIPE_CASE(25)
    ODT_PIPE_CASE(27)
    ODT_PIPE_CASE(35)
#undef ODT_PIPE_CASE
    default: return cudaErrorNotSupported;
  }
}

}  // namespace odt
