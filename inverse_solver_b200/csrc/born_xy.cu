// Fused xy-pass of the Born iteration: the whole x-y plane of one z and one
// illumination in shared memory, so one iteration moves 72 bytes per voxel
// (this pass: T, Field_n, Field read and written, V read; the z-pass: T read
// and written) instead of the 104 of separate x-, y- and y-passes.
//
// Per plane (FORWARD_SOLVER_CONVERGENT_BORN.m:577-647; jj = iteration):
//   inverse y-FFT and inverse x-FFT of the spectral array T (the last two
//   transforms of PSI = ifftn(G .* fftn(psi)) of iteration jj-1), update of
//   iteration jj-1 (:616-642), source term of iteration jj times the phase
//   ramp (:588-605), forward x-FFT and forward y-FFT (the first two of fftn).
// The z-pass (cols_pipe.cu) does the z-FFT, the Green's multiply and the
// inverse z-FFT in between.
//
// Transforms along an axis of length N = 8 R (11 <= R <= 20): index
// n = R n1 + n2 (n1 < 8, n2 < R), k = k1 + 8 k2 (k1 < 8, k2 < R).
//   forward  F1: 8-point DFT over n1 of the positions R n1 + n2 (stride R),
//                result k1 stored at R k1 + n2;
//            F2: times W_N^(n2 k1);
//            F3: R-point DFT over n2 of the contiguous positions R k1 + n2,
//                result k2 stored at R k1 + k2.
//   inverse  the same steps in reverse order with conjugate roots.
// Every step writes the positions it read, so the plane is transformed in
// place and needs one buffer; the spectrum is stored in this permuted order
// (spectral index k1 + 8 k2 at position R k1 + k2 along x and along y) and
// the z-pass maps each column to its (kx, ky) accordingly (BornArgs.perm_xy).
// Space-domain data is in natural order, so the pointwise work reads and
// writes Field_n / Field / V / the incident field in their global layout.
//
// Seven steps per plane:
//   1 y-F3^-1 + F2^-1  read T from global (one R-point column group per item)
//   2 y-F1^-1          shared memory
//   3 x-F3^-1 + F2^-1  shared memory
//   4 x-F1^-1, update + source, x-F1 (8 points per item; the global reads
//                      and writes of Field_n, Field, V, E_inc)
//   5 x-F2 + F3        shared memory
//   6 y-F1             shared memory
//   7 y-F2 + F3        write T to global
// One CTA per SM (the plane takes 8 N^2 bytes: 185 KB for N = 152) with 32 R
// threads -- R warps -- persistent over the planes (illumination fastest, so
// concurrent CTAs share V's planes in L2; prefetching the next plane's T,
// Field_n and Field into L2 with cp.async.bulk.prefetch made a step 5.4 ms
// slower, so there is none).  Steps 2-6 touch, for one n2, only
// the 8 rows R n1 + n2 (step 2 and 6 combine exactly those rows, steps 3-5
// work along rows), so warp w takes n2 = w and runs steps 2-6 on its own rows
// with warp-level synchronisation only; step 7 of a plane and step 1 of the
// next touch the same rows per item (see step1 below), so a plane needs two
// CTA barriers (after steps 1 and 6), and the warps drift apart so that one
// warp's global loads overlap other warps' transforms.
//
// Bank conflicts: rows have a pitch of N = 8 (mod 16) complex elements for
// odd R.  Steps 1, 2, 6, 7 put consecutive x on consecutive lanes; steps 3
// and 5 take R consecutive elements at R k1 (lanes over k1 and rows: the
// stride of 2R banks and the row pitch of 16 banks keep a half-warp's 8-byte
// accesses on distinct bank pairs); step 4 takes consecutive n2 on
// consecutive lanes.  For even R (N = 96, 128) a stride of R elements puts
// several k1 on the same banks (all eight at R = 16), so those planes carry
// one pad element after every R elements of a row (XYSmem::sx): group k1
// starts at (R + 1) k1, eight distinct bank pairs, and the pitch N + N / R
// is 8 (mod 16); the four rows of a warp's step-3 / -5 access still share
// banks (two wavefronts where one would do).
#include <cuda_runtime.h>

#include "b16.cuh"
#include "cbs_kernels.cuh"
#include "fft_core.cuh"
#include "tma.cuh"

namespace odt {
namespace {

constexpr size_t a16(size_t b) { return (b + 15) & ~(size_t)15; }
constexpr size_t a128(size_t b) { return (b + 127) & ~(size_t)127; }

template <int R>
struct XYSmem {
  static constexpr int N = 8 * R;
  static constexpr size_t kTw = 0;                                    // W_N^k, k < N
  static constexpr size_t kRampX = kTw + a16(sizeof(float2) * N);     // ramp along x
  static constexpr size_t kRampY = kRampX + a16(sizeof(float2) * N);  // ramp along y
  static constexpr size_t kMaskX = kRampY + a16(sizeof(float2) * N);
  static constexpr size_t kMaskY = kMaskX + a16(sizeof(float) * N);
  // W_N^(r k1) at twk[k1 * kTkS + r] (steps 3 and 5, whose lanes take 8
  // different k1): an odd stride puts the 8 addresses on distinct bank pairs
  static constexpr int kTkS = R | 1;
  static constexpr size_t kTk = kMaskY + a16(sizeof(float) * N);
  static constexpr size_t kPlane = a128(kTk + a16(sizeof(float2) * 8 * kTkS));
  // plane rows: for odd R a pitch of N (= 8 mod 16) elements; for even R
  // (N = 96, 128: 0 mod 16) one pad element after every R elements of a row,
  // so that the groups R k1 .. R k1 + R-1 of steps 3 and 5 start on
  // different banks ((R + 1) k1) and the pitch N + N / R is 8 mod 16 again
  static constexpr bool kPad = R % 2 == 0;
  static constexpr int P = kPad ? N + N / R : N;
  static constexpr size_t kTotal = kPlane + sizeof(float2) * N * P;
  // in-row position of x
  static __device__ __forceinline__ int sx(int x) { return kPad ? x + x / R : x; }
};

// KIND: which Born iterations a launch serves (compile time, so the steady
// kernel carries none of the other cases' work)
enum XYKind { kXYSteady = 0, kXYEarly = 1, kXYFinal = 2, kXYFirst = 3 };

// (i c) * v for real c: (-c v.y, c v.x), two products (a complex product
// with (0, c) would also form 0 * v.x and 0 * v.y)
__device__ __forceinline__ float2 mul_i(float c, float2 v) { return make_float2(-(c * v.y), c * v.x); }

// ST: storage of T and Field_n, 0 = complex64, 1 = 16-bit block floating
// point (b16.cuh; T's blocks are 8 consecutive x of a row, Field_n's are the
// values of one n1 in 8 consecutive step-4 work items of a warp, exponent
// index plane * N^2/8 + n1 * R^2 + w * R + item / 8)
// __launch_bounds__ lets the compiler fit the R warps of the one CTA per SM
// into the register file, which is split into four quarters of 16384
// registers (one per warp scheduler): 19 warps put five warps on a quarter,
// so at most 96 registers per thread for R = 19 (104 did not launch).
template <int R, int KIND, int ST>
__global__ void __launch_bounds__(32 * R, 1)
    born_xy_kernel(const BornArgs a, const int jj, const float2* __restrict__ twg, const int nplanes) {
#if defined(__CUDA_ARCH__)
  constexpr int N = 8 * R;
  constexpr int NT = 32 * R;
  using L = XYSmem<R>;
  extern __shared__ __align__(128) unsigned char sm[];
  float2* tw = reinterpret_cast<float2*>(sm + L::kTw);
  float2* rxt = reinterpret_cast<float2*>(sm + L::kRampX);
  float2* ryt = reinterpret_cast<float2*>(sm + L::kRampY);
  float* mxt = reinterpret_cast<float*>(sm + L::kMaskX);
  float* myt = reinterpret_cast<float*>(sm + L::kMaskY);
  float2* twk = reinterpret_cast<float2*>(sm + L::kTk);
  float2* pl = reinterpret_cast<float2*>(sm + L::kPlane);
  const int tid = threadIdx.x;
  const int w = tid >> 5, lane = tid & 31;   // warp w owns the rows R n1 + w in steps 2-6
  const float2 one = make_float2(1.f, 0.f);
  const float2 z2 = make_float2(0.f, 0.f);
  for (int i = tid; i < N; i += NT) {
    tw[i] = twg[i];
    rxt[i] = a.acyclic ? a.ramp[0][i] : one;
    ryt[i] = a.acyclic ? a.ramp[1][i] : one;
    mxt[i] = a.mask[0][i];
    myt[i] = a.mask[1][i];
  }
  for (int i = tid; i < 8 * L::kTkS; i += NT) {   // r k1 < 8 R = N
    const int k1 = i / L::kTkS, r = i - k1 * L::kTkS;
    twk[i] = r < R ? twg[r * k1] : make_float2(0.f, 0.f);
  }
  __syncthreads();

  constexpr bool kInv = KIND != kXYFirst;   // transforms T back (update of jj-1)
  constexpr bool kFwd = KIND != kXYFinal;   // forms the source and transforms it
  const int e = jj - 1;                     // iteration whose update completes here
  const long long plane_n = (long long)N * N;
  const long long est = (long long)a.rx * a.ry * a.rz;
  // Field_n / Field are read by the update from iteration 3 on (and Field by
  // the final pass of a 2-iteration series); the incident field by the
  // source of iteration 1 and 2 and by the final pass
  const bool need_fn = kInv && e >= 3;
  // the steady kind only adds Field_n to Field, with a reduction in L2
  // (red.global.add: no load of Field on the way)
  const bool need_f = KIND != kXYSteady && kInv && (e >= 3 || (KIND == kXYFinal && e == 2));
  const bool need_e = KIND == kXYFinal || ((KIND == kXYFirst || KIND == kXYEarly) && jj <= 2);

  // ---- 1: y-F3^-1 (R-point over k2 at rows R k1 + k2) and twiddles of item
  // i = (x, k1) of the plane at g0, from T into the plane buffer
  auto step1 = [&](int i, long long g0) {
    const int x = i % N, k1 = i / N;
    float2 v[R];
    if constexpr (ST == 0) {
      const float2* src = a.T + g0 + (long long)(R * k1) * N + x;
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = src[(long long)r * N];
    } else {
      const long long o = g0 + (long long)(R * k1) * N + x;
      const short2* src = a.T16 + o;
      const signed char* se = a.Te + (o >> 3);
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = b16_decode(src[(long long)r * N], se[r * (N >> 3)]);
    }
    Butterfly<R, true>::run(v, tw, N);
#pragma unroll
    for (int r = 1; r < R; ++r) v[r] = cmul(v[r], cconj(tw[r * k1]));
#pragma unroll
    for (int r = 0; r < R; ++r) pl[(R * k1 + r) * L::P + L::sx(x)] = v[r];
  };
  // Step 7 of item (x, k1) reads the rows R k1 + r of column x and step 1 of
  // the same item writes them, with the same item -> thread map: a thread
  // goes from its step-7 item of one plane straight to its step-1 item of
  // the next, with no CTA barrier in between.
  bool loaded = false;   // step 1 of this plane done during the previous plane's step 7
  for (int p = blockIdx.x; p < nplanes; p += gridDim.x) {
    const int b = p % a.nbatch;
    const int z = p / a.nbatch;
    const long long g0 = plane_n * (z + (long long)a.pz * b);   // plane (z, b) of T / Field_n / Field
    const long long v0 = plane_n * z;
    const int pn = p + gridDim.x;
    const long long gn = pn < nplanes ? plane_n * (pn / a.nbatch + (long long)a.pz * (pn % a.nbatch)) : -1;
    const float mz = a.mask[2][z];
    const float2 rz = a.acyclic ? a.ramp[2][z] : one;
    const bool zroi = (unsigned)(z - a.rz0) < (unsigned)a.rz;

    if constexpr (kInv) {
      // ---- 1 (unless the previous plane's step 7 did it item by item)
      if (!loaded)
        for (int i = tid; i < 8 * N; i += NT) step1(i, g0);
      __syncthreads();
      // ---- 2: y-F1^-1 (8-point over k1 at rows R k1 + w) -> natural rows R n1 + w
      for (int x = lane; x < N; x += 32) {
        float2 v[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) v[r] = pl[(R * r + w) * L::P + L::sx(x)];
        Butterfly<8, true>::run(v, tw, N);
#pragma unroll
        for (int r = 0; r < 8; ++r) pl[(R * r + w) * L::P + L::sx(x)] = v[r];
      }
      __syncwarp();
      // ---- 3: x-F3^-1 + F2^-1 on the contiguous groups R k1 .. R k1 + R-1 of the warp's rows
      for (int it = lane; it < 64; it += 32) {
        const int k1 = it & 7, y = R * (it >> 3) + w;
        float2* row = pl + y * L::P + (R + (L::kPad ? 1 : 0)) * k1;
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = row[r];
        Butterfly<R, true>::run(v, tw, N);
        const float2* tk = twk + k1 * L::kTkS;
#pragma unroll
        for (int r = 1; r < R; ++r) v[r] = cmul(v[r], cconj(tk[r]));
#pragma unroll
        for (int r = 0; r < R; ++r) row[r] = v[r];
      }
      __syncwarp();
    }

    // ---- 4: x-F1^-1 -> update of iteration jj-1 and source of jj -> x-F1, on
    //      the warp's rows (item it: row R (it / R) + w, n2 = it % R)
    for (int it = lane; it < 8 * R; it += 32) {
      const int n2 = it % R, y = R * (it / R) + w;
      // Field_n's exponent block of this item's n1 = r value: the 8 lanes of a
      // group (8 consecutive it) share one; block w R + it / 8 of n1's R^2
      const long long fe = (g0 >> 3) + w * R + (it >> 3);
      float2* row = pl + y * L::P;
      const long long gy = g0 + (long long)y * N;
      const long long vy = v0 + (long long)y * N;
      const bool yzroi = zroi && (unsigned)(y - a.ry0) < (unsigned)a.ry;
      const long long ebase = (long long)b * est + (long long)(y - a.ry0) * a.rx +
                              (long long)(z - a.rz0) * a.rx * a.ry - a.rx0;
      // the row's factors of the separable mask and phase ramp (mask(x) my mz,
      // ramp(x) ry rz: per element one product with the x factor)
      const float myz = myt[y] * mz;
      const float2 ryz = a.acyclic ? cmul(ryt[y], rz) : one;
      float2 V[8], Fo[8], Fp[8], Ei[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int x = R * r + n2;
        const bool in_roi = yzroi && (unsigned)(x - a.rx0) < (unsigned)a.rx;
        V[r] = a.V[vy + x];
        if constexpr (ST == 0) {
          Fo[r] = need_fn ? a.Fn[gy + x] : z2;
        } else {
          Fo[r] = need_fn ? b16_decode(a.Fn16[gy + x], a.Fe[fe + r * R * R]) : z2;
        }
        Fp[r] = need_f ? a.F[gy + x] : z2;
        Ei[r] = (need_e && in_roi) ? a.Einc[ebase + x] : z2;
      }
      // Field_n of element (x, y) of the item's r-th value (the 8 lanes of a
      // group take 8 consecutive items, so they share Field_n's blocks)
      auto store_fn = [&](int r, int x, float2 f) {
        if constexpr (ST == 0) {
          a.Fn[gy + x] = f;
        } else {
          const int ex = b16_group_exponent(f, __activemask());
          a.Fn16[gy + x] = b16_encode(f, ex);
          if ((it & 7) == 0) a.Fe[fe + r * R * R] = (signed char)ex;
        }
      };
      float2 v[8];
      if constexpr (kInv) {
#pragma unroll
        for (int r = 0; r < 8; ++r) v[r] = row[(R + (L::kPad ? 1 : 0)) * r + n2];
        Butterfly<8, true>::run(v, tw, N);
      }
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int x = R * r + n2;
        const float2 Vr = V[r];
        const float2 r0 = a.acyclic ? cmul(rxt[x], ryz) : one;
        const bool in_roi = yzroi && (unsigned)(x - a.rx0) < (unsigned)a.rx;
        float2 fn_new = z2, ftot = z2;
        if constexpr (kInv) {
          // PSI .* conj(phase ramp of iteration e)
          float2 P = v[r];
          if (a.acyclic) P = cmul(P, (e & 1) ? r0 : cconj(r0));
          const float m = mxt[x] * myz;
          const float2 vP = cmul(Vr, P);
          if (KIND != kXYSteady && e <= 2) {   // Field_n = (0 + V .* PSI) .* mask
            fn_new = cscale(vP, m);
            // Field = 0 + Field_n after iteration 1; after iteration 2 Field
            // keeps Field_n(1) until the e == 3 update
            ftot = e == 1 ? fn_new : cadd(Fp[r], fn_new);
            if (KIND != kXYFinal) {
              store_fn(r, x, fn_new);
              if (e == 1) a.F[gy + x] = fn_new;
            }
          } else {
            const float2 fo = Fo[r];
            const float2 fp = Fp[r];
            const float2 psi = cmul(mul_i(a.c_im, fo), Vr);
            const float2 fn = cscale(cadd(csub(fo, psi), vP), m);
            if (KIND == kXYSteady) {   // e >= 4: Field += Field_n (the same IEEE add, done in L2)
              fn_new = fn;
              red_add2(a.F + gy + x, fn);
              store_fn(r, x, fn_new);
            } else {
              if (e == 3) {  // Field = (Field_n1 + Field_n2) + Field_n3; Field_n = Field_n3 + Field_n1
                ftot = cadd(cadd(fp, fo), fn);
                fn_new = cadd(fn, fp);
              } else {
                ftot = cadd(fp, fn);
                fn_new = fn;
              }
              if (KIND != kXYFinal) {
                a.F[gy + x] = ftot;
                store_fn(r, x, fn_new);
              }
            }
          }
        }
        if constexpr (KIND == kXYFinal) {
          if (in_roi) a.Fout[ebase + x] = cadd(ftot, Ei[r]);
        } else {
          float2 src;
          if (jj <= 2) {  // (1i/eps) .* ((V(ROI) + 1i*eps) .* E_inc) / 2 inside the ROI
            src = in_roi ? cscale(mul_i(a.c_im, cmul(make_float2(Vr.x, Vr.y + a.eps), Ei[r])), 0.5f) : z2;
          } else {        // (1i/eps) .* Field_n .* V
            src = cmul(mul_i(a.c_im, fn_new), Vr);
          }
          if (a.acyclic) src = cmul(src, (jj & 1) ? cconj(r0) : r0);
          v[r] = src;
        }
      }
      if constexpr (kFwd) {
        Butterfly<8, false>::run(v, tw, N);
#pragma unroll
        for (int r = 0; r < 8; ++r) row[(R + (L::kPad ? 1 : 0)) * r + n2] = v[r];
      }
    }
    if constexpr (!kFwd) {
      __syncthreads();   // the next plane's step 1 overwrites the plane
      loaded = false;
      continue;
    }
    __syncwarp();
    // ---- 5: x-F2 + F3 on the contiguous groups of the warp's rows
    for (int it = lane; it < 64; it += 32) {
      const int k1 = it & 7, y = R * (it >> 3) + w;
      float2* row = pl + y * L::P + (R + (L::kPad ? 1 : 0)) * k1;
      float2 v[R];
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = row[r];
      const float2* tk = twk + k1 * L::kTkS;
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tk[r]);
      Butterfly<R, false>::run(v, tw, N);
#pragma unroll
      for (int r = 0; r < R; ++r) row[r] = v[r];
    }
    __syncwarp();
    // ---- 6: y-F1 (8-point over n1 at the warp's rows R n1 + w)
    for (int x = lane; x < N; x += 32) {
      float2 v[8];
#pragma unroll
      for (int r = 0; r < 8; ++r) v[r] = pl[(R * r + w) * L::P + L::sx(x)];
      Butterfly<8, false>::run(v, tw, N);
#pragma unroll
      for (int r = 0; r < 8; ++r) pl[(R * r + w) * L::P + L::sx(x)] = v[r];
    }
    __syncthreads();
    // ---- 7: y-F2 + F3 -> T
    for (int i = tid; i < 8 * N; i += NT) {
      const int x = i % N, k1 = i / N;
      float2 v[R];
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = pl[(R * k1 + r) * L::P + L::sx(x)];
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], tw[r * k1]);
      Butterfly<R, false>::run(v, tw, N);
      if constexpr (ST == 0) {
        float2* dst = a.T + g0 + (long long)(R * k1) * N + x;
#pragma unroll
        for (int r = 0; r < R; ++r) dst[(long long)r * N] = v[r];
      } else {   // the 8 lanes of a group hold 8 consecutive x of the same rows
        const long long o = g0 + (long long)(R * k1) * N + x;
        short2* dst = a.T16 + o;
        signed char* de = a.Te + (o >> 3);
        const unsigned mask = __activemask();
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int ex = b16_group_exponent(v[r], mask);
          dst[(long long)r * N] = b16_encode(v[r], ex);
          if ((x & 7) == 0) de[r * (N >> 3)] = (signed char)ex;
        }
      }
    }
    if (kInv && gn >= 0)   // the same items as this thread's step 7: no barrier needed
      for (int i = tid; i < 8 * N; i += NT) step1(i, gn);
    loaded = kInv && gn >= 0;
    if (!loaded) __syncthreads();   // the next plane's step 4 (first kind) writes other threads' rows
  }
#endif
}

template <int R, int KIND, int ST>
cudaError_t launch_r(const BornArgs& a, int jj, const float2* tw, cudaStream_t s) {
  using L = XYSmem<R>;
  static DeviceFlags configured;   // attribute raised once per device
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (!configured.test(dev)) {
    e = cudaFuncSetAttribute(born_xy_kernel<R, KIND, ST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)L::kTotal);
    if (e != cudaSuccess) return e;
    configured.set(dev);
  }
  int nsm = 0;
  e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  int per_sm = 0;   // the kernel needs one resident CTA per SM
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, born_xy_kernel<R, KIND, ST>, 32 * R, L::kTotal);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorLaunchOutOfResources;
  const long long nplanes = (long long)a.pz * a.nbatch;
  const int grid = (int)(nplanes < nsm ? nplanes : nsm);
  born_xy_kernel<R, KIND, ST><<<grid, 32 * R, L::kTotal, s>>>(a, jj, tw, (int)nplanes);
  return cudaGetLastError();
}

template <int R, int ST>
cudaError_t launch_kind_st(const BornArgs& a, int kind, int jj, const float2* tw, cudaStream_t s) {
  switch (kind) {
    case kXYSteady: return launch_r<R, kXYSteady, ST>(a, jj, tw, s);
    case kXYEarly: return launch_r<R, kXYEarly, ST>(a, jj, tw, s);
    case kXYFinal: return launch_r<R, kXYFinal, ST>(a, jj, tw, s);
    default: return launch_r<R, kXYFirst, ST>(a, jj, tw, s);
  }
}

template <int R>
cudaError_t launch_kind(const BornArgs& a, int kind, int jj, const float2* tw, cudaStream_t s) {
  return a.storage ? launch_kind_st<R, 1>(a, kind, jj, tw, s) : launch_kind_st<R, 0>(a, kind, jj, tw, s);
}

}  // namespace

bool born_xy_supported(const BornArgs& a, int max_smem) {
  if (a.px != a.py || a.px % 8 != 0) return false;
  const int r = a.px / 8;
  size_t need = 0;
  switch (r) {
    case 11: need = XYSmem<11>::kTotal; break;
    case 12: need = XYSmem<12>::kTotal; break;
    case 13: need = XYSmem<13>::kTotal; break;
    case 14: need = XYSmem<14>::kTotal; break;
    case 15: need = XYSmem<15>::kTotal; break;
    case 16: need = XYSmem<16>::kTotal; break;
    case 17: need = XYSmem<17>::kTotal; break;
    case 18: need = XYSmem<18>::kTotal; break;
    case 19: need = XYSmem<19>::kTotal; break;
    case 20: need = XYSmem<20>::kTotal; break;
    default: return false;
  }
  return need <= (size_t)max_smem && (long long)a.pz * a.nbatch < (1LL << 31);
}

int born_xy_perm_radix(const BornArgs& a) { return a.px / 8; }

cudaError_t launch_born_xy(const BornArgs& a, int mode, int jj, const DevFft& fx, cudaStream_t s) {
  int kind;
  if (mode == kBornFirst) kind = kXYFirst;
  else if (mode == kBornLast) kind = kXYFinal;
  else kind = jj <= 4 ? kXYEarly : kXYSteady;   // steady: e = jj - 1 >= 4 (Field += Field_n only)
  if ((mode == kBornFirst) != (jj == 1)) return cudaErrorInvalidValue;
  switch (a.px / 8) {
    case 11: return launch_kind<11>(a, kind, jj, fx.tw, s);
    case 12: return launch_kind<12>(a, kind, jj, fx.tw, s);
    case 13: return launch_kind<13>(a, kind, jj, fx.tw, s);
    case 14: return launch_kind<14>(a, kind, jj, fx.tw, s);
    case 15: return launch_kind<15>(a, kind, jj, fx.tw, s);
    case 16: return launch_kind<16>(a, kind, jj, fx.tw, s);
    case 17: return launch_kind<17>(a, kind, jj, fx.tw, s);
    case 18: return launch_kind<18>(a, kind, jj, fx.tw, s);
    case 19: return launch_kind<19>(a, kind, jj, fx.tw, s);
    case 20: return launch_kind<20>(a, kind, jj, fx.tw, s);
    default: return cudaErrorNotSupported;
  }
}

}  // namespace odt
