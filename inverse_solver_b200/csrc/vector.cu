// Dyadic (vector) branch of the CBS solver (vector_simulation, pole_num = 3):
//
//   * pol23 / pol32: the polarisation change of basis of transform_field_3D
//     (FORWARD_SOLVER.m:38-68) and transform_field_2D / _reflection
//     (:69-128) on the field spectrum, per pixel, after the pupil factor;
//   * the z-pass with the dyadic absorptive Green's function
//     (FORWARD_SOLVER_CONVERGENT_BORN.m:596-604):
//       PSI_i = sum_j Greenp (delta_ij - corr rads_i rads_j) fftn(psi_j)
//     The three components of a field are consecutive batch entries (entry
//     3 b + i), so the x- and y-passes of the Born iteration, which act on
//     each component alone, run unchanged; only here do the components meet.
//     A CTA takes 16 (x, y) columns of one illumination, z-transforms the
//     three components into shared memory, couples them voxel by voxel and
//     transforms each back.
//   * an RI tensor (size(RI,4) > 1, V [sim, 3, 3]): the x-pass's pointwise
//     work couples the components through V (:567-574, :588-594, :624-627),
//     so it runs as its own kernel between plain x-FFTs (born_tensor_point),
//     and the emitter of the output stage is sum_j Field_j pot_ij dV
//     (:451-455, born_tensor_emitter).
#include <cuda_runtime.h>

#include "cbs_kernels.cuh"
#include "fft_tile.cuh"
#include "tile_bodies.cuh"
#include "tile_launch.cuh"

namespace odt {
namespace {

constexpr int kThreads = 256;

int grid_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  if (b > 148LL * 32) b = 148LL * 32;
  return (int)(b < 1 ? 1 : b);
}

__device__ __forceinline__ float2 rmul(float2 a, float r) { return make_float2(a.x * r, a.y * r); }

// in [nF, 2, nb] -> out [nF, 3, nb]
__global__ void pol23_kernel(const float2* __restrict__ in, float2* __restrict__ out,
                             float2* __restrict__ keep, const float* __restrict__ radial,
                             const float* __restrict__ perp, const float* __restrict__ tan3,
                             const float* __restrict__ kmask, long long nF, long long nb) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nF * nb;
       i += (long long)gridDim.x * blockDim.x) {
    const long long b = i / nF, p = i - b * nF;
    const float k = kmask[p];
    const float2 f1 = rmul(in[(2 * b) * nF + p], k), f2 = rmul(in[(2 * b + 1) * nF + p], k);
    const float r1 = radial[p], r2 = radial[nF + p];
    const float p1 = perp[p], p2 = perp[nF + p];
    const float2 b1 = cadd(rmul(f1, r1), rmul(f2, r2));  // sum(f .* Radial_2D, 3)
    const float2 b2 = cadd(rmul(f1, p1), rmul(f2, p2));  // sum(f .* Perp_2D, 3)
    const float2 o0 = cadd(rmul(b1, tan3[p]), rmul(b2, p1));
    const float2 o1 = cadd(rmul(b1, tan3[nF + p]), rmul(b2, p2));
    const float2 o2 = rmul(b1, tan3[2 * nF + p]);
    float2* o = out + (3 * b) * nF + p;
    o[0] = o0;
    o[nF] = o1;
    o[2 * nF] = o2;
    if (keep) {
      float2* q = keep + (3 * b) * nF + p;
      q[0] = o0;
      q[nF] = o1;
      q[2 * nF] = o2;
    }
  }
}

// in [nF, 3, nb] -> out [nF, 2, nb]; tz = +1 (transmission) or -1 (reflection)
__global__ void pol32_kernel(const float2* __restrict__ in, float2* __restrict__ out,
                             const float* __restrict__ radial, const float* __restrict__ perp,
                             const float* __restrict__ tan3, const float* __restrict__ kmask, float tz,
                             long long nF, long long nb) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nF * nb;
       i += (long long)gridDim.x * blockDim.x) {
    const long long b = i / nF, p = i - b * nF;
    const float k = kmask[p];
    const float2* x = in + (3 * b) * nF + p;
    const float2 x0 = rmul(x[0], k), x1 = rmul(x[nF], k), x2 = rmul(x[2 * nF], k);
    const float p1 = perp[p], p2 = perp[nF + p];
    const float2 b1 = cadd(cadd(rmul(x0, tan3[p]), rmul(x1, tan3[nF + p])), rmul(x2, tz * tan3[2 * nF + p]));
    const float2 b2 = cadd(rmul(x0, p1), rmul(x1, p2));
    out[(2 * b) * nF + p] = cadd(rmul(b1, radial[p]), rmul(b2, p1));
    out[(2 * b + 1) * nF + p] = cadd(rmul(b1, radial[nF + p]), rmul(b2, p2));
  }
}

template <int CLS>
__global__ void __launch_bounds__(128) born_z_dyadic_kernel(const BornArgs a, const DyadArgs d, const int jj,
                                                            const FftPlan plan, const float2* twg,
                                                            const int lgW) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const Thr th{(int)threadIdx.x, (int)blockDim.x};
  const int n = plan.n;  // == pz
  const int W = 1 << lgW;
  const int ld = W + 1;
  float2* tw = reinterpret_cast<float2*>(smraw);
  float* colv = reinterpret_cast<float*>(smraw + align16(sizeof(float2) * n));  // gxy, rx, ry
  float2* Q = reinterpret_cast<float2*>(smraw + align16(sizeof(float2) * n) + align16(sizeof(float) * 3 * W));
  float2* cur = Q + 3 * (size_t)n * ld;
  float2* oth = cur + (size_t)n * ld;
  load_twiddles(th, tw, twg, n);
  const long long n0 = (long long)a.px * a.py;
  const long long ntile = (n0 + W - 1) >> lgW;
  const long long b = blockIdx.x / ntile;  // illumination (components 3b, 3b+1, 3b+2)
  const long long i00 = (blockIdx.x - b * ntile) << lgW;
  const int ncol = (int)lmin(W, n0 - i00);
  const bool flip = a.acyclic && (jj & 1);
  for (int c = th.tid; c < W; c += th.nthr) {
    const long long i0 = lmin(i00 + c, n0 - 1);
    const int kx = (int)(i0 % a.px), ky = (int)(i0 / a.px);
    const int ix = flip ? wrap_neg(kx, a.px) : kx;
    const int iy = flip ? wrap_neg(ky, a.py) : ky;
    colv[c] = a.kq2[0][ix] + a.kq2[1][iy];
    colv[W + c] = d.rad[0][ix];
    colv[2 * W + c] = d.rad[1][iy];
  }
  __syncthreads();
  const ColMap m{lgW};
  for (int j = 0; j < 3; ++j) {
    float2* base = a.T + (3 * b + j) * a.nvox + i00;
    const GlobalPlain g{base, nullptr, (int)n0, 1, ncol};
    tile_fft_io<CLS, false>(th, plan, m, tw, g, SmemCol{Q + (size_t)j * n * ld, ld}, SmemCol{cur, ld},
                            SmemCol{oth, ld});
  }
  for (int idx = th.tid; idx < W * n; idx += th.nthr) {
    const int c = idx & (W - 1), kz = idx >> lgW;
    const int iz = flip ? wrap_neg(kz, a.pz) : kz;
    float q = colv[c] + a.kq2[2][iz];
    q = a.g_scale * q - a.g_off;
    const float rden = frcp(q * q + a.eps * a.eps);
    const float2 G = make_float2(q * rden, a.eps * rden);  // Greenp = 1 / (q - i eps)
    const float r0 = colv[W + c], r1 = colv[2 * W + c], r2 = d.rad[2][iz];
    const float2 v0 = Q[kz * ld + c];
    const float2 v1 = Q[(size_t)n * ld + kz * ld + c];
    const float2 v2 = Q[2 * (size_t)n * ld + kz * ld + c];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const float ri = i == 0 ? r0 : (i == 1 ? r1 : r2);
      const float2 ci = rmul(d.absorb, ri);  // corr * rads_i
      // (eye - (corr rads_i) rads_j) for j = 0, 1, 2, times Greenp, times fftn(psi_j)
      float2 d0 = cscale(ci, -r0), d1 = cscale(ci, -r1), d2 = cscale(ci, -r2);
      if (i == 0) d0.x += 1.f;
      if (i == 1) d1.x += 1.f;
      if (i == 2) d2.x += 1.f;
      float2 acc = cmul(cmul(G, d0), v0);
      acc = cadd(acc, cmul(cmul(G, d1), v1));
      acc = cadd(acc, cmul(cmul(G, d2), v2));
      Q[(size_t)i * n * ld + kz * ld + c] = cscale(acc, a.inv_n);
    }
  }
  __syncthreads();
  for (int i = 0; i < 3; ++i) {
    float2* base = a.T + (3 * b + i) * a.nvox + i00;
    const GlobalPlain g{nullptr, base, (int)n0, 1, ncol};
    tile_fft_io<CLS, true>(th, plan, m, tw, SmemCol{Q + (size_t)i * n * ld, ld}, g, SmemCol{cur, ld},
                           SmemCol{oth, ld});
  }
}

// ---- RI tensor
// Pointwise work of the x-pass (the tensor counterpart of BornXOp in
// tile_bodies.cuh) for one voxel and one illumination, its three components
// at batch entries 3 b + i.  T holds the inverse x-FFT of the spectral array
// (modes Mid / Last) and receives the source term of iteration jj times the
// phase ramp (modes First / Mid).  V9[v + nvox (i + 3 j)] = V_ij, with
// -1i eps_imag on the diagonal.  Sums over j run in the reference's order
// (j = 1, 2, 3, starting from the value the reference starts from).
template <int MODE>
__global__ void born_tensor_point_kernel(BornArgs a, const float2* __restrict__ V9, int jj, long long total) {
  const long long nv = a.nvox;
  const long long est = (long long)a.rx * a.ry * a.rz;
  const float2 z2 = make_float2(0.f, 0.f);
  const float2 cc = make_float2(0.f, a.c_im);
  const int e = jj - 1;  // iteration whose update completes here
  const bool upd = MODE != kBornFirst && e >= 1;
  const bool need_fn = upd && e >= 3;
  const bool need_f = upd && (e >= 3 || (MODE == kBornLast && e == 2));
  const bool need_einc = MODE == kBornLast || jj <= 2;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const long long v = t % nv;
    const long long b = t / nv;
    const int x = (int)(v % a.px);
    const long long r = v / a.px;
    const int y = (int)(r % a.py);
    const int z = (int)(r / a.py);
    const bool in_roi = (unsigned)(x - a.rx0) < (unsigned)a.rx && (unsigned)(y - a.ry0) < (unsigned)a.ry &&
                        (unsigned)(z - a.rz0) < (unsigned)a.rz;
    const long long eo = in_roi ? (x - a.rx0) + (long long)a.rx * ((y - a.ry0) + (long long)a.ry * (z - a.rz0)) : 0;
    float2 V[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) V[i][j] = V9[v + nv * (i + 3 * j)];
    const float2 r0 = a.acyclic ? cmul(cmul(a.ramp[0][x], a.ramp[1][y]), a.ramp[2][z]) : make_float2(1.f, 0.f);
    const float m = (a.mask[0][x] * a.mask[1][y]) * a.mask[2][z];
    float2 P[3], Fo[3], Fp[3], Ei[3], fn_new[3], ftot[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const long long gi = v + nv * (3 * b + i);
      P[i] = upd ? a.T[gi] : z2;
      if (upd && a.acyclic) P[i] = cmul(P[i], (e & 1) ? r0 : cconj(r0));
      Fo[i] = need_fn ? a.Fn[gi] : z2;
      Fp[i] = need_f ? a.F[gi] : z2;
      Ei[i] = (need_einc && in_roi) ? a.Einc[(3 * b + i) * est + eo] : z2;
      fn_new[i] = z2;
      ftot[i] = z2;
    }
    if (upd) {
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const long long gi = v + nv * (3 * b + i);
        if (e <= 2) {  // Field_n = 0 + sum_j V_ij PSI_j, then the mask
          float2 acc = cmul(V[i][0], P[0]);
          acc = cadd(acc, cmul(V[i][1], P[1]));
          acc = cadd(acc, cmul(V[i][2], P[2]));
          fn_new[i] = cscale(acc, m);
          if (MODE == kBornMid) {
            a.Fn[gi] = fn_new[i];
            if (e == 1) a.F[gi] = fn_new[i];
          } else {
            ftot[i] = (e == 1) ? fn_new[i] : cadd(Fp[i], fn_new[i]);
          }
        } else {
          // psi of iteration e: sum_j (1i/eps) Field_n_j V_ij
          float2 psi = cmul(cmul(cc, Fo[0]), V[i][0]);
          psi = cadd(psi, cmul(cmul(cc, Fo[1]), V[i][1]));
          psi = cadd(psi, cmul(cmul(cc, Fo[2]), V[i][2]));
          float2 acc = csub(Fo[i], psi);
          acc = cadd(acc, cmul(V[i][0], P[0]));
          acc = cadd(acc, cmul(V[i][1], P[1]));
          acc = cadd(acc, cmul(V[i][2], P[2]));
          const float2 fn = cscale(acc, m);
          if (e == 3) {
            ftot[i] = cadd(cadd(Fp[i], Fo[i]), fn);
            fn_new[i] = cadd(fn, Fp[i]);
          } else {
            ftot[i] = cadd(Fp[i], fn);
            fn_new[i] = fn;
          }
          if (MODE == kBornMid) {
            a.F[gi] = ftot[i];
            a.Fn[gi] = fn_new[i];
          }
        }
      }
    }
    if (MODE == kBornLast) {
      if (in_roi) {
#pragma unroll
        for (int i = 0; i < 3; ++i) a.Fout[(3 * b + i) * est + eo] = cadd(ftot[i], Ei[i]);
      }
      continue;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      float2 psi = z2;
      if (jj <= 2) {  // (1i/eps) (sum_j V_ij(ROI) E_inc_j + 1i eps E_inc_i) / 2 inside the ROI
        if (in_roi) {
          float2 sv = cmul(V[i][0], Ei[0]);
          sv = cadd(sv, cmul(V[i][1], Ei[1]));
          sv = cadd(sv, cmul(V[i][2], Ei[2]));
          sv = cadd(sv, cmul(make_float2(0.f, a.eps), Ei[i]));
          psi = cscale(cmul(cc, sv), 0.5f);
        }
      } else {  // sum_j (1i/eps) Field_n_j V_ij
        psi = cmul(cmul(cc, fn_new[0]), V[i][0]);
        psi = cadd(psi, cmul(cmul(cc, fn_new[1]), V[i][1]));
        psi = cadd(psi, cmul(cmul(cc, fn_new[2]), V[i][2]));
      }
      if (a.acyclic) psi = cmul(psi, (jj & 1) ? cconj(r0) : r0);
      a.T[v + nv * (3 * b + i)] = psi;
    }
  }
}

// emitter_i = sum_j Field_j pot_ij dV on the [c0, c1, rz] plane stack of each
// component (entry 3 b + i), zero outside the RI window; pot = V + 1i eps on
// the diagonal
__global__ void born_tensor_emitter_kernel(BornArgs a, const float2* __restrict__ V9, float2* conv, int c0,
                                           int c1, int o0, int o1, float dV, long long total) {
  const long long est = (long long)a.rx * a.ry * a.rz;
  const long long nv = a.nvox;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int X = (int)(t % c0);
    long long q = t / c0;
    const int Y = (int)(q % c1);
    q /= c1;
    const int z = (int)(q % a.rz);
    const long long ent = q / a.rz;  // 3 b + i
    const int i = (int)(ent % 3);
    const long long b = ent / 3;
    const int x = X - o0, y = Y - o1;
    float2 out = make_float2(0.f, 0.f);
    if ((unsigned)x < (unsigned)a.rx && (unsigned)y < (unsigned)a.ry) {
      const long long eo = x + (long long)a.rx * (y + (long long)a.ry * z);
      const long long v = (x + a.rx0) + (long long)a.px * ((y + a.ry0) + (long long)a.py * (z + a.rz0));
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        float2 pot = V9[v + nv * (i + 3 * j)];
        if (j == i) pot.y += a.eps;
        const float2 f = a.Fout[(3 * b + j) * est + eo];
        const float2 term = cscale(cmul(f, pot), dV);
        out = j == 0 ? term : cadd(out, term);
      }
    }
    conv[t] = out;
  }
}

size_t dyad_smem(int n, int W) {
  return align16(sizeof(float2) * n) + align16(sizeof(float) * 3 * W) + 5 * sizeof(float2) * (size_t)n * (W + 1);
}

}  // namespace

cudaError_t launch_pol23(const float2* in, float2* out, float2* keep, const PolTables& t, long long nF,
                         long long nb, cudaStream_t s) {
  pol23_kernel<<<grid_for(nF * nb), kThreads, 0, s>>>(in, out, keep, t.radial, t.perp, t.tan3, t.kmask, nF, nb);
  return cudaGetLastError();
}

cudaError_t launch_pol32(const float2* in, float2* out, const PolTables& t, bool reflection, long long nF,
                         long long nb, cudaStream_t s) {
  pol32_kernel<<<grid_for(nF * nb), kThreads, 0, s>>>(in, out, t.radial, t.perp, t.tan3, t.kmask,
                                                      reflection ? -1.f : 1.f, nF, nb);
  return cudaGetLastError();
}

cudaError_t launch_born_tensor_point(const BornArgs& a, const float2* V9, int mode, int jj, cudaStream_t s) {
  const long long total = a.nvox * (a.nbatch / 3);
  switch (mode) {
    case kBornFirst: born_tensor_point_kernel<kBornFirst><<<grid_for(total), kThreads, 0, s>>>(a, V9, jj, total); break;
    case kBornMid: born_tensor_point_kernel<kBornMid><<<grid_for(total), kThreads, 0, s>>>(a, V9, jj, total); break;
    case kBornLast: born_tensor_point_kernel<kBornLast><<<grid_for(total), kThreads, 0, s>>>(a, V9, jj, total); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_born_tensor_emitter(const BornArgs& a, const float2* V9, float2* conv, int c0, int c1, int o0,
                                       int o1, float dV, cudaStream_t s) {
  const long long total = (long long)c0 * c1 * a.rz * a.nbatch;
  born_tensor_emitter_kernel<<<grid_for(total), kThreads, 0, s>>>(a, V9, conv, c0, c1, o0, o1, dV, total);
  return cudaGetLastError();
}

cudaError_t launch_born_z_dyadic(const BornArgs& a, const DyadArgs& d, int jj, const DevFft& fz, int max_smem,
                                 cudaStream_t s) {
  int lgW = 4;
  while (lgW > 0 && dyad_smem(fz.plan.n, 1 << lgW) > (size_t)max_smem) --lgW;
  const size_t sm = dyad_smem(fz.plan.n, 1 << lgW);
  if (sm > (size_t)max_smem) return cudaErrorInvalidValue;
  const long long n0 = (long long)a.px * a.py;
  const long long ntile = (n0 + (1 << lgW) - 1) >> lgW;
  const unsigned blocks = (unsigned)(ntile * (a.nbatch / 3));
  cudaError_t e = cudaSuccess;
  switch (fz.plan.rclass) {
#define ODT_DYAD_CASE(C)                                                                                \
  case C:                                                                                              \
    e = raise_smem_limit(reinterpret_cast<const void*>(born_z_dyadic_kernel<C>), sm);                  \
    if (e != cudaSuccess) return e;                                                                    \
    born_z_dyadic_kernel<C><<<blocks, 128, sm, s>>>(a, d, jj, fz.plan, fz.tw, lgW);                    \
    break;
    ODT_DYAD_CASE(0)
    ODT_DYAD_CASE(1)
    ODT_DYAD_CASE(2)
    ODT_DYAD_CASE(3)
#undef ODT_DYAD_CASE
    default:
      return cudaErrorNotSupported;
  }
  return cudaGetLastError();
}

}  // namespace odt
