// Bodies of the tile kernels, written once for the GPU (cbs_tiles.cu wraps
// them in __global__ functions) and for a sequential CPU check (one thread,
// barriers dropped; tests/native/tile_host_check.cpp runs every CTA in turn).
//
//   born_x_body : x-pass of Born iteration jj -- inverse x-FFT of the
//                 spectral array, completion of the update of iteration jj-1
//                 (FORWARD_SOLVER_CONVERGENT_BORN.m:616-642), the source term
//                 of iteration jj (:588-605) times the phase ramp, forward
//                 x-FFT.  Modes: First (jj = 1: source only), Mid, Last
//                 (update of the final iteration, writes Field(ROI) + incident
//                 field, :646-647).
//   born_z_body : forward z-FFT, Green's multiply G(k -/+ dk/4) with the
//                 1/N of ifftn folded in (:608-615), inverse z-FFT.
//   fft_lines_body / fft_cols_body : plain batched FFTs (y-pass of the Born
//                 loop, centred 2D FFTs of the field input/output paths).
#pragma once

#include "cbs_kernels.cuh"
#include "fft_tile.cuh"
#include "tile_launch.cuh"

#if defined(__CUDA_ARCH__)
#define ODT_SYNC() __syncthreads()
#else
#define ODT_SYNC() ((void)0)
#endif

namespace odt {

ODT_HD int wrap_neg(int i, int n) { return i == 0 ? 0 : n - i; }
ODT_HD long long lmin(long long a, long long b) { return a < b ? a : b; }

// correctly rounded single-precision reciprocal
ODT_HD float frcp(float x) {
#if defined(__CUDA_ARCH__)
  return __frcp_rn(x);
#else
  return 1.0f / x;
#endif
}

ODT_HD void load_twiddles(const Thr& th, float2* dst, const float2* src, int n) {
  for (int i = th.tid; i < n; i += th.nthr) dst[i] = src[i];
}

// ------------------------------------------------------------------ born_x
// Pointwise work of the x-pass on the R values v[r] at x = j + r*nb of line c.
template <int MODE>
struct BornXOp {
  const BornArgs* a;
  const LineInfo* lines;
  int jj;
  // Loads of all R elements are issued before any arithmetic or store (the
  // stores to Field_n / Field could alias the loads, so interleaving them
  // would serialise one memory latency per element).
  template <int R>
  ODT_HD void apply(int c, int j, int nb, float2* v) const {
    const LineInfo& L = lines[c];
    const BornArgs& A = *a;
    if (!L.valid) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = make_float2(0.f, 0.f);
      return;
    }
    const int e = jj - 1;  // iteration whose update completes here
    const bool upd = MODE != kBornFirst && e >= 1;
    const bool need_fn = upd && e >= 3;
    const bool need_f = upd && (e >= 3 || (MODE == kBornLast && e == 2));
    const bool need_einc = MODE == kBornLast || jj <= 2;
    const float2 z2 = make_float2(0.f, 0.f);
    float2 Vv[R], Fo[R], Fp[R], Ei[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int x = j + r * nb;
      const long long gi = L.g + x;
      const bool in_roi = L.roi && (unsigned)(x - A.rx0) < (unsigned)A.rx;
      Vv[r] = A.V[L.v + x];
      Fo[r] = need_fn ? A.Fn[gi] : z2;
      Fp[r] = need_f ? A.F[gi] : z2;
      Ei[r] = (need_einc && in_roi) ? A.Einc[L.einc + x] : z2;
    }
    const float2 cc = make_float2(0.f, A.c_im);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int x = j + r * nb;
      const long long gi = L.g + x;
      const float2 V = Vv[r];
      const float2 r0 = A.acyclic ? cmul(cmul(A.ramp[0][x], L.ry), L.rz) : make_float2(1.f, 0.f);
      const bool in_roi = L.roi && (unsigned)(x - A.rx0) < (unsigned)A.rx;
      float2 fn_new = z2;
      float2 ftot = z2;
      if (upd) {
        // PSI = ifftn(...) .* conj(phase_ramp_e), phase_ramp_e = conj(r0) for odd e
        float2 P = v[r];
        if (A.acyclic) P = cmul(P, (e & 1) ? r0 : cconj(r0));
        const float m = (A.mask[0][x] * L.my) * L.mz;
        const float2 vP = cmul(V, P);
        if (e <= 2) {
          fn_new = cscale(vP, m);  // (0 + V.*PSI) .* mask
          if (MODE == kBornMid) {
            A.Fn[gi] = fn_new;
            if (e == 1) A.F[gi] = fn_new;  // Field = 0 + Field_n
            // e == 2: Field keeps Field_n(1) until the e == 3 update
          } else {
            ftot = (e == 1) ? fn_new : cadd(Fp[r], fn_new);
          }
        } else {
          const float2 fo = Fo[r];
          const float2 psi = cmul(cmul(cc, fo), V);
          const float2 fn = cscale(cadd(csub(fo, psi), vP), m);
          const float2 fp = Fp[r];
          if (e == 3) {  // Field = (Field_n1 + Field_n2) + Field_n3; Field_n = Field_n3 + Field_n1
            ftot = cadd(cadd(fp, fo), fn);
            fn_new = cadd(fn, fp);
          } else {
            ftot = cadd(fp, fn);
            fn_new = fn;
          }
          if (MODE == kBornMid) {
            A.F[gi] = ftot;
            A.Fn[gi] = fn_new;
          }
        }
      }
      if (MODE == kBornLast) {
        if (in_roi) A.Fout[L.einc + x] = cadd(ftot, Ei[r]);
        continue;
      }
      float2 psi = z2;
      if (jj <= 2) {  // (1i/eps) .* ((V(ROI) + 1i*eps) .* E_inc) / 2 inside the ROI
        if (in_roi) {
          const float2 sv = cmul(make_float2(V.x, V.y + A.eps), Ei[r]);
          psi = cscale(cmul(cc, sv), 0.5f);
        }
      } else {  // (1i/eps) .* Field_n .* V
        psi = cmul(cmul(cc, fn_new), V);
      }
      if (A.acyclic) psi = cmul(psi, (jj & 1) ? cconj(r0) : r0);
      v[r] = psi;
    }
  }
};

// CTA -> (illumination b fastest, then y-tile, then z): the CTAs that read the
// same V lines run back to back, so V is served from L2 for all but the first.
template <int CLS, int MODE>
ODT_HD void born_x_body(const BornArgs& a, int jj, const FftPlan& plan, const float2* twg, int W,
                        unsigned char* smraw, unsigned block, const Thr& th) {
  const int n = plan.n;  // == px
  const int ld = smem_line_ld(n);
  float2* tw = reinterpret_cast<float2*>(smraw);
  LineInfo* lines = reinterpret_cast<LineInfo*>(smraw + align16(sizeof(float2) * n));
  float2* bufA = reinterpret_cast<float2*>(smraw + align16(sizeof(float2) * n) +
                                           align16(sizeof(LineInfo) * W));
  float2* bufB = bufA + (size_t)W * ld;
  load_twiddles(th, tw, twg, n);
  const int nty = (a.py + W - 1) / W;
  const int b = (int)(block % (unsigned)a.nbatch);
  const int t = (int)(block / (unsigned)a.nbatch);
  const int ty = t % nty;
  const int z = t / nty;
  const int y0 = ty * W;
  const int nl = (int)lmin(W, a.py - y0);
  const long long est = (long long)a.rx * a.ry * a.rz;
  for (int c = th.tid; c < W; c += th.nthr) {
    LineInfo L;
    L.valid = c < nl;
    const int yy = L.valid ? y0 + c : y0;
    L.g = ((long long)yy + (long long)a.py * (z + (long long)a.pz * b)) * n;
    L.v = (yy + a.py * z) * n;
    L.roi = (unsigned)(yy - a.ry0) < (unsigned)a.ry && (unsigned)(z - a.rz0) < (unsigned)a.rz;
    L.einc = (long long)b * est + (long long)(yy - a.ry0) * a.rx +
             (long long)(z - a.rz0) * a.rx * a.ry - a.rx0;
    L.my = a.mask[1][yy];
    L.mz = a.mask[2][z];
    L.ry = a.ramp[1][yy];
    L.rz = a.ramp[2][z];
    lines[c] = L;
  }
  ODT_SYNC();
  const LineMap m{W};
  float2* T0 = a.T + ((long long)y0 + (long long)a.py * (z + (long long)a.pz * b)) * n;
  const GlobalPlain g{T0, T0, 1, n, nl};
  const int P = plan.npass;
  const BornXOp<MODE> op{&a, lines, jj};
  SmemLine cur{bufA, ld}, oth{bufB, ld};
  if (MODE != kBornFirst) {
    int ns = 1;  // inverse passes, radices f[P-1] .. f[1]; result ends in `oth`
    for (int i = 0; i + 1 < P; ++i) {
      const int R = plan.radix[P - 1 - i];
      if (i == 0) tile_pass_any<CLS, true>(th, R, m, n, ns, tw, g, cur);
      else tile_pass_any<CLS, true>(th, R, m, n, ns, tw, oth, cur);
      ODT_SYNC();
      ns *= R;
      const SmemLine t2 = cur;
      cur = oth;
      oth = t2;
    }
  }
  const int R0 = plan.radix[0];
  if (MODE == kBornLast) {
    if (P == 1) tile_mid_any<CLS, true, kMidEnd>(th, R0, m, n, tw, g, g, op);
    else tile_mid_any<CLS, true, kMidEnd>(th, R0, m, n, tw, oth, g, op);
    return;
  }
  if (MODE == kBornFirst) {
    if (P == 1) tile_mid_any<CLS, true, kMidGen>(th, R0, m, n, tw, g, g, op);
    else tile_mid_any<CLS, true, kMidGen>(th, R0, m, n, tw, g, cur, op);
  } else {
    if (P == 1) tile_mid_any<CLS, true, kMidBoth>(th, R0, m, n, tw, g, g, op);
    else tile_mid_any<CLS, true, kMidBoth>(th, R0, m, n, tw, oth, cur, op);
  }
  if (P == 1) return;
  ODT_SYNC();
  {
    const SmemLine t2 = cur;
    cur = oth;
    oth = t2;
  }
  int ns = R0;  // forward passes f[1] .. f[P-1]; the last one writes T
  for (int p = 1; p < P; ++p) {
    const int R = plan.radix[p];
    if (p == P - 1) tile_pass_any<CLS, false>(th, R, m, n, ns, tw, oth, g);
    else tile_pass_any<CLS, false>(th, R, m, n, ns, tw, oth, cur);
    ODT_SYNC();
    ns *= R;
    const SmemLine t2 = cur;
    cur = oth;
    oth = t2;
  }
}

// ------------------------------------------------------------------ born_z
struct GreenOp {
  const BornArgs* a;
  const float* gxy;  // per column: kq2x + kq2y (at negated indices on odd jj)
  bool flip;
  template <int R>
  ODT_HD void apply(int c, int j, int nb, float2* v) const {
    const BornArgs& A = *a;
    const float qxy = gxy[c];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int kz = j + r * nb;
      const int iz = flip ? wrap_neg(kz, A.pz) : kz;
      float q = qxy + A.kq2[2][iz];
      q = A.g_scale * q - A.g_off;
      const float rden = frcp(q * q + A.eps * A.eps);
      const float2 G = make_float2(q * rden, A.eps * rden);  // 1 / (q - i eps)
      v[r] = cscale(cmul(G, v[r]), A.inv_n);
    }
  }
};

template <int CLS>
ODT_HD void born_z_body(const BornArgs& a, int jj, const FftPlan& plan, const float2* twg,
                        int lgW, unsigned char* smraw, unsigned block, const Thr& th) {
  const int n = plan.n;  // == pz
  const int W = 1 << lgW;
  float2* tw = reinterpret_cast<float2*>(smraw);
  float* gxy = reinterpret_cast<float*>(smraw + align16(sizeof(float2) * n));
  float2* bufA = reinterpret_cast<float2*>(smraw + align16(sizeof(float2) * n) +
                                           align16(sizeof(float) * W));
  float2* bufB = bufA + (size_t)n * (W + 1);
  load_twiddles(th, tw, twg, n);
  const long long n0 = (long long)a.px * a.py;
  const long long ntile = (n0 + W - 1) >> lgW;
  const long long b = block / ntile;
  const long long i00 = (block - b * ntile) << lgW;
  const int ncol = (int)lmin(W, n0 - i00);
  const bool flip = a.acyclic && (jj & 1);
  for (int c = th.tid; c < W; c += th.nthr) {
    const long long i0 = lmin(i00 + c, n0 - 1);
    int kx = (int)(i0 % a.px), ky = (int)(i0 / a.px);
    if (a.perm_xy) {   // fused xy-pass order: position R k1 + k2 holds index k1 + 8 k2
      const int rx = a.px >> 3, ry = a.py >> 3;
      kx = kx / rx + 8 * (kx % rx);
      ky = ky / ry + 8 * (ky % ry);
    }
    const int ix = flip ? wrap_neg(kx, a.px) : kx;
    const int iy = flip ? wrap_neg(ky, a.py) : ky;
    gxy[c] = a.kq2[0][ix] + a.kq2[1][iy];
  }
  ODT_SYNC();
  float2* base = a.T + b * a.nvox + i00;
  const GlobalPlain g{base, base, (int)n0, 1, ncol};
  const ColMap m{lgW};
  const GreenOp op{&a, gxy, flip};
  SmemCol cur{bufA, W + 1}, oth{bufB, W + 1};
  const int P = plan.npass;
  int ns = 1;
  for (int p = 0; p + 1 < P; ++p) {  // forward passes f[0] .. f[P-2]
    const int R = plan.radix[p];
    if (p == 0) tile_pass_any<CLS, false>(th, R, m, n, ns, tw, g, cur);
    else tile_pass_any<CLS, false>(th, R, m, n, ns, tw, oth, cur);
    ODT_SYNC();
    ns *= R;
    const SmemCol t2 = cur;
    cur = oth;
    oth = t2;
  }
  const int RL = plan.radix[P - 1];
  if (P == 1) {
    tile_mid_any<CLS, false, kMidBoth>(th, RL, m, n, tw, g, g, op);
    return;
  }
  tile_mid_any<CLS, false, kMidBoth>(th, RL, m, n, tw, oth, cur, op);
  ODT_SYNC();
  {
    const SmemCol t2 = cur;
    cur = oth;
    oth = t2;
  }
  ns = RL;
  for (int i = P - 2; i >= 0; --i) {  // inverse passes f[P-2] .. f[0]; the last writes T
    const int R = plan.radix[i];
    if (i == 0) tile_pass_any<CLS, true>(th, R, m, n, ns, tw, oth, g);
    else tile_pass_any<CLS, true>(th, R, m, n, ns, tw, oth, cur);
    ODT_SYNC();
    ns *= R;
    const SmemCol t2 = cur;
    cur = oth;
    oth = t2;
  }
}

// --------------------------------------------------------- generic FFTs
// Whole transform of a tile: forward in plan order, inverse in reverse order;
// the first pass reads `src`, the last writes `dst`.
template <int CLS, bool INV, class Map, class S, class G1, class G2>
ODT_HD void tile_fft_io(const Thr& th, const FftPlan& plan, const Map& m, const float2* tw,
                        const G1& src, const G2& dst, S cur, S oth) {
  const int n = plan.n;
  const int P = plan.npass;
  if (P == 0) {  // n == 1
    for (int idx = th.tid; idx < m.total(1); idx += th.nthr) {
      int c, j;
      m.decode(idx, 1, c, j);
      dst.store(0, c, src.load(0, c));
    }
    return;
  }
  int ns = 1;
  for (int i = 0; i < P; ++i) {
    const int R = INV ? plan.radix[P - 1 - i] : plan.radix[i];
    if (P == 1) tile_pass_any<CLS, INV>(th, R, m, n, ns, tw, src, dst);
    else if (i == 0) tile_pass_any<CLS, INV>(th, R, m, n, ns, tw, src, cur);
    else if (i == P - 1) tile_pass_any<CLS, INV>(th, R, m, n, ns, tw, oth, dst);
    else tile_pass_any<CLS, INV>(th, R, m, n, ns, tw, oth, cur);
    ODT_SYNC();
    ns *= R;
    const S t2 = cur;
    cur = oth;
    oth = t2;
  }
}

template <int CLS, bool INV>
ODT_HD void fft_lines_body(const float2* in, float2* out, long long nlines, int in_shift,
                           int out_shift, float scale, const FftPlan& plan, const float2* twg,
                           int W, unsigned char* smraw, unsigned block, const Thr& th) {
  const int n = plan.n;
  const int ld = smem_line_ld(n);
  float2* tw = reinterpret_cast<float2*>(smraw);
  float2* bufA = reinterpret_cast<float2*>(smraw + align16(sizeof(float2) * n));
  float2* bufB = bufA + (size_t)W * ld;
  load_twiddles(th, tw, twg, n);
  ODT_SYNC();
  const long long L0 = (long long)block * W;
  const int nl = (int)lmin(W, nlines - L0);
  const GlobalShift src{in + L0 * n, nullptr, 1, n, nl, n, in_shift, 1.f};
  const GlobalShift dst{nullptr, out + L0 * n, 1, n, nl, n, out_shift, scale};
  tile_fft_io<CLS, INV>(th, plan, LineMap{W}, tw, src, dst, SmemLine{bufA, ld}, SmemLine{bufB, ld});
}

template <int CLS, bool INV, bool SHIFT>
ODT_HD void fft_cols_body(const float2* in, float2* out, long long n0, int in_shift,
                          int out_shift, float scale, const FftPlan& plan, const float2* twg,
                          int lgW, unsigned char* smraw, unsigned block, const Thr& th) {
  const int n = plan.n;
  const int W = 1 << lgW;
  float2* tw = reinterpret_cast<float2*>(smraw);
  float2* bufA = reinterpret_cast<float2*>(smraw + align16(sizeof(float2) * n));
  float2* bufB = bufA + (size_t)n * (W + 1);
  load_twiddles(th, tw, twg, n);
  ODT_SYNC();
  const long long ntile = (n0 + W - 1) >> lgW;
  const long long o = block / ntile;
  const long long i00 = (block - o * ntile) << lgW;
  const int ncol = (int)lmin(W, n0 - i00);
  const long long off = o * n0 * n + i00;
  const ColMap m{lgW};
  if (SHIFT) {
    const GlobalShift src{in + off, nullptr, (int)n0, 1, ncol, n, in_shift, 1.f};
    const GlobalShift dst{nullptr, out + off, (int)n0, 1, ncol, n, out_shift, scale};
    tile_fft_io<CLS, INV>(th, plan, m, tw, src, dst, SmemCol{bufA, W + 1}, SmemCol{bufB, W + 1});
  } else {
    const GlobalPlain src{in + off, nullptr, (int)n0, 1, ncol};
    const GlobalPlain dst{nullptr, out + off, (int)n0, 1, ncol};
    tile_fft_io<CLS, INV>(th, plan, m, tw, src, dst, SmemCol{bufA, W + 1}, SmemCol{bufB, W + 1});
  }
}

}  // namespace odt
