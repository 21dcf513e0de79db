// Mixed-radix Stockham FFT building blocks for the CBS hot path.
//
// Every 1D transform in the solver runs through these device functions.  A
// "tile" is a block of W independent pencils of length n held in shared
// memory as rows: element (i, c) of pencil c lives at s[i * ld + c], with the
// row pitch ld = W + 1 so that both the column-wise butterfly accesses and the
// transposed global<->shared staging are bank-conflict free for 8-byte
// elements.  One pass of radix R reads the tile from `src`, applies the
// inter-pass twiddles and an R-point DFT in registers, and writes the
// self-sorting (Stockham) output to `dst`; passes ping-pong between two tiles,
// so no bit reversal is ever needed and the result is in natural order.
//
// Twiddles come from a table tw[k] = exp(-2*pi*i*k/n), k < n, computed in
// double on the host and rounded once to float (the accuracy of the table
// bounds the accuracy of the transform; nothing here calls sin/cos).
//
// Radices: 2, 4, 8 (closed-form butterflies) and any odd R <= 31 through the
// symmetric real-coefficient DFT (pairs v[m], v[R-m] so that an odd R-point
// DFT costs (R-1)^2 real multiply-adds instead of R^2 complex products).
//
// The functions are usable from host code as well (plain C++ when not
// compiled by nvcc) so the pass logic can be checked on a CPU by running each
// pass with one "thread" -- every pass is a pure src -> dst map, so the
// sequential schedule is exact.
#pragma once

#include <cuda_runtime.h>  // float2 / make_float2 for host and device code
#if defined(__CUDACC__)
#define ODT_HD __host__ __device__ __forceinline__
#else
#define ODT_HD inline
#endif

namespace odt {

constexpr int kMaxPasses = 8;

// One transform length: radix sequence and where its twiddles live.
struct FftPlan {
  int n;
  int npass;
  int radix[kMaxPasses];
  int rclass;  // radix class (largest radix: 0 -> <= 8, 1 -> <= 15, 2 -> <= 31)
};

// Device code on sm_100 adds, subtracts and multiply-adds complex values as
// packed FP32 pairs (one add.f32x2 / sub.f32x2 / fma.rn.f32x2 per complex
// operation instead of two scalar ones): the same IEEE operations on each
// component, so the results are the scalar code's, at half the instruction
// count.
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 1000
#define ODT_F32X2 1
__device__ __forceinline__ float2 fsub2(float2 a, float2 b) {
  float2 r;
  asm("{\n\t.reg .b64 x, y, d;\n\t"
      "mov.b64 x, {%2, %3};\n\tmov.b64 y, {%4, %5};\n\t"
      "sub.rn.f32x2 d, x, y;\n\tmov.b64 {%0, %1}, d;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
#endif
ODT_HD float2 cadd(float2 a, float2 b) {
#if defined(ODT_F32X2)
  return __fadd2_rn(a, b);
#else
  return make_float2(a.x + b.x, a.y + b.y);
#endif
}
ODT_HD float2 csub(float2 a, float2 b) {
#if defined(ODT_F32X2)
  return fsub2(a, b);
#else
  return make_float2(a.x - b.x, a.y - b.y);
#endif
}
// acc + c * v for real c (both components)
ODT_HD float2 cfma_real(float c, float2 v, float2 acc) {
#if defined(ODT_F32X2)
  return __ffma2_rn(make_float2(c, c), v, acc);
#else
  return make_float2(c * v.x + acc.x, c * v.y + acc.y);
#endif
}
ODT_HD float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
ODT_HD float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
ODT_HD float2 cscale(float2 a, float s) {
#if defined(ODT_F32X2)
  return __fmul2_rn(a, make_float2(s, s));
#else
  return make_float2(a.x * s, a.y * s);
#endif
}
// multiply by -i (forward) or +i (inverse)
template <bool INV>
ODT_HD float2 rot90(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// a + rot90<INV>(c) and a - rot90<INV>(c) as scalar pairs: the rotation
// swaps components, which a packed operation could only take after two moves
template <bool INV>
ODT_HD float2 addrot(float2 a, float2 c) {
  return INV ? make_float2(a.x - c.y, a.y + c.x) : make_float2(a.x + c.y, a.y - c.x);
}
template <bool INV>
ODT_HD float2 subrot(float2 a, float2 c) {
  return INV ? make_float2(a.x + c.y, a.y - c.x) : make_float2(a.x - c.y, a.y + c.x);
}

// ---------------------------------------------------------------- butterflies
template <int R, bool INV>
struct Butterfly;

template <bool INV>
struct Butterfly<2, INV> {
  ODT_HD static void run(float2* v, const float2*, int) {
    float2 a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <bool INV>
struct Butterfly<4, INV> {
  ODT_HD static void run(float2* v, const float2*, int) {
    float2 s02 = cadd(v[0], v[2]), d02 = csub(v[0], v[2]);
    float2 s13 = cadd(v[1], v[3]), c13 = csub(v[1], v[3]);
    v[0] = cadd(s02, s13);
    v[2] = csub(s02, s13);
    v[1] = addrot<INV>(d02, c13);   // d02 + rot90(c13)
    v[3] = subrot<INV>(d02, c13);
  }
};

template <bool INV>
struct Butterfly<8, INV> {
  ODT_HD static void run(float2* v, const float2*, int) {
    const float h = 0.70710678118654752440f;
    float2 e[4] = {v[0], v[2], v[4], v[6]};
    float2 o[4] = {v[1], v[3], v[5], v[7]};
    Butterfly<4, INV>::run(e, nullptr, 0);
    Butterfly<4, INV>::run(o, nullptr, 0);
    // W8^k, k = 1..3 applied to the odd half: o1 and o3 hold W8^k o[k] / h
    // (h enters through the multiply-adds below), W8^2 = -/+ i through addrot
    float2 o1 = INV ? make_float2(o[1].x - o[1].y, o[1].x + o[1].y)
                    : make_float2(o[1].x + o[1].y, o[1].y - o[1].x);
    float2 o3 = INV ? make_float2(-(o[3].x + o[3].y), o[3].x - o[3].y)
                    : make_float2(o[3].y - o[3].x, -(o[3].x + o[3].y));
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cfma_real(h, o1, e[1]);    // e1 +/- h o1 as one multiply-add each
    v[5] = cfma_real(-h, o1, e[1]);
    v[2] = addrot<INV>(e[2], o[2]);
    v[6] = subrot<INV>(e[2], o[2]);
    v[3] = cfma_real(h, o3, e[3]);
    v[7] = cfma_real(-h, o3, e[3]);
  }
};

// cos(2 pi t / R) and sin(2 pi t / R) at compile time, in double: the angle
// reduced to [-pi, pi] and Taylor series of 26 terms (the largest term is
// below 2^3, so the result is within a few units of 1e-16), rounded to float
// once -- the values the double-precision twiddle tables hold.
constexpr double kTwoPi = 6.283185307179586476925286766559;
constexpr double ce_sin_red(double x) {
  double term = x, sum = x;
  for (int k = 1; k < 26; ++k) {
    term *= -x * x / ((2.0 * k) * (2.0 * k + 1.0));
    sum += term;
  }
  return sum;
}
constexpr double ce_cos_red(double x) {
  double term = 1.0, sum = 1.0;
  for (int k = 1; k < 26; ++k) {
    term *= -x * x / ((2.0 * k - 1.0) * (2.0 * k));
    sum += term;
  }
  return sum;
}
constexpr double ce_angle(int t, int R) {   // 2 pi t / R reduced to [-pi, pi]
  const int u = ((t % R) + R) % R;
  return 2 * u > R ? kTwoPi * (double)(u - R) / (double)R : kTwoPi * (double)u / (double)R;
}
template <int R>
struct UnitRoots {   // cos / sin of 2 pi t / R, t < R, as float
  float c[R];
  float s[R];
  constexpr UnitRoots() : c(), s() {
    for (int t = 0; t < R; ++t) {
      c[t] = (float)ce_cos_red(ce_angle(t, R));
      s[t] = (float)ce_sin_red(ce_angle(t, R));
    }
  }
};

// R = 12 = 4 x 3 in registers (for the fused passes on lengths 96 = 8 x 12):
// n = 3 n1 + n2, k = k1 + 4 k2; 4-point DFTs over n1, twiddles W_12^(n2 k1)
// as compile-time constants, 3-point DFTs over n2.
template <bool INV>
struct Butterfly<12, INV> {
  ODT_HD static void run(float2* v, const float2* tw, int n) {
    constexpr UnitRoots<12> ur{};
    (void)tw;
    (void)n;
    float2 t[3][4];
#pragma unroll
    for (int n2 = 0; n2 < 3; ++n2) {
      float2 q[4] = {v[n2], v[3 + n2], v[6 + n2], v[9 + n2]};
      Butterfly<4, INV>::run(q, nullptr, 0);
#pragma unroll
      for (int k1 = 0; k1 < 4; ++k1) {
        const int e = n2 * k1;
        if (e == 0) {
          t[n2][k1] = q[k1];
        } else {   // exp(-/+ 2 pi i e / 12)
          const float2 w = make_float2(ur.c[e], INV ? ur.s[e] : -ur.s[e]);
          t[n2][k1] = cmul(q[k1], w);
        }
      }
    }
    // 3-point DFT: c = cos(2 pi / 3) = -1/2, s = sin(2 pi / 3)
    const float s3 = 0.86602540378443864676f;
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      const float2 a0 = t[0][k1], a1 = t[1][k1], a2 = t[2][k1];
      const float2 sum = cadd(a1, a2), dif = csub(a1, a2);
      const float2 m = make_float2(a0.x - 0.5f * sum.x, a0.y - 0.5f * sum.y);
      // forward: X1 = m - i s dif, X2 = m + i s dif
      const float2 j = make_float2(-s3 * dif.y, s3 * dif.x);   // i s dif
      v[k1] = cadd(a0, sum);
      v[k1 + 4] = INV ? cadd(m, j) : csub(m, j);
      v[k1 + 8] = INV ? csub(m, j) : cadd(m, j);
    }
  }
};

// Odd R: X[k] = v0 + sum_m a_m cos(2 pi m k / R) -/+ i sum_m b_m sin(2 pi m k / R)
// with a_m = v[m] + v[R-m], b_m = v[m] - v[R-m]; the cosines and sines are
// read from the transform's table at multiples of n / R.
template <int R, bool INV>
struct OddButterfly {
  ODT_HD static void run(float2* v, const float2* tw, int n) {
    constexpr int H = (R - 1) / 2;
    constexpr UnitRoots<R> ur{};   // compile-time coefficients (no table loads)
    (void)tw;
    (void)n;
    float cs[H + 1], sn[H + 1];
    cs[0] = 1.f;  // m*k can be a multiple of R when R is composite (9, 15, ...)
    sn[0] = 0.f;
#pragma unroll
    for (int t = 1; t <= H; ++t) {
      cs[t] = ur.c[t];   // exp(-2 pi i t / R) = cs - i sn
      sn[t] = ur.s[t];
    }
    // jb_m = i b_m = (-b_m.y, b_m.x), so that i * im = sum_m s jb_m is a sum
    // of packed products (negation is exact: the same values as i * (sum s b_m))
    float2 a[H + 1], jb[H + 1];
    float2 x0 = v[0];
    float2 sum = v[0];
#pragma unroll
    for (int m = 1; m <= H; ++m) {
      a[m] = cadd(v[m], v[R - m]);
      jb[m] = make_float2(v[R - m].y - v[m].y, v[m].x - v[R - m].x);
      sum = cadd(sum, a[m]);
    }
    v[0] = sum;
#pragma unroll
    for (int k = 1; k <= H; ++k) {
      float2 re = x0, jim = make_float2(0.f, 0.f);
#pragma unroll
      for (int m = 1; m <= H; ++m) {
        const int t = (m * k) % R;
        const float c = (t <= H) ? cs[t] : cs[R - t];
        const float s = (t <= H) ? sn[t] : -sn[R - t];
        re = cfma_real(c, a[m], re);
        jim = cfma_real(s, jb[m], jim);
      }
      // forward: X[k] = re - i*im, X[R-k] = re + i*im (jim = i * im)
      if (INV) {
        v[k] = cadd(re, jim);
        v[R - k] = csub(re, jim);
      } else {
        v[k] = csub(re, jim);
        v[R - k] = cadd(re, jim);
      }
    }
  }
};

// A * B points in registers (Cooley-Tukey with both factors as butterflies):
// n = B n1 + n2, k = k1 + A k2; A-point DFTs over n1, the twiddles
// W_AB^(n2 k1) as compile-time constants, B-point DFTs over n2.  For
// composite radices of the pipelined passes (35 = 5 x 7: the 280-point axes).
template <int A, int B, bool INV>
struct CompositeButterfly {
  ODT_HD static void run(float2* v, const float2* tw, int n) {
    constexpr int AB = A * B;
    constexpr UnitRoots<AB> ur{};
    float2 t[B][A];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) {
      float2 q[A];
#pragma unroll
      for (int n1 = 0; n1 < A; ++n1) q[n1] = v[B * n1 + n2];
      Butterfly<A, INV>::run(q, tw, n);
#pragma unroll
      for (int k1 = 0; k1 < A; ++k1) {
        const int e = (n2 * k1) % AB;
        if (e == 0) {
          t[n2][k1] = q[k1];
        } else {   // exp(-/+ 2 pi i e / AB)
          const float2 w = make_float2(ur.c[e], INV ? ur.s[e] : -ur.s[e]);
          t[n2][k1] = cmul(q[k1], w);
        }
      }
    }
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
      float2 q[B];
#pragma unroll
      for (int n2 = 0; n2 < B; ++n2) q[n2] = t[n2][k1];
      Butterfly<B, INV>::run(q, tw, n);
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = q[k2];
    }
  }
};

#define ODT_ODD_BUTTERFLY(R)                                      \
  template <bool INV>                                             \
  struct Butterfly<R, INV> {                                      \
    ODT_HD static void run(float2* v, const float2* tw, int n) {  \
      OddButterfly<R, INV>::run(v, tw, n);                        \
    }                                                             \
  };
ODT_ODD_BUTTERFLY(3)
ODT_ODD_BUTTERFLY(5)
ODT_ODD_BUTTERFLY(7)
ODT_ODD_BUTTERFLY(9)
ODT_ODD_BUTTERFLY(11)
ODT_ODD_BUTTERFLY(13)
ODT_ODD_BUTTERFLY(15)
ODT_ODD_BUTTERFLY(17)
ODT_ODD_BUTTERFLY(19)
ODT_ODD_BUTTERFLY(23)
ODT_ODD_BUTTERFLY(25)
ODT_ODD_BUTTERFLY(27)
ODT_ODD_BUTTERFLY(29)
ODT_ODD_BUTTERFLY(31)
#undef ODT_ODD_BUTTERFLY

template <bool INV>
struct Butterfly<35, INV> {
  ODT_HD static void run(float2* v, const float2* tw, int n) { CompositeButterfly<5, 7, INV>::run(v, tw, n); }
};

// even radices of the fused xy-pass and the pipelined z-pass (axes of
// 8 R = 112, 128, 144, 160 points): 14 = 2 x 7, 16 = 4 x 4, 18 = 2 x 9,
// 20 = 4 x 5
template <bool INV>
struct Butterfly<14, INV> {
  ODT_HD static void run(float2* v, const float2* tw, int n) { CompositeButterfly<2, 7, INV>::run(v, tw, n); }
};
template <bool INV>
struct Butterfly<16, INV> {
  ODT_HD static void run(float2* v, const float2* tw, int n) { CompositeButterfly<4, 4, INV>::run(v, tw, n); }
};
template <bool INV>
struct Butterfly<18, INV> {
  ODT_HD static void run(float2* v, const float2* tw, int n) { CompositeButterfly<2, 9, INV>::run(v, tw, n); }
};
template <bool INV>
struct Butterfly<20, INV> {
  ODT_HD static void run(float2* v, const float2* tw, int n) { CompositeButterfly<4, 5, INV>::run(v, tw, n); }
};

// ------------------------------------------------------------------ one pass
// Stockham radix-R pass over a tile of W pencils (W a power of two, lgW its
// log2).  ns = product of the radices of the passes already done.  Work item
// idx -> (column c, butterfly j); thread `tid` of `nthr` takes every nthr-th.
template <int R, bool INV>
ODT_HD void stockham_pass(const float2* __restrict__ src, float2* __restrict__ dst,
                          int n, int ns, int lgW, int ld, const float2* __restrict__ tw,
                          int tid, int nthr) {
  const int W = 1 << lgW;
  const int nb = n / R;
  const int total = nb << lgW;
  const int tstride = n / (ns * R);
  for (int idx = tid; idx < total; idx += nthr) {
    const int c = idx & (W - 1);
    const int j = idx >> lgW;
    const int k = j % ns;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[(j + r * nb) * ld + c];
    if (ns > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        float2 w = tw[r * k * tstride];
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    Butterfly<R, INV>::run(v, tw, n);
    const int d = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[(d + r * ns) * ld + c] = v[r];
  }
}

// Radix classes: a kernel instantiated for class K only contains the
// butterflies of classes <= K, so its register budget is set by the largest
// radix it can meet (class 0: 2, 3, 4, 5, 8; 1: adds 7, 9, 11, 13, 15;
// 2: adds 17, 19; 3: adds 23-31).
constexpr int kNumRadixClasses = 4;
inline int radix_class_of(int r) {
  switch (r) {
    case 2: case 3: case 4: case 5: case 8: return 0;  // closed-form / short butterflies
    case 7: case 9: case 11: case 13: case 15: return 1;
    case 17: case 19: return 2;
    default: return 3;
  }
}

template <int CLS, bool INV>
ODT_HD void run_pass(int R, const float2* src, float2* dst, int n, int ns, int lgW, int ld,
                     const float2* tw, int tid, int nthr) {
  switch (R) {
#define ODT_CASE(r) \
  case r: stockham_pass<r, INV>(src, dst, n, ns, lgW, ld, tw, tid, nthr); break;
    ODT_CASE(2) ODT_CASE(3) ODT_CASE(4) ODT_CASE(5) ODT_CASE(8)
#undef ODT_CASE
    default:
      if (CLS >= 1) {
        switch (R) {
#define ODT_CASE(r) \
  case r: stockham_pass<(CLS >= 1 ? r : 2), INV>(src, dst, n, ns, lgW, ld, tw, tid, nthr); break;
          ODT_CASE(7) ODT_CASE(9) ODT_CASE(11) ODT_CASE(13) ODT_CASE(15)
#undef ODT_CASE
          default:
            if (CLS >= 2) {
              switch (R) {
#define ODT_CASE(r) \
  case r: stockham_pass<(CLS >= 2 ? r : 2), INV>(src, dst, n, ns, lgW, ld, tw, tid, nthr); break;
                ODT_CASE(17) ODT_CASE(19)
#undef ODT_CASE
                default:
                  if (CLS >= 3) {
                    switch (R) {
#define ODT_CASE(r) \
  case r: stockham_pass<(CLS >= 3 ? r : 2), INV>(src, dst, n, ns, lgW, ld, tw, tid, nthr); break;
                      ODT_CASE(23) ODT_CASE(25) ODT_CASE(27) ODT_CASE(29) ODT_CASE(31)
#undef ODT_CASE
                      default: break;  // unreachable: plans are validated on the host
                    }
                  }
                  break;
              }
            }
            break;
        }
      }
      break;
  }
}

// Host-side dispatch by a plan's radix class, as the kernels dispatch.
template <bool INV>
inline void run_pass_any(int cls, int R, const float2* src, float2* dst, int n, int ns, int lgW,
                         int ld, const float2* tw, int tid, int nthr) {
  switch (cls) {
    case 0: run_pass<0, INV>(R, src, dst, n, ns, lgW, ld, tw, tid, nthr); break;
    case 1: run_pass<1, INV>(R, src, dst, n, ns, lgW, ld, tw, tid, nthr); break;
    case 2: run_pass<2, INV>(R, src, dst, n, ns, lgW, ld, tw, tid, nthr); break;
    default: run_pass<3, INV>(R, src, dst, n, ns, lgW, ld, tw, tid, nthr); break;
  }
}

inline bool radix_supported(int r) {
  switch (r) {
    case 2: case 3: case 4: case 5: case 7: case 8: case 9: case 11: case 13: case 15:
    case 17: case 19: case 23: case 25: case 27: case 29: case 31: return true;
    default: return false;
  }
}

}  // namespace odt
