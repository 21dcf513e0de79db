// Tile-level FFT passes with pluggable storage: the first pass of a
// transform may read straight from global memory and the last may write
// straight to it, so a pencil crosses shared memory only between passes.
//
// A tile is W pencils of length n.  A pass of radix R on it is W * n/R
// butterflies; `Map` assigns butterflies to threads, `Src`/`Dst` say where
// element (row, pencil) lives.  Stockham indexing (see fft_core.cuh): the
// butterfly j of a pass with ns = product of the earlier radices reads rows
// j + r*(n/R) and writes rows (j - j%ns)*R + j%ns + r*ns, r < R.
//
// tile_mid fuses the LAST pass of one transform with the FIRST pass of the
// next one when both have the same radix R: the last pass of a transform
// (ns = n/R) writes rows j + r*(n/R), which are exactly the rows the first
// pass (ns = 1) of the next transform reads, so the R values never leave
// registers and a pointwise operation can be applied in between.  Plans are
// therefore run forward in radix order f[0..P-1] and inverse in reverse
// order f[P-1..0].
#pragma once

#include "fft_core.cuh"

namespace odt {

// ------------------------------------------------------------------ maps
// column index fastest: coalesced when pencils are adjacent in memory
// (y / z pencils); blockDim.x must be a multiple of W.
struct ColMap {
  int lgW;
  ODT_HD int total(int nb) const { return nb << lgW; }
  ODT_HD void decode(int idx, int nb, int& c, int& j) const {
    c = idx & ((1 << lgW) - 1);
    j = idx >> lgW;
  }
  // (c, j) advance by `nthr` work items as c += dc, j += dj with the carry
  // from c into j (no carry when nthr is a multiple of W, as on the GPU)
  ODT_HD void step(int nthr, int nb, int& dc, int& dj) const {
    dc = nthr & ((1 << lgW) - 1);
    dj = nthr >> lgW;
  }
  // returns the carry into j
  ODT_HD int wrap(int& c, int& j, int nb) const {
    if (c >= (1 << lgW)) {
      c -= 1 << lgW;
      ++j;
      return 1;
    }
    return 0;
  }
};

// butterfly index fastest: coalesced when a pencil is contiguous (x lines)
struct LineMap {
  int W;
  ODT_HD int total(int nb) const { return nb * W; }
  ODT_HD void decode(int idx, int nb, int& c, int& j) const {
    c = idx / nb;
    j = idx - c * nb;
  }
  ODT_HD void step(int nthr, int nb, int& dc, int& dj) const {
    dc = nthr / nb;
    dj = nthr - dc * nb;
  }
  // j wraps at nb into the next pencil; j itself gains no carry
  ODT_HD int wrap(int& c, int& j, int nb) const {
    if (j >= nb) {
      j -= nb;
      ++c;
    }
    return 0;
  }
};

// --------------------------------------------------------------- storage
// shared memory, row-major over pencils: s[row * ld + c], ld = W + 1
struct SmemCol {
  float2* s;
  int ld;
  ODT_HD float2 load(int row, int c) const { return s[row * ld + c]; }
  ODT_HD void store(int row, int c, float2 v) const { s[row * ld + c] = v; }
};

// shared memory, pencil-major with one pad element every 8 rows (keeps the
// stride-R writes of small-ns passes off a single bank): s[c*ld + row + row/8].
// The pencil pitch ld is = 8 (mod 16) elements, so two pencils that share a
// half-warp (8-byte accesses, 16 threads) fall in opposite halves of the banks.
struct SmemLine {
  float2* s;
  int ld;
  ODT_HD int at(int row, int c) const { return c * ld + row + (row >> 3); }
  ODT_HD float2 load(int row, int c) const { return s[at(row, c)]; }
  ODT_HD void store(int row, int c, float2 v) const { s[at(row, c)] = v; }
};

ODT_HD int smem_line_ld(int n) {
  const int m = n + (n >> 3) + 1;
  return m + ((8 - (m & 15)) & 15);
}

// global memory, element (row, c) at p[row*rs + c*cs]; pencils c >= ncol
// read as zero and are not written
struct GlobalPlain {
  const float2* in;
  float2* out;
  int rs, cs;  // element strides (a tile spans < 2^31 elements)
  int ncol;
  ODT_HD float2 load(int row, int c) const {
    return c < ncol ? in[row * rs + c * cs] : make_float2(0.f, 0.f);
  }
  ODT_HD void store(int row, int c, float2 v) const {
    if (c < ncol) out[row * rs + c * cs] = v;
  }
};

// as GlobalPlain with a cyclic row shift (gather at (row+shift)%n on load,
// scatter to (row+shift)%n on store) and a scale applied on store: the
// fftshift / ifftshift pair around MATLAB's centred transforms
struct GlobalShift {
  const float2* in;
  float2* out;
  int rs, cs;
  int ncol, n, shift;
  float scale;
  ODT_HD int rot(int row) const {
    int r = row + shift;
    return r >= n ? r - n : r;
  }
  ODT_HD float2 load(int row, int c) const {
    return c < ncol ? in[rot(row) * rs + c * cs] : make_float2(0.f, 0.f);
  }
  ODT_HD void store(int row, int c, float2 v) const {
    if (c < ncol) out[rot(row) * rs + c * cs] = cscale(v, scale);
  }
};

// ------------------------------------------------------------------ passes
// Every pass / body takes the calling thread's index and the thread count,
// so the same code runs in a CUDA block and, with tid = 0 and nthr = 1 and
// the barriers dropped, sequentially on a CPU (exact: each pass completes all
// its butterflies before the next one starts).
struct Thr {
  int tid, nthr;
};

template <int R, bool INV, class Map, class Src, class Dst>
ODT_HD void tile_pass(const Thr& th, const Map& m, int n, int ns, const float2* tw,
                      const Src& src, const Dst& dst) {
  const int nb = n / R;
  const int tstride = n / (ns * R);
  const int total = m.total(nb);
  if (th.tid >= total) return;
  // (c, j, k = j % ns) advance incrementally: ns divides nb, so k is
  // unaffected when j wraps into the next pencil
  int c, j, dc, dj;
  m.decode(th.tid, nb, c, j);
  m.step(th.nthr, nb, dc, dj);
  int k = j % ns;
  const int dk = dj % ns;
  for (int idx = th.tid; idx < total; idx += th.nthr) {
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src.load(j + r * nb, c);
    if (ns > 1) {
      const int kt = k * tstride;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        float2 w = tw[r * kt];
        if (INV) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    Butterfly<R, INV>::run(v, tw, n);
    const int d = (j - k) * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst.store(d + r * ns, c, v[r]);
    c += dc;
    j += dj;
    k += dk + m.wrap(c, j, nb);  // a wrap of j past nb leaves k (ns divides nb)
    if (k >= ns) k -= ns;
  }
}

// MODE_BOTH: last pass (direction FIRST_INV) -> op -> first pass of the
//            other direction; MODE_GEN: op generates the inputs of a first
//            (forward) pass; MODE_END: last pass -> op, nothing stored.
enum MidMode { kMidBoth = 0, kMidGen = 1, kMidEnd = 2 };

template <int R, bool FIRST_INV, int MODE, class Map, class Src, class Dst, class Op>
ODT_HD void tile_mid(const Thr& th, const Map& m, int n, const float2* tw, const Src& src,
                     const Dst& dst, const Op& op) {
  const int nb = n / R;
  const int total = m.total(nb);
  if (th.tid >= total) return;
  int c, j, dc, dj;
  m.decode(th.tid, nb, c, j);
  m.step(th.nthr, nb, dc, dj);
  for (int idx = th.tid; idx < total; idx += th.nthr) {
    if (idx != th.tid) {
      c += dc;
      j += dj;
      m.wrap(c, j, nb);
    }
    float2 v[R];
    if (MODE != kMidGen) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = src.load(j + r * nb, c);
      if (nb > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          float2 w = tw[r * j];  // ns = nb, k = j, tstride = 1
          if (FIRST_INV) w.y = -w.y;
          v[r] = cmul(v[r], w);
        }
      }
      Butterfly<R, FIRST_INV>::run(v, tw, n);
    }
    op.template apply<R>(c, j, nb, v);
    if (MODE != kMidEnd) {
      if (MODE == kMidGen)
        Butterfly<R, false>::run(v, tw, n);
      else
        Butterfly<R, !FIRST_INV>::run(v, tw, n);
#pragma unroll
      for (int r = 0; r < R; ++r) dst.store(j * R + r, c, v[r]);
    }
  }
}

// -------------------------------------------------- radix dispatch by class
#define ODT_RADIX_SWITCH(R, CLS, CALL)                                             \
  switch (R) {                                                                     \
    case 2: { constexpr int RR = 2; CALL; } break;                                 \
    case 3: { constexpr int RR = 3; CALL; } break;                                 \
    case 4: { constexpr int RR = 4; CALL; } break;                                 \
    case 5: { constexpr int RR = 5; CALL; } break;                                 \
    case 8: { constexpr int RR = 8; CALL; } break;                                 \
    default:                                                                       \
      if (CLS == 1) {                                                              \
        switch (R) {                                                               \
          case 7: { constexpr int RR = (CLS == 1) ? 7 : 2; CALL; } break;           \
          case 9: { constexpr int RR = (CLS == 1) ? 9 : 2; CALL; } break;           \
          case 11: { constexpr int RR = (CLS == 1) ? 11 : 2; CALL; } break;         \
          case 13: { constexpr int RR = (CLS == 1) ? 13 : 2; CALL; } break;         \
          case 15: { constexpr int RR = (CLS == 1) ? 15 : 2; CALL; } break;         \
          default: break;                                                          \
        }                                                                          \
      } else if (CLS == 2) {                                                       \
        switch (R) {                                                               \
          case 7: { constexpr int RR = (CLS == 2) ? 7 : 2; CALL; } break;           \
          case 9: { constexpr int RR = (CLS == 2) ? 9 : 2; CALL; } break;           \
          case 11: { constexpr int RR = (CLS == 2) ? 11 : 2; CALL; } break;         \
          case 13: { constexpr int RR = (CLS == 2) ? 13 : 2; CALL; } break;         \
          case 15: { constexpr int RR = (CLS == 2) ? 15 : 2; CALL; } break;         \
          case 17: { constexpr int RR = (CLS == 2) ? 17 : 2; CALL; } break;         \
          case 19: { constexpr int RR = (CLS == 2) ? 19 : 2; CALL; } break;         \
          default: break;                                                          \
        }                                                                          \
      } else if (CLS == 3) {                                                         \
        switch (R) {                                                               \
          case 7: { constexpr int RR = (CLS == 3) ? 7 : 2; CALL; } break;           \
          case 9: { constexpr int RR = (CLS == 3) ? 9 : 2; CALL; } break;           \
          case 11: { constexpr int RR = (CLS == 3) ? 11 : 2; CALL; } break;         \
          case 13: { constexpr int RR = (CLS == 3) ? 13 : 2; CALL; } break;         \
          case 15: { constexpr int RR = (CLS == 3) ? 15 : 2; CALL; } break;         \
          case 17: { constexpr int RR = (CLS == 3) ? 17 : 2; CALL; } break;         \
          case 19: { constexpr int RR = (CLS == 3) ? 19 : 2; CALL; } break;         \
          case 23: { constexpr int RR = (CLS == 3) ? 23 : 2; CALL; } break;          \
          case 29: { constexpr int RR = (CLS == 3) ? 29 : 2; CALL; } break;          \
          case 31: { constexpr int RR = (CLS == 3) ? 31 : 2; CALL; } break;          \
          default: break;                                                          \
        }                                                                          \
      }                                                                            \
      break;                                                                       \
  }

template <int CLS, bool INV, class Map, class Src, class Dst>
ODT_HD void tile_pass_any(const Thr& th, int R, const Map& m, int n, int ns, const float2* tw,
                          const Src& src, const Dst& dst) {
  ODT_RADIX_SWITCH(R, CLS, (tile_pass<RR, INV>(th, m, n, ns, tw, src, dst)))
}

template <int CLS, bool FIRST_INV, int MODE, class Map, class Src, class Dst, class Op>
ODT_HD void tile_mid_any(const Thr& th, int R, const Map& m, int n, const float2* tw,
                         const Src& src, const Dst& dst, const Op& op) {
  ODT_RADIX_SWITCH(R, CLS, (tile_mid<RR, FIRST_INV, MODE>(th, m, n, tw, src, dst, op)))
}

}  // namespace odt
