// CPU run of the Born loop through the exact tile-kernel bodies of libodt
// (tile_bodies.cuh): every CTA of every launch runs in turn with one thread,
// in the launch order of odt_api.cu.  Test infrastructure only.
//
// usage: tile_host_check <in.bin> <out.bin>
//   in.bin : int32[16] header {px,py,pz, rx0,ry0,rz0, rx,ry,rz, nb, bornmax,
//            acyclic, Wx, lgWz, lgWy, 0}, float32[5] {eps, c_im, g_scale,
//            g_off, inv_n}, then mask x/y/z (f32), ramp x/y/z (c64),
//            kq2 x/y/z (f32), V (c64, nvox), Einc (c64, rx*ry*rz*nb)
//   out.bin: Fout (c64, rx*ry*rz*nb)
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "fft_plan.h"
#include "tile_bodies.cuh"

using namespace odt;

template <typename T>
static void rd(FILE* f, std::vector<T>& v, size_t n) {
  v.resize(n);
  if (fread(v.data(), sizeof(T), n, f) != n) { fprintf(stderr, "short read\n"); exit(3); }
}

struct Len {
  FftPlan plan;
  std::vector<float2> tw;
};

static Len make_len(int n, int order) {
  Len L;
  std::string why;
  if (!make_plan(n, &L.plan, &why, order)) { fprintf(stderr, "%s\n", why.c_str()); exit(4); }
  L.tw = make_twiddles(n);
  return L;
}

int main(int argc, char** argv) {
  if (argc != 3) return 2;
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 2;
  std::vector<int> h;
  std::vector<float> sc;
  rd(f, h, 16);
  rd(f, sc, 5);
  BornArgs a{};
  a.px = h[0]; a.py = h[1]; a.pz = h[2];
  a.rx0 = h[3]; a.ry0 = h[4]; a.rz0 = h[5];
  a.rx = h[6]; a.ry = h[7]; a.rz = h[8];
  a.nbatch = h[9];
  const int B = h[10];
  a.acyclic = h[11];
  const int Wx = h[12], lgWz = h[13], lgWy = h[14];
  a.eps = sc[0]; a.c_im = sc[1]; a.g_scale = sc[2]; a.g_off = sc[3]; a.inv_n = sc[4];
  const int P[3] = {a.px, a.py, a.pz};
  a.nvox = (long long)a.px * a.py * a.pz;
  std::vector<float> mask[3], kq2[3];
  std::vector<float2> ramp[3], V, Einc;
  for (int i = 0; i < 3; ++i) rd(f, mask[i], P[i]);
  for (int i = 0; i < 3; ++i) rd(f, ramp[i], P[i]);
  for (int i = 0; i < 3; ++i) rd(f, kq2[i], P[i]);
  rd(f, V, a.nvox);
  const long long est = (long long)a.rx * a.ry * a.rz;
  rd(f, Einc, est * a.nbatch);
  fclose(f);
  for (int i = 0; i < 3; ++i) { a.mask[i] = mask[i].data(); a.ramp[i] = ramp[i].data(); a.kq2[i] = kq2[i].data(); }
  std::vector<float2> T(a.nvox * a.nbatch), Fn(T.size()), F(T.size()), Fout(est * a.nbatch);
  a.T = T.data(); a.Fn = Fn.data(); a.F = F.data(); a.V = V.data(); a.Einc = Einc.data(); a.Fout = Fout.data();
  // radix orders as odt_api.cu: smallest radix first for the fused x-pass
  Len lx = make_len(a.px, kSmallFirst), ly = make_len(a.py, kLargeFirst), lz = make_len(a.pz, kLargeFirst);
  std::vector<unsigned char> sm(1 << 22);
  const Thr th{0, 1};
  const unsigned bx = (unsigned)(((a.py + Wx - 1) / Wx) * a.pz * a.nbatch);
  const long long n0z = (long long)a.px * a.py;
  const unsigned bz = (unsigned)(((n0z + (1 << lgWz) - 1) >> lgWz) * a.nbatch);
  const unsigned by = (unsigned)((((long long)a.px + (1 << lgWy) - 1) >> lgWy) * a.pz * a.nbatch);
  // every body is dispatched on its plan's radix class, as the launchers do
  if (lx.plan.rclass > 2 || ly.plan.rclass > 2 || lz.plan.rclass > 2) return 6;
  auto born_x = [&](int mode, int jj) {
    for (unsigned blk = 0; blk < bx; ++blk) {
#define BX(C)                                                                                   \
  if (mode == kBornFirst) born_x_body<C, kBornFirst>(a, jj, lx.plan, lx.tw.data(), Wx, sm.data(), blk, th); \
  else if (mode == kBornMid) born_x_body<C, kBornMid>(a, jj, lx.plan, lx.tw.data(), Wx, sm.data(), blk, th); \
  else born_x_body<C, kBornLast>(a, jj, lx.plan, lx.tw.data(), Wx, sm.data(), blk, th);
      if (lx.plan.rclass == 0) { BX(0) } else if (lx.plan.rclass == 1) { BX(1) } else { BX(2) }
#undef BX
    }
  };
  auto born_y = [&](bool inv) {
    for (unsigned blk = 0; blk < by; ++blk) {
#define BY(C)                                                                                                    \
  if (inv) fft_cols_body<C, true, false>(a.T, a.T, a.px, 0, 0, 1.f, ly.plan, ly.tw.data(), lgWy, sm.data(), blk, th); \
  else fft_cols_body<C, false, false>(a.T, a.T, a.px, 0, 0, 1.f, ly.plan, ly.tw.data(), lgWy, sm.data(), blk, th);
      if (ly.plan.rclass == 0) { BY(0) } else if (ly.plan.rclass == 1) { BY(1) } else { BY(2) }
#undef BY
    }
  };
  auto born_z = [&](int jj) {
    for (unsigned blk = 0; blk < bz; ++blk) {
      if (lz.plan.rclass == 0) born_z_body<0>(a, jj, lz.plan, lz.tw.data(), lgWz, sm.data(), blk, th);
      else if (lz.plan.rclass == 1) born_z_body<1>(a, jj, lz.plan, lz.tw.data(), lgWz, sm.data(), blk, th);
      else born_z_body<2>(a, jj, lz.plan, lz.tw.data(), lgWz, sm.data(), blk, th);
    }
  };
  for (int jj = 1; jj <= B; ++jj) {
    born_x(jj == 1 ? kBornFirst : kBornMid, jj);
    born_y(false);
    born_z(jj);
    born_y(true);
  }
  born_x(kBornLast, B + 1);
  FILE* o = fopen(argv[2], "wb");
  fwrite(Fout.data(), sizeof(float2), Fout.size(), o);
  fclose(o);
  return 0;
}
