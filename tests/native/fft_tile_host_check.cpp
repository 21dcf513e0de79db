// CPU run of the line / column FFT tile bodies (tile_bodies.cuh) with the
// centring shifts, CTA by CTA with one thread.  Test infrastructure only.
// usage: fft_tile_host_check <kind 0=lines 1=cols> <n0> <n> <n2> <inverse> <shift> <order>
// reads n0*n*n2 complex (column-major [n0, n, n2] for cols, [n, nlines] for
// lines with n0 = nlines) from stdin, writes the transformed array.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "fft_plan.h"
#include "tile_bodies.cuh"

using namespace odt;

int main(int argc, char** argv) {
  if (argc != 8) return 2;
  const int kind = atoi(argv[1]), n0 = atoi(argv[2]), n = atoi(argv[3]), n2 = atoi(argv[4]);
  const bool inv = atoi(argv[5]) != 0;
  const int shift = atoi(argv[6]), order = atoi(argv[7]);
  FftPlan plan;
  std::string why;
  if (!make_plan(n, &plan, &why, order)) { fprintf(stderr, "%s\n", why.c_str()); return 4; }
  std::vector<float2> tw = make_twiddles(n);
  const long long tot = (long long)n0 * n * n2;
  std::vector<float2> x(tot);
  for (long long i = 0; i < tot; ++i) if (scanf("%f %f", &x[i].x, &x[i].y) != 2) return 5;
  std::vector<float2> y(tot);
  std::vector<unsigned char> sm(1 << 22);
  const Thr th{0, 1};
  const float sc = inv ? 1.0f / n : 1.0f;
  // dispatch on the plan's radix class exactly as the kernels do
#define RUN_CLS(C)                                                                                  \
  if (kind == 0) {                                                                                  \
    const int W = 16;                                                                               \
    const long long nlines = (long long)n0 * n2;                                                    \
    const unsigned blocks = (unsigned)((nlines + W - 1) / W);                                       \
    for (unsigned b = 0; b < blocks; ++b) {                                                         \
      if (inv) fft_lines_body<C, true>(x.data(), y.data(), nlines, shift, shift, sc, plan, tw.data(), W, sm.data(), b, th); \
      else fft_lines_body<C, false>(x.data(), y.data(), nlines, shift, shift, sc, plan, tw.data(), W, sm.data(), b, th); \
    }                                                                                               \
  } else {                                                                                          \
    const int lgW = 4;                                                                              \
    const unsigned blocks = (unsigned)(((n0 + 15) / 16) * n2);                                      \
    for (unsigned b = 0; b < blocks; ++b) {                                                         \
      if (inv) fft_cols_body<C, true, true>(x.data(), y.data(), n0, shift, shift, sc, plan, tw.data(), lgW, sm.data(), b, th); \
      else fft_cols_body<C, false, true>(x.data(), y.data(), n0, shift, shift, sc, plan, tw.data(), lgW, sm.data(), b, th); \
    }                                                                                               \
  }
  if (plan.rclass > 2) return 6;
  if (plan.rclass == 0) { RUN_CLS(0) } else if (plan.rclass == 1) { RUN_CLS(1) } else { RUN_CLS(2) }
#undef RUN_CLS
  for (long long i = 0; i < tot; ++i) printf("%.9g %.9g\n", y[i].x, y[i].y);
  return 0;
}
