// CPU check of the FFT pass logic in fft_core.cuh: runs every Stockham pass
// with a single "thread" on a tile of pencils and prints the result so the
// Python test can compare it against numpy.  Test infrastructure only.
//
// usage: fft_host_check n W inverse [order]  (reads 2*n*W floats from stdin: pencil-
// major interleaved complex input, writes the same layout to stdout)
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "fft_plan.h"

int main(int argc, char** argv) {
  if (argc != 4 && argc != 5) return 2;
  const int order = argc == 5 ? std::atoi(argv[4]) : 0;
  int n = std::atoi(argv[1]), W = std::atoi(argv[2]), inv = std::atoi(argv[3]);
  int lgW = 0;
  while ((1 << lgW) < W) ++lgW;
  if ((1 << lgW) != W) return 3;
  odt::FftPlan plan;
  std::string why;
  if (!odt::make_plan(n, &plan, &why, order)) {
    std::fprintf(stderr, "%s\n", why.c_str());
    return 4;
  }
  auto tw = odt::make_twiddles(n);
  int ld = W + 1;
  std::vector<float2> a(n * ld), b(n * ld);
  for (int c = 0; c < W; ++c)
    for (int i = 0; i < n; ++i) {
      float re, im;
      if (std::scanf("%f %f", &re, &im) != 2) return 5;
      a[i * ld + c] = make_float2(re, im);
    }
  float2* src = a.data();
  float2* dst = b.data();
  int ns = 1;
  for (int p = 0; p < plan.npass; ++p) {
    int R = plan.radix[p];
    if (inv) odt::run_pass_any<true>(plan.rclass, R, src, dst, n, ns, lgW, ld, tw.data(), 0, 1);
    else odt::run_pass_any<false>(plan.rclass, R, src, dst, n, ns, lgW, ld, tw.data(), 0, 1);
    ns *= R;
    std::swap(src, dst);
  }
  std::fprintf(stderr, "plan:");
  for (int p = 0; p < plan.npass; ++p) std::fprintf(stderr, " %d", plan.radix[p]);
  std::fprintf(stderr, "\n");
  for (int c = 0; c < W; ++c)
    for (int i = 0; i < n; ++i) std::printf("%.9g %.9g\n", src[i * ld + c].x, src[i * ld + c].y);
  return 0;
}
