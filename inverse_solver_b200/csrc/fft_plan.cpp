#include "fft_plan.h"

#include <algorithm>
#include <cmath>

namespace odt {

bool make_plan(int n, FftPlan* plan, std::string* why, int order) {
  if (n < 1) {
    if (why) *why = "FFT length must be positive";
    return false;
  }
  std::vector<int> rad;
  int m = n;
  while (m % 8 == 0 && m > 1) { rad.push_back(8); m /= 8; }
  if (m % 4 == 0) { rad.push_back(4); m /= 4; }
  if (m % 2 == 0) { rad.push_back(2); m /= 2; }
  std::vector<int> odd;
  for (int p = 3; p * p <= m; p += 2) {
    while (m % p == 0) { odd.push_back(p); m /= p; }
  }
  if (m > 1) odd.push_back(m);
  for (int p : odd) {
    if (p > 31) {
      if (why) *why = "FFT length " + std::to_string(n) + " has prime factor " + std::to_string(p) +
                      " > 31 (unsupported)";
      return false;
    }
  }
  // merge small odd factors (3*3=9, 3*5=15) to save passes
  std::vector<int> merged;
  for (int p : odd) {
    if (!merged.empty() && merged.back() * p <= 15 && radix_supported(merged.back() * p)) {
      merged.back() *= p;
    } else {
      merged.push_back(p);
    }
  }
  std::vector<int> all = merged;
  all.insert(all.end(), rad.begin(), rad.end());
  if (all.empty()) all.push_back(1);
  std::stable_sort(all.begin(), all.end(), [order](int a, int b) {
    return order == kSmallFirst ? a < b : a > b;
  });
  if ((int)all.size() > kMaxPasses) {
    if (why) *why = "too many FFT passes for length " + std::to_string(n);
    return false;
  }
  plan->n = n;
  plan->npass = 0;
  plan->rclass = 0;
  for (int r : all) {
    if (r == 1) continue;
    plan->radix[plan->npass++] = r;
    plan->rclass = std::max(plan->rclass, radix_class_of(r));
  }
  return true;
}

std::vector<float2> make_twiddles(int n) {
  std::vector<float2> tw(n);
  const double two_pi = 6.283185307179586476925286766559;
  for (int k = 0; k < n; ++k) {
    // reduce the angle to the first octant pair for accuracy
    double a = two_pi * (double)k / (double)n;
    tw[k] = make_float2((float)std::cos(a), (float)(-std::sin(a)));
  }
  return tw;
}

}  // namespace odt
