// Host-side FFT planning: radix factorisation and twiddle tables.
#pragma once

#include <string>
#include <vector>

#include "fft_core.cuh"

namespace odt {

// Factor n into supported radices (8s, then 4, then 2, then odd factors,
// merging small odd primes while the product stays <= 15).  Returns false when
// n has a prime factor > 31 (those lengths are rejected with a clear error).
// order = kLargeFirst puts the largest radix first (f[0]); kSmallFirst the
// smallest.  Forward transforms run f[0..P-1], inverse f[P-1..0].
enum PlanOrder { kLargeFirst = 0, kSmallFirst = 1 };
bool make_plan(int n, FftPlan* plan, std::string* why, int order = kLargeFirst);

// tw[k] = exp(-2 pi i k / n), k = 0..n-1, evaluated in double, rounded once.
std::vector<float2> make_twiddles(int n);

}  // namespace odt
