// Test-infrastructure driver around the reference's own Goldstein code,
// compiled on the host from the sources where they lie (see Makefile):
//   ref_branches: get_branches_goldstein_compute (get_branches_goldstein_
//                 compute_v2.cpp:12-203, with update_v2.cpp and the host
//                 variant of search_universal.cpp)
//   ref_nearest:  the GPU nearest-residue search shortest_compute_kernel
//                 (search_universal.cpp with GPU_COMPUTE, as included by
//                 get_shortest_sort_cuda.cu), run one "thread" at a time on
//                 the host with the CUDA qualifiers defined away.
// The lookup table is passed with a block of -1 entries in front of it, so a
// read below its start would see an empty box (none is expected).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <vector>

#include "get_branches_goldstein_compute_v2.hpp"

namespace emu {
struct Dim3 {
  int x = 0, y = 0, z = 0;
};
Dim3 threadIdx, blockIdx, blockDim;
using std::abs;
using std::max;
using std::min;
#define __device__
#define __global__
#define GPU_COMPUTE
#include "search_universal.cpp"
#undef GPU_COMPUTE
#undef __global__
#undef __device__
}  // namespace emu

static std::vector<int32_t> guarded(const int32_t* lookup, int len) {
  std::vector<int32_t> g((size_t)2 * len + 1, -1);
  std::copy(lookup, lookup + len, g.begin() + len + 1);
  return g;
}

extern "C" {

int ref_nearest(const int32_t* rows, const int32_t* lookup, const int32_t* zstart, const int32_t* square,
                int R, int K, int M1, int M2, int nz, int lookup_len, int32_t* out) {
  std::vector<int32_t> g = guarded(lookup, lookup_len);
  const int32_t* lk = g.data() + lookup_len + 1;
  emu::blockDim.x = 1;
  emu::blockIdx.x = 0;
  for (int i = 0; i < R; ++i) {
    emu::threadIdx.x = i;
    emu::shortest_compute_kernel(rows, lk, zstart, square, out, R, K, M1, M2, nz, lookup_len);
  }
  return 0;
}

long long ref_branches(const int32_t* rows, const int32_t* nearest, const int32_t* square,
                       const int32_t* lookup, const int32_t* zstart, int R, int nz, int lookup_len, int K,
                       int M1, int M2, int M3, int32_t* out, long long cap) {
  std::vector<int32_t> g = guarded(lookup, lookup_len);
  const std::array<int, 3> size = {M1, M2, M3};
  std::vector<branche_coordinates> br = get_branches_goldstein_compute(
      rows, nearest, square, g.data() + lookup_len + 1, zstart, R, nz, lookup_len, K, size);
  const long long n = (long long)br.size();
  for (long long i = 0; i < n && i < cap; ++i) {
    int32_t* o = out + 6 * i;
    o[0] = br[i].point_1_x;
    o[1] = br[i].point_1_y;
    o[2] = br[i].point_2_x;
    o[3] = br[i].point_2_y;
    o[4] = br[i].point_z;
    o[5] = br[i].jump_value;
  }
  return n;
}

}  // extern "C"
