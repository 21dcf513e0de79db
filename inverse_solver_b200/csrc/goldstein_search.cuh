// Nearest-residue search of the Goldstein branch-cut unwrapper, shared by the
// GPU kernel that precomputes each residue's 8 nearest neighbours
// (get_shortest_sort_cuda.cu, search_universal.cpp:102-271 with
// GPU_COMPUTE) and the host linker's one-nearest search among the residues
// that are not active (search_universal.cpp with the host `states` mask).
//
// The residue table has the reference's layout: int32 rows of 6 (index,
// value, box id, x, y, z), sorted by (z, box id) with ties in index order.
// A slice of size M1 x M2 with residue count R_z is divided into ss x ss boxes
// (ss = ceil(sqrt((R_z + 1) / 16))) of side ceil(M1/ss) x ceil(M2/ss);
// lookup[zstart[z] + b1 + b2*ss] is the first row in box (b1, b2) or -1.
//
// The search grows square rings of boxes around the residue's box and keeps
// the K nearest (Euclidean distance truncated to int) that lie closer than
// the residue's distance to the nearest border; a box is searched only when
// its nearest edge is closer than the current K-th distance, and the rings
// stop when they reach past it.  Boxes outside the slice are either skipped
// (upper side) or never reached: a box left of / above the slice is at least
// the border distance away, which is never below the K-th distance.
#pragma once
#include <stdint.h>
#include <math.h>

#if defined(__CUDACC__)
#define GS_HD __host__ __device__ __forceinline__
#else
#define GS_HD inline
#endif

namespace odt {
namespace gs {

constexpr int kRowLen = 6;
constexpr int kColIdx = 0, kColVal = 1, kColBox = 2, kColX = 3, kColY = 4, kColZ = 5;
constexpr unsigned char kBalanced = 1, kActive = 2;

struct TableView {
  const int32_t* rows;     // [6, R]
  const int32_t* lookup;   // [lookup_len]
  const int32_t* zstart;   // [nz]
  const int32_t* square;   // [nz]
  int R, lookup_len, M1, M2;
};

GS_HD int gs_min(int a, int b) { return a < b ? a : b; }
GS_HD int gs_max(int a, int b) { return a > b ? a : b; }
GS_HD int gs_abs(int a) { return a < 0 ? -a : a; }

// ceil(size / ss) in single precision, as create_sort_value_cuda.cu:76-77.
GS_HD int box_side(int size, int ss) { return (int)ceilf((float)size / (float)ss); }

// Insertion point of distance x in the sorted (id, distance) pairs cur[0..K):
// a bisection that stops early on an equal distance
// (binarySearch_array_2_size, search_universal.cpp:1-27).
GS_HD int insertion_point(const int* cur, int x, int low, int high) {
  int mid = 0;
  while (low < high) {
    mid = (high + low) / 2;
    const int v = cur[2 * mid + 1];
    if (v == x) break;
    if (v > x) high = mid - 1;
    else low = mid + 1;
  }
  mid = (high + low) / 2;
  return x <= cur[2 * mid + 1] ? mid : mid + 1;
}

// Offer every residue of box (b1, b2) to the K-nearest list
// (search_in_case, search_universal.cpp:28-100).
template <int K>
GS_HD void scan_box(const TableView& T, const unsigned char* states, int* cur, int ss, int b1, int b2,
                    int start, int xc, int yc, int self) {
  if (b1 >= ss || b2 >= ss) return;
  const int box = start + b1 + b2 * ss;
  if (box < 0) return;  // unreachable (see the file comment); keeps reads in range
  const int first = T.lookup[box];
  if (first == -1) return;
  int last = T.R;
  for (int nxt = box + 1; nxt < T.lookup_len; ++nxt) {  // next non-empty box starts the next run
    const int v = T.lookup[nxt];
    if (v >= 0) {
      last = v;
      break;
    }
  }
  for (int i = first; i < last; ++i) {
    if (states && (states[i] & kActive)) continue;
    const int dx = gs_abs(xc - T.rows[kColX + kRowLen * i]);
    const int dy = gs_abs(yc - T.rows[kColY + kRowLen * i]);
    const int d = (int)sqrtf((float)(dx * dx + dy * dy));
    if (d < cur[2 * K - 1] && i != self) {
      const int at = insertion_point(cur, d, 0, K - 1);
      if (at < K) {
        for (int k = K - 1; k > at; --k) {
          cur[2 * k] = cur[2 * k - 2];
          cur[2 * k + 1] = cur[2 * k - 1];
        }
        cur[2 * at] = i;
        cur[2 * at + 1] = d;
      }
    }
  }
}

// The K nearest residues of row `self`: cur[2k] = row id (or -1), cur[2k+1] =
// distance (the border distance where no residue was found)
// (shortest_compute_kernel, search_universal.cpp:102-271).
template <int K>
GS_HD void nearest(const TableView& T, int self, const unsigned char* states, int* cur) {
  const int* r = T.rows + kRowLen * self;
  const int box = r[kColBox], xc = r[kColX], yc = r[kColY], z = r[kColZ];
  const int start = T.zstart[z];
  const int ss = T.square[z];
  const int s1 = box_side(T.M1, ss), s2 = box_side(T.M2, ss);
  const int c1 = box % ss, c2 = box / ss;
  const int rings = gs_max(gs_max(ss - c1, ss - c2), gs_max(c1, c2));
  const int cap = gs_min(gs_min(xc, yc), gs_min(T.M1 - xc, T.M2 - yc));
  for (int k = 0; k < K; ++k) {
    cur[2 * k] = -1;
    cur[2 * k + 1] = cap;
  }
  int reach = cap;
  for (int d = 0; d < rings && d < ss; ++d) {
    if (d == 0) {
      scan_box<K>(T, states, cur, ss, c1, c2, start, xc, yc, self);
    } else {
      for (int ii = 1 - d; ii <= d; ++ii) {
        const int on = ii == 0 ? 0 : 1;  // the ring's middle box has no offset along the ring
        const int up = ii > 0 ? 1 : 0, dn = ii > 0 ? 0 : 1;
        // four sides of the ring: box coordinates and nearest-edge distance
        const int b1[4] = {c1 - d, c1 + ii, c1 - ii, c1 + d};
        const int b2[4] = {c2 - ii, c2 - d, c2 + d, c2 + ii};
        const int near[4] = {
            gs_max(gs_abs((b1[0] + 1) * s1 - xc), gs_abs(((b2[0] + up) * s2 - yc) * on)),
            gs_max(gs_abs(((b1[1] + dn) * s1 - xc) * on), gs_abs((b2[1] + 1) * s2 - yc)),
            gs_max(gs_abs(((b1[2] + up) * s1 - xc) * on), gs_abs(b2[2] * s2 - yc)),
            gs_max(gs_abs(b1[3] * s1 - xc), gs_abs(((b2[3] + dn) * s2 - yc) * on))};
        const int lim = reach;  // all four sides are tested against the same bound
        for (int e = 0; e < 4; ++e)
          if (near[e] < lim) scan_box<K>(T, states, cur, ss, b1[e], b2[e], start, xc, yc, self);
        reach = cur[2 * K - 1];
      }
    }
    reach = cur[2 * K - 1];
    if (d * s1 >= reach && d * s2 >= reach) break;
  }
}

}  // namespace gs
}  // namespace odt
