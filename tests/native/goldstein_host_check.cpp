// CPU harness for the host stages of the library's Goldstein unwrapper:
// compiled as plain C++ together with inverse_solver_b200/csrc/goldstein_link.cpp
// into a shared library that the tests call through ctypes.  Exposes the
// residue-table builder, the nearest-residue search (the same function the
// GPU kernel runs, here on the host) and the multi-threaded branch linker.
#include <algorithm>
#include <cstring>
#include <vector>

#include "goldstein.h"
#include "goldstein_search.cuh"

using namespace odt::gs;

static Table g_table;

extern "C" {

// Builds the table; returns the lookup length.  rows [6*R], square/zstart [nz].
int gs_table(const int32_t* idx, const int32_t* val, long long R, int M1, int M2, int nz, int32_t* rows,
             int32_t* square, int32_t* zstart) {
  build_table(idx, val, R, M1, M2, nz, &g_table);
  std::memcpy(rows, g_table.rows.data(), g_table.rows.size() * 4);
  std::memcpy(square, g_table.square.data(), nz * 4);
  std::memcpy(zstart, g_table.zstart.data(), nz * 4);
  return (int)g_table.lookup.size();
}

void gs_lookup(int32_t* lookup) { std::memcpy(lookup, g_table.lookup.data(), g_table.lookup.size() * 4); }

// The 8 nearest residues of every row of the last table: [R][8][2].
void gs_nearest(int32_t* out) {
  const TableView T = view_of(g_table);
  for (int i = 0; i < T.R; ++i) nearest<8>(T, i, nullptr, out + 16 * (long long)i);
}

// Links the last table with the given [R][8][2] lists; returns the count.
long long gs_link(const int32_t* near, int threads, int32_t* out, long long cap) {
  std::vector<Branch> br;
  link_branches(g_table, near, 8, threads, &br);
  for (long long i = 0; i < (long long)br.size() && i < cap; ++i) {
    const Branch& b = br[i];
    const int32_t v[6] = {b.x1, b.y1, b.x2, b.y2, b.z, b.jump};
    std::memcpy(out + 6 * i, v, sizeof(v));
  }
  return (long long)br.size();
}

}  // extern "C"
