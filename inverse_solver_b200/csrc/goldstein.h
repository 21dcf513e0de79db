// Host-side data of the Goldstein branch-cut unwrapper (see goldstein.cu).
#pragma once
#include <stdint.h>

#include <vector>

namespace odt {
namespace gs {

struct TableView;

// Residue table sorted by (slice, box), in the reference's row layout.
struct Table {
  int M1 = 0, M2 = 0, nz = 0;           // residue-map size (phase size - 1) and slices
  std::vector<int32_t> rows;            // [6, R]: index, value, box, x, y, z
  std::vector<int32_t> square;          // [nz] boxes per side
  std::vector<int32_t> zstart;          // [nz] first lookup entry of each slice
  std::vector<int32_t> lookup;          // first row of each box, -1 if empty
  std::vector<int64_t> slice_begin;     // [nz + 1] row range of each slice
};

// A branch cut between two residues (x1 = y1 = -1: to the nearest border),
// with the charge that crosses it (branche_coordinates, struct_v2.hpp:8-15).
struct Branch {
  int32_t x1, y1, x2, y2, z, jump;
};

// idx/val: the non-zero residues in column-major index order.
void build_table(const int32_t* idx, const int32_t* val, int64_t R, int M1, int M2, int nz, Table* t);
TableView view_of(const Table& t);
// nearest: [2, K, R] (row id, distance) pairs of the K nearest residues.
void link_branches(const Table& t, const int32_t* nearest, int K, int threads, std::vector<Branch>* out);

}  // namespace gs
}  // namespace odt
