// Host stages of the Goldstein branch-cut unwrapper:
//   * the residue table (goldstein_branch_cut.m:10-33): per-slice counts
//     (histcounts), box grid size ss = int32(ceil(sqrt((count + 1) / 16))),
//     box ids (create_sort_value_cuda.cu:52-86), the stable sort by
//     (slice, box) (sortrows(..., [6, 3])) and the box lookup table
//     (get_lookup_mex.cpp:123-136, get_lookup_cuda.cu:60-88);
//   * the branch linker (get_branches_goldstein_compute_v2.cpp:12-203 with
//     get_branches_goldstein_update_v2.cpp:13-61), which grows a tree of
//     links from each unbalanced residue until its charge is cancelled by
//     other residues or by the border.
//
// The linker is sequential within a slice.  Slices are independent -- every
// neighbour list and every search stays inside the residue's own slice and
// the linker only changes the state of residues it links -- so slices run on
// a pool of host threads, and concatenating their branch lists in slice order
// gives exactly the list of the one-thread loop over all residues.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <thread>
#include <vector>

#include "goldstein.h"
#include "goldstein_search.cuh"

namespace odt {
namespace gs {

void build_table(const int32_t* idx, const int32_t* val, int64_t R, int M1, int M2, int nz, Table* t) {
  t->M1 = M1;
  t->M2 = M2;
  t->nz = nz;
  const int64_t m12 = (int64_t)M1 * M2;
  std::vector<int64_t> count(nz, 0);
  for (int64_t i = 0; i < R; ++i) count[idx[i] / m12]++;
  t->square.assign(nz, 0);
  t->zstart.assign(nz, 0);
  t->slice_begin.assign(nz + 1, 0);
  int64_t total = 0;
  for (int z = 0; z < nz; ++z) {
    t->square[z] = (int32_t)std::ceil(std::sqrt(((double)count[z] + 1.0) / 16.0));
    t->zstart[z] = (int32_t)total;
    total += (int64_t)t->square[z] * t->square[z];
    t->slice_begin[z + 1] = t->slice_begin[z] + count[z];
  }
  t->lookup.assign(total, -1);
  t->rows.assign(kRowLen * R, 0);
  // Input rows are in index order, hence grouped by slice; a counting sort by
  // box id within each slice keeps index order inside a box (stable sort).
  std::vector<int32_t> box(R);
  for (int z = 0; z < nz; ++z) {
    const int ss = t->square[z];
    const int s1 = box_side(M1, ss), s2 = box_side(M2, ss);
    const int64_t b = t->slice_begin[z], e = t->slice_begin[z + 1];
    std::vector<int64_t> fill((size_t)ss * ss + 1, 0);
    for (int64_t i = b; i < e; ++i) {
      const int64_t d12 = idx[i] % m12;
      const int x = (int)(d12 % M1), y = (int)(d12 / M1);
      box[i] = x / s1 + (y / s2) * ss;
      fill[box[i] + 1]++;
    }
    for (size_t k = 1; k < fill.size(); ++k) fill[k] += fill[k - 1];
    for (int k = 0; k < ss * ss; ++k)
      if (fill[k + 1] > fill[k]) t->lookup[t->zstart[z] + k] = (int32_t)(b + fill[k]);
    for (int64_t i = b; i < e; ++i) {
      const int64_t row = b + fill[box[i]]++;
      const int64_t d12 = idx[i] % m12;
      int32_t* r = &t->rows[kRowLen * row];
      r[kColIdx] = idx[i];
      r[kColVal] = val[i];
      r[kColBox] = box[i];
      r[kColX] = (int32_t)(d12 % M1);
      r[kColY] = (int32_t)(d12 / M1);
      r[kColZ] = z;
    }
  }
}

TableView view_of(const Table& t) {
  TableView v;
  v.rows = t.rows.data();
  v.lookup = t.lookup.data();
  v.zstart = t.zstart.data();
  v.square = t.square.data();
  v.R = (int)(t.rows.size() / kRowLen);
  v.lookup_len = (int)t.lookup.size();
  v.M1 = t.M1;
  v.M2 = t.M2;
  return v;
}

namespace {

constexpr int kFar = 200000;

// One node of the link tree grown from an unbalanced residue.
struct Node {
  int row;        // residue row, -1 for the border
  int parent;     // node index of the residue it was linked from
  int branch;     // index of the branch that links it to its parent
  int dist;       // distance to its nearest unused candidate
  int slot;       // position of that candidate in the precomputed list (K = searched)
  int searched;   // candidate found by the search beyond the list
};

struct Linker {
  const TableView& T;
  const int32_t* nearest;  // [2, K, R]
  int K;
  unsigned char* state;
  std::vector<Branch>* out;

  int candidate(const Node& n) const {
    return n.slot < K ? nearest[2 * (int64_t)K * n.row + 2 * n.slot] : n.searched;
  }

  // Move n to its next candidate: the next list entry that is empty, not
  // active, or the last of the list; past the list, search the slice for the
  // nearest residue that is not active (update_min_distance).
  void advance(Node& n) const {
    for (int s = n.slot + 1;; ++s) {
      if (s < K) {
        const int32_t* e = nearest + 2 * (int64_t)K * n.row + 2 * s;
        if (e[0] == -1 || s == K - 1 || !(state[e[0]] & kActive)) {
          n.slot = s;
          n.dist = e[1];
          return;
        }
      } else {
        n.slot = K;
        int cur[2];
        odt::gs::nearest<1>(T, n.row, state, cur);
        n.searched = cur[0];
        n.dist = cur[1];
        return;
      }
    }
  }

  void balance(int seed) {
    std::vector<Node> tree;
    tree.push_back(Node{seed, 0, 0, 0, 0, 0});
    state[seed] |= kActive;
    int charge = T.rows[kRowLen * seed + kColVal];
    int next_dist = 0;
    while (charge != 0) {
      int cur_dist = next_dist;
      next_dist = kFar;
      for (size_t a = 0; a < tree.size(); ++a) {
        if (tree[a].dist == cur_dist) {
          const int c = candidate(tree[a]);
          if (c == -1 || !(state[c] & kActive)) {
            const int before = charge;
            if (c != -1 && !(state[c] & kBalanced)) charge += T.rows[kRowLen * c + kColVal];
            if (c == -1) charge = 0;
            tree.push_back(Node{c, (int)a, (int)out->size(), 0, -1, 0});
            if (c != -1) state[c] |= kActive;
            const int32_t* src = T.rows + kRowLen * tree[a].row;
            Branch br;
            br.x1 = c != -1 ? T.rows[kRowLen * c + kColX] : -1;
            br.y1 = c != -1 ? T.rows[kRowLen * c + kColY] : -1;
            br.x2 = src[kColX];
            br.y2 = src[kColY];
            br.z = src[kColZ];
            br.jump = 0;
            out->push_back(br);
            if (c == -1 || !(state[c] & kBalanced)) {
              // the charge that now flows through every branch up to the seed
              const int jump = c != -1 ? T.rows[kRowLen * c + kColVal] : -before;
              for (int p = (int)tree.size() - 1; p != 0; p = tree[p].parent) (*out)[tree[p].branch].jump += jump;
            }
            advance(tree[a]);
            if (c != -1) advance(tree.back());
            // The reference lowers both bounds with the new node's distance
            // as it was when created (0), so the next pass re-runs at 0.
            if (0 < cur_dist) cur_dist = 0;
            if (0 < next_dist) next_dist = 0;
          } else {
            advance(tree[a]);
          }
        }
        if (tree[a].dist < next_dist) next_dist = tree[a].dist;
        if (charge == 0) break;
      }
    }
    for (const Node& n : tree)
      if (n.row != -1) state[n.row] = (unsigned char)((state[n.row] & ~kActive) | kBalanced);
  }
};

}  // namespace

void link_branches(const Table& t, const int32_t* nearest, int K, int threads, std::vector<Branch>* out) {
  const TableView T = view_of(t);
  std::vector<unsigned char> state(T.R, 0);
  std::vector<std::vector<Branch>> per(t.nz);
  std::atomic<int> next{0};
  auto work = [&]() {
    for (int z = next.fetch_add(1); z < t.nz; z = next.fetch_add(1)) {
      Linker L{T, nearest, K, state.data(), &per[z]};
      for (int64_t i = t.slice_begin[z]; i < t.slice_begin[z + 1]; ++i)
        if (!(state[i] & kBalanced)) L.balance((int)i);
    }
  };
  int nt = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
  nt = std::max(1, std::min(nt, t.nz));
  if (nt == 1) {
    work();
  } else {
    std::vector<std::thread> pool;
    for (int i = 0; i < nt; ++i) pool.emplace_back(work);
    for (auto& th : pool) th.join();
  }
  out->clear();
  for (auto& p : per) out->insert(out->end(), p.begin(), p.end());
}

}  // namespace gs
}  // namespace odt
