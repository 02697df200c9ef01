// phmg_setup.cpp -- host-side set-up of the ph-multigrid preconditioner's
// tree-AMG coarse solver: the aggregate hierarchy (tamg_mg_init,
// src/multigrid/tree_amg_multigrid.f90:111-228, with the greedy aggregation
// of src/multigrid/tree_amg_aggregate.f90) and the seeded start vectors.
//
// The aggregation keeps the reference's steps (first pass over a shuffled
// node order, second pass to the smallest neighbouring aggregate, adjacency
// of the aggregates in first-seen order for the next level), because the
// aggregates decide the coarse operator.  The shuffle and the power
// iteration's start vectors draw from splitmix64 seeded with 3901 where the
// reference draws from gfortran's random_number after random_seed(put =
// 3901), a compiler-runtime stream that has no portable restatement.
#include <cstdint>

#include "nb_phmg.h"

namespace nb {

namespace {

// splitmix64 (Steele, Lea and Flood, OOPSLA 2014); doubles from the top 53
// bits.
struct SplitMix64 {
  uint64_t s;
  explicit SplitMix64(uint64_t seed) : s(seed) {}
  double uniform() {
    s += 0x9E3779B97F4A7C15ull;
    uint64_t z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  }
};
constexpr uint64_t kSeed = 3901;

// Adjacency of one level's nodes: `width` slots per node, 0-based neighbour
// ids, -1 for none.
struct Adjacency {
  int width = 0;
  std::vector<int> nb;
  int at(int node, int side) const { return nb[(size_t)node * width + side]; }
};

// Greedy aggregation of `count` nodes into at least target aggregates
// (agg_greedy_first_pass / _second_pass / agg_fill_nhbr_info,
// tree_amg_aggregate.f90:113-357).  agg[i] = aggregate of node i.
bool greedy(int count, int target, const Adjacency &A, std::vector<int> &agg, int &naggs,
            Adjacency &next, std::string &err) {
  agg.assign(count, -1);
  std::vector<int> size(target > 0 ? target : 0, 0);
  int cap = target;
  naggs = 0;
  auto exists = [&](int v) { return v >= 0 && v < count; };
  // first pass: shuffled order (Fisher-Yates, from the last position down)
  std::vector<int> order(count);
  for (int i = 0; i < count; i++) order[i] = i;
  SplitMix64 g(kSeed);
  for (int i = count; i >= 2; i--) {
    const int j = (int)(g.uniform() * (double)i);
    std::swap(order[i - 1], order[j]);
  }
  for (int t = 0; t < count; t++) {
    const int i = order[t];
    if (agg[i] != -1) continue;
    bool free_nbhd = true;
    for (int s = 0; s < A.width; s++) {
      const int v = A.at(i, s);
      if (exists(v) && agg[v] != -1) free_nbhd = false;
    }
    if (!free_nbhd) continue;
    const int a = naggs++;
    if (cap < naggs) {
      cap = naggs + 20;
      size.resize(cap, 0);
    }
    agg[i] = a;
    size[a] = 1;
    for (int s = 0; s < A.width; s++) {
      const int v = A.at(i, s);
      if (exists(v) && agg[v] == -1) {
        agg[v] = a;
        size[a]++;
      }
    }
  }
  // second pass: every node left joins its smallest neighbouring aggregate
  // (the first of equal size in side order), else starts one
  for (int i = 0; i < count; i++) {
    if (agg[i] != -1) continue;
    int best = -1, best_size = 0x7fffffff;
    for (int s = 0; s < A.width; s++) {
      const int v = A.at(i, s);
      if (exists(v) && agg[v] != -1 && size[agg[v]] < best_size) {
        best_size = size[agg[v]];
        best = agg[v];
      }
    }
    if (best != -1) {
      agg[i] = best;
      size[best]++;
      continue;
    }
    const int a = naggs++;
    if (naggs > cap) {
      err = "phmg: the coarse-grid aggregation made more aggregates than it has room for";
      return false;
    }
    agg[i] = a;
    size[a] = 1;
    for (int s = 0; s < A.width; s++) {
      const int v = A.at(i, s);
      if (exists(v) && agg[v] == -1) {
        size[a]++;
        agg[v] = a;
      }
    }
  }
  // adjacency of the aggregates: width = the most cross-aggregate faces of
  // one aggregate, distinct neighbours in first-seen order
  std::vector<int> cross(naggs, 0);
  next.width = 0;
  for (int i = 0; i < count; i++) {
    for (int s = 0; s < A.width; s++) {
      const int v = A.at(i, s);
      if (exists(v) && agg[v] != agg[i]) cross[agg[i]]++;
    }
    if (cross[agg[i]] > next.width) next.width = cross[agg[i]];
  }
  next.nb.assign((size_t)next.width * naggs, -1);
  for (int i = 0; i < count; i++)
    for (int s = 0; s < A.width; s++) {
      const int v = A.at(i, s);
      if (!exists(v) || agg[v] == agg[i]) continue;
      int *row = &next.nb[(size_t)agg[i] * next.width];
      for (int k = 0; k < next.width; k++) {
        if (row[k] == agg[v]) break;
        if (row[k] == -1) {
          row[k] = agg[v];
          break;
        }
      }
    }
  return true;
}

// CSR of a node map: node -> its entries, ascending.
void invert(const std::vector<int> &node_of, int nnodes, std::vector<int> &ptr,
            std::vector<int> &idx) {
  ptr.assign(nnodes + 1, 0);
  for (int c : node_of) ptr[c + 1]++;
  for (int c = 0; c < nnodes; c++) ptr[c + 1] += ptr[c];
  idx.assign(node_of.size(), 0);
  std::vector<int> fill(nnodes, 0);
  for (size_t i = 0; i < node_of.size(); i++) {
    const int c = node_of[i];
    idx[ptr[c] + fill[c]++] = (int)i;
  }
}

}  // namespace

void phmg_start_vector(long n, std::vector<double> &d) {
  d.resize(n);
  SplitMix64 g(kSeed);
  for (long i = 0; i < n; i++) d[i] = g.uniform() + 10.0;
}

bool tamg_build(long nelv, int lx, const std::vector<int> &fn, int crs_lvls, TamgHost &H,
                std::string &err) {
  if (crs_lvls < 2) {
    err = "phmg: the coarse grid needs at least two AMG levels";
    return false;
  }
  const int l3 = lx * lx * lx;
  const long n0 = nelv * l3;
  H.nlvls = crs_lvls;
  H.lvl.assign(crs_lvls, TamgLevelHost());
  // level 1: one node per element
  {
    TamgLevelHost &L = H.lvl[1];
    L.nnodes = (int)nelv;
    L.nbelow = (int)n0;
    L.node_of.resize(n0);
    for (long i = 0; i < n0; i++) L.node_of[i] = (int)(i / l3);
  }
  Adjacency A;
  A.width = 6;
  A.nb.resize(6 * (size_t)nelv);
  for (size_t i = 0; i < A.nb.size(); i++) A.nb[i] = fn[i] - 1;
  for (int ml = 2; ml <= crs_lvls - 1; ml++) {
    const int target = H.lvl[ml - 1].nnodes / 8;
    if (target < 4) {  // too few nodes left for another level
      H.nlvls = ml;
      H.lvl.resize(ml);
      break;
    }
    TamgLevelHost &L = H.lvl[ml];
    Adjacency next;
    int naggs = 0;
    if (!greedy(H.lvl[ml - 1].nnodes, target, A, L.node_of, naggs, next, err)) return false;
    L.nnodes = naggs;
    L.nbelow = H.lvl[ml - 1].nnodes;
    A = std::move(next);
  }
  for (int l = 1; l < H.nlvls; l++) {
    TamgLevelHost &L = H.lvl[l];
    invert(L.node_of, L.nnodes, L.ptr, L.idx);
    L.finest.resize(n0);
    for (long i = 0; i < n0; i++)
      L.finest[i] = l == 1 ? L.node_of[i] : L.node_of[H.lvl[l - 1].finest[i]];
    invert(L.finest, L.nnodes, L.fptr, L.fidx);
  }
  return true;
}

}  // namespace nb
