// nb_phmg.h -- host-side set-up of the ph-multigrid preconditioner: the
// aggregation hierarchy of its tree-AMG coarse solver and the seeded start
// vectors of its eigenvalue estimates.
#pragma once

#include <string>
#include <vector>

namespace nb {

// Settings of phmg_init (phmg.f90:141-180 defaults).
struct PhmgSettings {
  int smoother_iterations = 3;      // Chebyshev steps a level
  std::vector<int> schedule{3, 1};  // polynomial degree of each coarser level
  int coarse_levels = 3;            // tree-AMG levels
  int coarse_iterations = 1;        // AMG V-cycles an application
  int cheby_degree = 4;             // Chebyshev degree on the AMG levels
};

// One aggregate level of the tree AMG.  Level 1 groups the lx^3 points of
// each element, level 2 and above group the nodes of the level below
// greedily (tree_amg_aggregate.f90).  All indices 0-based.
struct TamgLevelHost {
  int nnodes = 0;               // aggregates ("nodes") on this level
  int nbelow = 0;               // entries of the level below
  std::vector<int> node_of;     // entry below -> node
  std::vector<int> ptr, idx;    // node -> its entries below, ascending (CSR)
  std::vector<int> finest;      // level-0 point -> node
  std::vector<int> fptr, fidx;  // node -> its level-0 points, ascending (CSR)
};

struct TamgHost {
  int nlvls = 0;                    // cycle levels 0 .. nlvls-1
  std::vector<TamgLevelHost> lvl;   // [1 .. nlvls-1]; [0] unused
};

// Builds the aggregation for a mesh of nelv elements with lx^3 points each
// and face neighbours fn (6 per element, 1-based, 0 = none), asking for
// crs_lvls levels.  Returns false with a message where the reference stops
// with an error.
bool tamg_build(long nelv, int lx, const std::vector<int> &fn, int crs_lvls, TamgHost &H,
                std::string &err);

// n values u + 10 with u uniform in [0, 1) from splitmix64 seeded 3901: the
// start vector of every power iteration (and the stream behind the
// aggregation's element order), restarted on each call.
void phmg_start_vector(long n, std::vector<double> &d);

}  // namespace nb
