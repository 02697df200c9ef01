// nb_hsmg.h -- host-side data of the hybrid Schwarz multigrid preconditioner.
#pragma once

#include <vector>

#include "nb_internal.h"

namespace nb {

// FDM factors of one level: per element and direction the B-orthonormal
// eigenvectors S (nl x nl, col-major) and eigenvalues, and the per-element
// eps below which an eigenvalue sum is treated as zero.
struct FdmHost {
  int lx = 0, nl = 0;
  long nelv = 0;
  std::vector<double> S;    // (nl*nl, 3, nelv)
  std::vector<double> lam;  // (nl, 3, nelv)
  std::vector<double> eps;  // (nelv)
};

void fdm_build(int lx, long nelv, const std::vector<double> &x, const std::vector<double> &y,
               const std::vector<double> &z, const std::vector<int> &facet_type,
               const GsMaps &maps, FdmHost &F);
void schwarz_weights(int lx, long nelv, const std::vector<int> &facet_neigh, const GsMaps &maps,
                     std::vector<double> &wt);
void lagrange_matrix(const std::vector<double> &z_to, const std::vector<double> &z_from,
                     std::vector<double> &J);

}  // namespace nb
