// nb_internal.h -- shared declarations of the neko_b200 native library.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/neko_b200.h"

namespace nb {

// Last error message of the calling thread (nb_last_error()).
void set_error(const std::string &msg);

#define NB_CUDA_TRY(expr)                                                   \
  do {                                                                      \
    cudaError_t _e = (expr);                                                \
    if (_e != cudaSuccess) {                                                \
      ::nb::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e)); \
      return NB_ERR_CUDA;                                                   \
    }                                                                       \
  } while (0)

// Streaming multiprocessors of the current device (queried once per device).
int device_sms();

// Capacity, in blocks, of every partial-sum buffer of a grid reduction.
constexpr int kMaxRedBlocks = 2048;

// Reference-style fatal check for the drop-in cuda_* symbols, which return
// no status (the reference's CUDA_CHECK prints and exits).
void cuda_check_fatal(cudaError_t e, const char *what);

// ---------------------------------------------------------------------------
// Host-side setup (setup.cpp)
// ---------------------------------------------------------------------------

// GLL nodes, weights and derivative matrix (column-major D(i,j), Dt = D^T).
void gll_space(int lx, std::vector<double> &z, std::vector<double> &w,
               std::vector<double> &D, std::vector<double> &Dt);

// Element-local gather-scatter maps in the reference layout (1-based):
// dof_gs = gather-scatter id per entry, gs_dof = local dof per entry, blocks
// over the vertex/edge part, facet pairs after facet_offset.
struct GsMaps {
  int nlocal = 0;
  int facet_offset = 0;  // 1-based index of the first facet entry
  std::vector<int> dof_gs, gs_dof, blk_len, blk_off;
};

// Structured box of nel[0] x nel[1] x nel[2] hexahedra, elements ordered
// x fastest, optional periodicity per direction.
struct BoxSpec {
  int nel[3];
  double lo[3], hi[3];
  int periodic[3];
};

// Vertex coordinates of every element (8 per element, symmetric order).
void box_vertices(const BoxSpec &b, std::vector<double> &xyz8);
// facet_neigh (6 per element, 1-based neighbour id, 0 on the boundary).
void box_facet_neigh(const BoxSpec &b, std::vector<int> &fn);
// Gather-scatter maps of the box at polynomial size lx.
int box_gs_maps(const BoxSpec &b, int lx, const std::vector<int> &facet_neigh, GsMaps &g);
// Connectivity of an unstructured hex mesh (8 positive global vertex ids per
// element, symmetric order): faces and edges numbered in first-appearance
// order, neighbour per face (1-based, 0 on the boundary).  Returns non-zero
// with a message for an invalid mesh.
struct MeshConn {
  std::vector<int> fn, face_gid, edge_gid;
  int nfaces = 0, nedges = 0, max_vid = 0;
};
int mesh_connectivity(long nelv, const int *ids, MeshConn &c, std::string &err);
// Gather-scatter maps of the mesh at polynomial size lx (reference layout).
int mesh_gs_maps(long nelv, const int *ids, const MeshConn &c, int lx, GsMaps &g);
// Zero-Dirichlet mask of the mesh's faces without a neighbour.
void mesh_boundary_mask(long nelv, int lx, const std::vector<int> &fn, std::vector<int> &msk);
// Every face neighbour meets the element through the opposite face with the
// same orientation (what the direct Schwarz ghost exchange needs).
bool mesh_faces_aligned(long nelv, const int *ids, const std::vector<int> &fn);

// Zero-Dirichlet mask (1-based, ascending) of all faces with facet_neigh == 0.
void box_boundary_mask(const BoxSpec &b, int lx, const std::vector<int> &facet_neigh,
                       std::vector<int> &msk);

}  // namespace nb
