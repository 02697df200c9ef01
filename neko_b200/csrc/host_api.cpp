// host_api.cpp -- host-only setup helpers of the C ABI (no device needed).
#include <cstring>
#include <string>

#include "nb_internal.h"

using namespace nb;

extern "C" nb_status nb_gll(int lx, double *z, double *w, double *D) {
  if (lx < 2 || lx > 84 || !z || !w || !D) {
    set_error("nb_gll: lx must be in 2..84 and arrays non-null");
    return NB_ERR_ARG;
  }
  std::vector<double> zz, ww, dd, dt;
  gll_space(lx, zz, ww, dd, dt);
  std::memcpy(z, zz.data(), lx * sizeof(double));
  std::memcpy(w, ww.data(), lx * sizeof(double));
  std::memcpy(D, dd.data(), (size_t)lx * lx * sizeof(double));
  return NB_OK;
}

extern "C" nb_status nb_box_gs_maps(const int nel[3], const int periodic[3], int lx,
                                    int *nlocal, int *facet_offset, int *nblocks, int *dof_gs,
                                    int *gs_dof, int *blk_len, int *blk_off) {
  if (!nel || !periodic || !nlocal || !facet_offset || !nblocks) {
    set_error("nb_box_gs_maps: null argument");
    return NB_ERR_ARG;
  }
  if (lx < 2 || lx > 16) {
    set_error("nb_box_gs_maps: lx must be in 2..16");
    return NB_ERR_UNSUPPORTED;
  }
  BoxSpec b{};
  for (int d = 0; d < 3; d++) {
    if (nel[d] < 1 || (periodic[d] && nel[d] < 3)) {
      set_error("nb_box_gs_maps: bad element count (periodic directions need >= 3)");
      return NB_ERR_UNSUPPORTED;
    }
    b.nel[d] = nel[d];
    b.periodic[d] = periodic[d] ? 1 : 0;
    b.lo[d] = 0.0;
    b.hi[d] = 1.0;
  }
  std::vector<int> fn;
  box_facet_neigh(b, fn);
  GsMaps g;
  box_gs_maps(b, lx, fn, g);
  *nlocal = g.nlocal;
  *facet_offset = g.facet_offset;
  *nblocks = (int)g.blk_len.size();
  if (dof_gs) std::memcpy(dof_gs, g.dof_gs.data(), g.dof_gs.size() * 4);
  if (gs_dof) std::memcpy(gs_dof, g.gs_dof.data(), g.gs_dof.size() * 4);
  if (blk_len) std::memcpy(blk_len, g.blk_len.data(), g.blk_len.size() * 4);
  if (blk_off) std::memcpy(blk_off, g.blk_off.data(), g.blk_off.size() * 4);
  return NB_OK;
}

extern "C" nb_status nb_mesh_gs_maps(int nelv, const int *vertex_ids, int lx, int *nlocal,
                                     int *facet_offset, int *nblocks, int *facet_neigh,
                                     int *dof_gs, int *gs_dof, int *blk_len, int *blk_off) {
  if (!vertex_ids || !nlocal || !facet_offset || !nblocks || nelv < 1) {
    set_error("nb_mesh_gs_maps: null argument or no element");
    return NB_ERR_ARG;
  }
  if (lx < 2 || lx > 16) {
    set_error("nb_mesh_gs_maps: lx must be in 2..16");
    return NB_ERR_UNSUPPORTED;
  }
  MeshConn c;
  std::string err;
  if (mesh_connectivity(nelv, vertex_ids, c, err)) {
    set_error("nb_mesh_gs_maps: " + err);
    return NB_ERR_ARG;
  }
  GsMaps g;
  mesh_gs_maps(nelv, vertex_ids, c, lx, g);
  *nlocal = g.nlocal;
  *facet_offset = g.facet_offset;
  *nblocks = (int)g.blk_len.size();
  if (facet_neigh) std::memcpy(facet_neigh, c.fn.data(), c.fn.size() * 4);
  if (dof_gs) std::memcpy(dof_gs, g.dof_gs.data(), g.dof_gs.size() * 4);
  if (gs_dof) std::memcpy(gs_dof, g.gs_dof.data(), g.gs_dof.size() * 4);
  if (blk_len) std::memcpy(blk_len, g.blk_len.data(), g.blk_len.size() * 4);
  if (blk_off) std::memcpy(blk_off, g.blk_off.data(), g.blk_off.size() * 4);
  return NB_OK;
}
