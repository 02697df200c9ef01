// nmsh.cpp -- Neko's binary mesh format (.nmsh) for the unstructured-mesh
// problems: reader and writer of 3-D hexahedral meshes.
//
// Layout (nmsh_file_read / nmsh_file_write, src/io/nmsh_file.f90:70-207 and
// 650-760, records of src/io/format/nmsh.f90 written packed by MPI-IO with
// the types of src/comm/mpi_types.f90:120-200), native byte order:
//   int32 nelv, int32 gdim (3)
//   nelv x { int32 el_idx; 8 x { int32 v_idx; float64 x, y, z } }   228 B
//   int32 nzones, nzones x { int32 e, f, p_e, p_f, glb_pt_ids[4], type }
//   int32 ncurves, ncurves x curve records (not used here)
// The vertices of a record are in the file's cyclic order; the symmetric
// order of the hex is (1, 2, 4, 3, 5, 6, 8, 7) of it.  Zone type 5 is a
// periodic face: its four vertices take glb_pt_ids in face-node order, and
// as in mesh_apply_periodic_facet (src/mesh/mesh.f90:1837-1866) the change
// follows the point (every element holding that original vertex id sees the
// new id), later zones overriding earlier ones.  Zone type 7 (a labeled
// boundary face) carries no id change and is reported as a count only.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "nb_internal.h"

using namespace nb;

namespace {

const int kFaceNodesSym[6][4] = {{1, 5, 7, 3}, {2, 6, 8, 4}, {1, 2, 6, 5},
                                 {3, 4, 8, 7}, {1, 2, 4, 3}, {5, 6, 8, 7}};
const int kCycToSym[8] = {0, 1, 3, 2, 4, 5, 7, 6};  // file vertex j is symmetric vertex kCycToSym[j]

struct FileCloser {
  FILE *f;
  ~FileCloser() {
    if (f) fclose(f);
  }
};

nb_status err(nb_status s, const std::string &m) {
  set_error(m);
  return s;
}

bool rd(FILE *f, void *p, size_t bytes) { return fread(p, 1, bytes, f) == bytes; }
bool wr(FILE *f, const void *p, size_t bytes) { return fwrite(p, 1, bytes, f) == bytes; }

}  // namespace

extern "C" nb_status nb_mesh_read_nmsh(const char *path, int *nelv, int *vertex_ids,
                                       double *vertex_xyz, int *nperiodic, int *nlabeled) {
  if (!path || !nelv) return err(NB_ERR_ARG, "nb_mesh_read_nmsh: null argument");
  FileCloser fc{fopen(path, "rb")};
  if (!fc.f) return err(NB_ERR_ARG, std::string("nb_mesh_read_nmsh: cannot open ") + path);
  int32_t hdr[2];
  if (!rd(fc.f, hdr, sizeof(hdr))) return err(NB_ERR_ARG, "nb_mesh_read_nmsh: short header");
  if (hdr[1] != 3) return err(NB_ERR_UNSUPPORTED, "nb_mesh_read_nmsh: only 3-D meshes (gdim 3)");
  if (hdr[0] < 1) return err(NB_ERR_ARG, "nb_mesh_read_nmsh: no elements");
  const int ne = hdr[0];
  *nelv = ne;
  if (!vertex_ids && !vertex_xyz && !nperiodic && !nlabeled) return NB_OK;  // size query
  std::vector<int> ids((size_t)ne * 8);
  std::vector<double> xyz((size_t)ne * 24);
  std::unordered_map<int, int> elmap;  // global element id -> index
  for (int e = 0; e < ne; e++) {
    unsigned char rec[228];
    if (!rd(fc.f, rec, sizeof(rec))) return err(NB_ERR_ARG, "nb_mesh_read_nmsh: short element data");
    int32_t el_idx;
    memcpy(&el_idx, rec, 4);
    elmap[el_idx] = e;
    for (int j = 0; j < 8; j++) {
      const unsigned char *v = rec + 4 + 28 * j;
      const int s = kCycToSym[j];
      int32_t id;
      memcpy(&id, v, 4);
      ids[(size_t)e * 8 + s] = id;
      memcpy(&xyz[((size_t)e * 8 + s) * 3], v + 4, 24);
    }
  }
  int32_t nz = 0;
  if (!rd(fc.f, &nz, 4)) nz = 0;  // a file that ends after the elements has no zones
  // periodic faces: the id of each original vertex (the point) as changed by
  // the zones in order
  std::unordered_map<int, int> point_id;
  int np = 0, nl = 0;
  for (int z = 0; z < nz; z++) {
    int32_t r[9];
    if (!rd(fc.f, r, sizeof(r))) return err(NB_ERR_ARG, "nb_mesh_read_nmsh: short zone data");
    const int ze = r[0], zf = r[1], type = r[8];
    if (type == 7) {
      nl++;
      continue;
    }
    if (type != 5) continue;
    auto it = elmap.find(ze);
    if (it == elmap.end()) return err(NB_ERR_ARG, "nb_mesh_read_nmsh: zone of an unknown element");
    if (zf < 1 || zf > 6) return err(NB_ERR_ARG, "nb_mesh_read_nmsh: zone facet out of range");
    np++;
    const int e = it->second;
    for (int i = 0; i < 4; i++) {
      const int orig = ids[(size_t)e * 8 + kFaceNodesSym[zf - 1][i] - 1];
      point_id[orig] = r[4 + i];
    }
  }
  if (!point_id.empty())
    for (int &id : ids) {
      auto it = point_id.find(id);
      if (it != point_id.end()) id = it->second;
    }
  if (vertex_ids) memcpy(vertex_ids, ids.data(), ids.size() * sizeof(int));
  if (vertex_xyz) memcpy(vertex_xyz, xyz.data(), xyz.size() * sizeof(double));
  if (nperiodic) *nperiodic = np;
  if (nlabeled) *nlabeled = nl;
  return NB_OK;
}

extern "C" nb_status nb_mesh_write_nmsh(const char *path, int nelv, const int *vertex_ids,
                                        const double *vertex_xyz) {
  if (!path || !vertex_ids || !vertex_xyz || nelv < 1)
    return err(NB_ERR_ARG, "nb_mesh_write_nmsh: null argument or no element");
  FileCloser fc{fopen(path, "wb")};
  if (!fc.f) return err(NB_ERR_ARG, std::string("nb_mesh_write_nmsh: cannot create ") + path);
  const int32_t hdr[2] = {nelv, 3};
  if (!wr(fc.f, hdr, sizeof(hdr))) return err(NB_ERR_ARG, "nb_mesh_write_nmsh: write failed");
  for (int e = 0; e < nelv; e++) {
    unsigned char rec[228];
    const int32_t el_idx = e + 1;
    memcpy(rec, &el_idx, 4);
    for (int j = 0; j < 8; j++) {
      unsigned char *v = rec + 4 + 28 * j;
      const int s = kCycToSym[j];
      const int32_t id = vertex_ids[(size_t)e * 8 + s];
      memcpy(v, &id, 4);
      memcpy(v + 4, &vertex_xyz[((size_t)e * 8 + s) * 3], 24);
    }
    if (!wr(fc.f, rec, sizeof(rec))) return err(NB_ERR_ARG, "nb_mesh_write_nmsh: write failed");
  }
  const int32_t zero[2] = {0, 0};  // no zones, no curves
  if (!wr(fc.f, zero, sizeof(zero))) return err(NB_ERR_ARG, "nb_mesh_write_nmsh: write failed");
  return NB_OK;
}
