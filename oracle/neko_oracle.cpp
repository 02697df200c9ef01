// neko_oracle.cpp -- CPU restatement of Neko's pressure/Helmholtz solve path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker: it is linked and called
// by tests/, by __graft_entry__.smoke() and by bench.py's cpu_baseline leg,
// never by the neko_b200 product path.
//
// Every routine restates one routine of the reference (Neko, Fortran) and
// cites the file:line it follows.  Indices that are 1-based in the reference
// (gather-scatter maps, dof numbers, element ids) stay 1-based here so the
// arrays can be compared bit for bit with the product's.
//
// Parity pin: the reference cannot be compiled in this image (no Fortran
// compiler, no MPI).  The restatement is pinned by the reference's own
// known-answer tests for this path, re-expressed as fixtures under
// tests/golden/: the seven two-element gather-scatter face-orientation tests
// (tests/unit/gather_scatter/test_gather_scatter_parallel.pf:38-903), the GLL
// space tests (tests/unit/space) and the device-math glsc3 vectors
// (tests/unit/device_math/test_device_math_parallel.pf:614-647).

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <unordered_map>
#include <vector>

#include "neko_oracle.h"

namespace nko {

// ---------------------------------------------------------------------------
// Hex element topology (src/mesh/hex.f90:59-80).  Vertices are numbered in
// Neko's "symmetric" order: p1=(0,0,0) p2=(1,0,0) p3=(0,1,0) p4=(1,1,0),
// p5..p8 the same at z=1.
// ---------------------------------------------------------------------------
const int kFaceNodes[6][4] = {{1, 5, 7, 3}, {2, 6, 8, 4}, {1, 2, 6, 5},
                              {3, 4, 8, 7}, {1, 2, 4, 3}, {5, 6, 8, 7}};
const int kEdgeNodes[12][2] = {{1, 2}, {3, 4}, {5, 6}, {7, 8}, {1, 3}, {2, 4},
                               {5, 7}, {6, 8}, {1, 5}, {2, 6}, {3, 7}, {4, 8}};

struct Point {
  double x[3];
  int id;
};

using Face = std::array<int, 4>;
using Edge = std::array<int, 2>;

struct FaceHash {
  size_t operator()(const Face &f) const {
    uint64_t h = 1469598103934665603ull;
    for (int v : f) h = (h ^ (uint64_t)(uint32_t)v) * 1099511628211ull;
    return (size_t)h;
  }
};
struct EdgeHash {
  size_t operator()(const Edge &e) const {
    return (size_t)(((uint64_t)(uint32_t)e[0] << 32) | (uint32_t)e[1]) *
           0x9E3779B97F4A7C15ull;
  }
};

struct PeriodicZone {
  int f, e, pf, pe;
  int pids[4];
  int org_ids[4];
};

// mesh_t (src/mesh/mesh.f90:66-150), single rank (pe_size = 1).
struct Mesh {
  int nelv = 0;
  std::vector<Point> points;              // this%points(:) (slots)
  std::vector<std::array<int, 8>> el;     // element -> slot of each vertex
  std::vector<int> el_id;                 // element global id
  std::unordered_map<int, int> htp;       // point id -> slot
  int max_pts_id = 0;
  std::vector<PeriodicZone> periodic;
  std::vector<std::pair<int, int>> labeled[21];  // label -> (f, e)
  std::vector<int> facet_neigh;           // (6, nelv), 0 = boundary
  std::unordered_map<Face, int, FaceHash> htf;
  std::unordered_map<Edge, int, EdgeHash> hte;
  int mfcs = 0, meds = 0;
  std::vector<uint8_t> dfrmd_el;
  std::vector<int> facet_type;  // (6, nelv)

  int pid(int e, int v) const { return points[el[e][v - 1]].id; }
  const double *px(int e, int v) const { return points[el[e][v - 1]].x; }

  // mesh_add_point (mesh.f90:1566-1587)
  int add_point(const Point &p) {
    max_pts_id = std::max(max_pts_id, p.id);
    if (p.id <= 0) {
      fprintf(stderr, "oracle: invalid point id\n");
      abort();
    }
    auto it = htp.find(p.id);
    if (it != htp.end()) return it->second;
    points.push_back(p);
    int idx = (int)points.size() - 1;
    htp[p.id] = idx;
    return idx;
  }

  // mesh_add_hex (mesh.f90:1526-1563); vertices in symmetric order.
  void add_hex(int e, int glb, const Point p[8]) {
    for (int v = 0; v < 8; v++) el[e][v] = add_point(p[v]);
    el_id[e] = glb;
  }

  void init(int n) {
    nelv = n;
    el.assign(n, {});
    el_id.assign(n, 0);
    dfrmd_el.assign(n, 0);
    facet_type.assign(6 * (size_t)n, 0);
  }

  // hex_facet_id (hex.f90:109-137): sorted ids of the face's 4 vertices.
  Face facet_id(int e, int side) const {
    Face t;
    for (int i = 0; i < 4; i++) t[i] = pid(e, kFaceNodes[side - 1][i]);
    for (int i = 0; i < 3; i++)
      for (int j = i + 1; j < 4; j++)
        if (t[j] < t[i]) std::swap(t[i], t[j]);
    return t;
  }
  // hex_facet_order (hex.f90:140-157): ids in face_nodes order.
  Face facet_order(int e, int side) const {
    Face t;
    for (int i = 0; i < 4; i++) t[i] = pid(e, kFaceNodes[side - 1][i]);
    return t;
  }
  // hex_edge_id (hex.f90:161-180): (min id, max id).
  Edge edge_id(int e, int side) const {
    int a = pid(e, kEdgeNodes[side - 1][0]), b = pid(e, kEdgeNodes[side - 1][1]);
    return a < b ? Edge{a, b} : Edge{b, a};
  }

  // mesh_mark_periodic_facet (mesh.f90:1653-1664)
  void mark_periodic_facet(int f, int e, int pf, int pe, const int pids[4]) {
    PeriodicZone z;
    z.f = f;
    z.e = e;
    z.pf = pf;
    z.pe = pe;
    Face o = facet_order(e, f);
    for (int i = 0; i < 4; i++) {
      z.pids[i] = pids[i];
      z.org_ids[i] = o[i];
    }
    periodic.push_back(z);
  }
  // mesh_mark_labeled_facet (mesh.f90:1633-1650)
  void mark_labeled_facet(int f, int e, int label) {
    labeled[label].push_back({f, e});
    facet_type[(size_t)e * 6 + (f - 1)] = -label;
  }

  // mesh_create_periodic_ids (mesh.f90:1743-1833), tol = 1e-7.
  void create_periodic_ids(int f, int e, int pf, int pe) {
    const double tol = 1e-7;
    double L[3] = {0, 0, 0};
    for (int i = 0; i < 4; i++)
      for (int d = 0; d < 3; d++)
        L[d] += px(e, kFaceNodes[f - 1][i])[d] - px(pe, kFaceNodes[pf - 1][i])[d];
    for (int d = 0; d < 3; d++) L[d] /= 4;
    for (int i = 0; i < 4; i++) {
      Point &pi = points[el[e][kFaceNodes[f - 1][i] - 1]];
      int match = 0;
      for (int j = 0; j < 4; j++) {
        Point &pj = points[el[pe][kFaceNodes[pf - 1][j] - 1]];
        double s = 0;
        for (int d = 0; d < 3; d++) {
          double t = pi.x[d] - pj.x[d] - L[d];
          s += t * t;
        }
        if (std::sqrt(s) < tol) {
          int id = std::min(pi.id, pj.id);
          pi.id = id;
          pj.id = id;
          match++;
        }
      }
      if (match != 1) {
        fprintf(stderr, "oracle: periodic point match count %d\n", match);
        abort();
      }
    }
  }

  // mesh_reset_periodic_ids (mesh.f90:1690-1740)
  void reset_periodic_ids() {
    for (auto &z : periodic) {
      Face o = facet_order(z.e, z.f);
      for (int i = 0; i < 4; i++) z.pids[i] = o[i];
    }
    for (auto &z : periodic)
      for (int j = 0; j < 4; j++)
        points[el[z.e][kFaceNodes[z.f - 1][j] - 1]].id = z.org_ids[j];
  }

  // mesh_apply_periodic_facet (mesh.f90:1837-1866)
  void apply_periodic_facet(int f, int e, const int pids[4]) {
    for (int i = 0; i < 4; i++) {
      int slot = el[e][kFaceNodes[f - 1][i] - 1];
      points[slot].id = pids[i];
      Point copy = points[slot];
      add_point(copy);
    }
  }

  // mesh_generate_flags (mesh.f90:437-467)
  void generate_flags() {
    auto sub = [&](int e, int a, int b, double *o) {
      for (int d = 0; d < 3; d++) o[d] = px(e, a)[d] - px(e, b)[d];
    };
    auto dot = [](const double *a, const double *b) {
      return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
    };
    const double eps = 2.220446049250313e-16;
    for (int e = 0; e < nelv; e++) {
      double u[3], v[3], w[3];
      uint8_t f = 0;
      sub(e, 2, 1, u);
      sub(e, 3, 1, v);
      sub(e, 5, 1, w);
      if (!(std::fabs(dot(u, v)) < eps)) f = 1;
      if (!(std::fabs(dot(u, w)) < eps)) f = 1;
      sub(e, 7, 8, u);
      sub(e, 6, 8, v);
      sub(e, 4, 8, w);
      if (!(std::fabs(dot(u, v)) < eps)) f = 1;
      if (!(std::fabs(dot(u, w)) < eps)) f = 1;
      dfrmd_el[e] = f;
    }
  }

  // mesh_generate_conn (mesh.f90:476-687), hex branch, pe_size = 1.
  void generate_conn() {
    for (int e = 0; e < nelv; e++) {
      for (int i = 1; i <= 6; i++) {
        Face f = facet_id(e, i);
        if (!htf.count(f)) htf[f] = ++mfcs;  // mesh_add_face (1590-1600)
      }
      for (int i = 1; i <= 12; i++) {
        Edge ed = edge_id(e, i);
        if (!hte.count(ed)) hte[ed] = ++meds;  // mesh_add_edge (1603-1613)
      }
    }
    facet_neigh.assign(6 * (size_t)nelv, 0);
    std::unordered_map<Face, std::array<int, 2>, FaceHash> fmp;
    for (int k = 0; k < 2; k++) {
      for (int i = 0; i < nelv; i++) {
        int eg = i + 1;
        for (int j = 1; j <= 6; j++) {
          Face face = facet_id(i, j);
          int &neigh = facet_neigh[(size_t)i * 6 + (j - 1)];
          auto it = fmp.find(face);
          if (it != fmp.end()) {
            std::array<int, 2> fd = it->second;
            if (fd[0] == eg) {
              neigh = fd[1];
              Face comp = facet_id(i, j + (2 * (j % 2) - 1));
              if (comp == face) {
                fd[1] = eg;
                neigh = fd[0];
                it->second = fd;
              }
            } else if (fd[1] == eg) {
              neigh = fd[0];
            } else if (fd[0] > eg) {
              fd[1] = fd[0];
              fd[0] = eg;
              neigh = fd[1];
              it->second = fd;
            } else if (fd[0] < eg) {
              fd[1] = eg;
              neigh = fd[0];
              it->second = fd;
            }
          } else {
            fmp[face] = {eg, 0};
            neigh = 0;
          }
        }
      }
    }
  }

  // mesh_finalize (mesh.f90:419-435)
  void finalize() {
    generate_flags();
    generate_conn();
  }
};

// An nmsh-style element record: global id + 8 vertices in the file's
// cyclic order (src/io/nmsh_file.f90:652-720, vcyc_to_sym = [1,2,4,3,5,6,8,7]).
struct ElemRecord {
  int el_idx;
  Point v[8];
};
// nmsh zone record (src/io/format/nmsh.f90): type 5 periodic, 7 labeled.
struct ZoneRecord {
  int e, f, p_e, p_f, type;
  int glb_pt_ids[4];
};

// genmeshbox (contrib/genmeshbox/genmeshbox.f90:200-353) followed by
// nmsh_file_write (src/io/nmsh_file.f90:650-760): returns the records that
// the file would hold.
void genmeshbox(double x0, double x1, double y0, double y1, double z0, double z1,
                int nelx, int nely, int nelz, bool px, bool py, bool pz,
                std::vector<ElemRecord> &elems, std::vector<ZoneRecord> &zones) {
  Mesh m;
  int nel = nelx * nely * nelz;
  m.init(nel);
  std::vector<double> cx(nelx + 1), cy(nely + 1), cz(nelz + 1);
  double lxe = (x1 - x0) / nelx, lye = (y1 - y0) / nely, lze = (z1 - z0) / nelz;
  cx[0] = x0;
  for (int i = 0; i < nelx; i++) cx[i + 1] = cx[i] + lxe;
  cy[0] = y0;
  for (int i = 0; i < nely; i++) cy[i + 1] = cy[i] + lye;
  cz[0] = z0;
  for (int i = 0; i < nelz; i++) cz[i + 1] = cz[i] + lze;
  int i = 0;
  for (int ez = 0; ez < nelz; ez++)
    for (int ey = 0; ey < nely; ey++)
      for (int ex = 0; ex < nelx; ex++) {
        Point p[8];
        for (int iz = 0; iz < 2; iz++)
          for (int iy = 0; iy < 2; iy++)
            for (int ix = 0; ix < 2; ix++) {
              Point &q = p[ix + 2 * iy + 4 * iz];
              q.x[0] = cx[ex + ix];
              q.x[1] = cy[ey + iy];
              q.x[2] = cz[ez + iz];
              q.id = 1 + (ix + ex) + (iy + ey) * (nelx + 1) +
                     (iz + ez) * (nelx + 1) * (nely + 1);
            }
        m.add_hex(i, i + 1, p);
        i++;
      }
  const int dummy[4] = {0, 0, 0, 0};
  // x zones
  for (int zone = 1; zone <= 2; zone++)
    for (int ey = 0; ey < nely; ey++)
      for (int ez = 0; ez < nelz; ez++) {
        int el, pel;
        if (zone == 1) {
          el = 1 + ey * nelx + ez * nely * nelx;
          pel = 1 + (nelx - 1) + ey * nelx + ez * nely * nelx;
        } else {
          pel = 1 + ey * nelx + ez * nely * nelx;
          el = 1 + (nelx - 1) + ey * nelx + ez * nely * nelx;
        }
        if (px)
          m.mark_periodic_facet(zone, el - 1, 1 + zone % 2, pel, dummy);
        else
          m.mark_labeled_facet(zone, el - 1, zone);
      }
  for (int zone = 3; zone <= 4; zone++)
    for (int ex = 0; ex < nelx; ex++)
      for (int ez = 0; ez < nelz; ez++) {
        int el, pel;
        if (zone == 3) {
          el = 1 + ex + ez * nely * nelx;
          pel = 1 + ex + (nely - 1) * nelx + ez * nely * nelx;
        } else {
          el = 1 + ex + (nely - 1) * nelx + ez * nely * nelx;
          pel = 1 + ex + ez * nely * nelx;
        }
        if (py)
          m.mark_periodic_facet(zone, el - 1, 3 + zone % 2, pel, dummy);
        else
          m.mark_labeled_facet(zone, el - 1, zone);
      }
  for (int zone = 5; zone <= 6; zone++)
    for (int ex = 0; ex < nelx; ex++)
      for (int ey = 0; ey < nely; ey++) {
        int el, pel;
        if (zone == 5) {
          el = 1 + ex + ey * nelx;
          pel = 1 + ex + ey * nelx + (nelz - 1) * nely * nelx;
        } else {
          pel = 1 + ex + ey * nelx;
          el = 1 + ex + ey * nelx + (nelz - 1) * nely * nelx;
        }
        if (pz)
          m.mark_periodic_facet(zone, el - 1, 5 + zone % 2, pel, dummy);
        else
          m.mark_labeled_facet(zone, el - 1, zone);
      }
  // create_periodic_ids passes (genmeshbox.f90:279-350)
  if (px)
    for (int zone = 1; zone <= 2; zone++)
      for (int ey = 0; ey < nely; ey++)
        for (int ez = 0; ez < nelz; ez++) {
          int el, pel;
          if (zone == 1) {
            el = 1 + ey * nelx + ez * nely * nelx;
            pel = 1 + (nelx - 1) + ey * nelx + ez * nely * nelx;
          } else {
            pel = 1 + ey * nelx + ez * nely * nelx;
            el = 1 + (nelx - 1) + ey * nelx + ez * nely * nelx;
          }
          m.create_periodic_ids(zone, el - 1, 1 + zone % 2, pel - 1);
        }
  if (py)
    for (int zone = 3; zone <= 4; zone++)
      for (int ex = 0; ex < nelx; ex++)
        for (int ez = 0; ez < nelz; ez++) {
          int el, pel;
          if (zone == 3) {
            el = 1 + ex + ez * nely * nelx;
            pel = 1 + ex + (nely - 1) * nelx + ez * nely * nelx;
          } else {
            el = 1 + ex + (nely - 1) * nelx + ez * nely * nelx;
            pel = 1 + ex + ez * nely * nelx;
          }
          m.create_periodic_ids(zone, el - 1, 3 + zone % 2, pel - 1);
        }
  if (pz)
    for (int zone = 5; zone <= 6; zone++)
      for (int ex = 0; ex < nelx; ex++)
        for (int ey = 0; ey < nely; ey++) {
          int el, pel;
          if (zone == 5) {
            el = 1 + ex + ey * nelx;
            pel = 1 + ex + ey * nelx + (nelz - 1) * nely * nelx;
          } else {
            pel = 1 + ex + ey * nelx;
            el = 1 + ex + ey * nelx + (nelz - 1) * nely * nelx;
          }
          m.create_periodic_ids(zone, el - 1, 5 + zone % 2, pel - 1);
        }
  // nmsh_file_write: reset ids, then dump element and zone records.
  m.reset_periodic_ids();
  static const int vcyc_to_sym[8] = {1, 2, 4, 3, 5, 6, 8, 7};
  elems.resize(nel);
  for (int e = 0; e < nel; e++) {
    elems[e].el_idx = m.el_id[e];
    for (int j = 0; j < 8; j++) elems[e].v[j] = m.points[m.el[e][vcyc_to_sym[j] - 1]];
  }
  zones.clear();
  for (auto &z : m.periodic) {
    ZoneRecord r;
    r.e = m.el_id[z.e];
    r.f = z.f;
    r.p_e = z.pe;
    r.p_f = z.pf;
    r.type = 5;
    for (int k = 0; k < 4; k++) r.glb_pt_ids[k] = z.pids[k];
    zones.push_back(r);
  }
  for (int k = 1; k <= 20; k++)
    for (auto &fe : m.labeled[k]) {
      ZoneRecord r;
      r.e = m.el_id[fe.second];
      r.f = fe.first;
      r.p_e = 0;
      r.p_f = k;
      r.type = 7;
      for (int q = 0; q < 4; q++) r.glb_pt_ids[q] = 0;
      zones.push_back(r);
    }
}

// nmsh_file_read (src/io/nmsh_file.f90:70-207, zones 328-432), one rank.
void mesh_from_records(Mesh &m, const std::vector<ElemRecord> &elems,
                       const std::vector<ZoneRecord> &zones) {
  m.init((int)elems.size());
  for (size_t i = 0; i < elems.size(); i++) {
    const Point *p = elems[i].v;
    Point s[8] = {p[0], p[1], p[3], p[2], p[4], p[5], p[7], p[6]};
    m.add_hex((int)i, elems[i].el_idx, s);
  }
  std::unordered_map<int, int> htel;
  for (int i = 0; i < m.nelv; i++) htel[m.el_id[i]] = i;
  for (auto &z : zones) {
    auto it = htel.find(z.e);
    if (it == htel.end()) continue;
    if (z.type == 5)
      m.mark_periodic_facet(z.f, it->second, z.p_f, z.p_e, z.glb_pt_ids);
    else if (z.type == 7)
      m.mark_labeled_facet(z.f, it->second, z.p_f);
  }
  for (auto &z : zones) {
    auto it = htel.find(z.e);
    if (it == htel.end()) continue;
    if (z.type == 5) m.apply_periodic_facet(z.f, it->second, z.glb_pt_ids);
  }
  m.finalize();
}

// ---------------------------------------------------------------------------
// speclib (src/sem/speclib.f90) -- GLL points, weights and derivative matrix.
// ---------------------------------------------------------------------------
double gammaf(double x) {  // speclib.f90:446-462
  const double PI = 4.0 * std::atan(1.0);
  const double eps = 2.220446049250313e-16;
  auto eq = [&](double a) { return std::fabs(x - a) < eps; };
  double g = 1.0;
  if (eq(-0.5)) g = -2.0 * std::sqrt(PI);
  if (eq(0.5)) g = std::sqrt(PI);
  if (eq(1.0)) g = 1.0;
  if (eq(2.0)) g = 1.0;
  if (eq(1.5)) g = std::sqrt(PI) / 2.0;
  if (eq(2.5)) g = 1.5 * std::sqrt(PI) / 2.0;
  if (eq(3.5)) g = 0.5 * (2.5 * (1.5 * std::sqrt(PI)));
  if (eq(3.0)) g = 2.0;
  if (eq(4.0)) g = 6.0;
  if (eq(5.0)) g = 24.0;
  if (eq(6.0)) g = 120.0;
  return g;
}

double pnormj(int n, double alpha, double beta) {  // speclib.f90:465-492
  double dn = n, cnst = alpha + beta + 1.0;
  if (n <= 1) {
    double prod = gammaf(dn + alpha) * gammaf(dn + beta);
    prod = prod / (gammaf(dn) * gammaf(dn + alpha + beta));
    return prod * std::pow(2.0, cnst) / (2.0 * dn + cnst);
  }
  double prod = gammaf(alpha + 1.0) * gammaf(beta + 1.0);
  prod = prod / (2.0 * (1.0 + cnst) * gammaf(cnst + 1.0));
  prod = prod * (1.0 + alpha) * (2.0 + alpha);
  prod = prod * (1.0 + beta) * (2.0 + beta);
  for (int i = 3; i <= n; i++) {
    double di = i;
    double frac = (di + alpha) * (di + beta) / (di * (di + alpha + beta));
    prod = prod * frac;
  }
  return prod * std::pow(2.0, cnst) / (2.0 * dn + cnst);
}

// JACOBF (speclib.f90:559-602)
void jacobf(double &poly, double &pder, double &polym1, double &pderm1,
            double &polym2, double &pderm2, int n, double alp, double bet,
            double x) {
  double apb = alp + bet;
  poly = 1.0;
  pder = 0.0;
  if (n == 0) return;
  double polyl = poly, pderl = pder;
  poly = (alp - bet + (apb + 2.0) * x) / 2.0;
  pder = (apb + 2.0) / 2.0;
  if (n == 1) return;
  double psave = 0, pdsave = 0;
  for (int k = 2; k <= n; k++) {
    double dk = k;
    double a1 = 2.0 * dk * (dk + apb) * (2.0 * dk + apb - 2.0);
    double a2 = (2.0 * dk + apb - 1.0) * (alp * alp - bet * bet);
    double b3 = (2.0 * dk + apb - 2.0);
    double a3 = b3 * (b3 + 1.0) * (b3 + 2.0);
    double a4 = 2.0 * (dk + alp - 1.0) * (dk + bet - 1.0) * (2.0 * dk + apb);
    double polyn = ((a2 + a3 * x) * poly - a4 * polyl) / a1;
    double pdern = ((a2 + a3 * x) * pder - a4 * pderl + a3 * poly) / a1;
    psave = polyl;
    pdsave = pderl;
    polyl = poly;
    poly = polyn;
    pderl = pder;
    pder = pdern;
  }
  polym1 = polyl;
  pderm1 = pderl;
  polym2 = psave;
  pderm2 = pdsave;
}

// JACG (speclib.f90:500-555)
void jacg(double *xjac, int np, double alpha, double beta) {
  const int kstop = 10;
  const double eps = 1.0e-12;
  const double PI = 4.0 * std::atan(1.0);
  int n = np - 1;
  double dth = PI / (2.0 * n + 2.0);
  double xlast = 0;
  for (int j = 1; j <= np; j++) {
    double x;
    if (j == 1) {
      x = std::cos((2.0 * (j - 1.0) + 1.0) * dth);
    } else {
      double x1 = std::cos((2.0 * (j - 1.0) + 1.0) * dth);
      x = (x1 + xlast) / 2.0;
    }
    for (int k = 1; k <= kstop; k++) {
      double p, pd, pm1, pdm1, pm2, pdm2;
      jacobf(p, pd, pm1, pdm1, pm2, pdm2, np, alpha, beta, x);
      double recsum = 0.0;
      for (int i = 1; i <= j - 1; i++) recsum += 1.0 / (x - xjac[np - i]);
      double delx = -p / (pd - recsum * p);
      x = x + delx;
      if (std::fabs(delx) < eps) break;
    }
    xjac[np - j] = x;
    xlast = x;
  }
  for (int i = 0; i < np; i++) {
    double xmin = 2.0;
    int jmin = i;
    for (int j = i; j < np; j++)
      if (xjac[j] < xmin) {
        xmin = xjac[j];
        jmin = j;
      }
    if (jmin != i) std::swap(xjac[i], xjac[jmin]);
  }
}

// ZWGJD (speclib.f90:224-269)
void zwgjd(double *z, double *w, int np, double alpha, double beta) {
  int n = np - 1;
  double apb = alpha + beta;
  if (np == 1) {
    z[0] = (beta - alpha) / (apb + 2.0);
    w[0] = gammaf(alpha + 1.0) * gammaf(beta + 1.0) / gammaf(apb + 2.0) *
           std::pow(2.0, apb + 1.0);
    return;
  }
  jacg(z, np, alpha, beta);
  int np1 = n + 1, np2 = n + 2;
  double dnp1 = np1, dnp2 = np2;
  double fac1 = dnp1 + alpha + beta + 1.0;
  double fac2 = fac1 + dnp1;
  double fac3 = fac2 + 1.0;
  double fnorm = pnormj(np1, alpha, beta);
  double rcoef = (fnorm * fac2 * fac3) / (2.0 * fac1 * dnp2);
  for (int i = 0; i < np; i++) {
    double p, pd, pm1, pdm1, pm2, pdm2;
    jacobf(p, pd, pm1, pdm1, pm2, pdm2, np2, alpha, beta, z[i]);
    w[i] = -rcoef / (p * pdm1);
  }
}

double endw1(int n, double alpha, double beta) {  // speclib.f90:347-393
  if (n == 0) return 0.0;
  double apb = alpha + beta;
  double f1 = gammaf(alpha + 2.0) * gammaf(beta + 1.0) / gammaf(apb + 3.0);
  f1 = f1 * (apb + 2.0) * std::pow(2.0, apb + 2.0) / 2.0;
  if (n == 1) return f1;
  double fint1 = gammaf(alpha + 2.0) * gammaf(beta + 1.0) / gammaf(apb + 3.0);
  fint1 = fint1 * std::pow(2.0, apb + 2.0);
  double fint2 = gammaf(alpha + 2.0) * gammaf(beta + 2.0) / gammaf(apb + 4.0);
  fint2 = fint2 * std::pow(2.0, apb + 3.0);
  double f2 = (-2.0 * (beta + 2.0) * fint1 + (apb + 4.0) * fint2) * (apb + 3.0) / 4.0;
  if (n == 2) return f2;
  double f3 = 0;
  for (int i = 3; i <= n; i++) {
    double di = i - 1;
    double abn = alpha + beta + di, abnn = abn + di;
    double a1 = -(2.0 * (di + alpha) * (di + beta)) / (abn * abnn * (abnn + 1.0));
    double a2 = (2.0 * (alpha - beta)) / (abnn * (abnn + 2.0));
    double a3 = (2.0 * (abn + 1.0)) / ((abnn + 2.0) * (abnn + 1.0));
    f3 = -(a2 * f2 + a1 * f1) / a3;
    f1 = f2;
    f2 = f3;
  }
  return f3;
}

double endw2(int n, double alpha, double beta) {  // speclib.f90:396-443
  if (n == 0) return 0.0;
  double apb = alpha + beta;
  double f1 = gammaf(alpha + 1.0) * gammaf(beta + 2.0) / gammaf(apb + 3.0);
  f1 = f1 * (apb + 2.0) * std::pow(2.0, apb + 2.0) / 2.0;
  if (n == 1) return f1;
  double fint1 = gammaf(alpha + 1.0) * gammaf(beta + 2.0) / gammaf(apb + 3.0);
  fint1 = fint1 * std::pow(2.0, apb + 2.0);
  double fint2 = gammaf(alpha + 2.0) * gammaf(beta + 2.0) / gammaf(apb + 4.0);
  fint2 = fint2 * std::pow(2.0, apb + 3.0);
  double f2 = (2.0 * (alpha + 2.0) * fint1 - (apb + 4.0) * fint2) * (apb + 3.0) / 4.0;
  if (n == 2) return f2;
  double f3 = 0;
  for (int i = 3; i <= n; i++) {
    double di = i - 1;
    double abn = alpha + beta + di, abnn = abn + di;
    double a1 = -(2.0 * (di + alpha) * (di + beta)) / (abn * abnn * (abnn + 1.0));
    double a2 = (2.0 * (alpha - beta)) / (abnn * (abnn + 2.0));
    double a3 = (2.0 * (abn + 1.0)) / ((abnn + 2.0) * (abnn + 1.0));
    f3 = -(a2 * f2 + a1 * f1) / a3;
    f1 = f2;
    f2 = f3;
  }
  return f3;
}

// ZWGLJD (speclib.f90:307-344) with alpha = beta = 0 gives ZWGLL.
void zwgll(double *z, double *w, int np) {
  int n = np - 1;
  const double alpha = 0.0, beta = 0.0;
  if (n - 1 > 0) zwgjd(z + 1, w + 1, n - 1, alpha + 1.0, beta + 1.0);
  z[0] = -1.0;
  z[np - 1] = 1.0;
  for (int i = 1; i < np - 1; i++) w[i] = w[i] / (1.0 - z[i] * z[i]);
  double p, pd, pm1, pdm1, pm2, pdm2;
  jacobf(p, pd, pm1, pdm1, pm2, pdm2, n, alpha, beta, z[0]);
  w[0] = endw1(n, alpha, beta) / (2.0 * pd);
  jacobf(p, pd, pm1, pdm1, pm2, pdm2, n, alpha, beta, z[np - 1]);
  w[np - 1] = endw2(n, alpha, beta) / (2.0 * pd);
}

double pnleg(double z, int n) {  // speclib.f90:967-999
  double p1 = 1.0;
  if (n == 0) return p1;
  double p2 = z, p3 = p2;
  for (int k = 1; k <= n - 1; k++) {
    double fk = k;
    p3 = ((2.0 * fk + 1.0) * z * p2 - fk * p1) / (fk + 1.0);
    p1 = p2;
    p2 = p3;
  }
  return p3;
}

// DGLL (speclib.f90:880-919): D(i,j) column-major, dt = transpose.
void dgll(double *d, double *dt, const double *z, int nz) {
  int n = nz - 1;
  if (nz == 1) {
    d[0] = 0.0;
    return;
  }
  double fn = n, d0 = fn * (fn + 1.0) / 4.0;
  for (int i = 0; i < nz; i++)
    for (int j = 0; j < nz; j++) {
      double v;
      if (i != j)
        v = pnleg(z[i], n) / (pnleg(z[j], n) * (z[i] - z[j]));
      else if (i == 0)
        v = -d0;
      else if (i == nz - 1)
        v = d0;
      else
        v = 0.0;
      d[i + nz * j] = v;
      dt[j + nz * i] = v;
    }
}

// fd_weights_full (src/math/fast3d.f90:105-163): Fornberg weights of the
// interpolant through x[0..n] evaluated at xi, derivative order 0..m.
void fd_weights_full(double xi, const double *x, int n, int m, double *c) {
  std::vector<double> cx((n + 1) * (m + 1), 0.0);
  auto C = [&](int j, int k) -> double & { return cx[j + (n + 1) * k]; };
  double c1 = 1.0, c4 = x[0] - xi;
  C(0, 0) = 1.0;
  for (int i = 1; i <= n; i++) {
    int mn = std::min(i, m);
    double c2 = 1.0, c5 = c4;
    c4 = x[i] - xi;
    for (int j = 0; j <= i - 1; j++) {
      double c3 = x[i] - x[j];
      c2 = c2 * c3;
      for (int k = mn; k >= 1; k--)
        C(i, k) = c1 * (k * C(i - 1, k - 1) - c5 * C(i - 1, k)) / c2;
      C(i, 0) = -c1 * c5 * C(i - 1, 0) / c2;
      for (int k = mn; k >= 1; k--) C(j, k) = (c4 * C(j, k) - k * C(j, k - 1)) / c3;
      C(j, 0) = c4 * C(j, 0) / c3;
    }
    c1 = c2;
  }
  for (size_t i = 0; i < cx.size(); i++) c[i] = cx[i];
}

// mxm (src/math/mxm_wrapper.F90:30-62): c(n1,n3) = a(n1,n2) b(n2,n3),
// column-major, sequential sums.
void mxm(const double *a, int n1, const double *b, int n2, double *c, int n3) {
  for (int j = 0; j < n3; j++)
    for (int i = 0; i < n1; i++) {
      double t = 0.0;
      for (int k = 0; k < n2; k++) t += a[i + n1 * k] * b[k + n2 * j];
      c[i + n1 * j] = t;
    }
}

}  // namespace nko

using namespace nko;

namespace {

inline long lin(int i, int j, int k, int e, int lx) {  // 1-based -> 0-based
  return (long)(i - 1) + (long)lx * ((j - 1) + (long)lx * ((k - 1) + (long)lx * (e - 1)));
}

// dofmap_number_points/edges/faces (dofmap.f90:264-719), pe_size = 1.
void dofmap_number(OrProblem &P) {
  Mesh &m = (*P.meshp);
  int lx = P.lx;
  P.dof.assign(P.n, 0);
  auto D = [&](int i, int j, int k, int e) -> int64_t & { return P.dof[lin(i, j, k, e, lx)]; };
  for (int e = 1; e <= m.nelv; e++)
    for (int jl = 1; jl <= 8; jl++) {
      int ix = ((jl - 1) % 2) * (lx - 1) + 1;
      int iy = (((jl - 1) % 4) / 2) * (lx - 1) + 1;
      int iz = ((jl - 1) / 4) * (lx - 1) + 1;
      D(ix, iy, iz, e) = m.pid(e - 1, jl);
    }
  P.glb_mpts = m.max_pts_id;
  P.glb_meds = m.meds;
  int64_t nde = lx - 2;
  int64_t edge_offset = (int64_t)P.glb_mpts + 1;
  // (edge index, start corner (i,j,k), direction 0=r 1=s 2=t, and the
  // quirk of edge 8 that reverses with lz instead of ly).
  struct EdgeDef {
    int edge, i0, j0, k0, dir;
  };
  const int L = lx;
  const EdgeDef defs[12] = {{1, 1, 1, 1, 0}, {3, 1, 1, L, 0}, {2, 1, L, 1, 0},
                            {4, 1, L, L, 0}, {5, 1, 1, 1, 1}, {7, 1, 1, L, 1},
                            {6, L, 1, 1, 1}, {8, L, 1, L, 1}, {9, 1, 1, 1, 2},
                            {10, L, 1, 1, 2}, {11, 1, L, 1, 2}, {12, L, L, 1, 2}};
  for (int e = 1; e <= m.nelv; e++) {
    for (const EdgeDef &d : defs) {
      Edge ed = m.edge_id(e - 1, d.edge);
      int gid = m.hte.at(ed);
      int64_t eid = edge_offset + (int64_t)(gid - 1) * nde;
      bool rev = (int64_t)ed[0] != D(d.i0, d.j0, d.k0, e);
      for (int j = 2; j <= lx - 1; j++) {
        int k = rev ? lx + 1 - j : j;
        int ii = d.i0, jj = d.j0, kk = d.k0;
        if (d.dir == 0) ii = k;
        if (d.dir == 1) jj = k;
        if (d.dir == 2) kk = k;
        D(ii, jj, kk, e) = eid + (j - 2);
      }
    }
  }
  // faces
  int64_t facet_offset = (int64_t)P.glb_mpts + (int64_t)P.glb_meds * (lx - 2) + 1;
  int64_t ndf = (int64_t)(lx - 2) * (lx - 2);
  auto facetidx = [](const Face &fo, const Face &f, int64_t fid, int k1, int j1,
                     int lk1, int lj1) -> int64_t {
    // dofmap_facetidx (dofmap.f90:722-771)
    int k = k1 - 2, j = j1 - 2, lk = lk1 - 2, lj = lj1 - 2;
    int64_t r = 0;
    if (fo[0] == f[0]) {
      r = fo[1] < fo[3] ? fid + j + k * lj : fid + j * lk + k;
    } else if (fo[1] == f[0]) {
      r = fo[2] < fo[0] ? fid + lk * (lj - 1 - j) + k : fid + (lj - 1 - j) + k * lj;
    } else if (fo[2] == f[0]) {
      r = fo[3] < fo[1] ? fid + (lj - 1 - j) + lj * (lk - 1 - k)
                        : fid + lk * (lj - 1 - j) + (lk - 1 - k);
    } else if (fo[3] == f[0]) {
      r = fo[0] < fo[2] ? fid + lk * j + (lk - 1 - k) : fid + j + lj * (lk - 1 - k);
    }
    return r;
  };
  for (int e = 1; e <= m.nelv; e++) {
    for (int side = 1; side <= 6; side++) {
      Face f = m.facet_id(e - 1, side), fo = m.facet_order(e - 1, side);
      int gid = m.htf.at(f);
      int64_t fid = facet_offset + (int64_t)(gid - 1) * ndf;
      for (int a = 2; a <= lx - 1; a++)      // outer
        for (int b = 2; b <= lx - 1; b++) {  // inner
          switch (side) {
            case 1: D(1, b, a, e) = facetidx(fo, f, fid, b, a, lx, lx); break;
            case 2: D(lx, b, a, e) = facetidx(fo, f, fid, b, a, lx, lx); break;
            case 3: D(b, 1, a, e) = facetidx(fo, f, fid, a, b, lx, lx); break;
            case 4: D(b, lx, a, e) = facetidx(fo, f, fid, a, b, lx, lx); break;
            case 5: D(b, a, 1, e) = facetidx(fo, f, fid, a, b, lx, lx); break;
            case 6: D(b, a, lx, e) = facetidx(fo, f, fid, a, b, lx, lx); break;
          }
        }
    }
  }
}

// dofmap_xyzlin (dofmap.f90:868-939) with tensr3 (src/math/tensor.f90:93-120).
void dofmap_xyz(OrProblem &P) {
  int lx = P.lx;
  const double zlin[2] = {-1.0, 1.0};
  std::vector<double> jxt(2 * lx), jx(2 * lx);
  for (int j = 0; j < lx; j++) fd_weights_full(P.zg[j], zlin, 1, 0, &jxt[2 * j]);
  for (int i = 0; i < lx; i++)  // trsp(jx, lx, jxt, 2): jx(lx,2)
    for (int j = 0; j < 2; j++) jx[i + lx * j] = jxt[j + 2 * i];
  P.x.assign(P.n, 0);
  P.y.assign(P.n, 0);
  P.z.assign(P.n, 0);
  std::vector<double> v(lx * lx * lx), w(4 * lx * lx * lx), tmp(lx * lx * lx);
  double xyzb[8];
  Mesh &m = (*P.meshp);
  for (int e = 0; e < m.nelv; e++) {
    for (int c = 0; c < 3; c++) {
      for (int vtx = 0; vtx < 8; vtx++) xyzb[vtx] = m.px(e, vtx + 1)[c];
      // tensr3(v, lx, xyzb, 2, jx, jyt, jzt, w)
      mxm(jx.data(), lx, xyzb, 2, v.data(), 4);
      for (int j = 0; j < 2; j++)
        mxm(&v[lx * 2 * j], lx, jxt.data(), 2, &w[lx * lx * j], lx);
      mxm(w.data(), lx * lx, jxt.data(), 2, tmp.data(), lx);
      double *dst = c == 0 ? P.x.data() : (c == 1 ? P.y.data() : P.z.data());
      std::memcpy(dst + (size_t)e * lx * lx * lx, tmp.data(), sizeof(double) * lx * lx * lx);
    }
  }
}

// gs_init_mapping (gather_scatter.f90:513-1375), single rank: every dof is
// local, ids are assigned in traversal order, then Hoare-quicksorted.
void gs_init_mapping(OrProblem &P) {
  Mesh &m = (*P.meshp);
  int lx = P.lx;
  std::unordered_map<int64_t, int> dm;
  dm.reserve(P.n / lx);
  int max_id = 0;
  std::vector<int> local_dof, dof_local, face_dof, dof_face;
  auto add = [&](int64_t key) {  // gs_mapping_add_dof (1276-1288)
    auto it = dm.find(key);
    if (it != dm.end()) return it->second;
    dm[key] = ++max_id;
    return max_id;
  };
  auto push = [&](int i, int j, int k, int e) {
    long l = lin(i, j, k, e, lx);
    local_dof.push_back(add(P.dof[l]));
    dof_local.push_back((int)(l + 1));
  };
  for (int e = 1; e <= m.nelv; e++) {
    push(1, 1, 1, e);
    push(lx, 1, 1, e);
    push(1, lx, 1, e);
    push(lx, lx, 1, e);
    push(1, 1, lx, e);
    push(lx, 1, lx, e);
    push(1, lx, lx, e);
    push(lx, lx, lx, e);
  }
  dm.clear();
  for (int e = 1; e <= m.nelv; e++) {
    for (int j = 2; j <= lx - 1; j++) push(j, 1, 1, e);
    for (int j = 2; j <= lx - 1; j++) push(j, 1, lx, e);
    for (int j = 2; j <= lx - 1; j++) push(j, lx, 1, e);
    for (int j = 2; j <= lx - 1; j++) push(j, lx, lx, e);
    for (int k = 2; k <= lx - 1; k++) push(1, k, 1, e);
    for (int k = 2; k <= lx - 1; k++) push(1, k, lx, e);
    for (int k = 2; k <= lx - 1; k++) push(lx, k, 1, e);
    for (int k = 2; k <= lx - 1; k++) push(lx, k, lx, e);
    for (int l = 2; l <= lx - 1; l++) push(1, 1, l, e);
    for (int l = 2; l <= lx - 1; l++) push(lx, 1, l, e);
    for (int l = 2; l <= lx - 1; l++) push(1, lx, l, e);
    for (int l = 2; l <= lx - 1; l++) push(lx, lx, l, e);
  }
  dm.clear();
  auto fpush = [&](int i, int j, int k, int e) {
    long l = lin(i, j, k, e, lx);
    face_dof.push_back(add(P.dof[l]));
    dof_face.push_back((int)(l + 1));
  };
  for (int e = 1; e <= m.nelv; e++) {
    const int *fn = &m.facet_neigh[(size_t)(e - 1) * 6];
    if (fn[0] != 0)
      for (int l = 2; l <= lx - 1; l++)
        for (int k = 2; k <= lx - 1; k++) fpush(1, k, l, e);
    if (fn[1] != 0)
      for (int l = 2; l <= lx - 1; l++)
        for (int k = 2; k <= lx - 1; k++) fpush(lx, k, l, e);
    if (fn[2] != 0)
      for (int l = 2; l <= lx - 1; l++)
        for (int j = 2; j <= lx - 1; j++) fpush(j, 1, l, e);
    if (fn[3] != 0)
      for (int l = 2; l <= lx - 1; l++)
        for (int j = 2; j <= lx - 1; j++) fpush(j, lx, l, e);
    if (fn[4] != 0)
      for (int k = 2; k <= lx - 1; k++)
        for (int j = 2; j <= lx - 1; j++) fpush(j, k, 1, e);
    if (fn[5] != 0)
      for (int k = 2; k <= lx - 1; k++)
        for (int j = 2; j <= lx - 1; j++) fpush(j, k, lx, e);
  }
  P.nlocal = (int)(local_dof.size() + face_dof.size());
  P.local_facet_offset = (int)local_dof.size() + 1;
  P.local_dof_gs = local_dof;
  P.local_dof_gs.insert(P.local_dof_gs.end(), face_dof.begin(), face_dof.end());
  P.local_gs_dof = dof_local;
  P.local_gs_dof.insert(P.local_gs_dof.end(), dof_face.begin(), dof_face.end());
  // gs_qsort_dofmap (1291-1330), 1-based lo/hi; explicit stack keeps the
  // recursion order (left part fully before right part).
  int *dg = P.local_dof_gs.data() - 1, *gd = P.local_gs_dof.data() - 1;
  std::vector<std::pair<int, int>> stack;
  if (P.nlocal > 0) stack.push_back({1, P.nlocal});
  while (!stack.empty()) {
    auto [lo, hi] = stack.back();
    stack.pop_back();
    int i = lo - 1, j = hi + 1;
    int pivot = dg[(lo + hi) / 2];
    for (;;) {
      do { i++; } while (dg[i] < pivot);
      do { j--; } while (dg[j] > pivot);
      if (i < j) {
        std::swap(dg[i], dg[j]);
        std::swap(gd[i], gd[j]);
      } else if (i == j) {
        i++;
        break;
      } else {
        break;
      }
    }
    // recursion order: (lo, j) first, then (i, hi) -> push right then left.
    if (i < hi) stack.push_back({i, hi});
    if (lo < j) stack.push_back({lo, j});
  }
  // gs_find_blks (1333-1373)
  P.blk_len.clear();
  int i = 1, mm = P.local_facet_offset, nn = P.nlocal;
  while (i < mm) {
    int id = dg[i], count = 1, j = i;
    while (j + 1 <= nn && dg[j + 1] == id) {
      j++;
      count++;
    }
    P.blk_len.push_back(count);
    i = j + 1;
  }
  P.nlocal_blks = (int)P.blk_len.size();
  P.blk_off.assign(P.nlocal_blks, 0);
  for (int b = 1; b < P.nlocal_blks; b++) P.blk_off[b] = P.blk_off[b - 1] + P.blk_len[b - 1];
}

}  // namespace

// gs_op_vector with GS_OP_ADD (gather_scatter.f90:1613-1682) using the CPU
// gather/scatter kernels (src/gs/bcknd/cpu/gs_cpu.f90:98-138,292-322).
static void gs_add(const OrProblem &P, double *u, std::vector<double> &v) {
  int m = P.nlocal, o = P.local_facet_offset, nb = P.nlocal_blks;
  v.assign(std::max(m, 1), 0.0);
  const int *dg = P.local_dof_gs.data() - 1, *gd = P.local_gs_dof.data() - 1;
  double *U = u - 1, *V = v.data() - 1;
  // Each phase writes distinct entries per block / pair, so the phases
  // run element-parallel without changing any sum.
  parallel_for(nb, [&](long b0, long b1) {
    for (long b = b0; b < b1; b++) {
      int k = P.blk_off[b], bl = P.blk_len[b];
      double t = U[gd[k + 1]];
      for (int j = 2; j <= bl; j++) t = t + U[gd[k + j]];
      V[dg[k + 1]] = t;
    }
  });
  const long npair = m >= o ? (m - o + 2) / 2 : 0;
  parallel_for(npair, [&](long q0, long q1) {
    for (long q = q0; q < q1; q++) {
      const int i = o + 2 * (int)q;
      V[dg[i]] = U[gd[i]] + U[gd[i + 1]];
    }
  });
  parallel_for(nb, [&](long b0, long b1) {
    for (long b = b0; b < b1; b++) {
      int k = P.blk_off[b], bl = P.blk_len[b];
      double t = V[dg[k + 1]];
      for (int j = 1; j <= bl; j++) U[gd[k + j]] = t;
    }
  });
  int start = nb > 0 ? P.blk_off[nb - 1] + P.blk_len[nb - 1] + 1 : 1;
  parallel_for(m - start + 1, [&](long q0, long q1) {
    for (long q = q0; q < q1; q++) U[gd[start + q]] = V[dg[start + q]];
  });
}

namespace {

// coef_generate_dxyzdrst / geo / mass (coef.f90:714-1156) and mult (405-418).
void coef_init(OrProblem &P) {
  int lx = P.lx, lxy = lx * lx, lxyz = lx * lx * lx;
  long n = P.n;
  std::vector<double> xr(n), xs(n), xt(n), yr(n), ys(n), yt(n), zr(n), zs(n), zt(n);
  std::vector<double> dyt = P.dxt, dzt = P.dxt;  // GLL: dy = dz = dx
  for (int e = 0; e < P.nelv; e++) {
    size_t o = (size_t)e * lxyz;
    mxm(P.dx.data(), lx, &P.x[o], lx, &xr[o], lxy);
    mxm(P.dx.data(), lx, &P.y[o], lx, &yr[o], lxy);
    mxm(P.dx.data(), lx, &P.z[o], lx, &zr[o], lxy);
    for (int i = 0; i < lx; i++) {
      mxm(&P.x[o + i * lxy], lx, dyt.data(), lx, &xs[o + i * lxy], lx);
      mxm(&P.y[o + i * lxy], lx, dyt.data(), lx, &ys[o + i * lxy], lx);
      mxm(&P.z[o + i * lxy], lx, dyt.data(), lx, &zs[o + i * lxy], lx);
    }
    mxm(&P.x[o], lxy, dzt.data(), lx, &xt[o], lx);
    mxm(&P.y[o], lxy, dzt.data(), lx, &yt[o], lx);
    mxm(&P.z[o], lxy, dzt.data(), lx, &zt[o], lx);
  }
  P.jac.assign(n, 0);
  P.jacinv.assign(n, 0);
  std::vector<double> rx(n), ry(n), rz(n), sx(n), sy(n), sz(n), tx(n), ty(n), tz(n);
  for (long i = 0; i < n; i++) {
    double j = 0.0;
    j = j + (xr[i] * ys[i] * zt[i]);
    j = j + (xt[i] * yr[i] * zs[i]);
    j = j + (xs[i] * yt[i] * zr[i]);
    j = j - (xr[i] * yt[i] * zs[i]);
    j = j - (xs[i] * yr[i] * zt[i]);
    j = j - (xt[i] * ys[i] * zr[i]);
    P.jac[i] = j;
    rx[i] = ys[i] * zt[i] - yt[i] * zs[i];
    ry[i] = xt[i] * zs[i] - xs[i] * zt[i];
    rz[i] = xs[i] * yt[i] - xt[i] * ys[i];
    sx[i] = yt[i] * zr[i] - yr[i] * zt[i];
    sy[i] = xr[i] * zt[i] - xt[i] * zr[i];
    sz[i] = xt[i] * yr[i] - xr[i] * yt[i];
    tx[i] = yr[i] * zs[i] - ys[i] * zr[i];
    ty[i] = xs[i] * zr[i] - xr[i] * zs[i];
    tz[i] = xr[i] * ys[i] - xs[i] * yr[i];
    P.jacinv[i] = 1.0 / j;  // invers2
  }
  P.drdx = rx; P.drdy = ry; P.drdz = rz;
  P.dsdx = sx; P.dsdy = sy; P.dsdz = sz;
  P.dtdx = tx; P.dtdy = ty; P.dtdz = tz;
  P.g11.assign(n, 0);
  P.g22.assign(n, 0);
  P.g33.assign(n, 0);
  P.g12.assign(n, 0);
  P.g13.assign(n, 0);
  P.g23.assign(n, 0);
  for (long i = 0; i < n; i++) {
    double ji = P.jacinv[i], w = P.w3[i % lxyz];
    P.g11[i] = ((rx[i] * rx[i] + ry[i] * ry[i] + rz[i] * rz[i]) * ji) * w;
    P.g22[i] = ((sx[i] * sx[i] + sy[i] * sy[i] + sz[i] * sz[i]) * ji) * w;
    P.g33[i] = ((tx[i] * tx[i] + ty[i] * ty[i] + tz[i] * tz[i]) * ji) * w;
    P.g12[i] = ((rx[i] * sx[i] + ry[i] * sy[i] + rz[i] * sz[i]) * ji) * w;
    P.g13[i] = ((rx[i] * tx[i] + ry[i] * ty[i] + rz[i] * tz[i]) * ji) * w;
    P.g23[i] = ((sx[i] * tx[i] + sy[i] * ty[i] + sz[i] * tz[i]) * ji) * w;
  }
  P.B.assign(n, 0);
  double vol = 0.0;
  for (long i = 0; i < n; i++) {
    P.B[i] = P.jac[i] * P.w3[i % lxyz];
    vol += P.B[i];
  }
  P.volume = vol;
  P.h1.assign(n, 1.0);
  P.h2.assign(n, 1.0);
  P.ifh2 = false;
  P.mult.assign(n, 1.0);
  std::vector<double> v;
  gs_add(P, P.mult.data(), v);
  for (long i = 0; i < n; i++) P.mult[i] = 1.0 / P.mult[i];
}

}  // namespace

void or_gs_add_impl(const OrProblem &P, double *u) {
  std::vector<double> v;
  gs_add(P, u, v);
}
const int *or_facet_neigh(const OrProblem &P) { return P.meshp->facet_neigh.data(); }
int or_facet_type(const OrProblem &P, int f, int e) {
  return P.meshp->facet_type[(size_t)(e - 1) * 6 + (f - 1)];
}
void or_all_deformed(OrProblem &P) {
  std::fill(P.meshp->dfrmd_el.begin(), P.meshp->dfrmd_el.end(), 1);
}
void or_coef_init_impl(OrProblem &P) { coef_init(P); }
void fd_weights_full_impl(double xi, const double *x, int n, int m, double *c) {
  fd_weights_full(xi, x, n, m, c);
}
void zwgll_impl(double *z, double *w, int np) { zwgll(z, w, np); }
void mxm_impl(const double *a, int n1, const double *b, int n2, double *c, int n3) {
  mxm(a, n1, b, n2, c, n3);
}
int or_dfrmd_el(const OrProblem &P, int e) { return P.meshp->dfrmd_el[e]; }

// ---------------------------------------------------------------------------
// C ABI for the Python test harness.
// ---------------------------------------------------------------------------
extern "C" {

static OrProblem *build_common(OrProblem *P, int lx) {
  P->lx = lx;
  P->nelv = P->meshp->nelv;
  P->n = (long)lx * lx * lx * P->nelv;
  P->zg.assign(lx, 0);
  P->wx.assign(lx, 0);
  zwgll(P->zg.data(), P->wx.data(), lx);
  P->w3.assign(lx * lx * lx, 0);
  for (int k = 0; k < lx; k++)
    for (int j = 0; j < lx; j++)
      for (int i = 0; i < lx; i++)
        P->w3[i + lx * (j + lx * k)] = P->wx[i] * P->wx[j] * P->wx[k];
  P->dx.assign(lx * lx, 0);
  P->dxt.assign(lx * lx, 0);
  dgll(P->dx.data(), P->dxt.data(), P->zg.data(), lx);
  dofmap_number(*P);
  dofmap_xyz(*P);
  gs_init_mapping(*P);
  return P;
}

void or_deform_sine(OrProblem *P, double amp);
}  // extern "C"

OrProblem *or_level_create(const OrProblem &fine, int lx, bool with_coef) {
  OrProblem *P = new OrProblem();
  P->meshp = fine.meshp;
  P->owns_mesh = false;
  build_common(P, lx);
  if (fine.deform_amp != 0.0) or_deform_sine(P, fine.deform_amp);
  if (with_coef) coef_init(*P);
  return P;
}

extern "C" {

OrProblem *or_box_create(int nelx, int nely, int nelz, double x0, double x1,
                         double y0, double y1, double z0, double z1, int px,
                         int py, int pz, int lx) {
  std::vector<ElemRecord> elems;
  std::vector<ZoneRecord> zones;
  genmeshbox(x0, x1, y0, y1, z0, z1, nelx, nely, nelz, px, py, pz, elems, zones);
  OrProblem *P = new OrProblem();
  P->meshp = new Mesh();
  mesh_from_records(*P->meshp, elems, zones);
  return build_common(P, lx);
}

// genmeshbox followed by nmsh_file_write into `path` in the file layout of
// nmsh_file_write (src/io/nmsh_file.f90:650-760, packed MPI-IO records of
// src/comm/mpi_types.f90:120-200): header, element records (el_idx, 8 x
// (v_idx, xyz) in cyclic order), zone records, zero curves.  Returns 0.
int or_genmeshbox_nmsh(const char *path, int nelx, int nely, int nelz, double x0, double x1,
                       double y0, double y1, double z0, double z1, int px, int py, int pz) {
  std::vector<ElemRecord> elems;
  std::vector<ZoneRecord> zones;
  genmeshbox(x0, x1, y0, y1, z0, z1, nelx, nely, nelz, px, py, pz, elems, zones);
  FILE *f = fopen(path, "wb");
  if (!f) return 1;
  int32_t hdr[2] = {(int32_t)elems.size(), 3};
  fwrite(hdr, 4, 2, f);
  for (auto &r : elems) {
    int32_t id = r.el_idx;
    fwrite(&id, 4, 1, f);
    for (int j = 0; j < 8; j++) {
      int32_t v = r.v[j].id;
      fwrite(&v, 4, 1, f);
      fwrite(r.v[j].x, 8, 3, f);
    }
  }
  int32_t nz = (int32_t)zones.size();
  fwrite(&nz, 4, 1, f);
  for (auto &z : zones) {
    int32_t rec[9] = {z.e, z.f, z.p_e, z.p_f, z.glb_pt_ids[0], z.glb_pt_ids[1],
                      z.glb_pt_ids[2], z.glb_pt_ids[3], z.type};
    fwrite(rec, 4, 9, f);
  }
  int32_t nc = 0;
  fwrite(&nc, 4, 1, f);
  fclose(f);
  return 0;
}

// Two-element style meshes of the gs unit tests: point ids and coordinates
// given per element in symmetric vertex order, then mesh_generate_conn.
OrProblem *or_elements_create(int nelv, const int *ids, const double *xyz, int lx) {
  OrProblem *P = new OrProblem();
  P->meshp = new Mesh();
  P->meshp->init(nelv);
  for (int e = 0; e < nelv; e++) {
    Point p[8];
    for (int v = 0; v < 8; v++) {
      p[v].id = ids[e * 8 + v];
      for (int d = 0; d < 3; d++) p[v].x[d] = xyz[(e * 8 + v) * 3 + d];
    }
    P->meshp->add_hex(e, e + 1, p);
  }
  P->meshp->finalize();
  return build_common(P, lx);
}

// mesh_deform hook (src/mesh/mesh.f90:126) applied to the GLL coordinates:
// x += a sin(y) sin(z), y += a sin(z) sin(x), z += a sin(x) sin(y), all
// evaluated at the undeformed point.
void or_deform_sine(OrProblem *P, double amp) {
  P->deform_amp = amp;
  for (long i = 0; i < P->n; i++) {
    double x = P->x[i], y = P->y[i], z = P->z[i];
    P->x[i] = x + amp * std::sin(y) * std::sin(z);
    P->y[i] = y + amp * std::sin(z) * std::sin(x);
    P->z[i] = z + amp * std::sin(x) * std::sin(y);
  }
}

void or_coef_init(OrProblem *P) { coef_init(*P); }

// Mark every face with facet_neigh == 0 as zero-Dirichlet
// (examples/poisson/setup.f90:2-30) and build the mask as bc_finalize_base
// does (bc.f90:434-593): gs-add an indicator, keep entries > 0.5.
void or_bc_boundary(OrProblem *P) { or_bc_boundary_impl(*P); }

// Strong (Dirichlet) boundary faces get facet_type 1, as the pressure bc
// factory does for strong boundaries (src/fluid/fluid_pnpn_bc_fctry.f90:
// 158-167); the FDM of the Schwarz smoother then drops those rows
// (fdm.f90:417-441).  Applied to every face without a neighbour.
void or_mark_dirichlet_facets(OrProblem *P) {
  for (int e = 0; e < P->nelv; e++)
    for (int f = 0; f < 6; f++)
      if (P->meshp->facet_neigh[(size_t)e * 6 + f] == 0) P->meshp->facet_type[(size_t)e * 6 + f] = 1;
}
}  // extern "C"
void or_bc_boundary_impl(OrProblem &PP) {
  OrProblem *P = &PP;
  int lx = P->lx;
  std::vector<double> t(P->n, 0.0);
  for (int e = 1; e <= P->nelv; e++)
    for (int f = 1; f <= 6; f++) {
      if (P->meshp->facet_neigh[(size_t)(e - 1) * 6 + f - 1] != 0) continue;
      for (int a = 1; a <= lx; a++)
        for (int b = 1; b <= lx; b++) {
          long l = 0;
          switch (f) {
            case 1: l = lin(1, b, a, e, lx); break;
            case 2: l = lin(lx, b, a, e, lx); break;
            case 3: l = lin(b, 1, a, e, lx); break;
            case 4: l = lin(b, lx, a, e, lx); break;
            case 5: l = lin(b, a, 1, e, lx); break;
            case 6: l = lin(b, a, lx, e, lx); break;
          }
          t[l] = 1.0;
        }
    }
  std::vector<double> v;
  gs_add(*P, t.data(), v);
  P->msk.clear();
  for (long i = 0; i < P->n; i++)
    if (t[i] > 0.5) P->msk.push_back((int)(i + 1));
}
extern "C" {

void or_destroy(OrProblem *P) {
  if (P->owns_mesh) delete P->meshp;
  delete P;
}

long or_n(OrProblem *P) { return P->n; }
int or_nelv(OrProblem *P) { return P->nelv; }
int or_lx(OrProblem *P) { return P->lx; }
int or_nlocal(OrProblem *P) { return P->nlocal; }
int or_local_facet_offset(OrProblem *P) { return P->local_facet_offset; }
int or_nblks(OrProblem *P) { return P->nlocal_blks; }
int or_nmsk(OrProblem *P) { return (int)P->msk.size(); }
double or_volume(OrProblem *P) { return P->volume; }
int or_glb_mpts(OrProblem *P) { return P->glb_mpts; }
int or_glb_meds(OrProblem *P) { return P->glb_meds; }
int or_dfrmd(OrProblem *P, int e) { return P->meshp->dfrmd_el[e]; }

// Copy-out accessors (sizes known to the caller).
void or_get_i64(OrProblem *P, const char *name, int64_t *out) {
  if (!strcmp(name, "dof")) std::memcpy(out, P->dof.data(), P->dof.size() * 8);
}
void or_get_i32(OrProblem *P, const char *name, int *out) {
  const std::vector<int> *v = nullptr;
  if (!strcmp(name, "dof_gs")) v = &P->local_dof_gs;
  if (!strcmp(name, "gs_dof")) v = &P->local_gs_dof;
  if (!strcmp(name, "blk_len")) v = &P->blk_len;
  if (!strcmp(name, "blk_off")) v = &P->blk_off;
  if (!strcmp(name, "msk")) v = &P->msk;
  if (!strcmp(name, "facet_neigh")) v = &P->meshp->facet_neigh;
  if (v) std::memcpy(out, v->data(), v->size() * 4);
}
void or_get_f64(OrProblem *P, const char *name, double *out) {
  const std::vector<double> *v = nullptr;
  if (!strcmp(name, "x")) v = &P->x;
  if (!strcmp(name, "y")) v = &P->y;
  if (!strcmp(name, "z")) v = &P->z;
  if (!strcmp(name, "zg")) v = &P->zg;
  if (!strcmp(name, "wx")) v = &P->wx;
  if (!strcmp(name, "dx")) v = &P->dx;
  if (!strcmp(name, "dxt")) v = &P->dxt;
  if (!strcmp(name, "w3")) v = &P->w3;
  if (!strcmp(name, "g11")) v = &P->g11;
  if (!strcmp(name, "g22")) v = &P->g22;
  if (!strcmp(name, "g33")) v = &P->g33;
  if (!strcmp(name, "g12")) v = &P->g12;
  if (!strcmp(name, "g13")) v = &P->g13;
  if (!strcmp(name, "g23")) v = &P->g23;
  if (!strcmp(name, "jac")) v = &P->jac;
  if (!strcmp(name, "jacinv")) v = &P->jacinv;
  if (!strcmp(name, "drdx")) v = &P->drdx;
  if (!strcmp(name, "drdy")) v = &P->drdy;
  if (!strcmp(name, "drdz")) v = &P->drdz;
  if (!strcmp(name, "dsdx")) v = &P->dsdx;
  if (!strcmp(name, "dsdy")) v = &P->dsdy;
  if (!strcmp(name, "dsdz")) v = &P->dsdz;
  if (!strcmp(name, "dtdx")) v = &P->dtdx;
  if (!strcmp(name, "dtdy")) v = &P->dtdy;
  if (!strcmp(name, "dtdz")) v = &P->dtdz;
  if (!strcmp(name, "B")) v = &P->B;
  if (!strcmp(name, "mult")) v = &P->mult;
  if (!strcmp(name, "h1")) v = &P->h1;
  if (!strcmp(name, "h2")) v = &P->h2;
  if (v) std::memcpy(out, v->data(), v->size() * 8);
}
void or_set_f64(OrProblem *P, const char *name, const double *in) {
  std::vector<double> *v = nullptr;
  if (!strcmp(name, "x")) v = &P->x;
  if (!strcmp(name, "y")) v = &P->y;
  if (!strcmp(name, "z")) v = &P->z;
  if (!strcmp(name, "h1")) v = &P->h1;
  if (!strcmp(name, "h2")) v = &P->h2;
  if (v) std::memcpy(v->data(), in, v->size() * 8);
}
void or_set_ifh2(OrProblem *P, int ifh2) { P->ifh2 = ifh2 != 0; }

// fd_weights_full (src/math/fast3d.f90:105-163), c is (n+1) x (m+1).
void or_fd_weights_full(double xi, const double *x, int n, int m, double *c) {
  fd_weights_full(xi, x, n, m, c);
}
// zwgll / dgll (src/sem/speclib.f90:179-186, 880-919)
void or_zwgll(int np, double *z, double *w) { zwgll(z, w, np); }
void or_dgll(int nz, const double *z, double *d, double *dt) { dgll(d, dt, z, nz); }

void or_gs_add(OrProblem *P, double *u) {
  std::vector<double> v;
  gs_add(*P, u, v);
}

}  // extern "C"

// Solver half (Ax, bc, Jacobi, CG, hsmg) lives in neko_oracle_solve.cpp.
