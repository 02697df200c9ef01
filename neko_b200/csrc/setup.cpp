// setup.cpp -- host-side setup of a structured box problem: GLL space,
// vertex coordinates, facet neighbours, gather-scatter maps and the
// zero-Dirichlet mask.
//
// The gather-scatter maps must be identical, entry for entry, to the ones
// the reference builds in gs_init_mapping (src/gs/gather_scatter.f90:
// 513-1375): same traversal (vertices, then edges, then faces with a
// neighbour), ids handed out in first-appearance order, the same Hoare
// quicksort (gather_scatter.f90:1291-1330) and the same block scan
// (gather_scatter.f90:1333-1373).  Those steps are kept.  What differs is how
// shared points are recognised: the reference numbers them through its mesh
// connectivity (point, edge and face hash tables, dofmap.f90:264-795); on a
// structured box every GLL point has a closed-form position on the global
// (lx-1)-refined lattice, wrapped in periodic directions, and that lattice
// index is the key.  Two local points share a key exactly when the
// reference gives them the same global dof, so the ids -- and therefore the
// maps -- coincide, while the lookup is a dense array instead of a hash.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <string>
#include <unordered_map>
#include <utility>

#include "nb_internal.h"

namespace nb {

namespace {

// Legendre polynomial P_n and its first derivative at x (three-term
// recurrence).
void legendre(int n, double x, double &p, double &dp) {
  double p0 = 1.0, p1 = x, d0 = 0.0, d1 = 1.0;
  if (n == 0) {
    p = 1.0;
    dp = 0.0;
    return;
  }
  for (int k = 1; k < n; k++) {
    double p2 = ((2.0 * k + 1.0) * x * p1 - k * p0) / (k + 1.0);
    double d2 = d0 + (2.0 * k + 1.0) * p1;  // P'_{k+1} = P'_{k-1} + (2k+1) P_k
    p0 = p1;
    p1 = p2;
    d0 = d1;
    d1 = d2;
  }
  p = p1;
  dp = d1;
}

}  // namespace

// GLL nodes are the roots of (1 - x^2) P'_N(x); interior ones are found by
// Newton's method on P'_N using P''_N from Legendre's equation
// (1 - x^2) P'' = 2 x P' - N (N+1) P, starting from the Chebyshev-Gauss-
// Lobatto points.  Weights 2 / (N (N+1) P_N(x_j)^2); the derivative matrix
// is the standard Lagrange-derivative closed form.
void gll_space(int lx, std::vector<double> &z, std::vector<double> &w,
               std::vector<double> &D, std::vector<double> &Dt) {
  const int N = lx - 1;
  z.assign(lx, 0.0);
  w.assign(lx, 0.0);
  D.assign(lx * lx, 0.0);
  Dt.assign(lx * lx, 0.0);
  if (lx == 1) return;
  const double pi = 3.14159265358979323846;
  z[0] = -1.0;
  z[N] = 1.0;
  for (int j = 1; j < N; j++) {
    double x = -std::cos(pi * j / N);
    for (int it = 0; it < 100; it++) {
      double p, dp;
      legendre(N, x, p, dp);
      double d2 = (2.0 * x * dp - N * (N + 1.0) * p) / (1.0 - x * x);
      double dx = dp / d2;
      x -= dx;
      if (std::fabs(dx) < 1e-16) break;
    }
    z[j] = x;
  }
  // Symmetrise: GLL nodes are symmetric about 0.
  for (int j = 0; j < lx / 2; j++) {
    double a = 0.5 * (z[N - j] - z[j]);
    z[j] = -a;
    z[N - j] = a;
  }
  if (lx % 2 == 1) z[N / 2] = 0.0;
  std::vector<double> pn(lx);
  for (int j = 0; j < lx; j++) {
    double p, dp;
    legendre(N, z[j], p, dp);
    pn[j] = p;
    w[j] = 2.0 / (N * (N + 1.0) * p * p);
  }
  const double d0 = N * (N + 1.0) / 4.0;
  for (int i = 0; i < lx; i++)
    for (int j = 0; j < lx; j++) {
      double v;
      if (i != j)
        v = pn[i] / (pn[j] * (z[i] - z[j]));
      else if (i == 0)
        v = -d0;
      else if (i == N)
        v = d0;
      else
        v = 0.0;
      D[i + lx * j] = v;
      Dt[j + lx * i] = v;
    }
}

// Element vertex coordinates: the box's grid lines are the running sums
// lo + h + h + ... (the same sums genmeshbox forms,
// contrib/genmeshbox/genmeshbox.f90:200-225), vertices in symmetric order.
void box_vertices(const BoxSpec &b, std::vector<double> &xyz8) {
  std::vector<double> c[3];
  for (int d = 0; d < 3; d++) {
    double h = (b.hi[d] - b.lo[d]) / b.nel[d];
    c[d].resize(b.nel[d] + 1);
    c[d][0] = b.lo[d];
    for (int i = 0; i < b.nel[d]; i++) c[d][i + 1] = c[d][i] + h;
  }
  const long nelv = (long)b.nel[0] * b.nel[1] * b.nel[2];
  xyz8.resize(nelv * 24);
  long e = 0;
  for (int ez = 0; ez < b.nel[2]; ez++)
    for (int ey = 0; ey < b.nel[1]; ey++)
      for (int ex = 0; ex < b.nel[0]; ex++, e++)
        for (int v = 0; v < 8; v++) {
          int ix = v & 1, iy = (v >> 1) & 1, iz = v >> 2;
          xyz8[e * 24 + v * 3 + 0] = c[0][ex + ix];
          xyz8[e * 24 + v * 3 + 1] = c[1][ey + iy];
          xyz8[e * 24 + v * 3 + 2] = c[2][ez + iz];
        }
}

// Neighbour across each face (face order -x,+x,-y,+y,-z,+z as in the
// reference hex, src/mesh/hex.f90:59-64), 1-based, 0 on a non-periodic
// boundary.
void box_facet_neigh(const BoxSpec &b, std::vector<int> &fn) {
  const int nx = b.nel[0], ny = b.nel[1], nz = b.nel[2];
  fn.assign((size_t)nx * ny * nz * 6, 0);
  auto id = [&](int x, int y, int z) { return 1 + x + nx * (y + ny * z); };
  const int n[3] = {nx, ny, nz};
  long e = 0;
  for (int ez = 0; ez < nz; ez++)
    for (int ey = 0; ey < ny; ey++)
      for (int ex = 0; ex < nx; ex++, e++) {
        int c[3] = {ex, ey, ez};
        for (int d = 0; d < 3; d++)
          for (int s = 0; s < 2; s++) {
            int q[3] = {c[0], c[1], c[2]};
            q[d] += s ? 1 : -1;
            if (q[d] < 0 || q[d] >= n[d]) {
              if (!b.periodic[d]) continue;
              q[d] = (q[d] + n[d]) % n[d];
            }
            fn[e * 6 + 2 * d + s] = id(q[0], q[1], q[2]);
          }
      }
}

namespace {

// Lattice key of local point (i,j,k) (1-based) of element e.
struct Lattice {
  long G[3];
  int nel[3], lx, per[3];
  explicit Lattice(const BoxSpec &b, int lx_) : lx(lx_) {
    for (int d = 0; d < 3; d++) {
      nel[d] = b.nel[d];
      per[d] = b.periodic[d];
      G[d] = (long)b.nel[d] * (lx - 1) + (per[d] ? 0 : 1);
    }
  }
  long key(int i, int j, int k, long e) const {
    long ex = e % nel[0], ey = (e / nel[0]) % nel[1], ez = e / ((long)nel[0] * nel[1]);
    long g[3] = {ex * (lx - 1) + i - 1, ey * (lx - 1) + j - 1, ez * (lx - 1) + k - 1};
    for (int d = 0; d < 3; d++)
      if (per[d] && g[d] >= G[d]) g[d] -= G[d];
    return g[0] + G[0] * (g[1] + G[1] * g[2]);
  }
};

inline long lin(int i, int j, int k, long e, int lx) {
  return (long)(i - 1) + (long)lx * ((j - 1) + (long)lx * ((k - 1) + (long)lx * e));
}

}  // namespace

// The gather-scatter maps of gs_init_mapping from a key per shared local
// point: two local points share a key exactly when the reference gives them
// the same global dof.  key(i, j, k, e) in [0, nkeys), 1-based (i,j,k).
template <class KeyFn>
static void gs_maps_from_keys(long nelv, int lx, const std::vector<int> &fn, long nkeys,
                              KeyFn key, GsMaps &g) {
  std::vector<int> idmap(nkeys, 0);
  int max_id = 0;
  std::vector<int> &dg = g.dof_gs;
  std::vector<int> &gd = g.gs_dof;
  dg.clear();
  gd.clear();
  const long nv = nelv * 8, ne = nelv * 12 * (long)(lx - 2);
  const long nf = nelv * 6 * (long)(lx - 2) * (lx - 2);
  dg.reserve(nv + ne + nf);
  gd.reserve(nv + ne + nf);
  auto push = [&](int i, int j, int k, long e) {
    int &id = idmap[key(i, j, k, e)];
    if (id == 0) id = ++max_id;
    dg.push_back(id);
    gd.push_back((int)(lin(i, j, k, e, lx) + 1));
  };
  // vertices (gather_scatter.f90:558-657)
  for (long e = 0; e < nelv; e++) {
    push(1, 1, 1, e);
    push(lx, 1, 1, e);
    push(1, lx, 1, e);
    push(lx, lx, 1, e);
    push(1, 1, lx, e);
    push(lx, 1, lx, e);
    push(1, lx, lx, e);
    push(lx, lx, lx, e);
  }
  // edges (gather_scatter.f90:662-865)
  for (long e = 0; e < nelv; e++) {
    const int c2[4][2] = {{1, 1}, {1, lx}, {lx, 1}, {lx, lx}};
    for (auto &c : c2)
      for (int t = 2; t <= lx - 1; t++) push(t, c[0], c[1], e);
    for (auto &c : c2)
      for (int t = 2; t <= lx - 1; t++) push(c[0], t, c[1], e);
    const int c3[4][2] = {{1, 1}, {lx, 1}, {1, lx}, {lx, lx}};
    for (auto &c : c3)
      for (int t = 2; t <= lx - 1; t++) push(c[0], c[1], t, e);
  }
  const int n_nonfacet = (int)dg.size();
  // face interiors of faces with a neighbour (gather_scatter.f90:960-1110)
  for (long e = 0; e < nelv; e++) {
    const int *f = &fn[e * 6];
    for (int side = 0; side < 6; side++) {
      if (f[side] == 0) continue;
      const int fix = (side & 1) ? lx : 1;
      for (int a = 2; a <= lx - 1; a++)
        for (int c = 2; c <= lx - 1; c++) {
          if (side < 2) push(fix, c, a, e);
          else if (side < 4) push(c, fix, a, e);
          else push(c, a, fix, e);
        }
    }
  }
  g.nlocal = (int)dg.size();
  g.facet_offset = n_nonfacet + 1;
  // Hoare quicksort with middle pivot, 1-based bounds (gather_scatter.f90:
  // 1291-1330).  Disjoint subranges, so an explicit stack gives the same
  // permutation as the recursion.
  int *DG = dg.data() - 1, *GD = gd.data() - 1;
  std::vector<std::pair<int, int>> st;
  if (g.nlocal > 1) st.push_back({1, g.nlocal});
  while (!st.empty()) {
    const int lo = st.back().first, hi = st.back().second;
    st.pop_back();
    int i = lo - 1, j = hi + 1;
    const int pivot = DG[(lo + hi) / 2];
    for (;;) {
      do { ++i; } while (DG[i] < pivot);
      do { --j; } while (DG[j] > pivot);
      if (i < j) {
        std::swap(DG[i], DG[j]);
        std::swap(GD[i], GD[j]);
      } else {
        if (i == j) ++i;
        break;
      }
    }
    if (lo < j) st.push_back({lo, j});
    if (i < hi) st.push_back({i, hi});
  }
  // Runs of equal id over the non-facet part (gather_scatter.f90:1333-1373).
  g.blk_len.clear();
  for (int i = 1; i < g.facet_offset;) {
    int j = i;
    while (j + 1 <= g.nlocal && DG[j + 1] == DG[i]) ++j;
    g.blk_len.push_back(j - i + 1);
    i = j + 1;
  }
  g.blk_off.assign(g.blk_len.size(), 0);
  for (size_t k = 1; k < g.blk_len.size(); k++) g.blk_off[k] = g.blk_off[k - 1] + g.blk_len[k - 1];
}

int box_gs_maps(const BoxSpec &b, int lx, const std::vector<int> &fn, GsMaps &g) {
  const long nelv = (long)b.nel[0] * b.nel[1] * b.nel[2];
  Lattice L(b, lx);
  gs_maps_from_keys(nelv, lx, fn, L.G[0] * L.G[1] * L.G[2],
                    [&](int i, int j, int k, long e) { return L.key(i, j, k, e); }, g);
  return 0;
}

// A local point is zero-Dirichlet when it lies on a face without a
// neighbour; on the box that is a lattice plane at a non-periodic boundary.
// Same set as bc_finalize_base (src/bc/bc.f90:434-593), ascending.
void box_boundary_mask(const BoxSpec &b, int lx, const std::vector<int> &fn,
                       std::vector<int> &msk) {
  (void)fn;
  const long nelv = (long)b.nel[0] * b.nel[1] * b.nel[2];
  msk.clear();
  Lattice L(b, lx);
  for (long e = 0; e < nelv; e++) {
    long ec[3] = {e % b.nel[0], (e / b.nel[0]) % b.nel[1], e / ((long)b.nel[0] * b.nel[1])};
    for (int k = 1; k <= lx; k++)
      for (int j = 1; j <= lx; j++)
        for (int i = 1; i <= lx; i++) {
          int loc[3] = {i, j, k};
          bool on = false;
          for (int d = 0; d < 3 && !on; d++) {
            if (b.periodic[d]) continue;
            long gcoord = ec[d] * (lx - 1) + loc[d] - 1;
            on = gcoord == 0 || gcoord == L.G[d] - 1;
          }
          if (on) msk.push_back((int)(lin(i, j, k, e, lx) + 1));
        }
  }
}

// ---------------------------------------------------------------------------
// Unstructured hexahedral meshes given by the caller: eight global vertex
// ids per element (periodic partners already sharing ids) in the reference's
// symmetric vertex order.
// ---------------------------------------------------------------------------

// Vertices of each face and each edge of the reference hex
// (face_nodes / edge_nodes, src/mesh/hex.f90:93-106, 113-127), 1-based.
static const int kHexFaceNodes[6][4] = {{1, 5, 7, 3}, {2, 6, 8, 4}, {1, 2, 6, 5},
                                        {3, 4, 8, 7}, {1, 2, 4, 3}, {5, 6, 8, 7}};
static const int kHexEdgeNodes[12][2] = {{1, 2}, {3, 4}, {5, 6}, {7, 8}, {1, 3}, {2, 4},
                                         {5, 7}, {6, 8}, {1, 5}, {2, 6}, {3, 7}, {4, 8}};

namespace {
struct ArrHash4 {
  size_t operator()(const std::array<int, 4> &a) const {
    size_t h = 1469598103934665603ull;
    for (int v : a) h = (h ^ (size_t)(unsigned)v) * 1099511628211ull;
    return h;
  }
};
struct PairHash {
  size_t operator()(const std::pair<int, int> &p) const {
    return ((size_t)(unsigned)p.first << 32) ^ (size_t)(unsigned)p.second;
  }
};
// vertex (1-based, symmetric order) at corner (i,j,k) of an lx^3 element
inline int corner_vertex(int i, int j, int k, int lx) {
  return 1 + (i == lx ? 1 : 0) + (j == lx ? 2 : 0) + (k == lx ? 4 : 0);
}
}  // namespace

int mesh_connectivity(long nelv, const int *ids, MeshConn &c, std::string &err) {
  c.fn.assign(nelv * 6, 0);
  c.face_gid.assign(nelv * 6, 0);
  c.edge_gid.assign(nelv * 12, 0);
  c.max_vid = 0;
  for (long q = 0; q < nelv * 8; q++) {
    if (ids[q] <= 0) {
      err = "vertex ids must be positive";
      return 1;
    }
    c.max_vid = std::max(c.max_vid, ids[q]);
  }
  for (long e = 0; e < nelv; e++)
    for (int a = 0; a < 8; a++)
      for (int b = a + 1; b < 8; b++)
        if (ids[e * 8 + a] == ids[e * 8 + b]) {
          err = "element " + std::to_string(e + 1) + " repeats a vertex id";
          return 1;
        }
  // faces and edges numbered in order of first appearance
  // (mesh_generate_conn, src/mesh/mesh.f90:476-687); a face key is its four
  // sorted vertex ids, an edge key its two.
  std::unordered_map<std::array<int, 4>, std::array<long, 3>, ArrHash4> faces;  // id, e1, e2
  std::unordered_map<std::pair<int, int>, int, PairHash> edges;
  int nf = 0, ne = 0;
  for (long e = 0; e < nelv; e++) {
    for (int f = 0; f < 6; f++) {
      std::array<int, 4> k;
      for (int v = 0; v < 4; v++) k[v] = ids[e * 8 + kHexFaceNodes[f][v] - 1];
      std::sort(k.begin(), k.end());
      auto it = faces.find(k);
      if (it == faces.end()) {
        faces.emplace(k, std::array<long, 3>{nf, e + 1, 0});
        c.face_gid[e * 6 + f] = nf++;
      } else {
        if (it->second[2] != 0 || it->second[1] == e + 1) {
          err = "a face is shared by more than two element faces";
          return 1;
        }
        it->second[2] = e + 1;
        c.face_gid[e * 6 + f] = (int)it->second[0];
      }
    }
    for (int q = 0; q < 12; q++) {
      int a = ids[e * 8 + kHexEdgeNodes[q][0] - 1], b = ids[e * 8 + kHexEdgeNodes[q][1] - 1];
      std::pair<int, int> k = a < b ? std::make_pair(a, b) : std::make_pair(b, a);
      auto it = edges.find(k);
      if (it == edges.end()) {
        edges.emplace(k, ne);
        c.edge_gid[e * 12 + q] = ne++;
      } else {
        c.edge_gid[e * 12 + q] = it->second;
      }
    }
  }
  c.nfaces = nf;
  c.nedges = ne;
  // neighbour across each face: the other element holding the same face
  for (long e = 0; e < nelv; e++)
    for (int f = 0; f < 6; f++) {
      std::array<int, 4> k;
      for (int v = 0; v < 4; v++) k[v] = ids[e * 8 + kHexFaceNodes[f][v] - 1];
      std::sort(k.begin(), k.end());
      const std::array<long, 3> &r = faces.at(k);
      c.fn[e * 6 + f] = (int)(r[1] == e + 1 ? r[2] : r[1]);
    }
  return 0;
}

// Key of a shared local point: vertices by id, edge interiors by edge and
// position from the lower-id end, face interiors by face and position in a
// frame fixed by the face's vertex ids (origin at the lowest id, first axis
// towards its lower-id neighbour corner), the same position from either
// element whatever the relative rotation or mirroring of the two faces.
// Equal keys are exactly the local points the reference's dofmap numbering
// (src/sem/dofmap.f90:264-771) gives one global dof.
struct MeshKeys {
  const int *ids;
  const MeshConn *c;
  int lx;
  long off_e, off_f, nkeys;
  MeshKeys(const int *ids_, const MeshConn &c_, int lx_) : ids(ids_), c(&c_), lx(lx_) {
    const long m = lx - 2;
    off_e = (long)c_.max_vid + 1;
    off_f = off_e + (long)c_.nedges * m;
    nkeys = off_f + (long)c_.nfaces * m * m;
  }
  int vid(long e, int v) const { return ids[e * 8 + v - 1]; }
  long operator()(int i, int j, int k, long e) const {
    const int L = lx;
    const int loc[3] = {i, j, k};
    int nb = 0;
    for (int d = 0; d < 3; d++) nb += (loc[d] == 1 || loc[d] == L);
    if (nb == 3) return vid(e, corner_vertex(i, j, k, L));
    if (nb == 2) {
      int d = 0;
      while (loc[d] == 1 || loc[d] == L) d++;  // the free direction
      int a[3] = {i, j, k}, b[3] = {i, j, k};
      a[d] = 1;
      b[d] = L;
      const int va = corner_vertex(a[0], a[1], a[2], L), vb = corner_vertex(b[0], b[1], b[2], L);
      int q = 0;
      while (!((kHexEdgeNodes[q][0] == va && kHexEdgeNodes[q][1] == vb) ||
               (kHexEdgeNodes[q][0] == vb && kHexEdgeNodes[q][1] == va)))
        q++;
      const int t = loc[d];
      const long p = vid(e, va) < vid(e, vb) ? t - 2 : L - 1 - t;
      return off_e + (long)c->edge_gid[e * 12 + q] * (L - 2) + p;
    }
    // face interior: fixed direction d, free directions u < v
    int d = 0;
    while (!(loc[d] == 1 || loc[d] == L)) d++;
    const int side = 2 * d + (loc[d] == L ? 1 : 0);
    const int u = d == 0 ? 1 : 0, v = d == 2 ? 1 : 2;
    auto cv = [&](int cu, int cvv) {
      int p[3] = {i, j, k};
      p[u] = cu;
      p[v] = cvv;
      return vid(e, corner_vertex(p[0], p[1], p[2], L));
    };
    // corners (u, v) in {1, L}^2 and the one with the lowest id
    const int cu[4] = {1, L, 1, L}, cw[4] = {1, 1, L, L};
    int o = 0;
    for (int q = 1; q < 4; q++)
      if (cv(cu[q], cw[q]) < cv(cu[o], cw[o])) o = q;
    const int ou = cu[o], ow = cw[o];
    const int nu = cv(ou == 1 ? L : 1, ow), nw = cv(ou, ow == 1 ? L : 1);
    const long du = ou == 1 ? loc[u] - 2 : L - 1 - loc[u];
    const long dw = ow == 1 ? loc[v] - 2 : L - 1 - loc[v];
    const long m = L - 2;
    const long pq = nu < nw ? du * m + dw : dw * m + du;
    return off_f + (long)c->face_gid[e * 6 + side] * m * m + pq;
  }
};

int mesh_gs_maps(long nelv, const int *ids, const MeshConn &c, int lx, GsMaps &g) {
  MeshKeys K(ids, c, lx);
  gs_maps_from_keys(nelv, lx, c.fn, K.nkeys, K, g);
  return 0;
}

// Local points on faces without a neighbour, ascending (1-based).
void mesh_boundary_mask(long nelv, int lx, const std::vector<int> &fn, std::vector<int> &msk) {
  const long L3 = (long)lx * lx * lx;
  std::vector<unsigned char> mark(nelv * L3, 0);
  for (long e = 0; e < nelv; e++)
    for (int side = 0; side < 6; side++) {
      if (fn[e * 6 + side]) continue;
      const int d = side >> 1, fix = (side & 1) ? lx : 1;
      for (int a = 1; a <= lx; a++)
        for (int b = 1; b <= lx; b++) {
          int p[3];
          p[d] = fix;
          p[d == 0 ? 1 : 0] = a;
          p[d == 2 ? 1 : 2] = b;
          mark[lin(p[0], p[1], p[2], e, lx)] = 1;
        }
    }
  msk.clear();
  for (long q = 0; q < nelv * L3; q++)
    if (mark[q]) msk.push_back((int)(q + 1));
}

// True when every neighbour across face f is reached through its opposite
// face f^1 with the same vertex ids at the same face positions, so the
// element's and its neighbour's face parametrisations coincide (a
// structured-type mesh without rotated elements).
bool mesh_faces_aligned(long nelv, const int *ids, const std::vector<int> &fn) {
  for (long e = 0; e < nelv; e++)
    for (int f = 0; f < 6; f++) {
      const int nb = fn[e * 6 + f];
      if (!nb) continue;
      const long n = nb - 1;
      const int g = f ^ 1;
      if (fn[n * 6 + g] != e + 1) return false;
      for (int v = 0; v < 4; v++)
        if (ids[e * 8 + kHexFaceNodes[f][v] - 1] != ids[n * 8 + kHexFaceNodes[g][v] - 1])
          return false;
    }
  return true;
}

}  // namespace nb
