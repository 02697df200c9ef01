// Host-side check of the gather-scatter warp layout (gs_relayout) and of the
// lane arithmetic of gs_add_warp_kernel, run on the CPU: for box meshes with
// and without masks and periodic directions, every chunk has 32 lanes with
// lane 0 a segment head, the lanes hold every map entry exactly once, and
// the in-warp sum (position from the head mask, running sum passed up one
// lane a step, total read from the segment's last lane) gives the same bits
// as the sequential gather of the item form.
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "nb_gs.h"

using namespace nb;

static int clz32(unsigned x) { return x ? __builtin_clz(x) : 32; }
static int ffs32(unsigned x) { return x ? __builtin_ctz(x) + 1 : 0; }

static int check(int nx, int ny, int nz, int lx, int per, bool mask, bool use_scale) {
  BoxSpec b{{nx, ny, nz}, {0, 0, 0}, {1, 1, 1}, {per, per, per}};
  std::vector<int> fn;
  box_facet_neigh(b, fn);
  GsMaps m;
  if (box_gs_maps(b, lx, fn, m) != 0) return 1;
  const long n = (long)nx * ny * nz * lx * lx * lx;
  std::vector<int> msk;
  std::vector<unsigned char> masked;
  if (mask) {
    box_boundary_mask(b, lx, fn, msk);
    masked.assign(n, 0);
    for (int q : msk) masked[q - 1] = 1;
  }
  GsHostLayout h;
  gs_relayout(m, masked, n, h);
  const long nchunk = (long)h.lane_head.size();
  if ((long)h.lane_idx.size() != 32 * nchunk || (long)h.lane_zero.size() != nchunk) {
    printf("chunk arrays of unequal sizes\n");
    return 1;
  }
  std::vector<int> seen(n, 0);
  for (int x : h.lane_idx)
    if (x >= 0) seen[x]++;
  long entries = 0;
  for (long i = 0; i < n; i++) {
    if (seen[i] > 1) {
      printf("point %ld in %d lanes\n", i, seen[i]);
      return 1;
    }
    entries += seen[i];
  }
  if (entries != m.nlocal) {
    printf("lanes hold %ld of %d entries\n", entries, m.nlocal);
    return 1;
  }
  std::mt19937_64 rng(7);
  std::uniform_real_distribution<double> U(-1, 1);
  std::vector<double> u(n), sc(n);
  for (auto &x : u) x = U(rng);
  for (auto &x : sc) x = U(rng);
  const double *scale = use_scale ? sc.data() : nullptr;
  std::vector<double> a = u, w = u;
  // item form: sequential sums in map order
  for (size_t p = 0; p < h.pairs.size(); p++) {
    const int2 pr = h.pairs[p];
    double s = a[pr.x] + a[pr.y];
    if (mask && h.pair_masked[p]) s = 0;
    a[pr.x] = scale ? s * scale[pr.x] : s;
    a[pr.y] = scale ? s * scale[pr.y] : s;
  }
  for (size_t q = 0; q + 1 < h.seg_ptr.size(); q++) {
    const int s0 = h.seg_ptr[q], s1 = h.seg_ptr[q + 1];
    double s = a[h.seg_idx[s0]];
    for (int k = s0 + 1; k < s1; k++) s = s + a[h.seg_idx[k]];
    if (mask && h.seg_masked[q]) s = 0;
    for (int k = s0; k < s1; k++) a[h.seg_idx[k]] = scale ? s * scale[h.seg_idx[k]] : s;
  }
  if (mask)
    for (int q : h.extra_mask) a[q] = 0;
  // warp form, one chunk at a time (chunks own disjoint points)
  for (long c = 0; c < nchunk; c++) {
    const unsigned head = h.lane_head[c];
    if (!(head & 1u)) {
      printf("chunk %ld: lane 0 is not a head\n", c);
      return 1;
    }
    double v[32], acc[32];
    int pos[32], last[32], idx[32], steps = 0;
    for (int l = 0; l < 32; l++) {
      idx[l] = h.lane_idx[32 * c + l];
      v[l] = idx[l] >= 0 ? w[idx[l]] : 0.0;
      const unsigned upto = 0xffffffffu >> (31 - l);
      pos[l] = l - (31 - clz32(head & upto));
      const unsigned above = head & ~upto;
      last[l] = above ? ffs32(above) - 2 : 31;
      if (idx[l] < 0 && pos[l] != 0) {
        printf("chunk %ld: padding lane %d inside a segment\n", c, l);
        return 1;
      }
      steps = pos[l] > steps ? pos[l] : steps;
      acc[l] = v[l];
    }
    for (int k = 1; k <= steps; k++) {
      double up[32];
      for (int l = 0; l < 32; l++) up[l] = l > 0 ? acc[l - 1] : acc[l];
      for (int l = 0; l < 32; l++)
        if (pos[l] == k) acc[l] = up[l] + v[l];
    }
    for (int l = 0; l < 32; l++) {
      double s = acc[last[l]];
      if (mask && ((h.lane_zero[c] >> l) & 1u)) s = 0;
      if (idx[l] >= 0) w[idx[l]] = scale ? s * scale[idx[l]] : s;
    }
  }
  for (int sg : h.seg_long) {
    const int s0 = h.seg_ptr[sg], s1 = h.seg_ptr[sg + 1];
    double s = w[h.seg_idx[s0]];
    for (int k = s0 + 1; k < s1; k++) s = s + w[h.seg_idx[k]];
    if (mask && h.seg_masked[sg]) s = 0;
    for (int k = s0; k < s1; k++) w[h.seg_idx[k]] = scale ? s * scale[h.seg_idx[k]] : s;
  }
  if (mask)
    for (int q : h.extra_mask) w[q] = 0;
  const bool same = memcmp(a.data(), w.data(), n * sizeof(double)) == 0;
  printf("%dx%dx%d lx %d periodic %d mask %d scale %d: %d entries, %ld chunks, %s\n", nx, ny, nz,
         lx, per, mask, use_scale, m.nlocal, nchunk, same ? "bit-identical" : "MISMATCH");
  return same ? 0 : 1;
}

int main() {
  int bad = 0;
  bad |= check(3, 4, 5, 8, 0, true, false);
  bad |= check(3, 4, 5, 8, 0, false, true);
  bad |= check(4, 4, 4, 6, 1, false, false);
  bad |= check(2, 3, 2, 2, 0, true, false);
  bad |= check(5, 3, 3, 5, 1, false, true);
  bad |= check(3, 3, 3, 7, 1, true, false);
  bad |= check(8, 8, 8, 8, 1, false, false);
  return bad;
}
