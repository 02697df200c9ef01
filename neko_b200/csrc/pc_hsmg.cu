// pc_hsmg.cu -- three-level hybrid Schwarz multigrid preconditioner on the
// device: the additive V-cycle of hsmg_solve (src/krylov/pc_hsmg.f90:
// 574-625, CPU order) with levels lx -> 4 -> 2 (pc_hsmg.f90:208-219),
// overlapping Schwarz + FDM smoothing on the fine and middle levels
// (src/math/schwarz.f90:506-596) and a Jacobi-CG coarse solve of
// `coarse_iter` iterations.
//
// B200 form of the Schwarz step.  The reference builds extended
// (lx+2)^3 elements, fills the ghost layer through a gather-scatter on a
// second (lx+2)-point numbering of the mesh plus four extrude passes, runs
// the FDM, and routes the ghost results back the same way.  On the
// structured box every element face has the same orientation as its
// neighbour's, so those exchanges are direct: the FDM kernel reads its
// ghost layer straight from the neighbours' first interior layer of the
// input, and the post kernel adds the neighbours' ghost results to its own
// first interior layer.  The FDM kernel keeps the whole extended element in
// shared memory for its six tensor passes and rebuilds the inverse
// eigenvalue sums from the three per-direction spectra, so it reads
// 3 nl^2 + 3 nl values of factors per element instead of nl^3.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

#include "nb_hsmg.h"
#include "nb_kernels.h"
#include "nb_precond.h"
#include "nb_problem.h"
#include "nb_reduce.cuh"

namespace nb {

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------

// Orientation of a face pairing (general meshes): bits 0-2 the neighbour's
// face nf, bit 3 swaps the two in-face coordinates, bits 4 and 5 reverse the
// first / second.  Maps the position (s1, s2) (1-based, 1..lx; s1 along the
// lower of the two in-face axes) on this element's face to (t1, t2) on the
// neighbour's face nf.
__device__ __forceinline__ void face_map(unsigned code, int lx, int s1, int s2, int &nf, int &t1,
                                         int &t2) {
  nf = code & 7;
  int u1 = (code & 8) ? s2 : s1, u2 = (code & 8) ? s1 : s2;
  t1 = (code & 16) ? lx + 1 - u1 : u1;
  t2 = (code & 32) ? lx + 1 - u2 : u2;
}

// e = S (D^-1) S' r on the extended element (NL = lx + 2 points a side),
// ghost layer gathered from the neighbours (fn: 1-based neighbour per face,
// 0 = none).  One block (one warp; two for NL >= 13) per element holds the
// element in shared memory and runs the six tensor passes; for NL <= 7 one
// warp holds four elements, eight lanes each.  Each pass
// contracts the first index and writes its result with that index moved
// last (out(m,n,i) = sum_l M(i,l) in(l,m,n)), so after three passes the
// order is back to (i,j,k).  A lane owns M lines of the pass and all NL
// outputs of each: for every l it reads its M line values and the NL matrix
// entries M(., l), which are the same for the whole warp (broadcast reads),
// and updates M*NL independent sums, so a matrix read serves M lines.  Lines
// sit at pos(t, l) = NLP t + C (t >> G) + l, the padding chosen per NL so
// that the consecutive lines of a warp's reads and rotated writes fall in
// distinct banks.  The D^-1 scaling of the third forward pass is applied to
// each value as the first backward pass reads it (the same product, stored
// one pass later).  The ghost-layer gather and the factor loads are
// asynchronous copies straight into shared memory (zero-filled where a face
// has no neighbour) when the input needs no conversion.  Every sum runs over
// l in ascending order from zero; the eigenvalue scaling multiplies by
// 1/diag, zero where the sum of the three spectra is <= eps
// (fdm_setup_fast, src/math/fdm.f90:373-393).
template <typename T, int NL>
struct FdmCfg {
  static constexpr int N2 = NL * NL, N3 = N2 * NL;
  // small elements share a warp: EPW elements of LPE lanes each
  static constexpr int EPW = NL <= 7 ? 4 : 1;
  static constexpr int W = EPW > 1 ? 1 : ((N2 + 31) / 32) * NL <= 64 ? 1 : 2;  // warps
  static constexpr int TPE = 32 * W;                             // threads per block
  static constexpr int LPE = TPE / EPW;                          // lanes per element
  static constexpr int M = (N2 + LPE - 1) / LPE;                 // lines per lane
  static constexpr int LA = (N2 + M - 1) / M;                    // lanes with lines
  static constexpr int NLP = NL == 16 ? 17 : NL;
  static constexpr int G = NL == 8 ? 2 : NL == 12 ? 3 : 4;
  static constexpr int C = (NL % 2 == 0 && NL != 16) ? 1 : 0;
  static constexpr int BUF = (NLP * (N2 - 1) + ((N2 - 1) >> G) * C + NL + 1) / 2 * 2;
  // One element a block: the matrices are kept twice, each row l of the
  // forward (S(l, .)) and backward (S(., l)) forms contiguous with a pitch of
  // whole 16-byte vectors, so a lane reads a row with NL*sizeof(T)/16 vector
  // loads instead of NL scalar ones.
  static constexpr bool VEC = EPW == 1;
  static constexpr int VW = 16 / (int)sizeof(T);            // values per vector
  static constexpr int NLR = (NL + VW - 1) / VW * VW;        // row pitch
  // FP32 one-element blocks pass in place: every lane reads its lines, the
  // block meets at a barrier, then the rotated output overwrites the same
  // buffer; the second buffer shrinks to the matrix staging area (3 N2), so
  // more blocks fit an SM.  FP64 keeps two buffers (its registers, not its
  // shared memory, bound its residency).
  static constexpr bool INPLACE = VEC && sizeof(T) == 4;
  static constexpr int BUF2 = INPLACE ? (3 * N2 + 1) / 2 * 2 : BUF;
  static constexpr int OFFM = (BUF + BUF2 + VW - 1) / VW * VW;  // matrices, aligned
  static_assert(!INPLACE || BUF2 >= 3 * N2, "the staging area holds the three raw matrices");
  static constexpr int MAT = VEC ? 6 * NL * NLR : 3 * N2;
  static constexpr int STR0 = VEC ? OFFM + MAT + 3 * NL + 1 : 2 * BUF + 3 * N2 + 3 * NL + 1;
  // per-element stride; with several elements in a warp it is 9 mod 16
  // values, which keeps the line reads of neighbouring elements in distinct banks
  static constexpr int STR = EPW > 1 ? STR0 + ((9 - STR0 % 16) + 16) % 16 : STR0;
  static constexpr size_t SMEM = ((size_t)EPW * STR * sizeof(T) + 15) / 16 * 16;
  // resident blocks per SM the register allocation is sized for: what the
  // shared memory allows (228 KB, 1 KB reserved per block), fewer if the
  // M x NL sums and the operands in flight would not fit in the registers
  static constexpr int OCC = (int)(233472 / (SMEM + 1024));
  static constexpr int REGS = sizeof(T) == 8 ? 3 * M * NL + 48 : 2 * M * NL + 4;
  static constexpr int RB = 65536 / (TPE * REGS);
  static constexpr int MINB0 = OCC < RB ? OCC : RB;
  static constexpr int MINB = MINB0 < 1 ? 1 : MINB0 > 32 / W ? 32 / W : MINB0;
  __device__ static __forceinline__ int pos(int t, int l) { return NLP * t + (t >> G) * C + l; }
};

template <typename T>
__device__ __forceinline__ void cp_async_elem(T *sdst, const T *gsrc, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(sa), "l"(gsrc),
               "n"((int)sizeof(T)), "r"(valid ? (int)sizeof(T) : 0)
               : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// shared[dst] = (T) global[src] (zero when !valid): an asynchronous copy when
// no conversion is needed, else a load and a store.
template <typename TIN, typename T>
__device__ __forceinline__ void gather_elem(T *dst, const TIN *src, bool valid) {
  if constexpr (std::is_same<TIN, T>::value)
    cp_async_elem<T>(dst, src, valid);
  else
    *dst = valid ? (T)__ldg(src) : T(0);
}

// One pass over the element: FWD contracts with S(l,i) at Sd[l + NL*i],
// otherwise with S(i,l) at Sd[i + NL*l].  SCALE multiplies each value read
// by D^-1 (the first backward pass reads the third forward pass's output);
// `out` != nullptr writes the natural (i,j,k) order to global memory (last
// pass) instead of the rotated shared-memory layout.
template <typename T, int NL, bool FWD, bool SCALE>
__device__ __forceinline__ void fdm_pass(const T *__restrict__ src, T *__restrict__ dst,
                                         const T *__restrict__ Sd, const T *__restrict__ sL,
                                         T *__restrict__ out, int u) {
  using C = FdmCfg<T, NL>;
  constexpr int N2 = C::N2, M = C::M, LA = C::LA;
  // in place (src == dst), lanes without lines still meet the barrier
  // between the reads and the writes
  if (!C::INPLACE && u >= LA) return;
  const bool lines = u < LA;
  T o[M][NL];
  int base[M];
  T ljk[M];  // SCALE: spectra sum of the line's second index, added to the first's
  T lz[M];
  const T ep = sL[3 * NL];
#pragma unroll
  for (int j = 0; j < M; j++) {
    const int t = u + LA * j, tt = (LA * M == N2 || t < N2) ? t : N2 - 1;
    base[j] = C::pos(tt, 0);
    if (SCALE) {
      ljk[j] = sL[NL + tt % NL];
      lz[j] = sL[2 * NL + tt / NL];
    }
#pragma unroll
    for (int i = 0; i < NL; i++) o[j][i] = T(0);
  }
#pragma unroll 2
  for (int l = 0; l < (lines ? NL : 0); l++) {
    T x[M];
#pragma unroll
    for (int j = 0; j < M; j++) {
      x[j] = src[base[j] + l];
      if (SCALE) {  // (lx + ly) + lz, as the third forward pass forms it
        const T d = (sL[l] + ljk[j]) + lz[j];
        x[j] = x[j] * (d > ep ? T(1) / d : T(0));
      }
    }
    if constexpr (C::VEC) {
      // row l of the pass's matrix in 16-byte vector loads (broadcast)
      T mr[C::NLR];
      using V = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
      const V *row = reinterpret_cast<const V *>(Sd + C::NLR * l);
#pragma unroll
      for (int q = 0; q < C::NLR / C::VW; q++) reinterpret_cast<V *>(mr)[q] = row[q];
#pragma unroll
      for (int i = 0; i < NL; i++) {
#pragma unroll
        for (int j = 0; j < M; j++) o[j][i] += mr[i] * x[j];
      }
    } else {
#pragma unroll
      for (int i = 0; i < NL; i++) {
        const T mv = Sd[FWD ? l + NL * i : i + NL * l];
#pragma unroll
        for (int j = 0; j < M; j++) o[j][i] += mv * x[j];
      }
    }
  }
  if constexpr (C::INPLACE) {
    if (!out) __syncthreads();  // every read of src done before dst (= src) is written
    if (!lines) return;
  }
#pragma unroll
  for (int j = 0; j < M; j++) {
    const int t = u + LA * j;
    if (LA * M != N2 && t >= N2) continue;
    if (out) {
#pragma unroll
      for (int k = 0; k < NL; k++) out[t + N2 * k] = o[j][k];
    } else {
      const int m = t % NL, n = t / NL;
#pragma unroll
      for (int i = 0; i < NL; i++) dst[C::pos(n + NL * i, m)] = o[j][i];
    }
  }
}

template <typename TIN, typename T, int NL>
__global__ void __launch_bounds__(FdmCfg<T, NL>::TPE, FdmCfg<T, NL>::MINB)
    fdm_kernel(const TIN *__restrict__ r, const int *__restrict__ fn,
               const unsigned char *__restrict__ ornt, const T *__restrict__ S,
               const T *__restrict__ lam, const T *__restrict__ eps, T *__restrict__ out,
               int nelv, const int *__restrict__ skip) {
  if (skip && *skip) return;
  using C = FdmCfg<T, NL>;
  constexpr int LX = NL - 2, L2 = LX * LX, L3 = L2 * LX, N2 = C::N2, N3 = C::N3;
  extern __shared__ __align__(16) unsigned char fdm_smem[];
  const int es = threadIdx.x / C::LPE, ul = threadIdx.x - es * C::LPE;
  T *b0 = reinterpret_cast<T *>(fdm_smem) + es * C::STR, *b1 = b0 + C::BUF;
  // scalar form: S_x, S_y, S_z with S(l,i) at l + NL*i; vector form: the
  // forward rows (S(l, i) at i + NLR*l) then the backward rows (S(i, l) at
  // i + NLR*l), the factors staged in b1 first
  T *sS = C::VEC ? b0 + C::OFFM : b1 + C::BUF;
  T *sL = sS + C::MAT;  // spectra + eps
  T *stage = C::VEC ? b1 : sS;
  const long e = (long)blockIdx.x * C::EPW + es;
  if ((long)blockIdx.x * C::EPW >= nelv) return;
  const bool active = e < nelv;
  const int u = active ? ul : C::LPE;  // lanes of a missing element do no work
  constexpr int LPE = C::LPE;
  if (active) {
    const TIN *re = r + e * L3;
#pragma unroll 4
    for (int q = u; q < L3; q += LPE) {  // interior: ext(a+1, b+1, c+1) = r(a, b, c)
      const int a = q % LX, b = (q / LX) % LX, c = q / L2;
      gather_elem<TIN, T>(b0 + C::pos((b + 1) + NL * (c + 1), a + 1), re + q, true);
    }
#pragma unroll 2
    for (int q = u; q < 6 * L2; q += LPE) {  // faces: the neighbour's first interior layer
      const int f = q / L2, w = q - f * L2, s1 = w % LX + 1, s2 = w / LX + 1, dir = f >> 1;
      const int cb = (f & 1) ? NL - 1 : 0;   // ghost coordinate across the face
      const int a = dir == 0 ? cb : s1, b = dir == 1 ? cb : (dir == 0 ? s1 : s2),
                c = dir == 2 ? cb : s2;
      // its source: the neighbour's first interior layer behind its face nf,
      // at the face position (t1, t2) of (s1, s2) in the neighbour's frame
      int nf = f ^ 1, t1 = s1, t2 = s2;
      if (ornt) face_map(__ldg(ornt + e * 6 + f), LX, s1, s2, nf, t1, t2);
      const int ndir = nf >> 1, cs = (nf & 1) ? LX - 1 : 2;
      const int sa = ndir == 0 ? cs : t1, sb = ndir == 1 ? cs : (ndir == 0 ? t1 : t2),
                sc = ndir == 2 ? cs : t2;
      const int nb = __ldg(fn + e * 6 + f);
      gather_elem<TIN, T>(b0 + C::pos(b + NL * c, a),
                          nb ? r + (long)(nb - 1) * L3 + (sa - 1) + LX * (sb - 1) + L2 * (sc - 1)
                             : r,
                          nb != 0);
    }
    for (int q = u; q < 12 * LX + 8; q += LPE) {  // edges and corners: zero
      int a, b, c;
      if (q < 12 * LX) {
        const int E = q / LX, s = q - E * LX + 1, D = E >> 2;
        const int c1 = (E & 1) ? NL - 1 : 0, c2 = (E & 2) ? NL - 1 : 0;
        a = D == 0 ? s : c1;
        b = D == 1 ? s : (D == 0 ? c1 : c2);
        c = D == 2 ? s : c2;
      } else {
        const int k = q - 12 * LX;
        a = (k & 1) ? NL - 1 : 0;
        b = (k & 2) ? NL - 1 : 0;
        c = (k & 4) ? NL - 1 : 0;
      }
      b0[C::pos(b + NL * c, a)] = T(0);
    }
    for (int q = u; q < 3 * N2; q += LPE) cp_async_elem<T>(stage + q, S + e * 3 * N2 + q, true);
    for (int q = u; q < 3 * NL; q += LPE) cp_async_elem<T>(sL + q, lam + e * 3 * NL + q, true);
    if (u == 0) cp_async_elem<T>(sL + 3 * NL, eps + e, true);
  }
  cp_async_wait_all();
  __syncthreads();
  // matrix of direction d for the forward / backward passes
  constexpr int MS = C::VEC ? NL * C::NLR : N2;
  T *fwd = sS, *bwd = C::VEC ? sS + 3 * MS : sS;
  if constexpr (C::VEC) {
    if (active)
      for (int q = u; q < 3 * N2; q += LPE) {
        const int d = q / N2, r = q - d * N2, a = r % NL, b = r / NL;
        const T v = stage[q];  // S_d(a, b)
        fwd[d * MS + b + C::NLR * a] = v;
        bwd[d * MS + a + C::NLR * b] = v;
      }
    __syncthreads();
  }
  // forward: b0 -> b1 -> b0 -> b1; backward (D^-1 on the first read): b1 -> b0 -> b1 -> out
  // (in place: b0 -> b0 throughout)
  if constexpr (C::INPLACE) b1 = b0;
  fdm_pass<T, NL, true, false>(b0, b1, fwd, sL, nullptr, u);
  __syncthreads();
  fdm_pass<T, NL, true, false>(b1, b0, fwd + MS, sL, nullptr, u);
  __syncthreads();
  fdm_pass<T, NL, true, false>(b0, b1, fwd + 2 * MS, sL, nullptr, u);
  __syncthreads();
  fdm_pass<T, NL, false, true>(b1, b0, bwd, sL, nullptr, u);
  __syncthreads();
  fdm_pass<T, NL, false, false>(b0, b1, bwd + MS, sL, nullptr, u);
  __syncthreads();
  fdm_pass<T, NL, false, false>(b1, nullptr, bwd + 2 * MS, sL, out + e * N3, u);
}

// e(i,j,k) = ext interior + neighbours' ghost results on the first interior
// layers (x, then y, then z, as the extrude passes add them), times the
// overlap weight, for point q of element e.  The neighbour table is read up
// front and every operand load is issued before the first add, so a thread
// waits on one round trip.
template <typename T, int LX>
__device__ __forceinline__ T schwarz_post_point(const T *__restrict__ ext,
                                                const int *__restrict__ fn,
                                                const unsigned char *__restrict__ ornt,
                                                const T *__restrict__ wt, long e, int q) {
  constexpr int NL = LX + 2, L2 = LX * LX, L3 = L2 * LX, N2 = NL * NL, N3 = N2 * NL;
  const int i = q % LX, j = (q / LX) % LX, k = q / L2;
  const int2 *f2 = reinterpret_cast<const int2 *>(fn + e * 6);
  const int2 fa = __ldg(f2), fb = __ldg(f2 + 1), fc = __ldg(f2 + 2);
  const int f[6] = {fa.x, fa.y, fb.x, fb.y, fc.x, fc.y};
  // the six candidate neighbour contributions: (condition, address)
  const bool c[6] = {i == 1 && f[0], i == LX - 2 && f[1], j == 1 && f[2],
                     j == LX - 2 && f[3], k == 1 && f[4], k == LX - 2 && f[5]};
  const long in = (long)NL * (j + 1) + (long)N2 * (k + 1), jn = (i + 1) + (long)N2 * (k + 1),
             kn = (i + 1) + (long)NL * (j + 1);
  long off[6] = {(NL - 1) + in, 0 + in, NL * (NL - 1) + jn, 0 + jn, N2 * (NL - 1) + kn,
                 0 + kn};
  if (ornt) {  // general mesh: the ghost result sits on the neighbour's face nf
#pragma unroll
    for (int d = 0; d < 6; d++) {
      if (!c[d]) continue;
      const int dir = d >> 1;
      const int s1 = (dir == 0 ? j : i) + 1, s2 = (dir == 2 ? j : k) + 1;
      int nf, t1, t2;
      face_map(__ldg(ornt + e * 6 + d), LX, s1, s2, nf, t1, t2);
      const int nd = nf >> 1, cg = (nf & 1) ? NL - 1 : 0;
      const int a = nd == 0 ? cg : t1, b = nd == 1 ? cg : (nd == 0 ? t1 : t2),
                cc = nd == 2 ? cg : t2;
      off[d] = a + (long)NL * b + (long)N2 * cc;
    }
  }
  T g[6];
#pragma unroll
  for (int d = 0; d < 6; d++) g[d] = c[d] ? ext[(long)(f[d] - 1) * N3 + off[d]] : T(0);
  T v = ext[e * N3 + (i + 1) + NL * (j + 1) + N2 * (k + 1)];
  const T w = wt[e * L3 + q];
#pragma unroll
  for (int d = 0; d < 6; d++)
    if (c[d]) v += g[d];
  return v * w;
}

template <typename T, int LX>
__global__ void __launch_bounds__(256)
    schwarz_post_kernel(const T *__restrict__ ext, const int *__restrict__ fn,
                        const unsigned char *__restrict__ ornt, const T *__restrict__ wt,
                        T *__restrict__ out, long nelv, const int *__restrict__ skip) {
  if (skip && *skip) return;
  constexpr int L3 = LX * LX * LX;
  const long p = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (p >= nelv * L3) return;
  const long e = p / L3;
  out[p] = schwarz_post_point<T, LX>(ext, fn, ornt, wt, e, (int)(p - e * L3));
}

// out = (A x A x A) in per element, A(o, i) = TR ? M[i + NI*o] : M[o + NO*i];
// without ACC the input is multiplied by `scale` first when given; ACC adds
// the result to out, times `scale` at the output point when given.
// Computed in T; input/output converted on load/store.  One element per
// block of kT3Threads threads; every per-thread loop has a compile-time trip
// count, so a thread's global loads are all in flight together.
constexpr int kT3Threads = 128;

// With DOT (prolongation into the unassembled fine-level output), the
// block also forms sum(out r) and sum(out w) over its element's points in
// FP64 and writes them to dots[2e], dots[2e + 1]: the flexible CG's inner
// products (r, mult z) and (w, mult z) of the assembled z = gs(out), since
// r and w are continuous (see PrologDots).
struct PrologDots {
  const double *r = nullptr, *w = nullptr;
  double *part = nullptr;  // 2 per element
};

template <typename TIN, typename TOUT, typename T, int NI, int NO, bool TR, bool ACC,
          bool DOT = false>
__global__ void __launch_bounds__(kT3Threads)
    tensor3_kernel(const TIN *__restrict__ in, const TIN *__restrict__ scale,
                   const float *__restrict__ scale_f,
                   const T *__restrict__ M, TOUT *__restrict__ out, long nelv,
                   const int *__restrict__ skip, PrologDots dots = PrologDots{}) {
  if (skip && *skip) return;
  constexpr int I3 = NI * NI * NI, O3 = NO * NO * NO, NT = kT3Threads;
  __shared__ T su[I3], s1[NO * NI * NI], s2[NO * NO * NI], sA[NO * NI];
  const long e = blockIdx.x;
  const int tid = threadIdx.x;
  {
    constexpr int R = (I3 + NT - 1) / NT;
    TIN v[R], c[R];
#pragma unroll
    for (int g = 0; g < R; g++) {
      const int q = tid + g * NT;
      v[g] = q < I3 ? in[e * I3 + q] : TIN(0);
      c[g] = (!ACC && scale && q < I3)
                 ? (scale_f ? (TIN)scale_f[e * I3 + q] : scale[e * I3 + q])
                 : TIN(1);
    }
#pragma unroll
    for (int g = 0; g < R; g++) {
      const int q = tid + g * NT;
      if (q < I3) su[q] = (!ACC && scale) ? (T)(v[g] * c[g]) : (T)v[g];
    }
  }
  for (int q = tid; q < NO * NI; q += NT) {
    const int o = q % NO, i = q / NO;
    sA[q] = TR ? M[i + NI * o] : M[o + NO * i];  // sA(o, i) at o + NO*i
  }
  __syncthreads();
#pragma unroll
  for (int q0 = 0; q0 < NO * NI * NI; q0 += NT) {  // x: s1(o, j, k)
    const int q = q0 + tid;
    if (q < NO * NI * NI) {
      const int o = q % NO, jk = q / NO;
      T acc = 0;
#pragma unroll
      for (int i = 0; i < NI; i++) acc += sA[o + NO * i] * su[i + NI * jk];
      s1[q] = acc;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q0 = 0; q0 < NO * NO * NI; q0 += NT) {  // y: s2(o, p, k)
    const int q = q0 + tid;
    if (q < NO * NO * NI) {
      const int o = q % NO, p = (q / NO) % NO, k = q / (NO * NO);
      T acc = 0;
#pragma unroll
      for (int j = 0; j < NI; j++) acc += sA[p + NO * j] * s1[o + NO * j + NO * NI * k];
      s2[q] = acc;
    }
  }
  __syncthreads();
  constexpr int RO = (O3 + NT - 1) / NT;
  TOUT prev[RO];
  TIN oscale[RO];
  double dr[DOT ? RO : 1], dw[DOT ? RO : 1];
  if (ACC) {
#pragma unroll
    for (int g = 0; g < RO; g++) {
      const int q = tid + g * NT;
      prev[g] = q < O3 ? out[e * O3 + q] : TOUT(0);
      oscale[g] = (scale && q < O3)
                      ? (scale_f ? (TIN)scale_f[e * O3 + q] : scale[e * O3 + q])
                      : TIN(1);
      if constexpr (DOT) {
        dr[g] = q < O3 ? __ldg(dots.r + e * O3 + q) : 0.0;
        dw[g] = q < O3 ? __ldg(dots.w + e * O3 + q) : 0.0;
      }
    }
  }
  double s_r = 0.0, s_w = 0.0;
#pragma unroll
  for (int g = 0; g < RO; g++) {  // z
    const int q = tid + g * NT;
    if (q < O3) {
      const int op = q % (NO * NO), r = q / (NO * NO);
      T acc = 0;
#pragma unroll
      for (int k = 0; k < NI; k++) acc += sA[r + NO * k] * s2[op + NO * NO * k];
      TOUT v;
      if (ACC && scale)
        v = (TOUT)((T)prev[g] + (T)oscale[g] * acc);
      else if (ACC)
        v = (TOUT)((T)prev[g] + acc);
      else
        v = (TOUT)acc;
      out[e * O3 + q] = v;
      if constexpr (DOT) {
        s_r += (double)v * dr[g];
        s_w += (double)v * dw[g];
      }
    }
  }
  if constexpr (DOT) {
    __shared__ double sh[kT3Threads / 32];
    s_r = block_sum<kT3Threads>(s_r, sh);
    s_w = block_sum<kT3Threads>(s_w, sh);
    if (tid == 0) {
      dots.part[2 * e] = s_r;
      dots.part[2 * e + 1] = s_w;
    }
  }
}

template <typename TA, typename TB>
__global__ void convert_kernel(TB *__restrict__ b, const TA *__restrict__ a, long n,
                               const int *__restrict__ skip) {
  if (skip && *skip) return;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    b[i] = (TB)a[i];
}

__global__ void mask_kernel(double *x, const int *msk, int m, const int *skip) {
  if (skip && *skip) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) x[msk[i] - 1] = 0.0;
}

// ---------------------------------------------------------------------------
// Schwarz level (smoother precision T)
// ---------------------------------------------------------------------------
template <typename T>
struct SchwarzLevel {
  int lx = 0, nl = 0;
  long nelv = 0, n = 0;
  nb_problem *P = nullptr;  // the level's problem (gs maps, mask)
  T *S = nullptr, *lam = nullptr, *eps = nullptr, *wt = nullptr, *ext = nullptr;
  int *fn = nullptr;
  const unsigned char *ornt = nullptr;  // face pairings of a general mesh (null: aligned)
};

template <typename TIN, typename T, int LX>
static cudaError_t launch_fdm_post(const SchwarzLevel<T> &L, const TIN *r, T *e, const int *skip,
                                   cudaStream_t s) {
  constexpr int NL = LX + 2;
  using C = FdmCfg<T, NL>;
  auto kern = fdm_kernel<TIN, T, NL>;
  static bool attr_set = false;  // per instantiation
  if (!attr_set) {
    cudaError_t err =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
    if (err == cudaSuccess)
      err = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (err != cudaSuccess) return err;
    attr_set = true;
  }
  kern<<<(unsigned)((L.nelv + C::EPW - 1) / C::EPW), C::TPE, C::SMEM, s>>>(
      r, L.fn, L.ornt, L.S, L.lam, L.eps, L.ext, (int)L.nelv, skip);
  const long n = L.nelv * LX * LX * LX;
  schwarz_post_kernel<T, LX><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(
      L.ext, L.fn, L.ornt, L.wt, e, L.nelv, skip);
  return cudaGetLastError();
}

// e = Schwarz(r) on level L (r already masked): FDM + overlap + gs + mask.
template <typename TIN, typename T>
static cudaError_t schwarz_apply(const SchwarzLevel<T> &L, const TIN *r, T *e, const int *skip,
                                 cudaStream_t s, bool assemble = true) {
  cudaError_t err;
  switch (L.lx) {
#define NB_S(N) \
  case N: err = launch_fdm_post<TIN, T, N>(L, r, e, skip, s); break;
    NB_S(3) NB_S(4) NB_S(5) NB_S(6) NB_S(7) NB_S(8) NB_S(9) NB_S(10) NB_S(11) NB_S(12)
    NB_S(13) NB_S(14)
#undef NB_S
    default: return cudaErrorNotSupported;
  }
  if (err != cudaSuccess || !assemble) return err;
  return gs_add_fused<T>(L.P->gsd, e, true, s, skip);
}

// Drop-in form of the FDM (cuda_fdm_do_fast, src/math/bcknd/device/cuda/
// fdm_kernel.h): the input is the caller's extended element itself, the
// matrices are the caller's s(:,:,m,d) (m = 2, the transposed eigenvectors,
// for the forward transform; m = 1 for the backward one) and the scaling is
// the caller's full diagonal d, applied between the transforms and written
// back to r as the reference does.  The passes are those of fdm_kernel (one
// warp per element, vector matrix rows), so nl >= 8 only.
template <int NL>
__global__ void __launch_bounds__(FdmCfg<double, NL>::TPE, FdmCfg<double, NL>::MINB)
    fdm_dropin_kernel(double *__restrict__ eo, double *__restrict__ r,
                      const double *__restrict__ s, const double *__restrict__ d, int nelv) {
  using T = double;
  using C = FdmCfg<T, NL>;
  static_assert(C::VEC && C::EPW == 1, "vector form only");
  constexpr int N2 = C::N2, N3 = C::N3, LPE = C::LPE, MS = NL * C::NLR;
  static_assert(6 * N2 <= C::BUF, "matrix staging fits the second buffer");
  extern __shared__ __align__(16) unsigned char fdm_smem[];
  const int u = threadIdx.x;
  T *b0 = reinterpret_cast<T *>(fdm_smem), *b1 = b0 + C::BUF;
  T *sS = b0 + C::OFFM, *sL = sS + C::MAT, *stage = b1;
  const long e = blockIdx.x;
  if (e >= nelv) return;
  for (int q = u; q < N3; q += LPE) cp_async_elem<T>(b0 + C::pos(q / NL, q % NL), r + e * N3 + q, true);
  for (int q = u; q < 6 * N2; q += LPE) cp_async_elem<T>(stage + q, s + e * 6 * N2 + q, true);
  cp_async_wait_all();
  __syncthreads();
  // Row l of a pass's matrix holds the weights of input l for outputs
  // i = 0..nl-1.  The reference's transforms are tnsr3d(s(2,x), s(1,y),
  // s(1,z)) forward and tnsr3d(s(1,x), s(2,y), s(2,z)) backward, whose
  // first matrix contracts as A(i, l) and the other two as Bt(l, j).
  T *fwd = sS, *bwd = sS + 3 * MS;
  for (int q = u; q < 3 * N2; q += LPE) {
    const int dd = q / N2, rr = q - dd * N2, i = rr % NL, l = rr / NL;
    const T *s1 = stage + (2 * dd) * N2, *s2 = stage + (2 * dd + 1) * N2;
    fwd[dd * MS + i + C::NLR * l] = dd == 0 ? s2[i + NL * l] : s1[l + NL * i];
    bwd[dd * MS + i + C::NLR * l] = dd == 0 ? s1[i + NL * l] : s2[l + NL * i];
  }
  __syncthreads();
  fdm_pass<T, NL, true, false>(b0, b1, fwd, sL, nullptr, u);
  __syncthreads();
  fdm_pass<T, NL, true, false>(b1, b0, fwd + MS, sL, nullptr, u);
  __syncthreads();
  fdm_pass<T, NL, true, false>(b0, b1, fwd + 2 * MS, sL, nullptr, u);
  __syncthreads();
  for (int q = u; q < N3; q += LPE) {  // r = d * (forward transform), kept for the backward one
    const int p = C::pos(q / NL, q % NL);
    const T v = b1[p] * d[e * N3 + q];
    b1[p] = v;
    r[e * N3 + q] = v;
  }
  __syncthreads();
  fdm_pass<T, NL, false, false>(b1, b0, bwd, sL, nullptr, u);
  __syncthreads();
  fdm_pass<T, NL, false, false>(b0, b1, bwd + MS, sL, nullptr, u);
  __syncthreads();
  fdm_pass<T, NL, false, false>(b1, nullptr, bwd + 2 * MS, sL, eo + e * N3, u);
}

template <int NL>
static cudaError_t launch_fdm_dropin(double *eo, double *r, const double *s, const double *d,
                                     int nel, cudaStream_t st) {
  using C = FdmCfg<double, NL>;
  auto kern = fdm_dropin_kernel<NL>;
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t err =
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
    if (err != cudaSuccess) return err;
    attr_set = true;
  }
  kern<<<(unsigned)nel, C::TPE, C::SMEM, st>>>(eo, r, s, d, nel);
  return cudaGetLastError();
}

cudaError_t fdm_dropin(double *eo, double *r, const double *s, const double *d, int nl, int nel,
                       cudaStream_t st) {
  if (nel <= 0) return cudaSuccess;
  switch (nl) {
#define NB_FD(N) \
  case N: return launch_fdm_dropin<N>(eo, r, s, d, nel, st);
    NB_FD(8) NB_FD(9) NB_FD(10) NB_FD(11) NB_FD(12) NB_FD(13) NB_FD(14) NB_FD(15) NB_FD(16)
#undef NB_FD
    default: return cudaErrorNotSupported;
  }
}

// restriction (Jt x Jt x Jt)(in * scale) from ni to no points (J: ni x no);
// scale_f, when given, holds the same values as scale exactly in FP32 and is
// read instead
template <typename TIN, typename TOUT, typename T>
static cudaError_t restrict_level(int ni, int no, const TIN *in, const TIN *scale, const T *J,
                                  TOUT *out, long nelv, const int *skip, cudaStream_t s,
                                  const float *scale_f = nullptr) {
#define NB_R(A, B)                                                                          \
  if (ni == A && no == B) {                                                                 \
    tensor3_kernel<TIN, TOUT, T, A, B, true, false><<<(unsigned)nelv, kT3Threads, 0, s>>>(         \
        in, scale, scale_f, J, out, nelv, skip);                                            \
    return cudaGetLastError();                                                              \
  }
  NB_R(4, 2) NB_R(3, 2) NB_R(5, 4) NB_R(6, 4) NB_R(7, 4) NB_R(8, 4) NB_R(9, 4) NB_R(10, 4)
  NB_R(11, 4) NB_R(12, 4) NB_R(13, 4) NB_R(14, 4) NB_R(4, 3)
#undef NB_R
  return cudaErrorNotSupported;
}

// prolongation out += (J x J x J) in from ni to no points (J: no x ni)
template <typename TIN, typename TOUT, typename T>
static cudaError_t prolong_add(int ni, int no, const TIN *in, const T *J, TOUT *out, long nelv,
                               const int *skip, cudaStream_t s, const TIN *oscale = nullptr,
                               const float *oscale_f = nullptr,
                               const PrologDots *dots = nullptr) {
  const PrologDots d0 = dots ? *dots : PrologDots{};
#define NB_P(A, B)                                                                          \
  if (ni == A && no == B) {                                                                 \
    const unsigned g = (unsigned)nelv;                                                      \
    if (dots)                                                                               \
      tensor3_kernel<TIN, TOUT, T, A, B, false, true, true>                                 \
          <<<g, kT3Threads, 0, s>>>(in, oscale, oscale_f, J, out, nelv, skip, d0);          \
    else                                                                                    \
      tensor3_kernel<TIN, TOUT, T, A, B, false, true>                                       \
          <<<g, kT3Threads, 0, s>>>(in, oscale, oscale_f, J, out, nelv, skip);              \
    return cudaGetLastError();                                                              \
  }
  NB_P(2, 4) NB_P(2, 3) NB_P(4, 5) NB_P(4, 6) NB_P(4, 7) NB_P(4, 8) NB_P(4, 9) NB_P(4, 10)
  NB_P(4, 11) NB_P(4, 12) NB_P(4, 13) NB_P(4, 14) NB_P(3, 4)
#undef NB_P
  return cudaErrorNotSupported;
}

// ---------------------------------------------------------------------------
// The preconditioner.  T is the precision of the smoothing levels (double
// for the FP64 path, float for the mixed path); the coarse CG is FP64.
// ---------------------------------------------------------------------------
struct HsmgState : public Precond {
  nb_problem *fine = nullptr, *mid = nullptr, *crs = nullptr;
  void *arena = nullptr;
  int niter = 10;
  double tol = 1e-9;
  bool mixed = false;
  // The two branches of the additive scheme share only the input r: the
  // fine-level Schwarz runs on `side`, the middle level and the coarse solve
  // on `hi`, a stream of the greatest priority, so that the small,
  // latency-bound coarse-branch kernels get SM slots ahead of the pending
  // blocks of the large fine-level FDM launch instead of queueing behind it.
  cudaStream_t side = nullptr, hi = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_join_hi = nullptr;
  cudaError_t ensure_side() {
    if (side) return cudaSuccess;
    cudaError_t e;
    int lo_prio = 0, hi_prio = 0;
    if ((e = cudaDeviceGetStreamPriorityRange(&lo_prio, &hi_prio)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithPriority(&hi, cudaStreamNonBlocking, hi_prio)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ev_join_hi, cudaEventDisableTiming)) != cudaSuccess)
      return e;
    return cudaSuccess;
  }
  ~HsmgState() override {
    if (side) cudaStreamDestroy(side);
    if (hi) cudaStreamDestroy(hi);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (ev_join_hi) cudaEventDestroy(ev_join_hi);
    if (arena) cudaFree(arena);
    if (mid) nb_problem_destroy(mid);
    if (crs) nb_problem_destroy(crs);
  }
};

template <typename T>
struct HsmgImpl : public HsmgState {
  SchwarzLevel<T> sf, sm;
  T *Jfm = nullptr, *Jmc = nullptr;  // prolongations (fine x mid), (mid x crs)
  T *mult_f = nullptr, *mult_m = nullptr;
  T *zf = nullptr;                   // smoother-precision fine output (float path)
  T *w_mid = nullptr, *e_mid = nullptr;
  double *r_crs = nullptr, *e_crs = nullptr;
  double *rc = nullptr, *zc = nullptr, *pc = nullptr, *wc = nullptr;
  CgState *stc = nullptr;
  CoarseArgs<T> ca;

  // The fine level has no masked point: its Schwarz gather-scatter merges
  // into the final one.
  bool merged_assembly() const { return fine->nmask == 0; }

  int launches() const override {
    // 2 Schwarz x (fdm, post, gs) + restrict + gs + coarse (one launch) +
    // prolong + final gs (+ convert); one gs fewer when merged
    return 6 + 1 + 1 + 1 + 1 + 1 + (sizeof(T) == 4 ? 1 : 0) - (merged_assembly() ? 1 : 0);
  }

  int take_error() override {
    int v = 0;
    if (cudaMemcpy(&v, ca.err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    if (v) {  // leave the barrier words at rest for the next launch
      cudaMemset(ca.err, 0, sizeof(int));
      cudaMemset(ca.bar, 0, 2 * sizeof(unsigned));
      cudaDeviceSynchronize();
    }
    return v;
  }

  // FP32 smoothing levels: the output can stay in FP32 (zf)
  const float *output_f32() override {
    return sizeof(T) == 4 ? reinterpret_cast<const float *>(zf) : nullptr;
  }
  cudaError_t apply_f32(const double *r, const int *skip, cudaStream_t s) override {
    if (sizeof(T) != 4) return cudaErrorNotSupported;
    return apply_to(zf, r, skip, s);
  }

  // Without a mask the output is assembled by one final gather-scatter of
  // the prolongation's result, so the inner products with the continuous r
  // and w_prev can be formed by the prolongation itself.
  bool dots_in_apply() const override { return merged_assembly(); }
  cudaError_t apply_dots(double *z, const double *r, const double *w_prev, double *part,
                         const int *skip, cudaStream_t s) override {
    if (!merged_assembly()) return cudaErrorNotSupported;
    PrologDots d;
    d.r = r;
    d.w = w_prev;
    d.part = part;
    if (sizeof(T) == 4) return apply_to(zf, r, skip, s, &d);  // output stays in zf
    return apply_to(reinterpret_cast<T *>(z), r, skip, s, &d);
  }

  cudaError_t apply(double *z, const double *r, const int *skip, cudaStream_t s) override {
    T *zs = sizeof(T) == 8 ? reinterpret_cast<T *>(z) : zf;
    cudaError_t e = apply_to(zs, r, skip, s);
    if (e != cudaSuccess) return e;
    if (sizeof(T) == 4)
      convert_kernel<T, double><<<stream_grid(fine->n, 256), 256, 0, s>>>(z, zs, fine->n, skip);
    return cudaGetLastError();
  }

  // zs = M r in the smoothing precision (dots: see apply_dots)
  cudaError_t apply_to(T *zs, const double *r, const int *skip, cudaStream_t s,
                       const PrologDots *dots = nullptr) {
    cudaError_t e;
    const long nelv = fine->nelv;
    // fine Schwarz on the side stream: zs = S_f r
    if ((e = ensure_side()) != cudaSuccess || (e = cudaEventRecord(ev_fork, s)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(side, ev_fork, 0)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(hi, ev_fork, 0)) != cudaSuccess)
      return e;
    // middle and coarse levels first, on the high-priority stream:
    // restrict (r * mult) to the middle level, assemble, mask
    if ((e = restrict_level<double, T, T>(fine->lx, mid->lx, r, fine->mult, Jfm, w_mid, nelv,
                                          skip, hi, fine->multf)) != cudaSuccess)
      return e;
    if ((e = gs_add_fused<T>(mid->gsd, w_mid, true, hi, skip)) != cudaSuccess) return e;
    // middle Schwarz: e_mid = S_m w
    if ((e = schwarz_apply<T, T>(sm, w_mid, e_mid, skip, hi)) != cudaSuccess) return e;
    // restrict (w * mult_mid) to the coarse level (FP64), assemble, mask,
    // niter Jacobi-CG iterations (or abs tol), e_mid += J e_crs: one launch
    ca.skip = skip;
    if ((e = hsmg_coarse_solve<T>(ca, mid->lx, kCoarseMaxBlocks, hi)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(ev_join_hi, hi)) != cudaSuccess) return e;
    // fine Schwarz on the side stream: zs = S_f r (left unassembled when the
    // final gather-scatter takes it, see below)
    const bool merged = merged_assembly();
    if ((e = schwarz_apply<double, T>(sf, r, zs, skip, side, !merged)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(ev_join, side)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(s, ev_join, 0)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(s, ev_join_hi, 0)) != cudaSuccess)
      return e;
    // prolong: zs += J e_mid; z = mult * gs(zs).  Without a mask the fine
    // Schwarz output's own gather-scatter is folded into this one: wt and
    // mult are the same at every copy of a point, so
    // mult gs(gs(wt e) + J e_mid) = gs(wt e + mult J e_mid).
    if ((e = prolong_add<T, T, T>(mid->lx, fine->lx, e_mid, Jfm, zs, nelv, skip, s,
                                  merged ? mult_f : nullptr,
                                  merged && sizeof(T) == 8 ? fine->multf : nullptr,
                                  merged ? dots : nullptr)) !=
        cudaSuccess)
      return e;
    if ((e = gs_add_fused<T>(fine->gsd, zs, false, s, skip, merged ? nullptr : mult_f)) !=
        cudaSuccess)
      return e;
    return cudaGetLastError();
  }
};

void hsmg_free(nb_problem *p) {
  for (auto &h : p->hsmg) {
    delete h;
    h = nullptr;
  }
}

// hsmg_set_h (pc_hsmg.f90:367-379): the coarse h1 is the first n_crs values
// of the fine h1 and the coarse problem has no h2; its Jacobi diagonal
// follows.  The mesh is marked all-deformed (pc_hsmg.f90:267), which turns on
// the corner cross terms of that diagonal.
static cudaError_t hsmg_set_h(nb_problem *P, nb_problem *C) {
  cudaError_t e;
  if ((e = cudaMemcpy(C->h1, P->h1, C->n * 8, cudaMemcpyDeviceToDevice)) != cudaSuccess ||
      (e = cudaMemset(C->dfrmd, 1, C->nelv)) != cudaSuccess)
    return e;
  C->ifh2 = false;
  C->invalidate_solver_cache();
  return C->update_jacobi(nullptr);
}

// Constant h1 on the coarse levels of p's preconditioners, on stream s
// (hsmg_set_h with a constant fine h1: every coarse value is h1).
cudaError_t hsmg_set_h_const(nb_problem *p, double h1, cudaStream_t s) {
  for (auto *h : p->hsmg) {
    if (!h) continue;
    nb_problem *C = h->crs;
    cudaError_t e = fill_const(C->h1, h1, C->n, s);
    if (e != cudaSuccess) return e;
    if ((e = C->update_jacobi(s)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t hsmg_refresh_coefficients(nb_problem *p) {
  for (auto *h : p->hsmg) {
    if (!h) continue;
    cudaError_t e = hsmg_set_h(p, h->crs);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

static nb_status hfail(nb_status st, const std::string &m) {
  set_error(m);
  return st;
}

// facet_type per element face for the FDM: 0 with a neighbour, 1 on a
// strong (zero-Dirichlet) face, -(face) on an unlabeled boundary.
static void facet_types(const std::vector<int> &fn, bool dirichlet, std::vector<int> &ft) {
  ft.resize(fn.size());
  for (size_t q = 0; q < fn.size(); q++)
    ft[q] = fn[q] ? 0 : (dirichlet ? 1 : -(int)(q % 6 + 1));
}

struct SchwarzHost {
  std::vector<double> S, lam, eps, wt;
  std::vector<int> fn;
};

// Face pairings of a general mesh for the Schwarz ghost exchange: for every
// element face with a neighbour, the neighbour's face that meets it (its
// opposite face preferred when several qualify, as on a periodic direction
// one element wide) and the map of the in-face coordinates, found by
// matching the four corner vertex ids (symmetric vertex order: corner
// (i, j, k) is vertex 1 + i + 2 j + 4 k).  The reference reaches the same
// pairing through a gather-scatter on an (lx+2)-point numbering
// (schwarz_init, src/math/schwarz.f90:112-171).  Codes as face_map reads
// them; false when a face has no matching pairing.
static bool face_pairings(long nelv, const std::vector<int> &ids, const std::vector<int> &fn,
                          std::vector<unsigned char> &ornt) {
  ornt.assign((size_t)nelv * 6, 0);
  auto corner = [&](long e, int f, int b1, int b2) {
    const int dir = f >> 1, side = f & 1;
    const int a1 = dir == 0 ? 1 : 0, a2 = dir == 2 ? 1 : 2;
    const int v = (side << dir) | (b1 << a1) | (b2 << a2);
    return ids[(size_t)e * 8 + v];
  };
  for (long e = 0; e < nelv; e++)
    for (int f = 0; f < 6; f++) {
      const int nb = fn[e * 6 + f];
      if (!nb) continue;
      const long n = nb - 1;
      bool found = false;
      for (int gi = 0; gi < 6 && !found; gi++) {
        const int g = gi == 0 ? (f ^ 1) : (gi - 1 < (f ^ 1) ? gi - 1 : gi);
        if (fn[n * 6 + g] != e + 1) continue;
        for (int code = 0; code < 8 && !found; code++) {
          const int sw = code & 1, f1 = (code >> 1) & 1, f2 = (code >> 2) & 1;
          bool ok = true;
          for (int b1 = 0; b1 < 2 && ok; b1++)
            for (int b2 = 0; b2 < 2 && ok; b2++) {
              const int u1 = sw ? b2 : b1, u2 = sw ? b1 : b2;
              const int t1 = f1 ? 1 - u1 : u1, t2 = f2 ? 1 - u2 : u2;
              ok = corner(e, f, b1, b2) == corner(n, g, t1, t2);
            }
          if (ok) {
            ornt[e * 6 + f] = (unsigned char)(g | (sw << 3) | (f1 << 4) | (f2 << 5));
            found = true;
          }
        }
      }
      if (!found) return false;
    }
  return true;
}

static nb_status build_schwarz_host(nb_problem *L, bool dirichlet, SchwarzHost &H) {
  std::vector<double> x(L->n), y(L->n), z(L->n);
  if (cudaMemcpy(x.data(), L->x, L->n * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(y.data(), L->y, L->n * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(z.data(), L->z, L->n * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
    return hfail(NB_ERR_CUDA, "hsmg: coordinate copy failed");
  H.fn = L->fn;
  std::vector<int> ft;
  facet_types(H.fn, dirichlet, ft);
  FdmHost F;
  fdm_build(L->lx, L->nelv, x, y, z, ft, L->maps, F);
  H.S.swap(F.S);
  H.lam.swap(F.lam);
  H.eps.swap(F.eps);
  schwarz_weights(L->lx, L->nelv, H.fn, L->maps, H.wt);
  return NB_OK;
}

// Device arena layout helper: offsets in 256-byte slices.
struct Slicer {
  size_t off = 0;
  size_t take(size_t bytes) {
    size_t o = off;
    off += (bytes + 255) & ~size_t(255);
    return o;
  }
};

template <typename T>
static std::vector<T> cast_vec(const std::vector<double> &v) {
  return std::vector<T>(v.begin(), v.end());
}

// Allocates and fills the device side of HsmgImpl<T>.
template <typename T>
static nb_status upload_impl(HsmgImpl<T> *H, const SchwarzHost &hf, const SchwarzHost &hm,
                             const std::vector<double> &Jfm, const std::vector<double> &Jmc,
                             const std::vector<unsigned char> &ornt) {
  nb_problem *P = H->fine, *M = H->mid, *C = H->crs;
  const long nelv = P->nelv, n = P->n, nm = M->n, nc = C->n;
  const int nlf = P->lx + 2, nlm = M->lx + 2;
  const bool f32 = sizeof(T) == 4;
  Slicer c;
  const size_t o_Sf = c.take(hf.S.size() * sizeof(T)), o_Lf = c.take(hf.lam.size() * sizeof(T)),
               o_Ef = c.take(hf.eps.size() * sizeof(T)), o_Wf = c.take(hf.wt.size() * sizeof(T)),
               o_Ff = c.take(hf.fn.size() * 4),
               o_Xf = c.take((size_t)nelv * nlf * nlf * nlf * sizeof(T));
  const size_t o_Sm = c.take(hm.S.size() * sizeof(T)), o_Lm = c.take(hm.lam.size() * sizeof(T)),
               o_Em = c.take(hm.eps.size() * sizeof(T)), o_Wm = c.take(hm.wt.size() * sizeof(T)),
               o_Fm = c.take(hm.fn.size() * 4),
               o_Xm = c.take((size_t)nelv * nlm * nlm * nlm * sizeof(T));
  const size_t o_Jfm = c.take(Jfm.size() * sizeof(T)), o_Jmc = c.take(Jmc.size() * sizeof(T));
  const size_t o_or = c.take(ornt.size());
  const size_t o_mf = f32 ? c.take(n * sizeof(T)) : 0, o_mm = c.take(nm * sizeof(T));
  const size_t o_zf = f32 ? c.take(n * sizeof(T)) : 0;
  const size_t o_wm = c.take(nm * sizeof(T)), o_em = c.take(nm * sizeof(T));
  const size_t o_rc = c.take(nc * 8), o_ec = c.take(nc * 8), o_r = c.take(nc * 8),
               o_z = c.take(nc * 8), o_p = c.take(nc * 8), o_w = c.take(nc * 8);
  const size_t o_st = c.take(sizeof(CgState)),
               o_part = c.take(2 * 2 * kCoarseMaxBlocks * sizeof(double) + 64);
  if (cudaMalloc(&H->arena, c.off) != cudaSuccess) return hfail(NB_ERR_OOM, "hsmg: device arena");
  char *A = (char *)H->arena;
  auto Tp = [&](size_t o) { return (T *)(A + o); };
  auto Dp = [&](size_t o) { return (double *)(A + o); };
  auto setlev = [&](SchwarzLevel<T> &L, nb_problem *Q, size_t oS, size_t oL, size_t oE, size_t oW,
                    size_t oF, size_t oX) {
    L.P = Q;
    L.lx = Q->lx;
    L.nl = Q->lx + 2;
    L.nelv = Q->nelv;
    L.n = Q->n;
    L.S = Tp(oS), L.lam = Tp(oL), L.eps = Tp(oE), L.wt = Tp(oW), L.fn = (int *)(A + oF);
    L.ext = Tp(oX);
  };
  setlev(H->sf, P, o_Sf, o_Lf, o_Ef, o_Wf, o_Ff, o_Xf);
  setlev(H->sm, M, o_Sm, o_Lm, o_Em, o_Wm, o_Fm, o_Xm);
  if (!ornt.empty()) H->sf.ornt = H->sm.ornt = (const unsigned char *)(A + o_or);
  H->Jfm = Tp(o_Jfm), H->Jmc = Tp(o_Jmc);
  H->mult_f = f32 ? Tp(o_mf) : reinterpret_cast<T *>(P->mult);
  H->mult_m = Tp(o_mm);
  H->zf = f32 ? Tp(o_zf) : nullptr;
  H->w_mid = Tp(o_wm), H->e_mid = Tp(o_em);
  H->r_crs = Dp(o_rc), H->e_crs = Dp(o_ec), H->rc = Dp(o_r), H->zc = Dp(o_z), H->pc = Dp(o_p),
  H->wc = Dp(o_w);
  H->stc = (CgState *)(A + o_st);
  CoarseArgs<T> &ca = H->ca;
  ca.nelv = nelv;
  ca.w_mid = H->w_mid, ca.mult_m = H->mult_m, ca.J = H->Jmc, ca.e_mid = H->e_mid;
  ca.f = H->r_crs, ca.x = H->e_crs, ca.r = H->rc, ca.z = H->zc, ca.p = H->pc, ca.w = H->wc;
  ca.h1 = C->h1, ca.g11 = C->g11, ca.g22 = C->g22, ca.g33 = C->g33, ca.g12 = C->g12,
  ca.g13 = C->g13, ca.g23 = C->g23, ca.D = C->D, ca.Dt = C->Dt;
  ca.dinv = C->jdiag, ca.mult = C->mult;
  ca.gs = C->gsd;
  ca.st = H->stc;
  ca.part = Dp(o_part);
  ca.bar = (unsigned *)(A + o_part + 2 * 2 * kCoarseMaxBlocks * sizeof(double));
  ca.err = (int *)(ca.bar + 2);
  auto upv = [&](size_t o, const std::vector<double> &v) {
    std::vector<T> t = cast_vec<T>(v);
    return t.empty() ? cudaSuccess
                     : cudaMemcpy(A + o, t.data(), t.size() * sizeof(T), cudaMemcpyHostToDevice);
  };
  auto upi = [&](size_t o, const std::vector<int> &v) {
    return cudaMemcpy(A + o, v.data(), v.size() * 4, cudaMemcpyHostToDevice);
  };
  std::vector<double> hm_mult(nm), hf_mult;
  if (cudaMemcpy(hm_mult.data(), M->mult, nm * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
    return hfail(NB_ERR_CUDA, "hsmg: mult copy failed");
  if (f32) {
    hf_mult.resize(n);
    if (cudaMemcpy(hf_mult.data(), P->mult, n * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
      return hfail(NB_ERR_CUDA, "hsmg: mult copy failed");
  }
  CgState cs{};
  cs.norm_fac = 1.0 / std::sqrt(C->volume);
  cs.abs_tol = H->tol;
  cs.max_iter = H->niter;
  cs.done = 1;
  if (upv(o_Sf, hf.S) || upv(o_Lf, hf.lam) || upv(o_Ef, hf.eps) || upv(o_Wf, hf.wt) ||
      upi(o_Ff, hf.fn) || upv(o_Sm, hm.S) || upv(o_Lm, hm.lam) || upv(o_Em, hm.eps) ||
      upv(o_Wm, hm.wt) || upi(o_Fm, hm.fn) || upv(o_Jfm, Jfm) || upv(o_Jmc, Jmc) ||
      upv(o_mm, hm_mult) || (f32 && upv(o_mf, hf_mult)) ||
      (!ornt.empty() &&
       cudaMemcpy(A + o_or, ornt.data(), ornt.size(), cudaMemcpyHostToDevice) != cudaSuccess) ||
      cudaMemcpy(A + o_st, &cs, sizeof(cs), cudaMemcpyHostToDevice) ||
      cudaMemset(A + o_part, 0, 2 * 2 * kCoarseMaxBlocks * sizeof(double) + 64))
    return hfail(NB_ERR_CUDA, "hsmg: upload failed");
  return NB_OK;
}

nb_status hsmg_get(nb_problem *P, const nb_solve_opts &o, Precond **out) {
  const int niter = o.coarse_iter > 0 ? o.coarse_iter : 10;
  const double tol = o.coarse_tol > 0 ? o.coarse_tol : 1e-9;
  const bool mixed = o.mixed != 0;
  HsmgState *&slot = P->hsmg[mixed ? 1 : 0];
  if (slot && (slot->niter != niter || slot->tol != tol)) {
    P->invalidate_solver_cache();
    delete slot;
    slot = nullptr;
  }
  if (slot) {
    *out = slot;
    return NB_OK;
  }
  const int lx = P->lx;
  if (lx < 3 || lx > 14) return hfail(NB_ERR_UNSUPPORTED, "hsmg supports lx 3..14");
  std::vector<unsigned char> ornt;  // face pairings (general meshes only)
  if (!P->faces_aligned && !face_pairings(P->nelv, P->mesh_ids, P->fn, ornt))
    return hfail(NB_ERR_UNSUPPORTED,
                 "hsmg: a face neighbour shares no face with matching corner vertices");
  const int lx_mid = lx < 5 ? std::max(lx - 1, 3) : 4, lx_crs = 2;
  HsmgState *H = mixed ? (HsmgState *)new HsmgImpl<float>() : (HsmgState *)new HsmgImpl<double>();
  H->fine = P;
  H->niter = niter;
  H->tol = tol;
  H->mixed = mixed;
  const bool dirichlet = P->nmask > 0;
  // the coarser levels are the same mesh at lx_mid and lx_crs points a side
  auto level = [&](int lxl, nb_problem **q) {
    return P->from_mesh ? nb_problem_create_mesh(P->nelv, P->mesh_ids.data(),
                                                 P->mesh_xyz8.data(), lxl, P->deform_amp,
                                                 dirichlet, q)
                        : nb_problem_create_box(P->box.nel, P->box.lo, P->box.hi,
                                                P->box.periodic, lxl, P->deform_amp, dirichlet,
                                                q);
  };
  nb_status st = level(lx_mid, &H->mid);
  if (st == NB_OK) st = level(lx_crs, &H->crs);
  if (st != NB_OK) {
    delete H;
    return st;
  }
  if (hsmg_set_h(P, H->crs) != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
    delete H;
    return hfail(NB_ERR_CUDA, "hsmg: coarse coefficients failed");
  }
  SchwarzHost hf, hm;
  if ((st = build_schwarz_host(P, dirichlet, hf)) != NB_OK ||
      (st = build_schwarz_host(H->mid, dirichlet, hm)) != NB_OK) {
    delete H;
    return st;
  }
  std::vector<double> zf, zm, zc, tmp, t2, t3, Jfm, Jmc;
  gll_space(lx, zf, tmp, t2, t3);
  gll_space(lx_mid, zm, tmp, t2, t3);
  gll_space(lx_crs, zc, tmp, t2, t3);
  lagrange_matrix(zf, zm, Jfm);
  lagrange_matrix(zm, zc, Jmc);
  st = mixed ? upload_impl((HsmgImpl<float> *)H, hf, hm, Jfm, Jmc, ornt)
             : upload_impl((HsmgImpl<double> *)H, hf, hm, Jfm, Jmc, ornt);
  // The uploads ran on the legacy stream (a pageable cudaMemcpy may return
  // before its DMA lands); finish them before any caller stream reads them.
  if (st == NB_OK && cudaDeviceSynchronize() != cudaSuccess)
    st = hfail(NB_ERR_CUDA, "hsmg: upload failed");
  if (st != NB_OK) {
    delete H;
    return st;
  }
  slot = H;
  *out = H;
  return NB_OK;
}

// Exposed for tests: z = M r with the problem's hsmg (built on demand).
nb_status hsmg_apply_once(nb_problem *P, double *z, const double *r, cudaStream_t s, int mixed) {
  nb_solve_opts o{};
  const HsmgState *h = P->hsmg[mixed ? 1 : 0];
  o.coarse_iter = h ? h->niter : 10;
  o.coarse_tol = h ? h->tol : 1e-9;
  o.mixed = mixed;
  Precond *pc = nullptr;
  nb_status st = hsmg_get(P, o, &pc);
  if (st != NB_OK) return st;
  NB_CUDA_TRY(pc->apply(z, r, nullptr, s));
  NB_CUDA_TRY(cudaStreamSynchronize(s));
  if (pc->take_error()) {
    set_error("a bounded device wait expired (coarse-level grid barrier)");
    return NB_ERR_TIMEOUT;
  }
  return NB_OK;
}

}  // namespace nb

extern "C" nb_status nb_hsmg_init(nb_problem *p, int mixed, int coarse_iter,
                                  double coarse_tol) {
  using namespace nb;
  if (!p) {
    set_error("null argument");
    return NB_ERR_ARG;
  }
  nb_solve_opts o{};
  o.mixed = mixed != 0;
  o.coarse_iter = coarse_iter;
  o.coarse_tol = coarse_tol;
  Precond *pc = nullptr;
  return hsmg_get(p, o, &pc);
}

extern "C" nb_status nb_pc_apply(nb_problem *p, int pc, double *z, const double *r,
                                 void *stream) {
  using namespace nb;
  if (!p || !z || !r) {
    set_error("null argument");
    return NB_ERR_ARG;
  }
  if (pc == NB_PC_PHMG) {
    Precond *M = nullptr;
    nb_status st = phmg_get(p, &M);
    if (st != NB_OK) return st;
    NB_CUDA_TRY(M->apply(z, r, nullptr, (cudaStream_t)stream));
    NB_CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    if (M->take_error()) {
      set_error("a bounded device wait expired (phmg level operator)");
      return NB_ERR_TIMEOUT;
    }
    return NB_OK;
  }
  if (pc != NB_PC_HSMG && pc != NB_PC_HSMG_MIXED) {
    set_error("nb_pc_apply: pc must be NB_PC_HSMG, NB_PC_HSMG_MIXED or NB_PC_PHMG");
    return NB_ERR_ARG;
  }
  return hsmg_apply_once(p, z, r, (cudaStream_t)stream, pc == NB_PC_HSMG_MIXED);
}
