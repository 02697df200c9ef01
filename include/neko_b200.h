/*
 * neko_b200.h -- C ABI of libnekob200.so, a B200 (sm_100a) device backend for
 * the pressure/Helmholtz solve path of the Neko spectral-element code.
 *
 * Part 1 exports the symbols that Neko's Fortran device layer binds through
 * `bind(c, name='cuda_*')`, with the same signatures and semantics, so a Neko
 * build can link this library in place of its own CUDA objects.  As in the
 * reference, integers arrive by reference, device buffers as plain pointers,
 * the stream (where the reference passes one) as an opaque handle, and
 * `real` is double.  Errors in this part print a message and exit, as the
 * reference's CUDA_CHECK does.  Entry points that take no stream launch on
 * the stream given to nb_set_default_stream(), else on Neko's global
 * `void *glb_cmd_queue` when the program defines it (the library holds a
 * weak reference to that symbol, src/device/device_config.h.in:19), else on
 * the legacy default stream.
 *
 * Part 2 is a native handle API (nb_*) over device-resident problems: mesh,
 * geometric factors and gather-scatter maps built once and kept in HBM, then
 * operator applications and complete Krylov solves.  Every nb_* call returns
 * an nb_status; nb_last_error() describes the last failure of the thread.
 */
#ifndef NEKO_B200_H
#define NEKO_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------
 * Part 1: drop-in replacements for the reference's cuda_* entry points.
 * ---------------------------------------------------------------------- */

/* w = A u, the matrix-free Helmholtz operator (h1 part) on nelv elements of
 * lx^3 points.  Replaces cuda_ax_helm
 * (src/math/bcknd/device/cuda/ax_helm.cu:63), called from
 * src/math/bcknd/device/ax_helm_device.F90:234.  Launches on glb_cmd_queue
 * as the reference does (see the stream rule above).  A bounded device wait
 * that expires is reported, fatally, by the next synchronising drop-in
 * (cuda_glsc3, cuda_glsc2, cuda_glsum, cuda_fusedcg_part2). */
void cuda_ax_helm(void *w, void *u, void *dx, void *dy, void *dz, void *dxt,
                  void *dyt, void *dzt, void *h1, void *g11, void *g22,
                  void *g33, void *g12, void *g13, void *g23, int *nelv,
                  int *lx);

/* (au, av, aw) = A (u, v, w), the h1 part of the operator for the three
 * velocity components with one set of geometric factors.  Replaces
 * cuda_ax_helm_vector (src/math/bcknd/device/cuda/ax_helm.cu:184), called
 * from ax_helm_device_compute_vector (src/math/bcknd/device/
 * ax_helm_device.F90).  Launches on glb_cmd_queue (see the stream rule
 * above). */
void cuda_ax_helm_vector(void *au, void *av, void *aw, void *u, void *v, void *w,
                         void *dx, void *dy, void *dz, void *dxt, void *dyt, void *dzt,
                         void *h1, void *g11, void *g22, void *g33, void *g12, void *g13,
                         void *g23, int *nelv, int *lx);
/* au += h2 B u, av += h2 B v, aw += h2 B w over n points.  Replaces
 * cuda_ax_helm_vector_part2 (src/math/bcknd/device/cuda/ax_helm.cu:254);
 * launches on glb_cmd_queue. */
void cuda_ax_helm_vector_part2(void *au, void *av, void *aw, void *u, void *v, void *w,
                               void *h2, void *B, int *n);

/* The full-stress operator of the velocity solve with variable viscosity,
 * (au, av, aw) = A_stress (u, v, w): per point the symmetric gradient
 * h1 w3 / jac (G + G^T) of the three components, G = cofactors^T grad, back
 * through the cofactors and the transposed derivatives.  Replaces
 * cuda_ax_helm_stress_vector (src/math/bcknd/device/cuda/ax_helm_full.cu,
 * called from ax_helm_full_device_compute_vector,
 * src/math/bcknd/device/ax_helm_full_device.F90:190-259); dxt, dyt, dzt are
 * accepted and not read (the transposes come from dx, dy, dz, as in the
 * reference kernel).  lx 2..16; launches on glb_cmd_queue. */
void cuda_ax_helm_stress_vector(void *au, void *av, void *aw, void *u, void *v, void *w,
                                void *dx, void *dy, void *dz, void *dxt, void *dyt, void *dzt,
                                void *h1, void *drdx, void *drdy, void *drdz, void *dsdx,
                                void *dsdy, void *dsdz, void *dtdx, void *dtdy, void *dtdz,
                                void *jacinv, void *w3, int *nelv, int *lx);
/* au += h2 B u, av += h2 B v, aw += h2 B w.  Replaces
 * cuda_ax_helm_stress_vector_part2 (ax_helm_full.cu); launches on
 * glb_cmd_queue. */
void cuda_ax_helm_stress_vector_part2(void *au, void *av, void *aw, void *u, void *v,
                                      void *w, void *h2, void *B, int *n);

/* au += h2 B u for one component.  Replaces the addcol4 used for the h2
 * term of the scalar Ax (ax_helm_device.F90:253-255 ->
 * src/math/bcknd/device/cuda/math.cu:641). */
void cuda_addcol4(void *a, void *b, void *c, void *d, int *n, void *stream);

/* Gather: v(dg(k)) = sum of u(gd(k..k+len-1)) for each block, and
 * v(dg(i)) = u(gd(i)) + u(gd(i+1)) for facet pairs from offset o (op = 1,
 * add); min/max/mul analogues for op = 2,3,4.  1-based index arrays.
 * Replaces src/gs/bcknd/device/cuda/gs.cu:51. */
void cuda_gather_kernel(void *v, int *m, int *o, void *dg, void *u, int *n,
                        void *gd, int *nb, void *b, void *bo, int *op,
                        void *stream);

/* Scatter: u(gd(i)) = v(dg(i)).  Replaces src/gs/bcknd/device/cuda/gs.cu:96. */
void cuda_scatter_kernel(void *v, int *m, void *dg, void *u, int *n, void *gd,
                         int *nb, void *b, void *bo, void *stream);

/* sum(a*b*c) returned to the host after a stream synchronisation.
 * Replaces src/math/bcknd/device/cuda/math.cu:906 (cuda_glsc3). */
double cuda_glsc3(void *a, void *b, void *c, int *n, void *stream);
/* sum(a*b) -- math.cu:965 */
double cuda_glsc2(void *a, void *b, int *n, void *stream);
/* sum(a) -- math.cu:1023 */
double cuda_glsum(void *a, int *n, void *stream);

/* Vector updates of the Krylov loop (math.cu:60-660). */
void cuda_copy(void *a, void *b, int *n, void *stream);           /* a = b */
void cuda_rzero(void *a, int *n, void *stream);                   /* a = 0 */
void cuda_add2s1(void *a, void *b, double *c1, int *n, void *stream); /* a = c1 a + b */
void cuda_add2s2(void *a, void *b, double *c1, int *n, void *stream); /* a = a + c1 b */
void cuda_col2(void *a, void *b, int *n, void *stream);           /* a = a b */
void cuda_col3(void *a, void *b, void *c, int *n, void *stream);  /* a = b c */
void cuda_addcol3(void *a, void *b, void *c, int *n, void *stream); /* a += b c */
void cuda_invcol1(void *a, int *n, void *stream);                 /* a = 1/a */
void cuda_radd(void *a, double *c, int *n, void *stream);         /* a += c (math.cu:266) */

/* Fused CG helpers of fusedcg_device_solve
 * (src/krylov/bcknd/device/fusedcg_device.F90:328-414), launched on
 * glb_cmd_queue.  Replace src/krylov/bcknd/device/cuda/fusedcg_aux.cu:61-87.
 *   update_p: p = beta po + z.
 *   update_x: x += sum_{j < p_cur} alpha[j] p[j], p a device array of p_cur
 *             device pointers, alpha a device array.
 *   part2:    alpha_d[p_cur-1] = *alpha; a = a - alpha c; returns
 *             sum(a b a) of the updated a after synchronising the stream. */
void cuda_fusedcg_update_p(void *p, void *z, void *po, double *beta, int *n);
void cuda_fusedcg_update_x(void *x, void *p, void *alpha, int *p_cur, int *n);
double cuda_fusedcg_part2(void *a, void *b, void *c, void *alpha_d, double *alpha,
                          int *p_cur, int *n);

/* Point-wise parts of the Pn-Pn pressure and velocity residuals, the
 * caller of the pressure solve (pnpn_prs_res_device_compute /
 * pnpn_vel_res_device_compute, src/fluid/bcknd/device/pnpn_res_device.F90).
 * Replace src/fluid/bcknd/device/cuda/pnpn_res.cu:43-107; launched on
 * glb_cmd_queue.
 *   part1: h1 = 1/rho; ta_i = f_i / rho - (wa_i (mu / rho)) B
 *   part2: p_res = -p_res + (wa1 + wa2 + wa3)
 *   part3: p_res = p_res - dtbd (ta1 + ta2 + ta3)
 *   vel_res_update: res_i = -res_i - ta_i + f_i */
void pnpn_prs_res_part1_cuda(void *ta1, void *ta2, void *ta3, void *wa1, void *wa2, void *wa3,
                             void *f_u, void *f_v, void *f_w, void *B, void *h1, double *mu,
                             double *rho, int *n);
void pnpn_prs_res_part2_cuda(void *p_res, void *wa1, void *wa2, void *wa3, int *n);
void pnpn_prs_res_part3_cuda(void *p_res, void *ta1, void *ta2, void *ta3, double *dtbd,
                             int *n);
void pnpn_vel_res_update_cuda(void *u_res, void *v_res, void *w_res, void *ta1, void *ta2,
                              void *ta3, void *f_u, void *f_v, void *f_w, int *n);

/* Stream for the Part-1 entry points that take none, overriding
 * glb_cmd_queue (NULL selects the legacy default stream).  No counterpart in
 * the reference, where Neko's device layer owns glb_cmd_queue. */
void nb_set_default_stream(void *stream);

/* x(msk(i)) = 0 for i = 1..m-1 (msk(0) holds the count).  Replaces
 * src/bc/bcknd/device/cuda/zero_dirichlet.cu:44. */
void cuda_zero_dirichlet_apply_scalar(void *msk, void *x, int *m, void *stream);

/* Diagonal of the stiffness matrix from the geometric factors, with the
 * boundary cross terms of the reference device kernel.  Replaces
 * src/krylov/bcknd/device/cuda/pc_jacobi.cu:102. */
void cuda_jacobi_update(void *d, void *dxt, void *dyt, void *dzt, void *G11,
                        void *G22, void *G33, void *G12, void *G13, void *G23,
                        int *nel, int *lx);

/* v = (C x B x A) u on nel elements: u has nu^3 points per element, v nv^3;
 * A is nv x nu, Bt and Ct nu x nv (column-major).  Replaces cuda_tnsr3d
 * (src/math/bcknd/device/cuda/tensor.cu:60); nu, nv <= 16.  Launches on
 * glb_cmd_queue as the reference does (see the stream rule above). */
void cuda_tnsr3d(void *v, int *nv, void *u, int *nu, void *A, void *Bt, void *Ct, int *nel);

/* Fast-diagonalisation solve per element of nl^3 points: r <- d * (S_x^T,
 * S_y^T, S_z^T) r, then e <- (S_x, S_y, S_z) r, with s holding
 * s(nl,nl,2,3,nel) (eigenvectors and their transposes) and d the inverse
 * eigenvalue sums.  r is overwritten, as in the reference.  Replaces
 * src/math/bcknd/device/cuda/fdm.cu:42; nl <= 16. */
void cuda_fdm_do_fast(void *e, void *r, void *s, void *d, int *nl, int *nel, void *stream);

/* a1 = f1 a1 + f2 a2 on the interior points of face layers l1 (a1) and l2
 * (a2) from each side, x then y then z.  Replaces
 * src/math/bcknd/device/cuda/schwarz.cu:45. */
void cuda_schwarz_extrude(void *arr1, int *l1, double *f1, void *arr2, int *l2, double *f2,
                          int *nx, int *nel, void *stream);
/* a ((nx+2)^3 per element) = b (nx^3) inside a zero ghost layer; and back.
 * Replace schwarz.cu:82 and schwarz.cu:92. */
void cuda_schwarz_toext3d(void *a, void *b, int *nx, int *nel, void *stream);
void cuda_schwarz_toreg3d(void *b, void *a, int *nx, int *nel, void *stream);

/* ------------------------------------------------------------------------
 * Part 2: native handle API.
 * ---------------------------------------------------------------------- */

typedef enum {
  NB_OK = 0,
  NB_ERR_ARG = 1,          /* invalid argument */
  NB_ERR_UNSUPPORTED = 2,  /* lx or mesh outside the supported set */
  NB_ERR_OOM = 3,          /* device allocation failed */
  NB_ERR_CUDA = 4,         /* CUDA runtime error */
  NB_ERR_NOT_CONVERGED = 5,
  NB_ERR_NAN = 6,          /* residual became NaN/Inf */
  NB_ERR_TIMEOUT = 7       /* a bounded device wait expired */
} nb_status;

typedef struct nb_problem nb_problem;

/* Returns the message of the last failed nb_* call of this thread. */
const char *nb_last_error(void);

/* Library version string. */
const char *nb_version(void);

/* Host-only setup helpers (no device needed). */

/* GLL nodes z[lx], weights w[lx] and derivative matrix D[lx*lx]
 * (column-major, D(i,j) = l_j'(z_i)), the quantities space_t%init builds
 * with zwgll/dgll (src/sem/space.f90:149-320). */
nb_status nb_gll(int lx, double *z, double *w, double *D);

/* Gather-scatter maps of a structured box, in the reference layout of
 * gs_init_mapping (src/gs/gather_scatter.f90:513-1375): 1-based gs id and
 * local point per entry, block lengths/offsets over the vertex/edge part,
 * facet pairs from facet_offset on.  Call once with NULL arrays to get the
 * sizes, then with arrays of those sizes. */
nb_status nb_box_gs_maps(const int nel[3], const int periodic[3], int lx,
                         int *nlocal, int *facet_offset, int *nblocks,
                         int *dof_gs, int *gs_dof, int *blk_len, int *blk_off);

/* Reads a 3-D Neko mesh file (.nmsh; nmsh_file_read,
 * src/io/nmsh_file.f90:70-207) into the arrays nb_problem_create_mesh
 * takes: vertex ids with the periodic zones applied (the ids of periodic
 * faces replaced by their partners', mesh_apply_periodic_facet) and
 * coordinates, both in symmetric vertex order.  Call once with NULL arrays
 * to get nelv.  *nperiodic / *nlabeled (may be NULL) receive the number of
 * periodic and labeled-boundary zones.  Host only. */
nb_status nb_mesh_read_nmsh(const char *path, int *nelv, int *vertex_ids, double *vertex_xyz,
                            int *nperiodic, int *nlabeled);
/* Writes such a mesh as a .nmsh file (element ids 1..nelv, no zones, no
 * curved edges; periodic identification stays in the vertex ids).  Host
 * only. */
nb_status nb_mesh_write_nmsh(const char *path, int nelv, const int *vertex_ids,
                             const double *vertex_xyz);

/* Writes a field file in Neko's fld format (fld_file_write,
 * src/io/fld_file.f90:183-620; the Nek5000 layout): 132-byte header with
 * real size 8, lx, nelv, time, step and the record code, the byte-order
 * tag, element ids, the coordinates ('X', when x, y, z are given), one
 * scalar as the pressure ('P', when p is given), then the per-element
 * min/max metadata in single precision.  Host arrays of nelv lx^3 values in
 * element order.  Host only. */
nb_status nb_fld_write(const char *path, int nelv, int lx, const double *x, const double *y,
                       const double *z, const double *p, double time, int step);

/* Gather-scatter maps (and the neighbour per face, 6 per element, 1-based,
 * 0 on the boundary) of the unstructured mesh that nb_problem_create_mesh
 * takes, in the reference layout of gs_init_mapping.  Host only; call once
 * with NULL arrays to get the sizes. */
nb_status nb_mesh_gs_maps(int nelv, const int *vertex_ids, int lx, int *nlocal,
                          int *facet_offset, int *nblocks, int *facet_neigh, int *dof_gs,
                          int *gs_dof, int *blk_len, int *blk_off);

/* Builds a structured box problem on the current device: nel[3] hexahedra
 * on [lo,hi]^3 (x fastest), optional periodicity, polynomial size lx
 * (2..16), and an optional smooth deformation of the GLL points
 * x += a sin(y) sin(z), y += a sin(z) sin(x), z += a sin(x) sin(y).
 * Geometric factors (G11..G23, B, mult) are computed on the device; the
 * gather-scatter maps follow the reference's gs_init_mapping
 * (src/gs/gather_scatter.f90:513-1375) entry for entry.  Faces with no
 * neighbour become zero-Dirichlet when dirichlet_boundary is non-zero.
 * Periodic directions need at least 3 elements. */
nb_status nb_problem_create_box(const int nel[3], const double lo[3],
                                const double hi[3], const int periodic[3],
                                int lx, double deform_amp,
                                int dirichlet_boundary, nb_problem **out);
/* Builds a problem on the current device from a caller's unstructured
 * hexahedral mesh: nelv elements, each with 8 positive global vertex ids
 * (vertex_ids[8 e + v]) and coordinates (vertex_xyz[24 e + 3 v + d]) in the
 * reference's symmetric vertex order (src/mesh/hex.f90:40-57); vertices that
 * a periodic boundary identifies carry one id.  Faces, edges and neighbours
 * come from the ids (mesh_generate_conn, src/mesh/mesh.f90:476-687), the
 * GLL points by trilinear interpolation of the vertices (dofmap_xyzlin) and
 * the optional sine deformation of nb_problem_create_box, the gather-scatter
 * maps follow gs_init_mapping entry for entry for any relative rotation of
 * neighbouring elements.  Faces with no neighbour become zero-Dirichlet when
 * dirichlet_boundary is non-zero.  Every solver and preconditioner accepts
 * any conforming mesh; hsmg's Schwarz ghost exchange follows each face
 * pairing (neighbour face and in-face orientation from the corner ids). */
nb_status nb_problem_create_mesh(int nelv, const int *vertex_ids, const double *vertex_xyz,
                                 int lx, double deform_amp, int dirichlet_boundary,
                                 nb_problem **out);
nb_status nb_problem_destroy(nb_problem *p);

/* Sizes: n = lx^3 * nelv local dofs. */
nb_status nb_problem_sizes(const nb_problem *p, int64_t *n, int *nelv, int *lx,
                           int *nlocal, int *nblocks, int *nmask);

/* Device pointer to a named field of the problem: "x","y","z","g11",
 * "g22","g33","g12","g13","g23","h1","h2","B","mult","dx","dxt", or a map
 * "dof_gs","gs_dof","blk_len","blk_off","msk" (int32, 1-based), or the
 * problem's device error word "err" (one int32, see nb_problem_sync).  Every field
 * is read-only for the caller: the solver keeps derived copies (the Jacobi
 * diagonal, an FP32 copy of mult, the hsmg levels) that a write through this
 * pointer would not update.  Change h1/h2 with nb_problem_set_coefficients. */
nb_status nb_problem_field(const nb_problem *p, const char *name, void **dptr);

/* Volume (sum of B) of the problem's mesh. */
nb_status nb_problem_volume(const nb_problem *p, double *vol);

/* Sets the Helmholtz coefficients from device arrays (n values each; h2 may
 * be NULL).  ifh2 enables the h2 B u term.  Synchronous: waits for all
 * device work before reading the arrays and returns when the Jacobi
 * diagonal (and any hsmg coarse level) has been updated. */
nb_status nb_problem_set_coefficients(nb_problem *p, const double *h1,
                                      const double *h2, int ifh2);

/* Constant coefficients h1 > 0 and h2 >= 0 (h2 = 0 turns the h2 B u term
 * off), set asynchronously on `stream`: the h1/h2 fields, the Jacobi
 * diagonal and the coarse levels of the problem's hsmg preconditioners are
 * rewritten by kernels on that stream, with no device synchronisation (the
 * form a serving loop uses between the solves of one problem instance).
 * The same coefficients as nb_problem_set_coefficients with filled arrays. */
nb_status nb_problem_set_coefficients_const(nb_problem *p, double h1, double h2, void *stream);

/* w = A u (ax_helm incl. h2 term when enabled), element-local.
 * Asynchronous on `stream`; a bounded device wait that expires is recorded
 * in the problem's error word and reported by the next nb_problem_sync or
 * nb_solve on the same problem. */
nb_status nb_ax(nb_problem *p, double *w, const double *u, void *stream);
/* (au, av, aw) = A (u, v, w) for the three components of a vector field
 * (the velocity Helmholtz operator, incl. the h2 term when enabled), one
 * pass over the coefficients for the three.  ax_helm_t%compute_vector
 * (src/math/ax_helm.f90).  Asynchronous on `stream`. */
nb_status nb_ax_vector(nb_problem *p, double *au, double *av, double *aw, const double *u,
                       const double *v, const double *w, void *stream);
/* (au, av, aw) = A_stress (u, v, w), the full-stress operator (incl. the
 * h2 B term when enabled), ax_helm_full_t%compute_vector
 * (src/math/ax_helm_full.f90).  The cofactors of the coordinate map and
 * 1/jac (10 arrays of n doubles) are built on the first call and kept with
 * the problem; nb_problem_field also hands them out ("drdx" ... "dtdz",
 * "jacinv").  Asynchronous on `stream`. */
nb_status nb_ax_stress(nb_problem *p, double *au, double *av, double *aw, const double *u,
                       const double *v, const double *w, void *stream);
/* Synchronises `stream` and reports (then clears) the problem's error word:
 * NB_ERR_TIMEOUT when an earlier asynchronous call on this problem had a
 * bounded device wait expire.  No counterpart in the reference, whose
 * kernels have no bounded waits. */
nb_status nb_problem_sync(nb_problem *p, void *stream);
/* The direction update and operator of one CG iteration in one streaming
 * pass: pdir = z + beta pdir, w = A pdir (element-local, before the
 * gather-scatter), and *pap = sum over the local points of pdir * w (pap a
 * device double, may be NULL).  One launch when the problem has no mask and
 * no h2 term (lx 6, 8, 10); separate passes otherwise.  It fuses what
 * fusedcg_device_solve does with cuda_fusedcg_update_p followed by
 * ax_t%compute (src/krylov/bcknd/device/fusedcg_device.F90:382-384), and
 * adds the curvature sum.  Asynchronous on `stream`; calls on one problem
 * share its reduction scratch, so they must not overlap on the GPU. */
nb_status nb_ax_update_p(nb_problem *p, double *w, double *pdir, const double *z,
                         double beta, double *pap, void *stream);
/* u = gs_add(u): sum of all local copies of each shared point. */
nb_status nb_gs_add(nb_problem *p, double *u, void *stream);
/* x(msk) = 0 for the problem's Dirichlet mask. */
nb_status nb_bc_apply(nb_problem *p, double *x, void *stream);

typedef enum {
  NB_PC_JACOBI = 0,
  NB_PC_HSMG = 1,
  NB_PC_NONE = 2,
  NB_PC_HSMG_MIXED = 3, /* nb_pc_apply only: hsmg with FP32 smoothing levels */
  NB_PC_PHMG = 4        /* hybrid ph-multigrid (phmg_t): Chebyshev-Jacobi
                           smoothing on the polynomial levels, tree AMG on
                           the last (nb_phmg_init) */
} nb_pc_type;

typedef struct {
  int max_iter;        /* iteration cap */
  double abs_tol;      /* stop when sqrt(r'*mult*r)/sqrt(volume) < abs_tol */
  int pc;              /* nb_pc_type */
  int mixed;           /* 1: hsmg smoothing levels in FP32 (coarse CG, outer
                          Krylov, inner products in FP64); true residual
                          recomputed every 50 iterations */
  int coarse_iter;     /* hsmg coarse CG iterations (reference default 10) */
  double coarse_tol;   /* hsmg coarse CG absolute tolerance (default 1e-9) */
  int flexible;        /* 1: flexible CG (Polak-Ribiere beta) with a pc */
  int ksp;             /* NB_KSP_CG (default), NB_KSP_GMRES or NB_KSP_PIPECG */
  int m_restart;       /* GMRES vectors per restart cycle (<= 0: 30, the
                          reference's default; at most 64) */
} nb_solve_opts;

typedef enum {
  NB_KSP_CG = 0,     /* cg_device_solve (flexible when opts.flexible) */
  NB_KSP_GMRES = 1,  /* gmres_device_solve: restarted flexible GMRES,
                        src/krylov/bcknd/device/gmres_device.F90:319-487 */
  NB_KSP_PIPECG = 2  /* pipecg_device_solve: pipelined PCG, one fused
                        reduction an iteration (src/krylov/bcknd/device/
                        pipecg_device.F90); a symmetric preconditioner */
} nb_ksp_type;

typedef struct {
  int iter;
  double res_start;
  double res_final;
  int converged;
  int launches;  /* kernels this solve launched on the device */
} nb_solve_result;

/* Operators of the coupled three-component solve. */
typedef enum {
  NB_AX_HELM_VECTOR = 0, /* ax_helm on each component (ax_helm_t%compute_vector) */
  NB_AX_STRESS = 1       /* the full-stress operator (ax_helm_full_t) */
} nb_ax_op;

/* Solves the coupled system A (x, y, z) = (fx, fy, fz) for the three
 * velocity components from zero with CG sharing one set of scalars
 * (cg_cpld_device_solve, src/krylov/bcknd/device/cg_cpld_device.f90:
 * 292-417): inner products summed over the components, gs add and the
 * zero-Dirichlet mask on each component, opts.pc NB_PC_JACOBI (the
 * problem's Jacobi diagonal on each component) or NB_PC_NONE (anything
 * else: NB_ERR_UNSUPPORTED), opts.max_iter and opts.abs_tol as nb_solve;
 * the other options are ignored.  op is an nb_ax_op.  Device arrays of n
 * doubles; synchronous on `stream`.  The reference's three monitors carry
 * the same values; res is one of them. */
nb_status nb_solve_coupled(nb_problem *p, int op, double *x, double *y, double *z,
                           const double *fx, const double *fy, const double *fz,
                           const nb_solve_opts *opts, nb_solve_result *res, void *stream);

/* Builds (or rebuilds, when the settings changed) the problem's hsmg
 * preconditioner: levels lx -> 4 -> 2, Schwarz/FDM smoothers, coarse
 * Jacobi-CG of coarse_iter iterations to abs tol coarse_tol (<= 0: the
 * reference defaults 10 and 1e-9).  mixed = 1 builds the FP32-smoother
 * variant, kept beside the FP64 one.  Replaces hsmg_init /
 * hsmg_init_from_components (src/krylov/pc_hsmg.f90:145-365). */
nb_status nb_hsmg_init(nb_problem *p, int mixed, int coarse_iter, double coarse_tol);

/* Settings of the hybrid ph-multigrid preconditioner; a field <= 0 takes
 * the reference's default (src/multigrid/phmg.f90:141-180). */
typedef struct {
  int smoother_iterations; /* Chebyshev steps a level (default 3) */
  int n_schedule;          /* entries of schedule; 0: the default {3, 1} */
  int schedule[8];         /* polynomial degree of each coarser level, decreasing
                              (level lx = degree + 1; default lx -> 4 -> 2) */
  int coarse_levels;       /* tree-AMG levels on the last level (default 3) */
  int coarse_iterations;   /* AMG V-cycles an application (default 1) */
  int cheby_degree;        /* Chebyshev degree on the AMG levels (default 4) */
} nb_phmg_opts;

/* Builds (or rebuilds) the problem's phmg preconditioner: phmg_init_from_
 * components (src/multigrid/phmg.f90:184-421) with the tree-AMG set-up
 * (src/multigrid/tree_amg_multigrid.f90:111-228) and the eigenvalue
 * estimates of its first solve (150 power steps a smoothed level and a
 * level of the AMG).  The coarser levels take the first n values of the
 * problem's h1 at build time, as the reference does.  opts may be null
 * (defaults).  Synchronous.  The power steps' start vectors and the
 * aggregation's element order come from splitmix64 seeded 3901 (the
 * reference uses gfortran's random_number at seed 3901). */
nb_status nb_phmg_init(nb_problem *p, const nb_phmg_opts *opts);

/* Set-up figures of the problem's phmg (built with the defaults when
 * absent): what = 0 levels, 1 lx of level i, 2/3/4 the Chebyshev tha/dlt/
 * lambda_max of level i, 5 AMG levels, 6 entries of AMG level i, 7/8/9
 * tha/dlt/lambda_max of AMG level i, 10 kernels an application launches. */
nb_status nb_phmg_describe(nb_problem *p, int what, int i, double *out);

/* The tree-AMG aggregation alone, on the host (no device use): for nelv
 * elements of lx^3 points with face neighbours facet_neigh (6 per element,
 * 1-based, 0 = none), asking for coarse_levels levels.  Writes *nlvls (the
 * levels kept), nnodes[l-1] = aggregates of level l and finest[(l-1) * n0
 * + i] = the 0-based aggregate of level-0 point i (n0 = nelv lx^3) for l =
 * 1 .. nlvls-1.  aggregate_finest_level / aggregate_greedy
 * (src/multigrid/tree_amg_aggregate.f90). */
nb_status nb_tamg_aggregate(int nelv, int lx, const int *facet_neigh, int coarse_levels,
                            int *nlvls, int *nnodes, int *finest);

/* z = M r for preconditioner pc (NB_PC_HSMG, or NB_PC_HSMG_MIXED for the
 * FP32-smoother variant, or NB_PC_PHMG), r masked; uses the settings of
 * the last nb_hsmg_init / nb_phmg_init of that preconditioner (the
 * defaults when there was none).  The hsmg_solve of the reference
 * (src/krylov/pc_hsmg.f90:481-627); phmg_solve (src/multigrid/
 * phmg.f90:462-498). */
nb_status nb_pc_apply(nb_problem *p, int pc, double *z, const double *r, void *stream);

/* Solves A x = f (f already assembled and masked) from x0 = 0 with
 * preconditioned CG (opts.ksp = NB_KSP_CG; cg_device_solve,
 * src/krylov/bcknd/device/cg_device.f90:162-238), restarted flexible
 * GMRES (NB_KSP_GMRES; gmres_device_solve) or pipelined CG (NB_KSP_PIPECG;
 * pipecg_device_solve), entirely on the device with device-resident
 * scalars.  x and f are device arrays of n doubles. */
nb_status nb_solve(nb_problem *p, double *x, const double *f,
                   const nb_solve_opts *opts, nb_solve_result *res,
                   void *stream);

/* Projection of the right-hand side onto earlier solutions, the step around
 * the pressure solve of a time step (projection_t,
 * src/common/projection.f90): a basis X of up to L earlier solutions and
 * B = A X, A-orthonormal in the mult-weighted inner product.  Every call is
 * asynchronous on `stream` (the basis size and coefficients stay on the
 * device) except nb_projection_info and nb_projection_reorthogonalize.
 *   project_on:  b -= B (X^T b) twice, xbar = X (X^T b) (device_project_on,
 *                :553-622); call it on the assembled, masked right-hand side.
 *   project_back: x += xbar; x enters the basis (bcknd_project_back and
 *                device_proj_ortho, :317-358, :638-714), dropped when it is
 *                not independent to 1e-7.
 *   reorthogonalize: B = A X with the current coefficients, then modified
 *                Gram-Schmidt (device_reorthogonalize_basis, :426-473).
 *   clear: empty basis (bcknd_clear).  The activation step and time-step
 *   control of pre_solving/post_solving stay with the caller. */
typedef struct nb_projection nb_projection;
nb_status nb_projection_create(nb_problem *p, int L, nb_projection **out);
nb_status nb_projection_destroy(nb_projection *j);
nb_status nb_projection_clear(nb_projection *j, void *stream);
nb_status nb_projection_project_on(nb_projection *j, double *b, void *stream);
nb_status nb_projection_project_back(nb_projection *j, double *x, void *stream);
nb_status nb_projection_reorthogonalize(nb_projection *j, void *stream);
nb_status nb_projection_info(nb_projection *j, int *m, int *proj_m, double *proj_res,
                             void *stream);

/* x -= sum(x) / n over the n local points: the mean removal of a singular
 * (all-Neumann or periodic) pressure problem, device_ortho
 * (src/math/operators.f90:349-368 with glb_n_points = n), with the mean kept
 * on the device.  Asynchronous on `stream`. */
nb_status nb_ortho(nb_problem *p, double *x, void *stream);

/* Batched solves.  A batch advances many independent Jacobi-PCG solves
 * (same iteration as nb_solve with NB_PC_JACOBI) together: one iteration
 * of every active solve is one persistent Ax launch over a work queue of
 * (solve, element range) items sorted by lx, one gather-scatter launch and
 * one vector/reduction launch, replayed from a CUDA graph.  Problems may
 * differ in size and lx (4, 6, 8, 10); the Ax k-split per lx is chosen by
 * timing on first use.  Solves can be submitted and released between runs
 * (continuous batching); each solve's work vectors (4 n doubles) are
 * charged against hbm_budget_bytes (<= 0: unlimited), and a submit over
 * budget returns NB_ERR_OOM without side effects.  No counterpart in the
 * reference, which runs one ksp solve at a time. */
typedef struct nb_batch nb_batch;
nb_status nb_batch_create(int64_t hbm_budget_bytes, nb_batch **out);
void nb_batch_destroy(nb_batch *b);
/* Adds a solve of p with right-hand side f (assembled, masked) into x
 * (device buffers that stay valid until release); returns its slot. */
nb_status nb_batch_submit(nb_batch *b, nb_problem *p, const double *f, double *x,
                          double abs_tol, int max_iter, int *slot);
/* The same with constant coefficients h1 > 0, h2 >= 0 (h2 > 0 adds h2 B)
 * held by the slot instead of the problem's h1/h2 fields; the slot keeps
 * its own Jacobi diagonal (5 n doubles charged), so one problem's mesh,
 * geometric factors and gs maps can serve solves with different
 * coefficients. */
nb_status nb_batch_submit_coef(nb_batch *b, nb_problem *p, const double *f, double *x,
                               double abs_tol, int max_iter, double h1, double h2, int *slot);
/* Adds a solve of problem instance p run as its own Krylov solve inside the
 * batch's run loop, concurrently with the other slots on a pool of streams:
 * opts chooses CG or flexible CG, Jacobi or hsmg, FP64 or mixed precision
 * (opts->ksp must be NB_KSP_CG).  The constant coefficients h1 > 0, h2 >= 0
 * are set on p when the slot starts (nb_problem_set_coefficients_const).  p
 * belongs to the slot until it is released: give concurrent slots of one
 * mesh distinct problem instances.  The slot's Krylov vectors (4 n doubles)
 * are charged against the budget; its result is bit-identical to nb_solve
 * of the same problem with the same options.  Slot ids of these solves
 * start at 2^24. */
nb_status nb_batch_submit_solve(nb_batch *b, nb_problem *p, const double *f, double *x,
                                const nb_solve_opts *opts, double h1, double h2, int *slot);
/* Frees a slot (finished or not) and its budget. */
nb_status nb_batch_release(nb_batch *b, int slot);
/* Runs up to max_chunks graph replays (<= 0: until every solve finished);
 * *active receives the number of solves still running. */
nb_status nb_batch_run(nb_batch *b, int max_chunks, int *active, void *stream);
/* State of a slot: *done = 1 once it stopped (converged, NaN or max_iter). */
nb_status nb_batch_result(nb_batch *b, int slot, int *done, nb_solve_result *res);
/* Self-test of the library's bounded device waits (no counterpart in the
 * reference): a grid barrier that one block never reaches and an mbarrier
 * that nothing arrives on, each with a short poll limit; both must return
 * with their timeout flag set (1) instead of hanging.  Leaves the device
 * usable. */
nb_status nb_selftest_bounded_waits(int *barrier_timed_out, int *mbarrier_timed_out);

/* Autotuner record for lx: chosen k-split and the candidates' times (ms). */
nb_status nb_batch_tuning(nb_batch *b, int lx, int *ks, float *ms, int *ncand);

/* sum(a*b*c) over n device values, written to the host double *result,
 * allocating nothing.  No counterpart in the reference: it is cuda_glsc3 for
 * callers that must not call cudaMalloc (a solve running under a fixed,
 * pre-committed device-memory budget; a thread that must not trigger the
 * device synchronisation cudaMalloc can imply).  Scratch is a static
 * device array of 128 KB (+256 B) held on every device that loads the
 * library until exit; n above 33,554,432 is rejected with NB_ERR_ARG.  All
 * calls share that array, so calls that overlap on the GPU race.  The first
 * call on a device looks up the array's address (cudaGetSymbolAddress) and
 * should come before any stream capture.  Synchronises `stream`. */
nb_status nb_glsc3_noalloc(const double *a, const double *b, const double *c,
                           int n, double *result, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* NEKO_B200_H */
