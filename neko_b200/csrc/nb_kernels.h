// nb_kernels.h -- launchers shared between the CUDA translation units.
#pragma once

#include <cuda_runtime.h>

#include "nb_internal.h"

namespace nb {

// Stream used by drop-in entry points that take none: the one set by
// nb_set_default_stream, else Neko's glb_cmd_queue when the program defines
// it, else the legacy default stream.
cudaStream_t default_stream();
void set_default_stream(cudaStream_t s);

template <typename T>
cudaError_t ax_helm(T *w, const T *u, const T *dx, const T *dy, const T *dz, const T *dxt,
                    const T *dyt, const T *dzt, const T *h1, const T *g11, const T *g22,
                    const T *g33, const T *g12, const T *g13, const T *g23, int nelv, int lx,
                    cudaStream_t s, const int *skip = nullptr);

// Persistent bulk-copy variant of ax_helm (dx = dy = dz); returns
// cudaErrorNotSupported when it has no instantiation for (T, lx) or the
// pointers are not 16-byte aligned.
template <typename T>
cudaError_t ax_helm_stream(T *w, const T *u, const T *D, const T *Dt, const T *h1,
                           const T *g11, const T *g22, const T *g33, const T *g12,
                           const T *g13, const T *g23, int nelv, int lx, cudaStream_t s,
                           const int *skip = nullptr, int *err = nullptr);

// True when dx, dy, dz (and dxt, dyt, dzt) hold the same lx x lx matrix
// (pointer-equal, or equal contents, compared once per pointer set).
bool same_derivatives(const void *dx, const void *dy, const void *dz, const void *dxt,
                      const void *dyt, const void *dzt, int lx);

// Reads and clears the error word of the drop-in cuda_ax_helm (0 = no
// error); kernels given a null error word record their timeouts there.
int take_dropin_error();
// Device address of that word on the current device (looked up once).
int *dropin_error_word();

// (au, av, aw) = A (u, v, w), h1 part, one set of coefficients
// (ax_vector.cu).
cudaError_t ax_helm_vector(double *au, double *av, double *aw, const double *u,
                           const double *v, const double *w, const double *D,
                           const double *Dt, const double *h1, const double *g11,
                           const double *g22, const double *g33, const double *g12,
                           const double *g13, const double *g23, int nelv, int lx,
                           cudaStream_t s, int *err, const int *skip = nullptr);

// (au, av, aw) = A_stress (u, v, w): the full-stress operator with
// cofactors cof[0..8] = drdx, drdy, drdz, dsdx, dsdy, dsdz, dtdx, dtdy, dtdz
// (ax_stress.cu), plus h2 B (u, v, w) when h2 is given (in the same pass on
// the streaming kernel).  Returns at once when *skip is set.
cudaError_t ax_stress(double *au, double *av, double *aw, const double *u, const double *v,
                      const double *w, const double *dx, const double *dy, const double *dz,
                      const double *h1, const double *jacinv, const double *const cof[9],
                      const double *w3, int nelv, int lx, cudaStream_t s, int *err,
                      const int *skip, const double *h2 = nullptr, const double *Bm = nullptr);
// au += h2 B u, av += h2 B v, aw += h2 B w
cudaError_t ax_stress_part2(double *au, double *av, double *aw, const double *u,
                            const double *v, const double *w, const double *h2,
                            const double *B, long n, cudaStream_t s, const int *skip);

struct CgState;
// p = z + beta p, w = A p (no gather-scatter) and pap = sum p * w in one
// streaming launch (ax_helm.cu).  With a CG state, beta is read from it,
// the launch returns at once when st->done is set, and pap and alpha =
// rtz / pap are written to it; without one, beta is the argument and pap
// goes to *pap_out (device, may be null).  cudaErrorNotSupported when lx or
// alignment is not covered.
// z may be FP32 (a mixed-precision preconditioner's output), widened as read.
template <typename TZ>
cudaError_t ax_cg_fused(double *w, double *p, const TZ *z, const double *D, const double *Dt,
                        const double *h1, const double *g11, const double *g22, const double *g33,
                        const double *g12, const double *g13, const double *g23, int nelv, int lx,
                        CgState *st, double beta, double *pap_out, double *partials,
                        unsigned *counter, int max_grid, cudaStream_t s, int *err);

// cuda_fdm_do_fast for nl 8..16 with the native FDM passes (pc_hsmg.cu);
// cudaErrorNotSupported for other nl.
cudaError_t fdm_dropin(double *eo, double *r, const double *s, const double *d, int nl, int nel,
                       cudaStream_t st);

// Grid size for streaming kernels: a multiple of the SM count.
int stream_grid(long n, int threads);

}  // namespace nb
