// pc_hsmg.cu -- three-level hybrid Schwarz multigrid preconditioner
// (src/krylov/pc_hsmg.f90).  Placeholder until the levels are built.
#include <string>

#include "nb_precond.h"

namespace nb {

struct HsmgState {};

void hsmg_free(nb_problem *p) {
  delete p->hsmg;
  p->hsmg = nullptr;
}

nb_status hsmg_get(nb_problem *P, const nb_solve_opts &o, Precond **out) {
  (void)P;
  (void)o;
  *out = nullptr;
  set_error("hsmg preconditioner not available yet");
  return NB_ERR_UNSUPPORTED;
}

}  // namespace nb
