// ctc_adjoint.cu -- adjoint of (rho, grad rho) (placeholder).
#include "ctc_internal.h"

namespace ctc {

int eval_adjoint(ctc_molecule* mol, const double* d_points, int64_t n, const double* v_rho,
                 const double* v_grad, double* dLdD, double* dLdR, cudaStream_t st) {
  (void)mol; (void)d_points; (void)n; (void)v_rho; (void)v_grad; (void)dLdD; (void)dLdR; (void)st;
  return fail(CTC_ERR_UNSUPPORTED, "adjoint not built yet");
}

}  // namespace ctc
