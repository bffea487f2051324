// ctc_tc.cu -- tensor-core split-precision contraction (placeholder until the tcgen05 kernel lands).
#include "ctc_internal.h"

namespace ctc {

int prepare_tc(ctc_molecule* mol, cudaStream_t st) {
  (void)mol; (void)st;
  return fail(CTC_ERR_UNSUPPORTED, "tensor-core split path not built yet");
}

int tc_local_chunk(ctc_molecule* mol, const LocalPlan& plan, const double* ao, int64_t n,
                   int64_t out_offset, const ctc_params* prm, const ctc_outputs* out,
                   cudaStream_t st) {
  (void)mol; (void)plan; (void)ao; (void)n; (void)out_offset; (void)prm; (void)out; (void)st;
  return fail(CTC_ERR_UNSUPPORTED, "tensor-core split path not built yet");
}

}  // namespace ctc
