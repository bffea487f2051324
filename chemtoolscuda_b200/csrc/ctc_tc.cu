// ctc_tc.cu -- tensor-core split-precision contraction (placeholder until the tcgen05 kernel lands).
#include "ctc_internal.h"

namespace ctc {

int prepare_tc(ctc_molecule* mol, cudaStream_t st) {
  (void)mol; (void)st;
  return fail(CTC_ERR_UNSUPPORTED, "tensor-core split path not built yet");
}

int tc_local_tiles(ctc_molecule* mol, const LocalPlan& plan, const TileBatch& tb,
                   const ctc_params* prm, const ctc_outputs* out, cudaStream_t st) {
  (void)mol; (void)plan; (void)tb; (void)prm; (void)out; (void)st;
  return fail(CTC_ERR_UNSUPPORTED, "tensor-core split path not built yet");
}

}  // namespace ctc
