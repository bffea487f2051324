// ctc_local.cu -- local descriptors: planning, chunk loop, FP64 fused contraction.
//
// The reference evaluates every descriptor with its own sequence of AO kernel,
// cublasDgemm, Hadamard product and cublasDgemv, re-uploading D each time
// (src/evaluate_density.cu:663-840, src/evaluate_gradient.cu:1197-1422,
// src/evaluate_hessian.cu:1906-2307, src/evaluate_laplacian.cu:479-841,
// src/evaluate_kinetic_dens.cu:12-214, src/evaluate_densbased.cu:44-222).
// All of them are contractions of four products with D:
//     G0 = Phi D,  Gk = (d_k Phi) D   (k = x, y, z)
//     rho     = sum_nu G0 phi                     grad_k = 2 sum_nu G0 d_k phi
//     H_ij    = 2 [sum_nu Gi d_j phi + sum_nu G0 d_i d_j phi]
//     lap     = tr H                              tau_PD = 1/2 sum_k sum_nu Gk d_k phi
//
// Screening.  An AO contributes only where its shell reaches: on the
// 200-atom benchmark molecule ~9% of the AOs exceed 1e-14 at a typical grid
// point.  Points are therefore grouped into spatially compact tiles (3-D
// blocks of a cubic grid, or sort-tile-recursive runs of points), every tile builds
// its own list of significant segments (distance from the tile's bounding
// sphere below the segment's screening radius, where every AO value and
// derivative has dropped below 1e-18), and the contraction of that tile runs
// over its compacted AO set only: G_t = A_t D[S_t, S_t] with D gathered from
// L2 by index.  The AOs left out are below 1e-18 on the whole tile.
//
// Per chunk of tiles: screen -> AO block (compact) -> contraction + epilogue.
// The FP64 contraction runs on the double-precision matrix units (mma.sync
// m8n8k4 f64); the tensor-core split form is in ctc_tc.cu.
#include "ctc_tiles.cuh"

namespace ctc {

LocalPlan plan_local(const ctc_outputs* o) {
  bool need_rows4 = o->hess || o->lap || o->tau_pd || o->tau_alpha || o->gge || o->general_ked;
  bool need_d2 = o->hess || o->lap || o->tau_alpha || o->gge || o->general_ked;
  bool need_d1 = o->grad || o->rdg || o->weizsacker || o->gge || need_rows4;
  LocalPlan p;
  p.deriv = need_d2 ? 2 : (need_d1 ? 1 : 0);
  p.nq_ao = need_d2 ? 10 : (need_d1 ? 4 : 1);
  p.nqa = need_rows4 ? 4 : 1;
  return p;
}

int fp64_local_tiles(ctc_molecule* mol, const LocalPlan& plan, const TileBatch& tb,
                     const ctc_params* prm, const ctc_outputs* out, cudaStream_t st) {
  if (tb.C <= 0) return CTC_OK;
  int rc;
  if (plan.nqa == 4) {
    if ((rc = ensure_smem_attr((const void*)fp64_tile_kernel<4, 0>, (int)kSmemFp64)) != CTC_OK) return rc;
    fp64_tile_kernel<4, 0><<<tb.C, kThreads, kSmemFp64, st>>>(tb, mol->d_D, mol->Mpad, *out, *prm, ForceArgs{});
  } else {
    if ((rc = ensure_smem_attr((const void*)fp64_tile_kernel<1, 0>, (int)kSmemFp64)) != CTC_OK) return rc;
    fp64_tile_kernel<1, 0><<<tb.C, kThreads, kSmemFp64, st>>>(tb, mol->d_D, mol->Mpad, *out, *prm, ForceArgs{});
  }
  CTC_CUDA_TRY(cudaGetLastError());
  return CTC_OK;
}

int eval_local(ctc_molecule* mol, const PointSrc& src, int64_t n, int precision,
               const ctc_params* prm, const ctc_outputs* out, cudaStream_t st) {
  if (n < 0) return fail(CTC_ERR_INVALID, "eval_local: negative point count");
  if (n == 0) return CTC_OK;
  if (precision != CTC_PREC_FP64 && precision != CTC_PREC_TC_SPLIT)
    return fail(CTC_ERR_INVALID, "eval_local: unknown precision " + std::to_string(precision));
  if (!src.cubic && n > (int64_t)INT32_MAX)
    return fail(CTC_ERR_INVALID, "eval_local: at most 2^31-1 points per call");
  const LocalPlan plan = plan_local(out);
  // a failure an earlier stream-ordered call recorded on the device
  if (int rc = poll_status(mol, st); rc != CTC_OK) return rc;
  if (precision == CTC_PREC_TC_SPLIT) {
    if (int rc = prepare_tc(mol, st); rc != CTC_OK) return rc;
  }
  // points per tile: 128 rows of the contraction (32 points x 4 quantities or
  // 128 points x phi)
  const int TP = 128 / plan.nqa;
  const int rows = TP * plan.nqa;
  // tensor-core path: the AO kernel also writes the int8 digit planes
  const std::function<int(const TileBatch&)> sliced_ao = [&](const TileBatch& tb) {
    int8_t* planes = nullptr;
    int32_t* eexp = nullptr;
    const int32_t* order = nullptr;
    int r = tc_slice_workspace(mol, tb, plan.nqa, st, &planes, &eexp, &order);
    if (r != CTC_OK) return r;
    return launch_ao_tiles_sliced(mol, tb, plan.deriv, plan.nqa, planes, eexp, order, st);
  };
  int rc = run_tiles(
      mol, src, n, TP, plan.nq_ao, plan.deriv, st,
      [&](const TileBatch& tb) {
        int r;
        if (precision == CTC_PREC_FP64) {
          ProfScope ps(mol, 0, st);
          r = fp64_local_tiles(mol, plan, tb, prm, out, st);
        } else {
          r = tc_local_tiles(mol, plan, tb, prm, out, st);
        }
        mol->host_launches += 1;
        return r;
      },
      precision == CTC_PREC_TC_SPLIT ? &sliced_ao : nullptr, rows);
  if (rc != CTC_OK) return rc;
  // kernels report failures (bounded-wait timeouts of the tensor-core
  // kernels, a tile beyond the workspace capacity) through the status word:
  // its copy is enqueued here and read by a later call (no wait now)
  return post_status(mol, st);
}

}  // namespace ctc
