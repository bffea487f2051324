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
// so one pass computes the AO block of a chunk of points, then one kernel per
// chunk forms the G tiles and reduces them against the AO values in its
// epilogue: G never leaves the SM and each point's descriptors are finished
// in registers.  The FP64 contraction runs on the double-precision matrix
// units (mma.sync m8n8k4 f64); the tensor-core split form is in ctc_tc.cu.
#include <algorithm>
#include <cmath>

#include "ctc_internal.h"

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

namespace {

constexpr double kPi = 3.14159265358979323846;

// Per-point partial sums produced by the contraction epilogues:
//   s[0] rho, s[1..3] sum G0 d_k phi, s[4..9] Hb_ij = sum G0 d_i d_j phi,
//   s[10..15] Ha_ij = sum Gi d_j phi  (ij = xx xy xz yy yz zz)
__device__ __forceinline__ void finalize_point(const double* s, int nqa, int nq_ao,
                                               const ctc_outputs& o, int64_t idx,
                                               const ctc_params& prm) {
  const double rho = s[0];
  const double g0 = 2.0 * s[1], g1 = 2.0 * s[2], g2 = 2.0 * s[3];
  double H[6] = {0, 0, 0, 0, 0, 0};
  double tau = 0.0;
  if (nqa == 4) {
    for (int i = 0; i < 6; ++i) H[i] = 2.0 * (s[10 + i] + (nq_ao == 10 ? s[4 + i] : 0.0));
    tau = 0.5 * (s[10] + s[13] + s[15]);
  }
  const double lap = H[0] + H[3] + H[5];
  if (o.rho) o.rho[idx] = rho;
  if (o.grad) {
    o.grad[3 * idx] = g0;
    o.grad[3 * idx + 1] = g1;
    o.grad[3 * idx + 2] = g2;
  }
  if (o.hess) {
    double* h = o.hess + 9 * idx;
    h[0] = H[0]; h[1] = H[1]; h[2] = H[2];
    h[3] = H[1]; h[4] = H[3]; h[5] = H[4];
    h[6] = H[2]; h[7] = H[4]; h[8] = H[5];
  }
  if (o.lap) o.lap[idx] = lap;
  if (o.tau_pd) o.tau_pd[idx] = tau;
  if (o.tau_alpha) o.tau_alpha[idx] = tau + prm.alpha * lap;
  const double gsq = g0 * g0 + g1 * g1 + g2 * g2;
  if (o.rdg) {
    // s = 1/(2 (3 pi^2)^(1/3)) |grad rho| / rho^(4/3), ratio set to 1e-20 where
    // rho^(4/3) <= 1e-20 (src/evaluate_densbased.cu:44-89, src/cuda_utils.cu:71-84)
    const double pref = 0.5 / cbrt(3.0 * kPi * kPi);
    const double d43 = pow(rho, 4.0 / 3.0);
    const double q = d43 > 1e-20 ? sqrt(gsq) / d43 : 1e-20;
    o.rdg[idx] = pref * q;
  }
  if (o.shannon) o.shannon[idx] = rho * log(rho);
  double w = 0.0, tf = 0.0;
  if (o.weizsacker || o.gge) {
    const double den = 8.0 * rho;
    w = den > 1e-20 ? gsq / den : 1e-20;
  }
  if (o.thomas_fermi || o.gge) tf = 0.3 * pow(3.0 * kPi * kPi, 2.0 / 3.0) * pow(rho, 5.0 / 3.0);
  if (o.weizsacker) o.weizsacker[idx] = w;
  if (o.thomas_fermi) o.thomas_fermi[idx] = tf;
  if (o.gge) o.gge[idx] = tf + prm.gge_a * w + prm.gge_b * lap;
  if (o.general_ked) o.general_ked[idx] = tau + 0.25 * (prm.ked_a - 1.0) * lap;
}

// ------------------------------------------------------------------ FP64 contraction kernel
constexpr int BM = 128, BN = 64, BK = 32, STAGES = 3;
constexpr int A_LD = BK + 4;  // 36 doubles: conflict-free fragment loads
constexpr int B_LD = BN + 4;  // 68 doubles
constexpr int C_LD = BN + 1;
constexpr int A_STAGE = BM * A_LD, B_STAGE = BK * B_LD;
constexpr int kThreads = 256;
constexpr size_t kSmemPipe = sizeof(double) * STAGES * (A_STAGE + B_STAGE);
constexpr size_t kSmemC = sizeof(double) * BM * C_LD;
constexpr size_t kSmemFp64 = kSmemPipe > kSmemC ? kSmemPipe : kSmemC;

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int sz = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// One CTA owns PTS = 128/NQA points; tile row r holds quantity r / PTS of
// point r % PTS (quantity 0 = phi, 1..3 = d_k phi).  It sweeps all nu tiles
// of 64 columns, each with a full K loop over mu, and reduces every finished
// G tile against the AO values of its columns.
template <int NQA>
__global__ void __launch_bounds__(kThreads)
    fp64_local_kernel(const double* __restrict__ ao, int nq_ao, int ld,
                      const double* __restrict__ D, int Mpad, int64_t n, ctc_outputs out,
                      int64_t out_off, ctc_params prm) {
  constexpr int PTS = BM / NQA;
  constexpr int TPP = kThreads / PTS;  // epilogue threads per point
  constexpr int NS = NQA == 4 ? 16 : 4;
  extern __shared__ __align__(16) double smem[];
  double* sA = smem;
  double* sB = smem + STAGES * A_STAGE;
  double* sC = smem;  // aliases the pipeline after the K loop

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 3, wn = warp >> 2;
  const int64_t p0 = (int64_t)blockIdx.x * PTS;

  // epilogue ownership
  const int epl = tid / TPP, esub = tid % TPP;
  const int64_t ep = p0 + epl;
  double acc_s[NS];
#pragma unroll
  for (int i = 0; i < NS; ++i) acc_s[i] = 0.0;

  const int nkb = Mpad / BK;
  for (int n0 = 0; n0 < Mpad; n0 += BN) {
    double c[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) c[i][j][0] = c[i][j][1] = 0.0;

    auto load_stage = [&](int stage, int kb) {
      double* a = sA + stage * A_STAGE;
      double* b = sB + stage * B_STAGE;
      const int k0 = kb * BK;
      // A: 128 rows x 32 doubles = 2048 chunks of 16 B, 8 per thread
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        int ch = tid + i * kThreads;
        int r = ch >> 4, cc = (ch & 15) * 2;
        int q = r / PTS, pl = r % PTS;
        int64_t p = p0 + pl;
        bool v = p < n;
        const double* src = ao + ((v ? p : 0) * nq_ao + q) * (int64_t)ld + k0 + cc;
        cp_async16(a + r * A_LD + cc, src, v);
      }
      // B: 32 rows (k) x 64 doubles = 1024 chunks, 4 per thread
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        int ch = tid + i * kThreads;
        int r = ch >> 5, cc = (ch & 31) * 2;
        cp_async16(b + r * B_LD + cc, D + (int64_t)(k0 + r) * Mpad + n0 + cc, true);
      }
    };

    load_stage(0, 0);
    cp_async_commit();
    if (nkb > 1) load_stage(1, 1);
    cp_async_commit();
    for (int kb = 0; kb < nkb; ++kb) {
      if (kb + 2 < nkb) load_stage((kb + 2) % STAGES, kb + 2);
      cp_async_commit();
      cp_async_wait<2>();
      __syncthreads();
      const double* a = sA + (kb % STAGES) * A_STAGE;
      const double* b = sB + (kb % STAGES) * B_STAGE;
#pragma unroll
      for (int ks = 0; ks < BK; ks += 4) {
        double af[4], bf[4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
          af[i] = a[(wm * 32 + i * 8 + (lane >> 2)) * A_LD + ks + (lane & 3)];
#pragma unroll
        for (int j = 0; j < 4; ++j)
          bf[j] = b[(ks + (lane & 3)) * B_LD + wn * 32 + j * 8 + (lane >> 2)];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) dmma(c[i][j][0], c[i][j][1], af[i], bf[j]);
      }
      __syncthreads();
    }
    cp_async_wait<0>();
    __syncthreads();
    // stage the G tile
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        int r = wm * 32 + i * 8 + (lane >> 2);
        int cc = wn * 32 + j * 8 + 2 * (lane & 3);
        sC[r * C_LD + cc] = c[i][j][0];
        sC[r * C_LD + cc + 1] = c[i][j][1];
      }
    __syncthreads();
    if (ep < n) {
      const double* aop = ao + ep * (int64_t)nq_ao * ld + n0;
      for (int v = esub; v < BN; v += TPP) {
        const double G0 = sC[(0 * PTS + epl) * C_LD + v];
        const double phi = aop[v];
        acc_s[0] += G0 * phi;
        if (nq_ao >= 4) {
          const double d0 = aop[ld + v], d1 = aop[2 * ld + v], d2 = aop[3 * ld + v];
          acc_s[1] += G0 * d0;
          acc_s[2] += G0 * d1;
          acc_s[3] += G0 * d2;
          if (NQA == 4) {
            const double G1 = sC[(1 * PTS + epl) * C_LD + v];
            const double G2 = sC[(2 * PTS + epl) * C_LD + v];
            const double G3 = sC[(3 * PTS + epl) * C_LD + v];
            acc_s[10] += G1 * d0;
            acc_s[11] += G1 * d1;
            acc_s[12] += G1 * d2;
            acc_s[13] += G2 * d1;
            acc_s[14] += G2 * d2;
            acc_s[15] += G3 * d2;
            if (nq_ao == 10) {
#pragma unroll
              for (int h = 0; h < 6; ++h) acc_s[4 + h] += G0 * aop[(4 + h) * ld + v];
            }
          }
        }
      }
    }
    __syncthreads();
  }
  // reduce the TPP partial sums of each point (consecutive lanes)
#pragma unroll
  for (int i = 0; i < NS; ++i)
#pragma unroll
    for (int off = TPP / 2; off > 0; off >>= 1)
      acc_s[i] += __shfl_xor_sync(0xffffffffu, acc_s[i], off);
  if (esub == 0 && ep < n) {
    double s[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) s[i] = i < NS ? acc_s[i] : 0.0;
    finalize_point(s, NQA, nq_ao, out, out_off + ep, prm);
  }
}

}  // namespace

int fp64_local_chunk(ctc_molecule* mol, const LocalPlan& plan, const double* ao, int64_t n,
                     int64_t out_off, const ctc_params* prm, const ctc_outputs* out,
                     cudaStream_t st) {
  if (n <= 0) return CTC_OK;
  static bool attr_set[2] = {false, false};
  if (plan.nqa == 4) {
    if (!attr_set[1]) {
      CTC_CUDA_TRY(cudaFuncSetAttribute(fp64_local_kernel<4>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemFp64));
      attr_set[1] = true;
    }
    int64_t grid = (n + (BM / 4) - 1) / (BM / 4);
    fp64_local_kernel<4><<<(unsigned)grid, kThreads, kSmemFp64, st>>>(
        ao, plan.nq_ao, mol->Mpad, mol->d_D, mol->Mpad, n, *out, out_off, *prm);
  } else {
    if (!attr_set[0]) {
      CTC_CUDA_TRY(cudaFuncSetAttribute(fp64_local_kernel<1>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemFp64));
      attr_set[0] = true;
    }
    int64_t grid = (n + BM - 1) / BM;
    fp64_local_kernel<1><<<(unsigned)grid, kThreads, kSmemFp64, st>>>(
        ao, plan.nq_ao, mol->Mpad, mol->d_D, mol->Mpad, n, *out, out_off, *prm);
  }
  CTC_CUDA_TRY(cudaGetLastError());
  return CTC_OK;
}

int eval_local(ctc_molecule* mol, const PointSrc& src0, int64_t n, int precision,
               const ctc_params* prm, const ctc_outputs* out, cudaStream_t st) {
  if (n < 0) return fail(CTC_ERR_INVALID, "eval_local: negative point count");
  if (n == 0) return CTC_OK;
  if (precision != CTC_PREC_FP64 && precision != CTC_PREC_TC_SPLIT)
    return fail(CTC_ERR_INVALID, "eval_local: unknown precision " + std::to_string(precision));
  const LocalPlan plan = plan_local(out);
  if (precision == CTC_PREC_TC_SPLIT) {
    int rc = prepare_tc(mol, st);
    if (rc != CTC_OK) return rc;
  }
  const int64_t chunk = std::min<int64_t>(chunk_points(mol, plan.nq_ao), n);
  const size_t ao_bytes = sizeof(double) * (size_t)chunk * plan.nq_ao * mol->Mpad;
  int rc = mol->ws_ao.ensure(ao_bytes, st);
  if (rc != CTC_OK) return rc;
  double* ao = (double*)mol->ws_ao.p;
  for (int64_t c0 = 0; c0 < n; c0 += chunk) {
    const int64_t nc = std::min(chunk, n - c0);
    PointSrc src = src0;
    src.offset += c0;
    if (mol->Mpad > mol->M) {
      CTC_CUDA_TRY(cudaMemset2DAsync(ao + mol->M, sizeof(double) * mol->Mpad, 0,
                                     sizeof(double) * (mol->Mpad - mol->M), nc * plan.nq_ao, st));
    }
    rc = launch_ao(mol, src, nc, plan.deriv, ao, plan.nq_ao, mol->Mpad, st);
    if (rc != CTC_OK) return rc;
    if (precision == CTC_PREC_FP64)
      rc = fp64_local_chunk(mol, plan, ao, nc, c0, prm, out, st);
    else
      rc = tc_local_chunk(mol, plan, ao, nc, c0, prm, out, st);
    if (rc != CTC_OK) return rc;
  }
  return CTC_OK;
}

}  // namespace ctc
