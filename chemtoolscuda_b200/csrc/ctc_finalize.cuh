// ctc_finalize.cuh -- the per-point end of every contraction kernel: the
// descriptors of one point from its partial sums (FP64 path, ctc_tiles.cuh,
// and tensor-core path, ctc_tc.cu, share this code).
//
// Formulas and masks follow the reference's drivers: rho, grad rho, Hessian
// and Laplacian (src/evaluate_density.cu:663-840, src/evaluate_gradient.cu:1197-1422,
// src/evaluate_hessian.cu:1906-2307, src/evaluate_laplacian.cu:479-841),
// tau_PD and tau_alpha (src/evaluate_kinetic_dens.cu:12-214), RDG, Shannon,
// Weizsacker, Thomas-Fermi, GGE and general(ish) KED
// (src/evaluate_densbased.cu:44-222, masked divides src/cuda_utils.cu:71-84).
#pragma once

#include <cstdint>

#include "ctc_internal.h"

namespace ctc {
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

__device__ __forceinline__ bool finite_point(const double* p) {
  return isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]);
}

// Every output of a point with a non-finite coordinate is NaN (the reference's
// kernels evaluate exp and powers of such a point and return NaN too).
__device__ __forceinline__ void nan_point(const ctc_outputs& o, int64_t idx) {
  const double q = __longlong_as_double(0x7ff8000000000000LL);
  if (o.rho) o.rho[idx] = q;
  if (o.grad)
    for (int k = 0; k < 3; ++k) o.grad[3 * idx + k] = q;
  if (o.hess)
    for (int k = 0; k < 9; ++k) o.hess[9 * idx + k] = q;
  double* one[] = {o.lap, o.tau_pd, o.tau_alpha, o.rdg, o.shannon, o.weizsacker,
                   o.thomas_fermi, o.gge, o.general_ked};
  for (double* p : one)
    if (p) p[idx] = q;
}

}  // namespace
}  // namespace ctc
