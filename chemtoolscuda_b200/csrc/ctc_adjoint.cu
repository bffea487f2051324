// ctc_adjoint.cu -- adjoint of (rho, grad rho) for grid functionals (no counterpart in the reference).
//
// For L = sum_g f(rho_g, grad rho_g) with v_rho = dL/drho_g and
// v_grad = dL/d(grad rho)_g (weights included; grid points and weights held
// fixed):
//   dL/dD_{mu nu} = sum_g v_rho phi_mu phi_nu
//                   + v_grad . (grad phi_mu phi_nu + phi_mu grad phi_nu)
//                 = 1/2 (Phi^T W + W^T Phi)_{mu nu},  W_g = v_rho phi_g + 2 v_grad . grad phi_g
//   (entries of D treated as independent), the XC-matrix build: a GEMM with
//   K = points, run here on the FP64 matrix units over the screened AO blocks
//   of each chunk scattered into dense rows;
//   dL/dR_{A,j} = sum_g sum_{mu on A} -2 v_rho d_j phi_mu G0_mu
//                 - 2 sum_k v_k (d_j d_k phi_mu G0_mu + d_j phi_mu Gk_mu),
//   with G0 = Phi D and Gk = (d_k Phi) D -- the forward contraction with a
//   force epilogue (ctc_tiles.cuh), since d phi_mu / d R_A = -grad phi_mu for
//   mu on atom A.
#include "ctc_tiles.cuh"

namespace ctc {

namespace {

// Dense rows of a chunk: Phi[p][mu], W[p][mu] (p = tile * TP + j) from the compact AO block.
__global__ void densify_kernel(TileBatch tb, const double* __restrict__ v_rho,
                               const double* __restrict__ v_grad, double* __restrict__ Phi,
                               double* __restrict__ W, int Mpad) {
  const int t = blockIdx.x;
  const int TP = tb.TP, kt = tb.kt[t];
  const int64_t ldq = (int64_t)TP * tb.Kcap;
  const double* A = tb.ao + (int64_t)t * tb.nq * ldq;
  const int32_t* am = tb.aomap + (int64_t)t * tb.Kcap;
  for (int idx = threadIdx.x; idx < TP * kt; idx += blockDim.x) {
    const int j = idx % TP, k = idx / TP;
    const int mu = am[k];
    const int64_t oi = tb.out[(int64_t)t * TP + j];
    if (mu < 0 || oi < 0) continue;
    const double phi = A[(int64_t)k * TP + j];
    double w = v_rho[oi] * phi;
    if (v_grad)
      for (int d = 0; d < 3; ++d) w += 2.0 * v_grad[3 * oi + d] * A[(1 + d) * ldq + (int64_t)k * TP + j];
    const int64_t row = ((int64_t)t * TP + j) * Mpad;
    Phi[row + mu] = phi;
    W[row + mu] = w;
  }
}

// C[mu][nu] += sum_p A[p][mu] B[p][nu] over p in [k_begin, k_end): 128 x 64 tiles,
// split K across blockIdx.z, double-precision MMA, atomic accumulation of the tile.
constexpr int TN_BM = 128, TN_BN = 64, TN_BK = 32;
constexpr int TN_ALD = TN_BM + 4, TN_BLD = TN_BN + 4;
constexpr int kSmemTn = (int)sizeof(double) * 2 * TN_BK * (TN_ALD + TN_BLD);

__global__ void __launch_bounds__(256)
    gemm_tn_kernel(const double* __restrict__ A, const double* __restrict__ B, int64_t P, int Mpad,
                   int64_t kchunk, double* __restrict__ C) {
  extern __shared__ __align__(16) double tn_smem[];
  double (*sA)[TN_BK * TN_ALD] = reinterpret_cast<double (*)[TN_BK * TN_ALD]>(tn_smem);
  double (*sB)[TN_BK * TN_BLD] = reinterpret_cast<double (*)[TN_BK * TN_BLD]>(tn_smem + 2 * TN_BK * TN_ALD);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 3, wn = warp >> 2;
  const int m0 = blockIdx.y * TN_BM, n0 = blockIdx.x * TN_BN;
  const int64_t kb0 = (int64_t)blockIdx.z * kchunk;
  const int64_t kb1 = min(P, kb0 + kchunk);
  double c[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) c[i][j][0] = c[i][j][1] = 0.0;
  auto load = [&](int stage, int64_t k0) {
    // A: 32 rows (points) x 128 doubles = 2048 chunks of 16 B, 8 per thread
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int ch = tid + i * 256;
      const int r = ch >> 6, cc = (ch & 63) * 2;
      const int64_t p = k0 + r;
      const bool v = p < kb1;
      cp_async16(&sA[stage][r * TN_ALD + cc], A + (v ? p : 0) * Mpad + m0 + cc, v);
    }
    // B: 32 rows x 64 doubles = 1024 chunks, 4 per thread
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int ch = tid + i * 256;
      const int r = ch >> 5, cc = (ch & 31) * 2;
      const int64_t p = k0 + r;
      const bool v = p < kb1;
      cp_async16(&sB[stage][r * TN_BLD + cc], B + (v ? p : 0) * Mpad + n0 + cc, v);
    }
  };
  if (kb0 < kb1) load(0, kb0);
  cp_async_commit();
  int stage = 0;
  for (int64_t k0 = kb0; k0 < kb1; k0 += TN_BK, stage ^= 1) {
    if (k0 + TN_BK < kb1) load(stage ^ 1, k0 + TN_BK);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    const double* a = sA[stage];
    const double* b = sB[stage];
#pragma unroll
    for (int ks = 0; ks < TN_BK; ks += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) af[i] = a[(ks + (lane & 3)) * TN_ALD + wm * 32 + i * 8 + (lane >> 2)];
#pragma unroll
      for (int j = 0; j < 4; ++j) bf[j] = b[(ks + (lane & 3)) * TN_BLD + wn * 32 + j * 8 + (lane >> 2)];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(c[i][j][0], c[i][j][1], af[i], bf[j]);
    }
    __syncthreads();
  }
  cp_async_wait<0>();
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int r = m0 + wm * 32 + i * 8 + (lane >> 2);
      const int cc = n0 + wn * 32 + j * 8 + 2 * (lane & 3);
      if (c[i][j][0] != 0.0) atomicAdd(&C[(int64_t)r * Mpad + cc], c[i][j][0]);
      if (c[i][j][1] != 0.0) atomicAdd(&C[(int64_t)r * Mpad + cc + 1], c[i][j][1]);
    }
}

// dLdD in the caller's AO order from the accumulator in internal order.
__global__ void symmetrize_add_kernel(const double* __restrict__ Cacc, int M, int Mpad,
                                      const int32_t* __restrict__ iperm, double* __restrict__ dLdD) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)M * M) return;
  const int r = iperm[i / M], c = iperm[i % M];
  dLdD[i] += 0.5 * (Cacc[(int64_t)r * Mpad + c] + Cacc[(int64_t)c * Mpad + r]);
}

}  // namespace

int eval_adjoint(ctc_molecule* mol, const double* d_points, int64_t n, const double* v_rho,
                 const double* v_grad, double* dLdD, double* dLdR, cudaStream_t st) {
  if (n > (int64_t)INT32_MAX) return fail(CTC_ERR_INVALID, "adjoint: at most 2^31-1 points per call");
  PointSrc src{};
  src.pts = d_points;
  const int deriv = v_grad ? 2 : 1;
  const int nq = v_grad ? 10 : 4;
  const int nqa = (dLdR && v_grad) ? 4 : 1;
  const int TP = 128 / nqa;
  const int Mpad = mol->Mpad;
  double* Cacc = nullptr;
  double* Phi = nullptr;
  double* W = nullptr;
  int rc;
  if (dLdD) {
    // accumulator, then room for the densified rows of the largest chunk
    const size_t cbytes = sizeof(double) * (size_t)Mpad * Mpad;
    if ((rc = mol->ws_sl.ensure(cbytes, st)) != CTC_OK) return rc;
    Cacc = (double*)mol->ws_sl.p;
    CTC_CUDA_TRY(cudaMemsetAsync(Cacc, 0, cbytes, st));
  }
  if (dLdR) {
    rc = nqa == 4 ? ensure_smem_attr((const void*)fp64_tile_kernel<4, 1>, (int)kSmemFp64)
                  : ensure_smem_attr((const void*)fp64_tile_kernel<1, 1>, (int)kSmemFp64);
    if (rc != CTC_OK) return rc;
  }
  if (dLdD && (rc = ensure_smem_attr((const void*)gemm_tn_kernel, kSmemTn)) != CTC_OK) return rc;
  ForceArgs fa;
  fa.v_rho = v_rho;
  fa.v_grad = v_grad;
  fa.ao_atom = mol->d_ao_atom;
  fa.dLdR = dLdR;
  fa.natom = mol->natom;
  rc = run_tiles(mol, src, n, TP, nq, deriv, st, [&](const TileBatch& tb) -> int {
    if (dLdD) {
      const int64_t rows = (int64_t)tb.C * tb.TP;
      const size_t dbytes = sizeof(double) * (size_t)rows * Mpad;
      if (!Phi) {
        // dense rows live after the accumulator in the same scratch (grown once)
        const size_t cbytes = sizeof(double) * (size_t)Mpad * Mpad;
        const size_t need = cbytes + 2 * dbytes + 512;
        if (mol->ws_sl.bytes < need) {
          // grow preserving the accumulator contents
          void* old = mol->ws_sl.p;
          void* fresh = nullptr;
          CTC_CUDA_TRY(cudaMallocAsync(&fresh, need, st));
          CTC_CUDA_TRY(cudaMemcpyAsync(fresh, old, cbytes, cudaMemcpyDeviceToDevice, st));
          CTC_CUDA_TRY(cudaFreeAsync(old, st));
          mol->ws_sl.p = fresh;
          mol->ws_sl.bytes = need;
          Cacc = (double*)fresh;
        }
        Phi = (double*)((char*)mol->ws_sl.p + (cbytes + 255) / 256 * 256);
        W = (double*)((char*)Phi + (dbytes + 255) / 256 * 256);
      }
      CTC_CUDA_TRY(cudaMemsetAsync(Phi, 0, dbytes, st));
      CTC_CUDA_TRY(cudaMemsetAsync(W, 0, dbytes, st));
      densify_kernel<<<tb.C, 256, 0, st>>>(tb, v_rho, v_grad, Phi, W, Mpad);
      CTC_CUDA_TRY(cudaGetLastError());
      const int tiles = (Mpad / TN_BM) * (Mpad / TN_BN);
      int splits = (int)std::max<int64_t>(1, std::min<int64_t>((2 * 148 + tiles - 1) / tiles, rows / 256));
      int64_t kchunk = (rows + splits - 1) / splits;
      kchunk = (kchunk + TN_BK - 1) / TN_BK * TN_BK;
      splits = (int)((rows + kchunk - 1) / kchunk);
      dim3 grid(Mpad / TN_BN, Mpad / TN_BM, splits);
      gemm_tn_kernel<<<grid, 256, kSmemTn, st>>>(Phi, W, rows, Mpad, kchunk, Cacc);
      CTC_CUDA_TRY(cudaGetLastError());
      mol->host_launches += 2;
    }
    if (dLdR) {
      if (nqa == 4)
        fp64_tile_kernel<4, 1><<<tb.C, kThreads, kSmemFp64, st>>>(tb, mol->d_D, Mpad, ctc_outputs{},
                                                                 ctc_params{}, fa);
      else
        fp64_tile_kernel<1, 1><<<tb.C, kThreads, kSmemFp64, st>>>(tb, mol->d_D, Mpad, ctc_outputs{},
                                                                 ctc_params{}, fa);
      CTC_CUDA_TRY(cudaGetLastError());
      mol->host_launches += 1;
    }
    return CTC_OK;
  });
  if (rc != CTC_OK) return rc;
  if (dLdD) {
    const int64_t MM = (int64_t)mol->M * mol->M;
    symmetrize_add_kernel<<<(unsigned)((MM + 255) / 256), 256, 0, st>>>(Cacc, mol->M, Mpad,
                                                                         mol->d_ao_iperm, dLdD);
    CTC_CUDA_TRY(cudaGetLastError());
  }
  return CTC_OK;
}

}  // namespace ctc
