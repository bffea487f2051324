// ctc_adjoint.cu -- adjoint of (rho, grad rho) for grid functionals (no counterpart in the reference).
//
// For L = sum_g f(rho_g, grad rho_g) with v_rho = dL/drho_g and
// v_grad = dL/d(grad rho)_g (weights included; grid points and weights held
// fixed):
//   dL/dD_{mu nu} = sum_g v_rho phi_mu phi_nu
//                   + v_grad . (grad phi_mu phi_nu + phi_mu grad phi_nu)
//                 = 1/2 (Phi^T W + W^T Phi)_{mu nu},  W_g = v_rho phi_g + 2 v_grad . grad phi_g
//   (entries of D treated as independent), the XC-matrix build: a GEMM with
//   K = points, run here tile by tile on the FP64 matrix units over each
//   tile's screened (compact) AO set only, so its cost follows the screened
//   work and not M^2 per point;
//   dL/dR_{A,j} = sum_g sum_{mu on A} -2 v_rho d_j phi_mu G0_mu
//                 - 2 sum_k v_k (d_j d_k phi_mu G0_mu + d_j phi_mu Gk_mu),
//   with G0 = Phi D and Gk = (d_k Phi) D -- the forward contraction with a
//   force epilogue (ctc_tiles.cuh), since d phi_mu / d R_A = -grad phi_mu for
//   mu on atom A.
#include "ctc_tiles.cuh"

namespace ctc {

namespace {

// dL/dD on each tile's compact AO set.  With A[p][k] = phi_k(p) and
// W[p][k] = v_rho(p) phi_k(p) + 2 v_grad(p) . grad phi_k(p) for the tile's
// points p and compact AOs k, the tile adds S = A^T W + W^T A (symmetric) to
// the accumulator: blocks of 64 x 64 compact indices on and above the
// diagonal only, FP64 matrix units (mma.sync m8n8k4), scattered with atomics
// into the upper triangle (internal AO order; compact indices follow it, so
// an upper block holds mu <= nu).  Work items are (tile, block pair), listed
// tile by tile (adj_pair_offsets_kernel) and taken in that order by a
// persistent grid: the CTAs running at any moment share one or two tiles, so
// each tile's AO block (up to ~11 MB at the centre of a 1 000-atom molecule,
// where a tile keeps ~2 800 AOs and ~990 block pairs) is read from DRAM once
// and re-read from L2 by its block pairs.  (One CTA per tile walking all of
// its pairs re-read the block from DRAM once per block row: 555 MB per tile,
// L2 hit rate 10%.)  The tile's points are streamed 16 at a time through
// shared memory.
constexpr int kAdjThreads = 128;
constexpr int kAdjB = 64;          // compact indices per block side
constexpr int kAdjK = 16;          // points per shared-memory stage
constexpr int kAdjLd = kAdjB + 4;  // padded row of a stage (conflict-free fragment loads)

// offsets[t] = block pairs of tiles 0 .. t-1 (nb (nb + 1) / 2 per tile, nb =
// kt / 64), offsets[C] = all of them.  One block of 1024 threads.
constexpr int kAdjScanThreads = 1024;
__global__ void __launch_bounds__(kAdjScanThreads) adj_pair_offsets_kernel(TileBatch tb, int32_t* offsets) {
  using Scan = cub::BlockScan<int, kAdjScanThreads>;
  __shared__ typename Scan::TempStorage tmp;
  const int per = (tb.C + kAdjScanThreads - 1) / kAdjScanThreads;
  const int t0 = threadIdx.x * per, t1 = min(tb.C, t0 + per);
  int sum = 0;
  for (int t = t0; t < t1; ++t) {
    const int nb = tb.kt[t] / kAdjB;
    sum += nb * (nb + 1) / 2;
  }
  int before = 0, total = 0;
  Scan(tmp).ExclusiveSum(sum, before, total);
  for (int t = t0; t < t1; ++t) {
    offsets[t] = before;
    const int nb = tb.kt[t] / kAdjB;
    before += nb * (nb + 1) / 2;
  }
  if (threadIdx.x == 0) offsets[tb.C] = total;
}

__global__ void __launch_bounds__(kAdjThreads)
    adjoint_dd_kernel(TileBatch tb, const int32_t* __restrict__ offsets, const double* __restrict__ v_rho,
                      const double* __restrict__ v_grad, double* __restrict__ Cacc, int Mpad) {
  __shared__ double sA[2][kAdjK * kAdjLd];  // A of the row block, A of the column block
  __shared__ double sW[2][kAdjK * kAdjLd];  // W of the row block, W of the column block
  __shared__ double sv[128][4];             // v_rho, 2 v_x, 2 v_y, 2 v_z per point
  const int TP = tb.TP;
  const int64_t ldq = (int64_t)TP * tb.Kcap;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 1, wn = warp >> 1;  // 32 x 32 sub-block of the 64 x 64 block
  const int total = offsets[tb.C];
  int cur = -1;  // tile whose point weights are in sv
  for (int item = blockIdx.x; item < total; item += gridDim.x) {
    // tile of the item: the last t with offsets[t] <= item
    int lo = 0, hi = tb.C;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (offsets[mid] <= item) lo = mid;
      else hi = mid;
    }
    const int t = lo;
    const int nb = tb.kt[t] / kAdjB;
    int pq = item - offsets[t], bi = 0;  // pair index within the tile, row-major over bj >= bi
    while (pq >= nb - bi) {
      pq -= nb - bi;
      ++bi;
    }
    const int bj = bi + pq;
    const double* ao = tb.ao + (int64_t)t * tb.nq * ldq;  // (q, k, p) at ao[q * ldq + k * TP + p]
    const int32_t* am = tb.aomap + (int64_t)t * tb.Kcap;
    if (t != cur) {     // uniform across the block, as item is
      __syncthreads();  // every reader of the previous tile's sv is done
      for (int j = tid; j < TP; j += kAdjThreads) {
        const int64_t oi = tb.out[(int64_t)t * TP + j];
        const bool ok = oi >= 0 && finite_point(tb.xyz + 3 * ((int64_t)t * TP + j));
        sv[j][0] = ok ? v_rho[oi] : 0.0;
        for (int d = 0; d < 3; ++d) sv[j][1 + d] = (ok && v_grad) ? 2.0 * v_grad[3 * oi + d] : 0.0;
      }
      cur = t;
    }
    {
      double c[4][4][2];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) c[i][j][0] = c[i][j][1] = 0.0;
      for (int p0 = 0; p0 < TP; p0 += kAdjK) {
        __syncthreads();
        // stage A and W of both blocks for points p0 .. p0 + 15 ([point][k])
        for (int e = tid; e < 2 * kAdjK * kAdjB; e += kAdjThreads) {
          const int side = e / (kAdjK * kAdjB), r = e % (kAdjK * kAdjB);
          const int k = r / kAdjK, p = r % kAdjK;  // lanes run along points: coalesced
          const int kk = (side ? bj : bi) * kAdjB + k;
          const int64_t o = (int64_t)kk * TP + p0 + p;
          const double phi = ao[o];
          const double* v = sv[p0 + p];
          double w = v[0] * phi;
          if (v_grad) w += v[1] * ao[ldq + o] + v[2] * ao[2 * ldq + o] + v[3] * ao[3 * ldq + o];
          sA[side][p * kAdjLd + k] = phi;
          sW[side][p * kAdjLd + k] = w;
        }
        __syncthreads();
        // S_block += A_i^T W_j + W_i^T A_j over the stage's points
#pragma unroll
        for (int ks = 0; ks < kAdjK; ks += 4) {
          const int pr = (ks + (lane & 3)) * kAdjLd;
          double ai[4], wi[4], aj[4], wj[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            ai[i] = sA[0][pr + wm * 32 + i * 8 + (lane >> 2)];
            wi[i] = sW[0][pr + wm * 32 + i * 8 + (lane >> 2)];
          }
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            aj[j] = sA[1][pr + wn * 32 + j * 8 + (lane >> 2)];
            wj[j] = sW[1][pr + wn * 32 + j * 8 + (lane >> 2)];
          }
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              dmma(c[i][j][0], c[i][j][1], ai[i], wj[j]);
              dmma(c[i][j][0], c[i][j][1], wi[i], aj[j]);
            }
        }
      }
      // scatter the block (on the diagonal block only its upper half)
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int r = wm * 32 + i * 8 + (lane >> 2);
            const int cc = wn * 32 + j * 8 + 2 * (lane & 3) + h;
            if (bi == bj && r > cc) continue;
            const int mu = am[bi * kAdjB + r], nu = am[bj * kAdjB + cc];
            const double val = c[i][j][h];
            if (mu >= 0 && nu >= 0 && val != 0.0) atomicAdd(&Cacc[(int64_t)mu * Mpad + nu], val);
          }
    }
  }
}

// dLdD (caller's AO order) += 1/2 S, S held in the upper triangle of Cacc
// (internal order; mu <= nu).
__global__ void upper_to_dldd_kernel(const double* __restrict__ Cacc, int M, int Mpad,
                                     const int32_t* __restrict__ iperm, double* __restrict__ dLdD) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)M * M) return;
  const int r = iperm[i / M], c = iperm[i % M];
  dLdD[i] += 0.5 * Cacc[(int64_t)min(r, c) * Mpad + max(r, c)];
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
  int rc;
  if (dLdD) {
    // accumulator of S = A^T W + W^T A (upper triangle used)
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
  ForceArgs fa;
  fa.v_rho = v_rho;
  fa.v_grad = v_grad;
  fa.ao_atom = mol->d_ao_atom;
  fa.dLdR = dLdR;
  fa.natom = mol->natom;
  int nsm = 148;
  if ((rc = device_sm_count(&nsm)) != CTC_OK) return rc;
  rc = run_tiles(mol, src, n, TP, nq, deriv, st, [&](const TileBatch& tb) -> int {
    if (dLdD) {
      int r2;
      if ((r2 = mol->ws_adj.ensure(sizeof(int32_t) * ((size_t)tb.C + 1), st)) != CTC_OK) return r2;
      int32_t* offsets = (int32_t*)mol->ws_adj.p;
      adj_pair_offsets_kernel<<<1, kAdjScanThreads, 0, st>>>(tb, offsets);
      CTC_CUDA_TRY(cudaGetLastError());
      adjoint_dd_kernel<<<4 * nsm, kAdjThreads, 0, st>>>(tb, offsets, v_rho, v_grad, Cacc, Mpad);
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
    upper_to_dldd_kernel<<<(unsigned)((MM + 255) / 256), 256, 0, st>>>(Cacc, mol->M, Mpad,
                                                                        mol->d_ao_iperm, dLdD);
    CTC_CUDA_TRY(cudaGetLastError());
  }
  return CTC_OK;
}

}  // namespace ctc
