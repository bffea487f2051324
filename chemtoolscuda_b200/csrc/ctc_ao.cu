// ctc_ao.cu -- contracted Gaussian AOs and their first/second derivatives on points.
//
// Restates the reference's AO evaluation (src/evaluate_density.cu:25-393,
// src/evaluate_gradient.cu:18-1127, src/evaluate_hessian.cu:17-1835) in one
// generic form.  Every AO component of a segment is
//     phi_j(r) = sum_t c_t x^a y^b z^c * R0(r^2),   R0 = sum_k coef_k exp(-alpha_k r^2)
// (x, y, z relative to the shell centre; c_t from ctc_terms.inc).  With
// R1 = sum_k alpha_k coef_k exp(..) and R2 = sum_k alpha_k^2 coef_k exp(..),
//     d/dx   [x^a e] = a x^(a-1) R0 - 2 x^(a+1) R1
//     d2/dx2 [x^a e] = a(a-1) x^(a-2) R0 - 2(2a+1) x^a R1 + 4 x^(a+2) R2
//     d2/dxdy[x^a y^b e] = (a x^(a-1))(b y^(b-1)) R0 - 2(a x^(a-1) y^(b+1) + b x^(a+1) y^(b-1)) R1
//                         + 4 x^(a+1) y^(b+1) R2
// so one exponential per primitive serves every component and derivative.
//
// One thread evaluates one segment at a few points.  Segments are visited in
// an order sorted by type and primitive count, so a warp runs one code path.
// A segment whose centre is farther than its screening radius from the point
// (every value and derivative below 1e-18) writes zeros without evaluating
// exponentials.  Arithmetic is FP64 throughout.
#include "ctc_internal.h"
#include "ctc_split.cuh"

#include "ctc_terms.inc"

namespace ctc {

namespace {

constexpr int kAoThreads = 128;

__device__ __forceinline__ int ncomp_dev(int type) {
  switch (type) {
    case 0: return 1;
    case 1: return 3;
    case 2: return 6;
    case 3: return 5;
    case 4: return 10;
    case 5: return 7;
    case 6: return 15;
    default: return 9;
  }
}

// Evaluate one segment at one point: o[i * ld_q + j] for quantity i < nq_out
// and component j.  Outside the screening radius every entry is zero.
template <int DERIV>
__device__ __forceinline__ void eval_segment(const DevSeg& sg, const double* __restrict__ alpha,
                                             const double* __restrict__ coef, double px, double py,
                                             double pz, double* __restrict__ o, int64_t ld_q,
                                             int nq_out) {
  constexpr int NQ = DERIV == 0 ? 1 : (DERIV == 1 ? 4 : 10);
  const int nc = ncomp_dev(sg.type);
  const double x = px - sg.cx, y = py - sg.cy, z = pz - sg.cz;
  const double r2 = x * x + y * y + z * z;
  if (r2 > sg.rcut2) {
    for (int q = 0; q < nq_out; ++q)
      for (int j = 0; j < nc; ++j) o[q * ld_q + j] = 0.0;
    return;
  }
  double R0 = 0.0, R1 = 0.0, R2 = 0.0;
  for (int k = 0; k < sg.nprim; ++k) {
    const double a = alpha[sg.prim0 + k];
    const double e = coef[sg.prim0 + k] * exp(-a * r2);
    R0 += e;
    if (DERIV >= 1) R1 += a * e;
    if (DERIV >= 2) R2 += a * a * e;
  }
  // powers with two leading zeros: P[i] = x^(i-2), P[0] = P[1] = 0
  double X[9], Y[9], Z[9];
  X[0] = X[1] = Y[0] = Y[1] = Z[0] = Z[1] = 0.0;
  X[2] = Y[2] = Z[2] = 1.0;
#pragma unroll
  for (int i = 3; i < 9; ++i) {
    X[i] = X[i - 1] * x;
    Y[i] = Y[i - 1] * y;
    Z[i] = Z[i - 1] * z;
  }
  for (int j = 0; j < nc; ++j) {
    double q[NQ];
#pragma unroll
    for (int i = 0; i < NQ; ++i) q[i] = 0.0;
    const int tb = c_comp_off[sg.type][j], te = c_comp_off[sg.type][j + 1];
    for (int t = tb; t < te; ++t) {
      const Term T = c_terms[t];
      const int a = T.a, b = T.b, c = T.z;
      const double X0 = X[a + 2], Y0 = Y[b + 2], Z0 = Z[c + 2];
      q[0] += T.c * X0 * Y0 * Z0 * R0;
      if (DERIV >= 1) {
        const double Xa = a * X[a + 1], Xb = X[a + 3];
        const double Ya = b * Y[b + 1], Yb = Y[b + 3];
        const double Za = c * Z[c + 1], Zb = Z[c + 3];
        q[1] += T.c * Y0 * Z0 * (Xa * R0 - 2.0 * Xb * R1);
        q[2] += T.c * X0 * Z0 * (Ya * R0 - 2.0 * Yb * R1);
        q[3] += T.c * X0 * Y0 * (Za * R0 - 2.0 * Zb * R1);
        if (DERIV >= 2) {
          const double Xaa = a * (a - 1) * X[a], Xd = X[a + 4];
          const double Yaa = b * (b - 1) * Y[b], Yd = Y[b + 4];
          const double Zaa = c * (c - 1) * Z[c], Zd = Z[c + 4];
          q[4] += T.c * Y0 * Z0 * (Xaa * R0 - 2.0 * (2 * a + 1) * X0 * R1 + 4.0 * Xd * R2);
          q[5] += T.c * Z0 * (Xa * Ya * R0 - 2.0 * (Xa * Yb + Xb * Ya) * R1 + 4.0 * Xb * Yb * R2);
          q[6] += T.c * Y0 * (Xa * Za * R0 - 2.0 * (Xa * Zb + Xb * Za) * R1 + 4.0 * Xb * Zb * R2);
          q[7] += T.c * X0 * Z0 * (Yaa * R0 - 2.0 * (2 * b + 1) * Y0 * R1 + 4.0 * Yd * R2);
          q[8] += T.c * X0 * (Ya * Za * R0 - 2.0 * (Ya * Zb + Yb * Za) * R1 + 4.0 * Yb * Zb * R2);
          q[9] += T.c * X0 * Y0 * (Zaa * R0 - 2.0 * (2 * c + 1) * Z0 * R1 + 4.0 * Zd * R2);
        }
      }
    }
#pragma unroll
    for (int i = 0; i < NQ; ++i)
      if (i < nq_out) o[i * ld_q + j] = q[i];
  }
}

template <int DERIV>
__global__ void __launch_bounds__(kAoThreads)
    ao_kernel(const DevSeg* __restrict__ segs, const int32_t* __restrict__ order, int nseg,
              const double* __restrict__ alpha, const double* __restrict__ coef, PointSrc src,
              int64_t n, int ppb, double* __restrict__ out, int nq_out, int64_t ld_point,
              int64_t ld_q) {
  int si = blockIdx.x * kAoThreads + threadIdx.x;
  if (si >= nseg) return;
  const DevSeg sg = segs[order[si]];
  int64_t p_begin = (int64_t)blockIdx.y * ppb;
  int64_t p_end = min(p_begin + ppb, n);
  for (int64_t p = p_begin; p < p_end; ++p) {
    double px, py, pz;
    point_of(src, p, px, py, pz);
    eval_segment<DERIV>(sg, alpha, coef, px, py, pz, out + p * ld_point + sg.orig_ao0, ld_q, nq_out);
  }
}

// High 32 bits of |x| (sign cleared): ordered like |x|, and bits 20..30 hold
// the biased exponent.
__device__ __forceinline__ unsigned abs_hi(double x) {
  return (unsigned)__double2hiint(x) & 0x7fffffffu;
}

#include "ctc_ao_poly.inc"

// Type-specialised evaluation of one segment at one point: the polynomial
// code of every component has literal exponents (ctc_ao_poly.inc), so the
// powers stay in registers.  Same arithmetic as eval_segment.
template <int DERIV, int TYPE, int TRACK>
__device__ __forceinline__ void eval_typed(const DevSeg& sg, const double* __restrict__ alpha,
                                           const double* __restrict__ coef, double px, double py,
                                           double pz, double* __restrict__ o, int64_t ld_q,
                                           int64_t ldc, int nq_out, unsigned* mx) {
  constexpr int L = TYPE == 0 ? 0 : (TYPE == 1 ? 1 : (TYPE <= 3 ? 2 : (TYPE <= 5 ? 3 : 4)));
  constexpr int NC = TYPE == 0 ? 1 : TYPE == 1 ? 3 : TYPE == 2 ? 6 : TYPE == 3 ? 5
                     : TYPE == 4 ? 10 : TYPE == 5 ? 7 : TYPE == 6 ? 15 : 9;
  constexpr int NP = L + 5;  // powers x^(i-2) for i < NP
  const double x = px - sg.cx, y = py - sg.cy, z = pz - sg.cz;
  const double r2 = x * x + y * y + z * z;
  if (r2 > sg.rcut2) {
    for (int q = 0; q < nq_out; ++q)
#pragma unroll
      for (int j = 0; j < NC; ++j) o[q * ld_q + j * ldc] = 0.0;
    return;
  }
  double R0 = 0.0, R1 = 0.0, R2 = 0.0;
  for (int k = 0; k < sg.nprim; ++k) {
    const double a = alpha[sg.prim0 + k];
    const double e = coef[sg.prim0 + k] * exp(-a * r2);
    R0 += e;
    if (DERIV >= 1) R1 += a * e;
    if (DERIV >= 2) R2 += a * a * e;
  }
  double X[NP], Y[NP], Z[NP];
  X[0] = X[1] = Y[0] = Y[1] = Z[0] = Z[1] = 0.0;
  X[2] = Y[2] = Z[2] = 1.0;
#pragma unroll
  for (int i = 3; i < NP; ++i) {
    X[i] = X[i - 1] * x;
    Y[i] = Y[i - 1] * y;
    Z[i] = Z[i - 1] * z;
  }
  if constexpr (TYPE == 0) ao_poly_0<DERIV, TRACK>(X, Y, Z, R0, R1, R2, o, ld_q, ldc, nq_out, mx);
  else if constexpr (TYPE == 1) ao_poly_1<DERIV, TRACK>(X, Y, Z, R0, R1, R2, o, ld_q, ldc, nq_out, mx);
  else if constexpr (TYPE == 2) ao_poly_2<DERIV, TRACK>(X, Y, Z, R0, R1, R2, o, ld_q, ldc, nq_out, mx);
  else if constexpr (TYPE == 3) ao_poly_3<DERIV, TRACK>(X, Y, Z, R0, R1, R2, o, ld_q, ldc, nq_out, mx);
  else if constexpr (TYPE == 4) ao_poly_4<DERIV, TRACK>(X, Y, Z, R0, R1, R2, o, ld_q, ldc, nq_out, mx);
  else if constexpr (TYPE == 5) ao_poly_5<DERIV, TRACK>(X, Y, Z, R0, R1, R2, o, ld_q, ldc, nq_out, mx);
  else if constexpr (TYPE == 6) ao_poly_6<DERIV, TRACK>(X, Y, Z, R0, R1, R2, o, ld_q, ldc, nq_out, mx);
  else ao_poly_7<DERIV, TRACK>(X, Y, Z, R0, R1, R2, o, ld_q, ldc, nq_out, mx);
}

template <int DERIV, int TRACK>
__device__ __forceinline__ void eval_dispatch(const DevSeg& sg, const double* __restrict__ alpha,
                                              const double* __restrict__ coef, double px, double py,
                                              double pz, double* __restrict__ o, int64_t ld_q,
                                              int64_t ldc, int nq_out, unsigned* mx) {
  switch (sg.type) {
    case 0: eval_typed<DERIV, 0, TRACK>(sg, alpha, coef, px, py, pz, o, ld_q, ldc, nq_out, mx); break;
    case 1: eval_typed<DERIV, 1, TRACK>(sg, alpha, coef, px, py, pz, o, ld_q, ldc, nq_out, mx); break;
    case 2: eval_typed<DERIV, 2, TRACK>(sg, alpha, coef, px, py, pz, o, ld_q, ldc, nq_out, mx); break;
    case 3: eval_typed<DERIV, 3, TRACK>(sg, alpha, coef, px, py, pz, o, ld_q, ldc, nq_out, mx); break;
    case 4: eval_typed<DERIV, 4, TRACK>(sg, alpha, coef, px, py, pz, o, ld_q, ldc, nq_out, mx); break;
    case 5: eval_typed<DERIV, 5, TRACK>(sg, alpha, coef, px, py, pz, o, ld_q, ldc, nq_out, mx); break;
    case 6: eval_typed<DERIV, 6, TRACK>(sg, alpha, coef, px, py, pz, o, ld_q, ldc, nq_out, mx); break;
    default: eval_typed<DERIV, 7, TRACK>(sg, alpha, coef, px, py, pz, o, ld_q, ldc, nq_out, mx); break;
  }
}

// One CTA per tile; each warp takes one significant segment at a time and
// its lanes take the tile's points, so a warp always runs one segment type
// and its stores of one (quantity, AO) cover consecutive points.  Layout of
// the tile block: A[q][k][point] (point fastest).  Padding columns
// [ktrue, kt) are zeroed.
//
// SLICE = 4 or 1 also produces the row exponents of the tensor-core split
// operands of the tile (ctc_split.cuh): the rows are the tile's points x {phi,
// d_x, d_y, d_z phi} (SLICE = 4, blocks of 32 points x 4 quantities, TP = 32)
// or its points x phi (SLICE = 1, TP <= 256).  Every lane keeps the running
// maximum of its values while it evaluates, so the exponents cost no second
// pass over the block; slice_rows_kernel then writes the digit planes.
template <int DERIV, int SLICE>
__global__ void __launch_bounds__(kAoThreads, 3)
    ao_tile_kernel(const DevSeg* __restrict__ segs, int nseg, const double* __restrict__ alpha,
                   const double* __restrict__ coef, TileBatch tb, int32_t* __restrict__ eexp,
                   const int32_t* __restrict__ order) {
  // per-warp maxima of the high word of |value| per row, [warp][row]
  constexpr int kMaxRows = 256;
  __shared__ unsigned s_mx[SLICE ? kAoThreads / 32 : 1][SLICE ? kMaxRows : 1];
  const int t = order ? order[blockIdx.x] : blockIdx.x;
  const int ns = tb.nsig[t], TP = tb.TP;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int32_t* sl = tb.segs + (int64_t)t * nseg;
  const int32_t* k0 = tb.k0 + (int64_t)t * nseg;
  const double* xyz = tb.xyz + (int64_t)t * TP * 3;
  double* A = tb.ao + (int64_t)t * tb.nq * TP * tb.Kcap;
  const int64_t ld_q = (int64_t)TP * tb.Kcap;
  for (int pg = 0; pg < TP; pg += 32) {
    const int j = pg + lane;
    const double px = xyz[3 * j], py = xyz[3 * j + 1], pz = xyz[3 * j + 2];
    unsigned mx[4] = {0u, 0u, 0u, 0u};
    for (int i = warp; i < ns; i += kAoThreads / 32) {
      const DevSeg sg = segs[sl[i]];
      eval_dispatch<DERIV, SLICE>(sg, alpha, coef, px, py, pz, A + (int64_t)k0[i] * TP + j, ld_q, TP,
                                  tb.nq, mx);
    }
    if (SLICE == 4) {
#pragma unroll
      for (int q = 0; q < 4; ++q) s_mx[SLICE ? warp : 0][SLICE ? (pg / 32) * 128 + q * 32 + lane : 0] = mx[q];
    } else if (SLICE == 1) {
      s_mx[SLICE ? warp : 0][SLICE ? j : 0] = mx[0];
    }
  }
  const int kt_true = tb.ktrue[t], kt = tb.kt[t];
  const int npad = (kt - kt_true) * TP;
  for (int idx = threadIdx.x; idx < tb.nq * npad; idx += kAoThreads) {
    const int q = idx / npad, r = idx % npad;
    A[q * ld_q + (int64_t)kt_true * TP + r] = 0.0;
  }
  if (SLICE != 0) {
    __syncthreads();  // row maxima of every warp are in shared memory
    const int rows = split_tile_rows(TP, SLICE);
    for (int r = threadIdx.x; r < rows; r += kAoThreads) {
      unsigned m = 0u;
#pragma unroll
      for (int w = 0; w < kAoThreads / 32; ++w) m = max(m, s_mx[SLICE ? w : 0][SLICE ? r : 0]);
      // |x| = 1.f 2^(E - 1023) < 2^(E - 1022) for the biased exponent E of the
      // largest |x| (frexp's exponent); a row of zeros gets 0
      const int E = (int)(m >> 20);
      const int e = m == 0u ? 0 : E - 1022;
      eexp[(int64_t)t * rows + r] = e < kMinScaleExponent ? kMinScaleExponent : e;
    }
  }
}

// Digit planes of the tile rows (ctc_split.cuh) with the exponents found by
// ao_tile_kernel.  One block per tile, the tiles taken in the chunk's order
// (largest compact K first) when one is given.  Work items are (32-row
// group, 32-column chunk); the block's warps take them in turn: a warp reads
// one 256-byte line per column (32 consecutive rows = points of one
// quantity), all 32 lines before any conversion so that they are in flight
// together, and each lane writes 32 bytes per plane of its own row.
constexpr int kSliceThreads = 256;

__global__ void __launch_bounds__(kSliceThreads, 2)
    slice_rows_kernel(TileBatch tb, int nqa, const int32_t* __restrict__ eexp,
                      int8_t* __restrict__ planes, const int32_t* __restrict__ order) {
  const int t = order ? order[blockIdx.x] : blockIdx.x;
  const int kt = tb.kt[t];
  const int TP = tb.TP;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t ld_q = (int64_t)TP * tb.Kcap;
  const double* A = tb.ao + (int64_t)t * tb.nq * ld_q;
  const int rows = split_tile_rows(TP, nqa);
  int8_t* P = planes + (int64_t)t * kSplitPlanesA * rows * tb.Kcap;
  const int nitem = (rows / 32) * (kt / 32);  // warp-sized items
  for (int it = warp; it < nitem; it += kSliceThreads / 32) {
    const int rg = it % (rows / 32), c = it / (rows / 32);
    const int r = rg * 32 + lane;             // tile row
    const int blk = r / kSplitRows;           // 128-row block of the row
    const int q = nqa == 4 ? rg % 4 : 0;      // quantity
    const int p = nqa == 4 ? blk * 32 + lane : r;  // point
    const double f = split_row_factor(eexp[(int64_t)t * rows + r], kFixedBitsA);
    const double* col = A + q * ld_q + p + (int64_t)(c * 32) * TP;
    double v[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __ldg(col + (int64_t)i * TP);
    write_row_digits32([&](int i) { return v[i]; }, f,
                       P + (int64_t)blk * kSplitPlanesA * kSplitRows * tb.Kcap, r % kSplitRows,
                       tb.Kcap, c * 32);
  }
}

}  // namespace

static int launch_ao_impl(const ctc_molecule* mol, const PointSrc& src, int64_t n, int deriv,
                          double* out, int nq_out, int64_t ld_point, int64_t ld_q, cudaStream_t st) {
  if (n <= 0) return CTC_OK;
  int ppb = 4;
  int64_t gy = (n + ppb - 1) / ppb;
  if (gy > 65535) {
    ppb = (int)((n + 65534) / 65535);
    gy = (n + ppb - 1) / ppb;
  }
  dim3 grid((mol->nseg + kAoThreads - 1) / kAoThreads, (unsigned)gy);
  switch (deriv) {
    case 0:
      ao_kernel<0><<<grid, kAoThreads, 0, st>>>(mol->d_segs, mol->d_order, mol->nseg, mol->d_alpha,
                                                mol->d_coef, src, n, ppb, out, nq_out, ld_point, ld_q);
      break;
    case 1:
      ao_kernel<1><<<grid, kAoThreads, 0, st>>>(mol->d_segs, mol->d_order, mol->nseg, mol->d_alpha,
                                                mol->d_coef, src, n, ppb, out, nq_out, ld_point, ld_q);
      break;
    default:
      ao_kernel<2><<<grid, kAoThreads, 0, st>>>(mol->d_segs, mol->d_order, mol->nseg, mol->d_alpha,
                                                mol->d_coef, src, n, ppb, out, nq_out, ld_point, ld_q);
  }
  CTC_CUDA_TRY(cudaGetLastError());
  return CTC_OK;
}

// Local-descriptor layout: out[(p * nq_out + q) * ld + ao]; AO columns beyond
// M (padding up to Mpad) are left untouched and must be zeroed by the caller.
int launch_ao(const ctc_molecule* mol, const PointSrc& src, int64_t n, int deriv, double* out,
              int nq_out, int ld, cudaStream_t st) {
  return launch_ao_impl(mol, src, n, deriv, out, nq_out, (int64_t)nq_out * ld, ld, st);
}

int launch_ao_tiles(const ctc_molecule* mol, const TileBatch& tb, int deriv, cudaStream_t st) {
  if (tb.C <= 0) return CTC_OK;
  const auto* sg = mol->d_segs;
  switch (deriv) {
    case 0: ao_tile_kernel<0, 0><<<tb.C, kAoThreads, 0, st>>>(sg, mol->nseg, mol->d_alpha, mol->d_coef, tb, nullptr, nullptr); break;
    case 1: ao_tile_kernel<1, 0><<<tb.C, kAoThreads, 0, st>>>(sg, mol->nseg, mol->d_alpha, mol->d_coef, tb, nullptr, nullptr); break;
    default: ao_tile_kernel<2, 0><<<tb.C, kAoThreads, 0, st>>>(sg, mol->nseg, mol->d_alpha, mol->d_coef, tb, nullptr, nullptr);
  }
  CTC_CUDA_TRY(cudaGetLastError());
  return CTC_OK;
}

int launch_ao_tiles_sliced(const ctc_molecule* mol, const TileBatch& tb, int deriv, int nqa,
                           int8_t* planes, int32_t* eexp, const int32_t* order, cudaStream_t st) {
  if (tb.C <= 0) return CTC_OK;
  if (!(nqa == 4 && tb.TP == 32 && deriv >= 1) && !(nqa == 1 && tb.TP == 128))
    return fail(CTC_ERR_INVALID, "sliced AO tiles: unsupported row layout");
  if (planes == nullptr || eexp == nullptr)
    return fail(CTC_ERR_INVALID, "sliced AO tiles: null workspace");
  const auto* sg = mol->d_segs;
  const double *al = mol->d_alpha, *co = mol->d_coef;
  if (nqa == 4) {
    if (deriv == 1) ao_tile_kernel<1, 4><<<tb.C, kAoThreads, 0, st>>>(sg, mol->nseg, al, co, tb, eexp, order);
    else ao_tile_kernel<2, 4><<<tb.C, kAoThreads, 0, st>>>(sg, mol->nseg, al, co, tb, eexp, order);
  } else {
    switch (deriv) {
      case 0: ao_tile_kernel<0, 1><<<tb.C, kAoThreads, 0, st>>>(sg, mol->nseg, al, co, tb, eexp, order); break;
      case 1: ao_tile_kernel<1, 1><<<tb.C, kAoThreads, 0, st>>>(sg, mol->nseg, al, co, tb, eexp, order); break;
      default: ao_tile_kernel<2, 1><<<tb.C, kAoThreads, 0, st>>>(sg, mol->nseg, al, co, tb, eexp, order);
    }
  }
  CTC_CUDA_TRY(cudaGetLastError());
  slice_rows_kernel<<<tb.C, kSliceThreads, 0, st>>>(tb, nqa, eexp, planes, order);
  CTC_CUDA_TRY(cudaGetLastError());
  return CTC_OK;
}

// Public layout (nq, n, M).
int launch_ao_public(const ctc_molecule* mol, const PointSrc& src, int64_t n, int deriv,
                     double* out, cudaStream_t st) {
  int nq = deriv == 0 ? 1 : (deriv == 1 ? 4 : 10);
  return launch_ao_impl(mol, src, n, deriv, out, nq, mol->M, n * (int64_t)mol->M, st);
}

}  // namespace ctc
