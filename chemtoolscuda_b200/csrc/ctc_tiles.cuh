// ctc_tiles.cuh -- the screened point-tile pipeline shared by the local
// descriptors (ctc_local.cu) and the adjoint (ctc_adjoint.cu).
//
// Points are grouped into spatially compact tiles (3-D blocks of a cubic grid,
// or sort-tile-recursive runs of explicit points); every tile lists the segments whose
// screening sphere (every AO value and derivative below 1e-18 outside it)
// meets the tile's bounding sphere, and works on that compacted AO set only.
// Per chunk of tiles: tile points -> screen -> AO block (compact) -> a
// contraction kernel supplied by the caller.
#pragma once

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <functional>

#include <cub/block/block_scan.cuh>
#include <cub/device/device_radix_sort.cuh>

#include "ctc_internal.h"
#include "ctc_finalize.cuh"

namespace ctc {

namespace {

__device__ __forceinline__ int ncomp_of_type_dev(int type) {
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

// ------------------------------------------------------------------ tiles
constexpr int kTileThreads = 256;
constexpr int kSortCap = 2048;  // segment lists up to this length are ordered by type

__device__ __forceinline__ uint32_t spread10(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

// 30-bit Morton key of each point (the single-sort order of small calls and
// of the fixed-scratch entry point, ctc_noalloc.cu); a point with a
// non-finite coordinate gets
// kNonFiniteKey, so the sort puts such points after every finite one and they
// share tiles only with each other (and at most one tile's finite points).
constexpr uint32_t kNonFiniteKey = 1u << 30;
constexpr int kMortonSortBits = 31;

__global__ void morton_kernel(const double* __restrict__ pts, int64_t n, double lox, double loy,
                              double loz, double inv_cell, uint32_t* keys, int32_t* vals) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  auto q = [&](double v, double lo) {
    double c = (v - lo) * inv_cell;
    c = c < 0.0 ? 0.0 : (c > 1023.0 ? 1023.0 : c);
    return (uint32_t)c;
  };
  const double x = pts[3 * i], y = pts[3 * i + 1], z = pts[3 * i + 2];
  keys[i] = isfinite(x) && isfinite(y) && isfinite(z)
                ? spread10(q(x, lox)) | (spread10(q(y, loy)) << 1) | (spread10(q(z, loz)) << 2)
                : kNonFiniteKey;
  vals[i] = (int32_t)i;
}

// Sort-tile-recursive packing of explicit points (Leutenegger, Lopez and
// Edgington, "STR: a simple and efficient algorithm for R-tree packing",
// ICDE 1997): sort by x and cut into sx slabs of whole tiles; sort each slab
// by y and cut it into sy columns; sort each column by z; tiles are then runs
// of TP consecutive points.  sx and sy follow the points' bounding box
// (edge a = (volume / P)^(1/3) for P tiles, sx ~ Lx / a, sy ~ Ly / a), so the
// tiles are close to cubes also for slab-shaped point sets such as a
// few-plane slice of a grid.  The box and the cut counts are formed on the
// device (every thread of the key kernel derives the same counts), so the
// host never waits.  Three radix sorts of 64-bit keys (group id << 32 |
// coordinate key); a point with a non-finite coordinate gets the largest
// coordinate key on every axis, so it sorts after every finite point and
// shares tiles only with its kind (and at most one tile's finite points).
__device__ __forceinline__ unsigned long long ordered_key(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double ordered_value(unsigned long long k) {
  return __longlong_as_double((long long)((k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k));
}
// box[0..2] = ordered keys of the minima, box[3..5] of the maxima (start at
// all-ones and zero); finite points only
__global__ void point_box_kernel(const double* __restrict__ pts, int64_t n, unsigned long long* box) {
  unsigned long long mn[3] = {~0ull, ~0ull, ~0ull}, mx[3] = {0ull, 0ull, 0ull};
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double* x = pts + 3 * i;
    if (!finite_point(x)) continue;
    for (int d = 0; d < 3; ++d) {
      const unsigned long long k = ordered_key(x[d]);
      mn[d] = k < mn[d] ? k : mn[d];
      mx[d] = k > mx[d] ? k : mx[d];
    }
  }
  for (int d = 0; d < 3; ++d)
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long a = __shfl_xor_sync(0xffffffffu, mn[d], o), b = __shfl_xor_sync(0xffffffffu, mx[d], o);
      mn[d] = a < mn[d] ? a : mn[d];
      mx[d] = b > mx[d] ? b : mx[d];
    }
  if ((threadIdx.x & 31) == 0)
    for (int d = 0; d < 3; ++d) {
      atomicMin(&box[d], mn[d]);
      atomicMax(&box[3 + d], mx[d]);
    }
}
struct StrShape {
  double lo[3], scale[3];  // coordinate key = (x - lo) * scale, clamped
  int64_t Sx, Scol, c;     // points per slab, points per column, columns per slab
};
__device__ StrShape str_shape(const unsigned long long* __restrict__ box, int64_t P, int TP) {
  StrShape sh;
  double L[3];
  bool any = box[0] <= box[3];
  double Lmax = 0.0;
  for (int d = 0; d < 3; ++d) {
    sh.lo[d] = any ? ordered_value(box[d]) : 0.0;
    L[d] = any ? ordered_value(box[3 + d]) - sh.lo[d] : 0.0;
    Lmax = fmax(Lmax, L[d]);
  }
  if (!(Lmax > 0.0)) Lmax = 1.0;
  for (int d = 0; d < 3; ++d) {
    L[d] = fmax(L[d], 1e-3 * Lmax);  // planar or linear sets: keep the volume positive
    sh.scale[d] = 4294967040.0 / L[d];
  }
  const double a = cbrt(L[0] * L[1] * L[2] / (double)P);
  int64_t sx = (int64_t)fmin(fmax(rint(L[0] / a), 1.0), (double)P);
  const int64_t Tsl = (P + sx - 1) / sx;
  int64_t sy = (int64_t)fmin(fmax(rint(L[1] / a), 1.0), (double)Tsl);
  const int64_t Tcol = (Tsl + sy - 1) / sy;
  sy = (Tsl + Tcol - 1) / Tcol;
  sh.Sx = Tsl * TP;
  sh.Scol = Tcol * TP;
  sh.c = sy;
  return sh;
}
__device__ __forceinline__ uint32_t axis_key(double v, double lo, double scale) {
  double c = (v - lo) * scale;
  c = c < 0.0 ? 0.0 : (c > 4294967040.0 ? 4294967040.0 : c);
  return (uint32_t)c;
}
__global__ void str_key_kernel(const double* __restrict__ pts, const int32_t* __restrict__ perm,
                               int64_t n, int pass, const unsigned long long* __restrict__ box,
                               int64_t P, int TP, uint64_t* __restrict__ keys, int32_t* __restrict__ vals) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const StrShape sh = str_shape(box, P, TP);
  const int64_t p = perm ? perm[i] : i;
  const double* x = pts + 3 * p;
  uint64_t g = 0;
  if (pass == 1) g = (uint64_t)(i / sh.Sx);
  if (pass == 2) g = (uint64_t)(i / sh.Sx) * (uint64_t)sh.c + (uint64_t)((i % sh.Sx) / sh.Scol);
  const uint32_t k = finite_point(x) ? axis_key(x[pass], sh.lo[pass], sh.scale[pass]) : 0xFFFFFFFFu;
  keys[i] = (g << 32) | k;
  vals[i] = (int32_t)p;
}

// Tiles of TP consecutive sorted points; padding slots repeat the tile's first point.
__global__ void tile_gather_kernel(const double* __restrict__ pts, const int32_t* __restrict__ perm,
                                   int64_t n, int64_t t0, TileBatch tb) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (int64_t)tb.C * tb.TP) return;
  const int64_t t = gid / tb.TP;
  const int j = (int)(gid % tb.TP);
  const int64_t g = (t0 + t) * tb.TP + j;
  const bool v = g < n;
  const int64_t p = perm[v ? g : (t0 + t) * tb.TP];
  tb.xyz[3 * gid] = pts[3 * p];
  tb.xyz[3 * gid + 1] = pts[3 * p + 1];
  tb.xyz[3 * gid + 2] = pts[3 * p + 2];
  tb.out[gid] = v ? p : -1;
}

// Cubic grid: tile = TX x TY x TZ block of grid points (z fastest).
__global__ void tile_cubic_kernel(PointSrc src, int nx, int TX, int TY, int TZ, int nby, int nbz,
                                  int64_t t0, TileBatch tb) {
  const int64_t gid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (int64_t)tb.C * tb.TP) return;
  const int64_t t = t0 + gid / tb.TP;
  const int j = (int)(gid % tb.TP);
  const int64_t bz = t % nbz, by = (t / nbz) % nby, bx = t / ((int64_t)nbz * nby);
  const int iz = j % TZ, iy = (j / TZ) % TY, ix = j / (TZ * TY);
  int64_t i = bx * TX + ix, k = by * TY + iy, l = bz * TZ + iz;
  const bool v = i < nx && k < src.ny && l < src.nz;
  if (!v) { i = bx * TX; k = by * TY; l = bz * TZ; }
  const double fi = (double)i, fj = (double)k, fk = (double)l;
  tb.xyz[3 * gid] = src.o[0] + fi * src.ax[0] + fj * src.ax[3] + fk * src.ax[6];
  tb.xyz[3 * gid + 1] = src.o[1] + fi * src.ax[1] + fj * src.ax[4] + fk * src.ax[7];
  tb.xyz[3 * gid + 2] = src.o[2] + fi * src.ax[2] + fj * src.ax[5] + fk * src.ax[8];
  tb.out[gid] = v ? (i * src.ny + k) * (int64_t)src.nz + l : -1;
}

// Bounding sphere of one tile's points, computed by a whole block of
// kTileThreads threads: centre = mean of the finite points (padding repeats a
// real point; a point with a non-finite coordinate gets NaN outputs and must
// not move the sphere of its tile mates), radius = largest distance from it,
// widened by a relative 1e-12 plus 1e-9 bohr; -1e300 when no point is finite.
// The screening kernel and the capacity pre-pass both use this code, so they
// see the same sphere to the last bit.
__device__ void tile_sphere(const double* __restrict__ xyz, int TP, double* sctr, double* srad) {
  __shared__ double red[3][kTileThreads / 32];
  __shared__ int s_nfin;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_nfin = 0;
  __syncthreads();
  double c[3] = {0, 0, 0};
  int nfin = 0;
  for (int j = threadIdx.x; j < TP; j += kTileThreads)
    if (finite_point(xyz + 3 * j)) {
      ++nfin;
      for (int d = 0; d < 3; ++d) c[d] += xyz[3 * j + d];
    }
  for (int o = 16; o > 0; o >>= 1) nfin += __shfl_xor_sync(0xffffffffu, nfin, o);
  if (lane == 0 && nfin) atomicAdd(&s_nfin, nfin);
  for (int d = 0; d < 3; ++d) {
    for (int o = 16; o > 0; o >>= 1) c[d] += __shfl_xor_sync(0xffffffffu, c[d], o);
    if (lane == 0) red[d][warp] = c[d];
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double acc = 0;
    for (int w = 0; w < kTileThreads / 32; ++w) acc += red[threadIdx.x][w];
    sctr[threadIdx.x] = s_nfin ? acc / s_nfin : 0.0;
  }
  __syncthreads();
  double r2 = 0.0;
  for (int j = threadIdx.x; j < TP; j += kTileThreads) {
    if (!finite_point(xyz + 3 * j)) continue;
    const double dx = xyz[3 * j] - sctr[0], dy = xyz[3 * j + 1] - sctr[1], dz = xyz[3 * j + 2] - sctr[2];
    r2 = fmax(r2, dx * dx + dy * dy + dz * dz);
  }
  for (int o = 16; o > 0; o >>= 1) r2 = fmax(r2, __shfl_xor_sync(0xffffffffu, r2, o));
  if (lane == 0) red[0][warp] = r2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0;
    for (int w = 0; w < kTileThreads / 32; ++w) m = fmax(m, red[0][w]);
    // a tile without a finite point keeps no segment
    *srad = s_nfin ? sqrt(m) * (1.0 + 1e-12) + 1e-9 : -1e300;
  }
  __syncthreads();
}

// Is segment sg significant on the tile sphere (ctr, rad)?  Every AO value and
// derivative of the segment is below 1e-18 beyond sqrt(rcut2) of its centre.
__device__ __forceinline__ bool seg_significant(const DevSeg& sg, const double* ctr, double rad) {
  const double dx = sg.cx - ctr[0], dy = sg.cy - ctr[1], dz = sg.cz - ctr[2];
  const double d = sqrt(dx * dx + dy * dy + dz * dz);
  return d <= sqrt(sg.rcut2) + rad;
}

// Status code of a tile whose compact AO set exceeds the batch's capacity
// (cannot happen when the capacity comes from tile_capacity_kernel).
constexpr int32_t kStatusCapacity = 0x7201;

// Capacity pre-pass: the largest padded compact AO count of a batch of tiles
// (atomicMax into *kmax).  One block per tile.
__global__ void __launch_bounds__(kTileThreads)
    tile_capacity_kernel(const DevSeg* __restrict__ segs, int nseg, TileBatch tb, int* kmax) {
  __shared__ double sctr[3], srad;
  __shared__ int part[kTileThreads / 32];
  const int t = blockIdx.x;
  tile_sphere(tb.xyz + (int64_t)t * tb.TP * 3, tb.TP, sctr, &srad);
  int cnt = 0;
  for (int s = threadIdx.x; s < nseg; s += kTileThreads) {
    const DevSeg sg = segs[s];
    if (seg_significant(sg, sctr, srad)) cnt += ncomp_of_type_dev(sg.type);
  }
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    int tot = 0;
    for (int w = 0; w < kTileThreads / 32; ++w) tot += part[w];
    atomicMax(kmax, (tot + kKtAlign - 1) / kKtAlign * kKtAlign);
  }
}

// One CTA per tile: bounding sphere of the tile's points, then the ordered
// list of segments whose screening sphere meets it.
__global__ void __launch_bounds__(kTileThreads)
    screen_kernel(const DevSeg* __restrict__ segs, int nseg, TileBatch tb, int rows,
                  double* __restrict__ stats, int32_t* __restrict__ status) {
  using Scan = cub::BlockScan<int, kTileThreads>;
  __shared__ typename Scan::TempStorage scan_tmp;
  __shared__ int s_sl[kSortCap], s_k0[kSortCap], s_cnt[8];
  __shared__ double sctr[3], srad;
  __shared__ int base_s, base_k;
  __shared__ int s_over_s, s_over_k;  // first segment beyond the capacity
  const int t = blockIdx.x, TP = tb.TP;
  tile_sphere(tb.xyz + (int64_t)t * TP * 3, TP, sctr, &srad);
  if (threadIdx.x == 0) {
    base_s = 0;
    base_k = 0;
    s_over_s = INT_MAX;
    s_over_k = INT_MAX;
  }
  __syncthreads();
  const double rad = srad;
  int32_t* sl = tb.segs + (int64_t)t * nseg;
  int32_t* k0 = tb.k0 + (int64_t)t * nseg;
  int32_t* am = tb.aomap + (int64_t)t * tb.Kcap;
  for (int s0 = 0; s0 < nseg; s0 += kTileThreads) {
    const int s = s0 + threadIdx.x;
    int sig = 0, nc = 0;
    DevSeg sg;
    if (s < nseg) {
      sg = segs[s];
      if (seg_significant(sg, sctr, rad)) {
        sig = 1;
        nc = ncomp_of_type_dev(sg.type);
      }
    }
    // pack (segment count, AO count) into one int: both sums stay below 2^16
    int packed, ptot;
    Scan(scan_tmp).ExclusiveSum((sig << 16) | nc, packed, ptot);
    const int2 pos = make_int2(packed >> 16, packed & 0xffff);
    const int2 tot = make_int2(ptot >> 16, ptot & 0xffff);
    if (sig) {
      const int ks = base_k + pos.y;
      sl[base_s + pos.x] = s;
      k0[base_s + pos.x] = ks;
      if (ks + nc <= tb.Kcap) {
        for (int q = 0; q < nc; ++q) am[ks + q] = sg.ao0 + q;
      } else {
        // never with a capacity from the pre-pass or Kcap = Mpad: the tile is
        // cut at this segment and the call reports kStatusCapacity
        atomicMin(&s_over_s, base_s + pos.x);
        atomicMin(&s_over_k, ks);
        atomicExch(status, kStatusCapacity);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      base_s += tot.x;
      base_k += tot.y;
    }
    __syncthreads();
  }
  // Visit order for the AO kernel: the significant segments grouped by type
  // (counting sort; compact positions k0 keep the AO order), so that the
  // warps of a CTA run one type's evaluation code at a time instead of
  // alternating between the types' large unrolled bodies.
  const int ns = min(base_s, s_over_s);
  if (ns <= kSortCap) {
    if (threadIdx.x < 8) s_cnt[threadIdx.x] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < ns; i += kTileThreads) {
      const int sg = sl[i];
      s_sl[i] = sg;
      s_k0[i] = k0[i];
      atomicAdd(&s_cnt[segs[sg].type & 7], 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int acc = 0;
      for (int ty = 0; ty < 8; ++ty) {
        const int c = s_cnt[ty];
        s_cnt[ty] = acc;
        acc += c;
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < ns; i += kTileThreads) {
      const int sg = s_sl[i];
      const int pos = atomicAdd(&s_cnt[segs[sg].type & 7], 1);
      sl[pos] = sg;
      k0[pos] = s_k0[i];
    }
  }
  const int kt_true = min(base_k, s_over_k);
  const int kt = min((kt_true + kKtAlign - 1) / kKtAlign * kKtAlign, tb.Kcap);
  for (int k = kt_true + threadIdx.x; k < kt; k += kTileThreads) am[k] = -1;
  if (threadIdx.x == 0) {
    tb.nsig[t] = ns;
    tb.ktrue[t] = kt_true;
    tb.kt[t] = kt;
    int npts = 0;
    for (int j = 0; j < TP; ++j) npts += tb.out[(int64_t)t * TP + j] >= 0;
    atomicAdd(&stats[0], 1.0);
    atomicAdd(&stats[1], (double)npts);
    atomicAdd(&stats[2], (double)kt_true);
    atomicAdd(&stats[3], (double)rows * (double)kt * (double)kt);
  }
}

// ------------------------------------------------------------------ FP64 contraction kernel
constexpr int BM = 128, BN = 64, BK = 32, STAGES = 3;
constexpr int A_LD = BM + 4;  // A stage stored [k][row], 132 doubles: conflict-free fragment loads
constexpr int B_LD = BN + 4;  // 68 doubles
constexpr int C_LD = BN + 1;
constexpr int A_STAGE = BK * A_LD, B_STAGE = BK * B_LD;
constexpr int kThreads = 256;
constexpr size_t kSmemPipe = sizeof(double) * STAGES * (A_STAGE + B_STAGE);
constexpr size_t kSmemC = sizeof(double) * BM * C_LD;
constexpr size_t kSmemFp64 = kSmemPipe > kSmemC ? kSmemPipe : kSmemC;
static_assert(kKtAlign % BN == 0 && kKtAlign % BK == 0, "tile K alignment");

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int sz = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int sz = valid ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
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

// One CTA per tile of PTS = 128/NQA points; tile row r holds quantity r / PTS
// of point r % PTS (quantity 0 = phi, 1..3 = d_k phi).  It sweeps the tile's
// compact nu range in 64-column slices, each with a full K loop over the
// compact mu range (B = D gathered by index), and reduces every finished G
// slice against the AO values of its columns.
// Inputs of the force epilogue (EPI = 1): per-point dL/drho and dL/dgrad rho
// indexed by the original point index, AO -> atom map, dL/dR accumulator.
struct ForceArgs {
  const double* v_rho = nullptr;
  const double* v_grad = nullptr;
  const int32_t* ao_atom = nullptr;
  double* dLdR = nullptr;
  int natom = 0;
};
constexpr int kMaxSmemAtoms = 1024;

template <int NQA, int EPI>
__global__ void __launch_bounds__(kThreads)
    fp64_tile_kernel(TileBatch tb, const double* __restrict__ D, int Mpad, ctc_outputs out,
                     ctc_params prm, ForceArgs fa) {
  constexpr int PTS = BM / NQA;
  constexpr int TPP = kThreads / PTS;  // epilogue threads per point
  constexpr int NS = NQA == 4 ? 16 : 4;
  extern __shared__ __align__(16) double smem[];
  double* sA = smem;
  double* sB = smem + STAGES * A_STAGE;
  double* sC = smem;  // aliases the pipeline after the K loop
  __shared__ int s_colmap[BN];
  __shared__ double s_force[EPI == 1 ? 3 * kMaxSmemAtoms : 1];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 3, wn = warp >> 2;
  const int t = blockIdx.x;
  const int kt = tb.kt[t];
  const int nq_ao = tb.nq;
  const int64_t ldq = (int64_t)PTS * tb.Kcap;  // stride between quantities
  const double* A = tb.ao + (int64_t)t * nq_ao * ldq;
  const int32_t* am = tb.aomap + (int64_t)t * tb.Kcap;

  // epilogue ownership: lanes take consecutive points (coalesced AO reads),
  // esub selects the column subset; partial sums meet in shared memory
  const int epl = tid % PTS, esub = tid / PTS;
  double acc_s[NS];
#pragma unroll
  for (int i = 0; i < NS; ++i) acc_s[i] = 0.0;
  // force epilogue: per-point weights, per-CTA atom accumulators
  const bool force_smem = EPI == 1 && fa.natom <= kMaxSmemAtoms;
  double fvr = 0.0, fvg[3] = {0.0, 0.0, 0.0};
  if constexpr (EPI == 1) {
    for (int i = tid; i < 3 * fa.natom && force_smem; i += kThreads) s_force[i] = 0.0;
    const int64_t oi = tb.out[(int64_t)t * PTS + epl];
    if (oi >= 0) {
      fvr = fa.v_rho[oi];
      if (fa.v_grad)
        for (int k = 0; k < 3; ++k) fvg[k] = fa.v_grad[3 * oi + k];
    }
  }

  const int nkb = kt / BK;
  for (int n0 = 0; n0 < kt; n0 += BN) {
    if (tid < BN) s_colmap[tid] = am[n0 + tid];
    __syncthreads();
    double c[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) c[i][j][0] = c[i][j][1] = 0.0;

    auto load_stage = [&](int stage, int kb) {
      double* a = sA + stage * A_STAGE;
      double* b = sB + stage * B_STAGE;
      const int k0 = kb * BK;
      // A stage [k][row]: 32 k x 128 rows, each (q, k) a run of PTS points
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int ch = tid + i * kThreads;
        const int kk = ch >> 6, r = (ch & 63) * 2;
        const int q = r / PTS, pl = r % PTS;
        cp_async16(a + kk * A_LD + r, A + q * ldq + (int64_t)(k0 + kk) * PTS + pl, true);
      }
      // B gather: 32 rows (compact mu) x 64 columns (compact nu), 8 bytes each
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int e = tid + i * kThreads;
        const int r = e >> 6, cc = e & 63;
        const int mu = am[k0 + r], nu = s_colmap[cc];
        const bool v = mu >= 0 && nu >= 0;
        cp_async8(b + r * B_LD + cc, D + (v ? (int64_t)mu * Mpad + nu : 0), v);
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
          af[i] = a[(ks + (lane & 3)) * A_LD + wm * 32 + i * 8 + (lane >> 2)];
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
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int r = wm * 32 + i * 8 + (lane >> 2);
        const int cc = wn * 32 + j * 8 + 2 * (lane & 3);
        sC[r * C_LD + cc] = c[i][j][0];
        sC[r * C_LD + cc + 1] = c[i][j][1];
      }
    __syncthreads();
    if constexpr (EPI == 0) {
      {
        // AO value of quantity q at column n0 + v for this point: A[q][n0 + v][epl]
        const double* aop = A + (int64_t)n0 * PTS + epl;
        for (int v = esub; v < BN; v += TPP) {
          const double G0 = sC[(0 * PTS + epl) * C_LD + v];
          const double phi = aop[v * PTS];
          acc_s[0] += G0 * phi;
          if (nq_ao >= 4) {
            const double d0 = aop[ldq + v * PTS], d1 = aop[2 * ldq + v * PTS], d2 = aop[3 * ldq + v * PTS];
            acc_s[1] += G0 * d0;
            acc_s[2] += G0 * d1;
            acc_s[3] += G0 * d2;
            if constexpr (NQA == 4) {
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
                for (int h = 0; h < 6; ++h) acc_s[4 + h] += G0 * aop[(4 + h) * ldq + v * PTS];
              }
            }
          }
        }
      }
    } else {
      // dL/dR_A,j += sum over nu on atom A of
      //   -2 v_rho d_j phi G0 - 2 sum_k v_k (d_j d_k phi G0 + d_j phi G_k)
      const double* aop = A + (int64_t)n0 * PTS + epl;
      const int hidx[3][3] = {{4, 5, 6}, {5, 7, 8}, {6, 8, 9}};
      for (int v = esub; v < BN; v += TPP) {
        const int nu = s_colmap[v];
        if (nu < 0 || (fvr == 0.0 && fvg[0] == 0.0 && fvg[1] == 0.0 && fvg[2] == 0.0)) continue;
        const int atom = fa.ao_atom[nu];
        if (atom < 0) continue;
        const double G0 = sC[(0 * PTS + epl) * C_LD + v];
        double Gk[3] = {0.0, 0.0, 0.0};
        if constexpr (NQA == 4) {
          Gk[0] = sC[(1 * PTS + epl) * C_LD + v];
          Gk[1] = sC[(2 * PTS + epl) * C_LD + v];
          Gk[2] = sC[(3 * PTS + epl) * C_LD + v];
        }
        for (int j = 0; j < 3; ++j) {
          const double dj = aop[(1 + j) * ldq + v * PTS];
          double c = -2.0 * fvr * dj * G0;
          if (fa.v_grad) {
            for (int k = 0; k < 3; ++k)
              c -= 2.0 * fvg[k] * (aop[hidx[j][k] * ldq + v * PTS] * G0 + dj * Gk[k]);
          }
          if (force_smem) atomicAdd(&s_force[3 * atom + j], c);
          else atomicAdd(&fa.dLdR[3 * atom + j], c);
        }
      }
    }
    __syncthreads();
  }
  if constexpr (EPI == 1) {
    __syncthreads();
    if (force_smem)
      for (int i = tid; i < 3 * fa.natom; i += kThreads)
        if (s_force[i] != 0.0) atomicAdd(&fa.dLdR[i], s_force[i]);
    return;
  }
  // sum the TPP column subsets of each point (sC is free after the last tile)
  double* red = sC;
#pragma unroll
  for (int i = 0; i < NS; ++i) red[(esub * NS + i) * PTS + epl] = acc_s[i];
  __syncthreads();
  const int64_t oidx = tb.out[(int64_t)t * PTS + epl];
  if (esub == 0 && oidx >= 0 && !finite_point(tb.xyz + 3 * ((int64_t)t * PTS + epl))) {
    nan_point(out, oidx);
  } else if (esub == 0 && oidx >= 0) {
    double s[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      double v = 0.0;
      if (i < NS)
        for (int e = 0; e < TPP; ++e) v += red[(e * NS + i) * PTS + epl];
      s[i] = v;
    }
    finalize_point(s, NQA, nq_ao, out, oidx, prm);
  }
}

// ------------------------------------------------------------------ chunk scratch

struct Carve {
  char* p;
  size_t off = 0;
  template <class T>
  T* take(size_t count) {
    off = (off + 255) / 256 * 256;
    T* r = (T*)(p + off);
    off += sizeof(T) * count;
    return r;
  }
};

size_t tile_bytes(const ctc_molecule* mol, int C, int TP, int Kcap_) {
  const size_t Kcap = Kcap_;
  size_t b = 0;
  auto add = [&](size_t x) { b = (b + 255) / 256 * 256 + x; };
  add(sizeof(double) * C * TP * 3);
  add(sizeof(int64_t) * C * TP);
  add(sizeof(int32_t) * C);
  add(sizeof(int32_t) * C);
  add(sizeof(int32_t) * C);
  add(sizeof(int32_t) * (size_t)C * mol->nseg);
  add(sizeof(int32_t) * (size_t)C * mol->nseg);
  add(sizeof(int32_t) * (size_t)C * Kcap);
  return b + 256;
}


// Tile builder + chunk loop.  For every chunk: tile points, screen, AO block
// (derivative order deriv, nq quantities; ao_launch replaces the plain AO
// kernel launch when given), then compute(tb).
inline int run_tiles(ctc_molecule* mol, const PointSrc& src, int64_t n, int TP, int nq, int deriv,
                     cudaStream_t st, const std::function<int(const TileBatch&)>& compute,
                     const std::function<int(const TileBatch&)>* ao_launch = nullptr,
                     int rows = 128) {
  if (n <= 0) return CTC_OK;  // (no zero-sized grids below)
  // cubic-grid tiles: blocks of 2x4x4 or 4x4x8 grid points
  int TX = 2, TY = 4, TZ = 4;
  if (TP == 128) { TX = 4; TY = 4; TZ = 8; }
  int64_t ntiles, nbx = 0, nby = 0, nbz = 0;
  int nx = 0;
  if (src.cubic) {
    nx = (int)(n / ((int64_t)src.ny * src.nz));
    nbx = (nx + TX - 1) / TX;
    nby = (src.ny + TY - 1) / TY;
    nbz = (src.nz + TZ - 1) / TZ;
    ntiles = nbx * nby * nbz;
  } else {
    ntiles = (n + TP - 1) / TP;
  }
  int rc;
  // explicit points: sort-tile-recursive order over the points' own box for
  // calls of kStrMinPoints points or more; below that, one sort of 30-bit
  // Morton keys over the molecule's box padded by 12 bohr (three sorts cost
  // ~0.4 ms, as much as a whole 1e5-point density call of a small molecule,
  // while the tiles' shape matters little there)
  constexpr int64_t kStrMinPoints = (int64_t)1 << 18;
  int32_t* perm = nullptr;
  if (!src.cubic) {
    const bool str = n >= kStrMinPoints;
    size_t tmp_bytes = 0, tmp32 = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, (uint64_t*)nullptr, (uint64_t*)nullptr,
                                    (int32_t*)nullptr, (int32_t*)nullptr, (int)n, 0, 64, st);
    cub::DeviceRadixSort::SortPairs(nullptr, tmp32, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (int32_t*)nullptr, (int32_t*)nullptr, (int)n, 0, kMortonSortBits, st);
    tmp_bytes = std::max(tmp_bytes, tmp32);
    const size_t need = 2 * sizeof(uint64_t) * (size_t)n + 2 * sizeof(int32_t) * (size_t)n + tmp_bytes + 4096;
    if ((rc = mol->ws_part.ensure(need, st)) != CTC_OK) return rc;
    Carve cv{(char*)mol->ws_part.p};
    unsigned long long* box = cv.take<unsigned long long>(6);
    uint64_t* k_in = cv.take<uint64_t>(n);
    uint64_t* k_out = cv.take<uint64_t>(n);
    int32_t* v_in = cv.take<int32_t>(n);
    perm = cv.take<int32_t>(n);
    void* tmp = cv.take<char>(tmp_bytes);
    if (str) {
      CTC_CUDA_TRY(cudaMemsetAsync(box, 0xFF, 3 * sizeof(unsigned long long), st));
      CTC_CUDA_TRY(cudaMemsetAsync(box + 3, 0, 3 * sizeof(unsigned long long), st));
      point_box_kernel<<<(unsigned)std::min<int64_t>((n + 255) / 256, 4 * 148), 256, 0, st>>>(src.pts, n, box);
      CTC_CUDA_TRY(cudaGetLastError());
      // group ids of passes 2 and 3 are below sx * sy <= sx * ceil(P / sx) < P + sx <= 2 P
      const int gbits = 64 - __builtin_clzll((unsigned long long)(2 * ntiles));
      const unsigned g = (unsigned)((n + 255) / 256);
      for (int pass = 0; pass < 3; ++pass) {
        str_key_kernel<<<g, 256, 0, st>>>(src.pts, pass ? perm : nullptr, n, pass, box, ntiles, TP, k_in, v_in);
        CTC_CUDA_TRY(cudaGetLastError());
        CTC_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, k_in, k_out, v_in, perm, (int)n, 0,
                                                     32 + (pass ? gbits : 0), st));
      }
      mol->host_launches += 7;
    } else {
      double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
      for (int a = 0; a < mol->natom; ++a)
        for (int d = 0; d < 3; ++d) {
          lo[d] = std::min(lo[d], mol->atom_xyz[3 * a + d]);
          hi[d] = std::max(hi[d], mol->atom_xyz[3 * a + d]);
        }
      if (mol->natom == 0)
        for (int d = 0; d < 3; ++d) { lo[d] = -1; hi[d] = 1; }
      double ext = 0;
      for (int d = 0; d < 3; ++d) ext = std::max(ext, hi[d] - lo[d] + 24.0);
      uint32_t* k32_in = (uint32_t*)k_in;
      uint32_t* k32_out = (uint32_t*)k_out;
      morton_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(src.pts, n, lo[0] - 12.0, lo[1] - 12.0,
                                                                  lo[2] - 12.0, 1024.0 / ext, k32_in, v_in);
      CTC_CUDA_TRY(cudaGetLastError());
      CTC_CUDA_TRY(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, k32_in, k32_out, v_in, perm, (int)n, 0,
                                                   kMortonSortBits, st));
      mol->host_launches += 2;
    }
  }
  // tile points of tiles [t0, t0 + tb.C)
  auto tile_points = [&](const TileBatch& tb, int64_t t0) -> int {
    const int64_t npts = (int64_t)tb.C * TP;
    const unsigned g = (unsigned)((npts + 255) / 256);
    if (src.cubic)
      tile_cubic_kernel<<<g, 256, 0, st>>>(src, nx, TX, TY, TZ, (int)nby, (int)nbz, t0, tb);
    else
      tile_gather_kernel<<<g, 256, 0, st>>>(src.pts, perm, n, t0, tb);
    CTC_CUDA_TRY(cudaGetLastError());
    return CTC_OK;
  };
  // chunk of tiles: AO block (nq x TP x Kcap doubles per tile) within
  // min(12 GiB, a quarter of the free device memory) (CTC_CHUNK_BYTES
  // overrides), at least one full wave of CTAs on 148 SMs.  Larger chunks
  // amortise the per-chunk launches and tails: on the 215^3 benchmark cube
  // 6 GiB gave 20.95 M points/s, 12 GiB 21.46 M, 24 GiB 21.60 M.
  size_t budget = (size_t)12 << 30;
  {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) budget = std::min(budget, free_b / 4);
    else cudaGetLastError();  // clear the error; keep the default
  }
  if (const char* env = std::getenv("CTC_CHUNK_BYTES")) {
    const long long v = std::atoll(env);
    if (v > 0) budget = (size_t)v;
  }
  // Capacity of a tile's compact AO set: Mpad always suffices.  When a chunk
  // sized for Mpad columns would hold fewer than four waves of tiles (large
  // bases: the 1 000-atom molecule keeps ~350 of 16 128 functions per tile), a
  // count-only screening pass over every tile of the call finds the largest
  // compact set and the workspace is sized for that instead.  It waits for
  // the stream once (to read the count back); smaller bases skip it.
  int Kcap = mol->Mpad;
  if ((int64_t)(budget / (sizeof(double) * (size_t)nq * TP * mol->Mpad)) < 4 * 148 && ntiles > 148) {
    const int64_t PB = std::min<int64_t>(ntiles, 16384);
    const size_t pb_bytes = sizeof(double) * (size_t)PB * TP * 3 + sizeof(int64_t) * (size_t)PB * TP + 1024;
    if ((rc = mol->ws_cap.ensure(pb_bytes, st)) != CTC_OK) return rc;
    TileBatch pb;
    pb.TP = TP;
    Carve cv{(char*)mol->ws_cap.p};
    int* d_kmax = cv.take<int>(1);
    pb.xyz = cv.take<double>((size_t)PB * TP * 3);
    pb.out = cv.take<int64_t>((size_t)PB * TP);
    CTC_CUDA_TRY(cudaMemsetAsync(d_kmax, 0, sizeof(int), st));
    for (int64_t t0 = 0; t0 < ntiles; t0 += PB) {
      pb.C = (int)std::min<int64_t>(PB, ntiles - t0);
      if ((rc = tile_points(pb, t0)) != CTC_OK) return rc;
      tile_capacity_kernel<<<pb.C, kTileThreads, 0, st>>>(mol->d_segs, mol->nseg, pb, d_kmax);
      CTC_CUDA_TRY(cudaGetLastError());
      mol->host_launches += 2;
    }
    CTC_CUDA_TRY(cudaMemcpyAsync(mol->h_status + 1, d_kmax, sizeof(int), cudaMemcpyDeviceToHost, st));
    CTC_CUDA_TRY(cudaStreamSynchronize(st));
    Kcap = std::min(mol->Mpad, std::max(kKtAlign, (int)mol->h_status[1]));
  }
  const size_t ao_per_tile = sizeof(double) * (size_t)nq * TP * Kcap;
  int64_t C = std::max<int64_t>(148, (int64_t)(budget / ao_per_tile));
  C = std::min<int64_t>(C, ntiles);
  if ((rc = mol->ws_ao.ensure(ao_per_tile * C, st)) != CTC_OK) return rc;
  if ((rc = mol->ws_misc.ensure(tile_bytes(mol, (int)C, TP, Kcap), st)) != CTC_OK) return rc;
  TileBatch tb;
  tb.TP = TP;
  tb.Kcap = Kcap;
  tb.nq = nq;
  tb.ao = (double*)mol->ws_ao.p;
  {
    Carve cv{(char*)mol->ws_misc.p};
    tb.xyz = cv.take<double>((size_t)C * TP * 3);
    tb.out = cv.take<int64_t>((size_t)C * TP);
    tb.nsig = cv.take<int32_t>(C);
    tb.ktrue = cv.take<int32_t>(C);
    tb.kt = cv.take<int32_t>(C);
    tb.segs = cv.take<int32_t>((size_t)C * mol->nseg);
    tb.k0 = cv.take<int32_t>((size_t)C * mol->nseg);
    tb.aomap = cv.take<int32_t>((size_t)C * tb.Kcap);
  }
  for (int64_t t0 = 0; t0 < ntiles; t0 += C) {
    tb.C = (int)std::min<int64_t>(C, ntiles - t0);
    if ((rc = tile_points(tb, t0)) != CTC_OK) return rc;
    screen_kernel<<<tb.C, kTileThreads, 0, st>>>(mol->d_segs, mol->nseg, tb, rows, mol->d_stats,
                                                 mol->d_status);
    CTC_CUDA_TRY(cudaGetLastError());
    {
      ProfScope ps(mol, 1, st);
      rc = ao_launch ? (*ao_launch)(tb) : launch_ao_tiles(mol, tb, deriv, st);
      if (rc != CTC_OK) return rc;
    }
    mol->host_launches += 3;
    mol->host_chunks += 1;
    if ((rc = compute(tb)) != CTC_OK) return rc;
  }
  return CTC_OK;
}

}  // namespace
}  // namespace ctc
