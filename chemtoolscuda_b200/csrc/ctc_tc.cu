// ctc_tc.cu -- tensor-core split-precision contraction (tcgen05, INT8, sm_100a).
//
// G_t = A_t D[S_t, S_t] of the screened tile pipeline (ctc_local.cu) on the
// 5th-generation tensor cores with results equal to the FP64 contraction to
// ~1e-9 of the sum of absolute terms (measured against the FP64 oracle;
// 1e-8 is the target).
//
// Split (an Ozaki-type scheme with exact integer accumulation, ctc_split.cuh):
//   * every A row r is scaled by 2^-e_r (e_r from the row's largest |value|)
//     and rounded to I_A = rint(x 2^(38 - e_r)), five balanced base-256 digits
//     a_0..a_4 (|a_i| <= 128, I_A = sum_i a_i 256^(4-i)); every D row nu by
//     2^-f_nu, I_D = rint(y 2^(38 - f_nu)), five digits b_0..b_4; one int8
//     plane per digit;
//   * the 15 digit products with i + j <= 4 are accumulated on INT8 tensor
//     cores (tcgen05.mma kind::i8, int32 accumulators in TMEM), one TMEM
//     accumulator per level L = i + j;  int32 accumulation is exact as long
//     as the compact K of a tile stays below 16 384;
//   * the epilogue forms G = 2^(e_r + f_nu - 76) sum_L acc_L 2^(64 - 8 L) in
//     FP64 and reduces it against the FP64 AO values (same epilogue sums as
//     the FP64 path).
// The dropped products (i + j >= 5) are below 2^-40 of the row/column scale.
//
// Kernel roles (288 threads, one persistent CTA per SM taking the chunk's
// tiles largest first from a launch-wide counter): warps 0-3 produce the
// operands of each K block (one thread issues the TMA loads of the five A
// planes; all 128 threads gather the five D planes by compact index from the
// packed copy of D and write them in the 64-byte-swizzled K-major layout),
// warps 4-7 drain the TMEM accumulators (one 32-lane quarter each) into an
// FP64 copy of G in shared memory and run the epilogue while the next nu
// tile's MMAs run, warp 8 issues the MMAs from one thread and commits them to
// mbarriers.  Registers move from the producer warpgroup (104 each) to the
// epilogue warpgroup (232 each), whose AO loads in flight are bounded by
// registers (setmaxnreg; 128 x 104 + 128 x 232 + 32 x 168 = the 288 x 168 of
// the launch, and per SM sub-partition 104 + 232 + 168 registers x 32 lanes
// stay within 16 384).  Every mbarrier wait is bounded: on timeout the kernel records a
// status code, stops issuing work, and the allocating warp still frees its
// TMEM.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#include <cstdio>
#include <cstdlib>

#include <cub/device/device_radix_sort.cuh>

#include "ctc_internal.h"
#include "ctc_split.cuh"
#include "ctc_finalize.cuh"

namespace ctc {

namespace {

constexpr int kN = 64;          // nu columns per TMEM accumulator
constexpr int kBK = 64;         // K bytes per pipeline stage
constexpr int kStages = 2;
constexpr int kRows = kSplitRows;  // tile rows (MMA M)
constexpr int kLevels = 5;
constexpr int kPlanesA = kSplitPlanesA;  // A digit planes (tile rows)
constexpr int kPlanes = kSplitPlanesD;   // D digit planes
constexpr int kAPlaneBytes = kRows * kBK;       // 8 KB
constexpr int kBPlaneBytes = kN * kBK;          // 4 KB
constexpr int kAStageBytes = kPlanesA * kAPlaneBytes;
constexpr int kBStageBytes = kPlanes * kBPlaneBytes;
constexpr int kGBytes = kN * kRows * 8;         // FP64 copy of one nu tile of G (64 KB)
constexpr int kSmemTc = kStages * (kAStageBytes + kBStageBytes) + kGBytes + 1024;  // + alignment slack
constexpr int kThreadsTc = 288;
constexpr int kMmaWarp = 8;             // warps 0-3 producers, 4-7 epilogue, 8 MMA
constexpr int kProducerRegs = 104;      // setmaxnreg shares (launch: 168 each)
constexpr int kEpilogueRegs = 232;
static_assert(4 * 32 * kProducerRegs + 4 * 32 * kEpilogueRegs + 32 * 168 <= kThreadsTc * 168,
              "register split above the launch's total");
constexpr int kMaxKt = 16384;
constexpr uint32_t kStatusTimeout = 0x7101;
// readers of a tile-ring slot: 4 producer warps, the MMA warp, one epilogue thread
constexpr uint32_t kTileReaders = 6;

// ------------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}\n" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(
                   smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Bounded wait on an mbarrier phase: false once `limit` SM cycles have passed
// (the pipeline's waits take the launch's limit, by default kWaitCycles).
constexpr long long kWaitCycles = 4000000000LL;  // ~2 s at 1.9-2.0 GHz
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit = kWaitCycles) {
  const uint32_t a = smem_u32(bar);
  const long long t0 = clock64();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > limit) return false;
  }
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}

// L2 eviction policies: the tile's int8 A planes (re-read once per nu tile)
// and the packed D (read by every tile) are kept; the FP64 AO values read once
// by the epilogue are evicted first.
__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}

__device__ __forceinline__ void tma_load_2d_hint(void* dst, const CUtensorMap* map, int c0, int c1,
                                                 uint64_t* bar, uint64_t policy) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1, {%2, %3}], [%4], %5;\n" ::"r"(smem_u32(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(smem_u32(bar)), "l"(policy)
      : "memory");
}

__device__ __forceinline__ uint64_t ldg_u64_hint(const uint64_t* p, uint64_t policy) {
  uint64_t v;
  asm("ld.global.nc.L2::cache_hint.u64 %0, [%1], %2;\n" : "=l"(v) : "l"(p), "l"(policy));
  return v;
}

__device__ __forceinline__ double ldg_f64_stream(const double* p, uint64_t policy) {
  double v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;\n"
               : "=d"(v)
               : "l"(p), "l"(policy));
  return v;
}

// K-major, 64-byte swizzle: 8-row atoms of 512 B, rows 64 B apart.
__device__ __forceinline__ uint64_t umma_desc_sw64(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3fff);        // start address
  d |= (uint64_t)1 << 16;                         // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(512 >> 4) << 32;                // stride byte offset: 8 rows x 64 B
  d |= (uint64_t)1 << 46;                         // descriptor version (sm_100)
  d |= (uint64_t)4 << 61;                         // layout: SWIZZLE_64B
  return d;
}

// byte offset of (row, k) inside a K-major SW64 plane (k < 64)
__device__ __forceinline__ uint32_t sw64_offset(int row, int k) {
  const int r8 = row & 7;
  const int chunk = (k >> 4) ^ ((r8 >> 1) & 3);
  return (uint32_t)((row >> 3) * 512 + r8 * 64 + chunk * 16 + (k & 15));
}

__device__ __forceinline__ void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                        uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, int32_t* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() {
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}
// Orders the use of tcgen05.ld results after tcgen05.wait::ld: the values pass
// through an empty volatile asm placed after the wait.
__device__ __forceinline__ void after_wait16(int32_t* v) {
  asm volatile(""
               : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]),
                 "+r"(v[7]), "+r"(v[8]), "+r"(v[9]), "+r"(v[10]), "+r"(v[11]), "+r"(v[12]),
                 "+r"(v[13]), "+r"(v[14]), "+r"(v[15]));
}

// x 2^S exactly, for int32 x and 0 <= S <= 48, with one integer and one FP64
// add (the exponent-bias construction of integer-to-double conversion): the
// bit pattern (1075 + S) << 52 | (x + 2^31) is the double 2^(52+S) + (x + 2^31) 2^S,
// and subtracting 2^(52+S) + 2^(31+S) leaves x 2^S.
template <int S>
__device__ __forceinline__ double i32_times_pow2(int32_t x) {
  const long long hi = (long long)(1075 + S) << 52;
  const double t = __longlong_as_double(hi | (long long)((uint32_t)x ^ 0x80000000u));
  return t - __longlong_as_double(hi | (1ll << 31));
}

// Epilogue contraction roles for tiles of 32 points x {phi, d_x, d_y, d_z}
// (NQA = 4).  Per point the epilogue needs 16 row sums
//   s[q'] = sum_nu G0 A_q'        (q' = 0..9: phi, first and second derivatives)
//   s[10..12] = sum_nu Gx A_{x,y,z},  s[13..14] = sum_nu Gy A_{y,z},  s[15] = sum_nu Gz A_z
// where A_q' is the AO quantity q' at the point and G0..Gz the rows of G.  Each
// of the four epilogue warps loads two or three AO quantities and forms the
// sums that use them (4-5 dot products per point each):
//   role 0: q' = 3 (rows 0,1,2,3 -> s3, s12, s14, s15), q' = 4 (s4)
//   role 1: q' = 2 (rows 0,1,2 -> s2, s11, s13),        q' = 5 (s5)
//   role 2: q' = 1 (rows 0,1 -> s1, s10), q' = 6 (s6), q' = 7 (s7)
//   role 3: q' = 0 (s0), q' = 8 (s8), q' = 9 (s9)
__device__ __forceinline__ constexpr int role_nslot(int role) { return role < 2 ? 2 : 3; }
__device__ __forceinline__ constexpr int role_q(int role, int slot) {
  return role == 0 ? (slot == 0 ? 3 : 4)
       : role == 1 ? (slot == 0 ? 2 : 5)
       : role == 2 ? (slot == 0 ? 1 : (slot == 1 ? 6 : 7))
                   : (slot == 0 ? 0 : (slot == 1 ? 8 : 9));
}
// number of G rows (0, 1, ...) paired with the slot's quantity
__device__ __forceinline__ constexpr int role_nrow(int role, int slot) {
  return slot == 0 ? (role == 0 ? 4 : (role == 1 ? 3 : (role == 2 ? 2 : 1))) : 1;
}
// index into the 16 per-point sums of (slot, G row)
__device__ __forceinline__ constexpr int role_sum(int role, int slot, int row) {
  return row == 0 ? role_q(role, slot)
       : role == 0 ? (row == 1 ? 12 : (row == 2 ? 14 : 15))
       : role == 1 ? (row == 1 ? 11 : 13)
                   : 10;
}

// One nu tile of the contraction for NQA = 4 and one role: acc[i] accumulates
// the role's i-th sum (slot-major, rows in order).  G is the FP64 copy in
// shared memory, [column][row]; ao points at AO quantity 0, column 0 of the nu
// tile for this thread's point (element (q, c) at ao[q * ldq + c * 32]).
// AO columns per load group of the epilogue contraction: kEpiColumns / GW
// register buffers keep kEpiColumns - GW columns of AO values in flight per
// thread while one group is reduced (measured on the 215^3 cube with 16
// columns: GW = 2 beat 8 (335 -> 317 ms), 4 (328 ms) and 1 (318 ms); the loads
// are latency-bound on tiles with few columns, so the epilogue warpgroup takes
// the producers' spare registers for 28)
constexpr int kEpiGroup = 2;
constexpr int kEpiColumns = 28;

template <int ROLE, int GW>
__device__ __forceinline__ void contract_role(const double* __restrict__ ao, int64_t ldq,
                                              const double* __restrict__ sG, int lane, int nq_ao,
                                              uint64_t stream, double* acc) {
  constexpr int NS = role_nslot(ROLE);
  constexpr int NG = kN / GW;    // groups of GW columns
  constexpr int NB = kEpiColumns / GW;  // register buffers of one group each
  bool live[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) live[s] = role_q(ROLE, s) < nq_ao;
  // NB register buffers: the loads of groups g + 1 .. g + NB - 1 are in flight
  // while group g is reduced
  double a[NB][NS][GW];
  auto load = [&](int buf, int cg) {
#pragma unroll
    for (int s = 0; s < NS; ++s)
#pragma unroll
      for (int j = 0; j < GW; ++j)
        a[buf][s][j] = live[s] ? ldg_f64_stream(ao + role_q(ROLE, s) * ldq + (cg + j) * 32, stream) : 0.0;
  };
#pragma unroll
  for (int g = 0; g < NB - 1; ++g) load(g, g * GW);
#pragma unroll
  for (int g = 0; g < NG; ++g) {
    if (g + NB - 1 < NG) load((g + NB - 1) % NB, (g + NB - 1) * GW);
    const int cg = g * GW;
#pragma unroll
    for (int j = 0; j < GW; ++j) {
      const double* gp = sG + (cg + j) * kRows + lane;
      int i = 0;
#pragma unroll
      for (int s = 0; s < NS; ++s)
#pragma unroll
        for (int rr = 0; rr < role_nrow(ROLE, s); ++rr, ++i)
          acc[i] = fma(gp[rr * 32], a[g % NB][s][j], acc[i]);
    }
  }
}

// One nu tile of the contraction for NQA = 1 (rows are the tile's 128
// points; thread etid owns point etid): acc[q] += sum_nu G[nu][etid] A_q[nu]
// for the NQ AO quantities, the columns in order.  The AO values stream in
// groups of GW columns through 4 register buffers (3 groups in flight).
template <int NQ, int GW>
__device__ __forceinline__ void contract_rows(const double* __restrict__ ao, int64_t ldq,
                                              const double* __restrict__ sG, int etid, uint64_t stream,
                                              double* acc) {
  constexpr int NB = 4;
  constexpr int NG = kN / GW;
  double a[NB][NQ][GW];
  auto load = [&](int buf, int cg) {
#pragma unroll
    for (int q = 0; q < NQ; ++q)
#pragma unroll
      for (int j = 0; j < GW; ++j) a[buf][q][j] = ldg_f64_stream(ao + q * ldq + (cg + j) * kRows, stream);
  };
#pragma unroll
  for (int g = 0; g < NB - 1; ++g) load(g, g * GW);
#pragma unroll
  for (int g = 0; g < NG; ++g) {
    if (g + NB - 1 < NG) load((g + NB - 1) % NB, (g + NB - 1) * GW);
#pragma unroll
    for (int j = 0; j < GW; ++j) {
      const double gv = sG[(g * GW + j) * kRows + etid];
#pragma unroll
      for (int q = 0; q < NQ; ++q) acc[q] = fma(gv, a[g % NB][q][j], acc[q]);
    }
  }
}

template <int ROLE>
__device__ __forceinline__ void store_role(double (*s_sums)[16], int lane, const double* acc) {
  constexpr int NS = role_nslot(ROLE);
  int i = 0;
#pragma unroll
  for (int s = 0; s < NS; ++s)
#pragma unroll
    for (int rr = 0; rr < role_nrow(ROLE, s); ++rr, ++i) s_sums[lane][role_sum(ROLE, s, rr)] = acc[i];
}

// ------------------------------------------------------------------ preparation kernels
// D (Mpad x Mpad, symmetric) -> one 64-bit word of five digits per element
// (pack_digits5), exponent per row.
__global__ void slice_d_kernel(const double* __restrict__ D, int Mpad, uint64_t* __restrict__ Dp,
                               int32_t* __restrict__ fexp) {
  const int row = blockIdx.x;
  const double* d = D + (int64_t)row * Mpad;
  double m = 0.0;
  for (int k = threadIdx.x; k < Mpad; k += blockDim.x) m = fmax(m, fabs(d[k]));
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    m = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (threadIdx.x == 0) red[0] = m;
  }
  __syncthreads();
  const int e = scale_exponent(red[0]);
  if (threadIdx.x == 0) fexp[row] = e;
  const double f = split_row_factor(e, kFixedBitsD);
  for (int k = threadIdx.x; k < Mpad; k += blockDim.x)
    Dp[(int64_t)row * Mpad + k] = pack_digits5(rint_i64(d[k] * f));
}

// Atom pairs with a non-zero element of D: nz[a * natom + b] = 1 for every
// D[mu][nu] != 0 with mu on atom a, nu on atom b (internal AO order).
__global__ void atom_pair_nonzero_kernel(const double* __restrict__ D, int M, int Mpad,
                                         const int32_t* __restrict__ ao_atom, int natom,
                                         uint8_t* __restrict__ nz) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)M * M) return;
  const int i = (int)(e / M), j = (int)(e % M);
  if (D[(int64_t)i * Mpad + j] != 0.0) nz[(int64_t)ao_atom[i] * natom + ao_atom[j]] = 1;
}

// Active K stages of each tile: bit nt * nb + kb of tile t's mask is set when
// the D block of nu block nt and mu block kb (64 compact AOs each) has a
// non-zero atom pair, and always for kb = 0 (the stage that initialises the
// accumulators of a nu tile).  One block per tile; a 64-AO block with more
// than kMaskAtoms distinct atoms is taken as non-zero.
constexpr int kMaskAtoms = 16;
__global__ void __launch_bounds__(256)
    stage_mask_kernel(TileBatch tb, const int32_t* __restrict__ ao_atom, const uint8_t* __restrict__ nz,
                      int natom, uint32_t* __restrict__ mask, int mask_words) {
  __shared__ int s_at[256][kMaskAtoms + 1];  // per 64-AO block: count, then atoms
  const int t = blockIdx.x;
  const int nb = tb.kt[t] / 64;
  const int32_t* am = tb.aomap + (int64_t)t * tb.Kcap;
  uint32_t* mk = mask + (int64_t)t * mask_words;
  for (int w = threadIdx.x; w < mask_words; w += blockDim.x) mk[w] = 0u;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    int cnt = 0;
    for (int k = 0; k < 64 && cnt <= kMaskAtoms; ++k) {
      const int ao = am[b * 64 + k];
      if (ao < 0) continue;
      const int a = ao_atom[ao];
      bool seen = false;
      for (int i = 0; i < cnt && i < kMaskAtoms; ++i) seen |= s_at[b][1 + i] == a;
      if (!seen) {
        if (cnt < kMaskAtoms) s_at[b][1 + cnt] = a;
        ++cnt;
      }
    }
    s_at[b][0] = cnt;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
    const int bi = e / nb, bj = e % nb;  // nu block, mu block
    bool on = bj == 0;
    const int ci = s_at[bi][0], cj = s_at[bj][0];
    if (ci > kMaskAtoms || cj > kMaskAtoms) on = true;
    for (int i = 0; i < ci && !on; ++i)
      for (int j = 0; j < cj && !on; ++j) on = nz[(int64_t)s_at[bi][1 + i] * natom + s_at[bj][1 + j]] != 0;
    if (on) atomicOr(&mk[e >> 5], 1u << (e & 31));
  }
}

// ------------------------------------------------------------------ main kernel
struct TcArgs {
  TileBatch tb;
  int nqa;
  const uint64_t* Dp;    // packed D digits (pack_digits5), Mpad x Mpad
  const int32_t* fexp;   // D row exponents
  const int32_t* eexp;   // A row exponents [C][128]
  int Mpad;
  ctc_outputs out;
  ctc_params prm;
  int32_t* status;
  // tile schedule: order[0..C) lists the chunk's tiles (largest compact K
  // first); tile_counter (zero at launch) hands them out to the CTAs
  const int32_t* order;
  int32_t* tile_counter;
  // limit of every pipeline wait, in SM cycles (kWaitCycles unless a caller
  // shortens it to exercise the timeout path)
  long long wait_cycles;
  // active K stages per tile (stage_mask_kernel), mask_words words per tile;
  // nullptr: every stage is active
  const uint32_t* stage_mask;
  int mask_words;
  // optional per-CTA cycle counters (CTC_TC_TRACE): [grid][8] = total,
  // producer wait on empty, producer stage work, MMA wait on full, MMA wait
  // on tempty, epilogue wait on tfull, drain, contraction
  long long* trace;
};

template <int NQA>
__global__ void __launch_bounds__(kThreadsTc, 1)
    tc_tile_kernel(const __grid_constant__ CUtensorMap amap, TcArgs args) {
  extern __shared__ uint8_t smem_raw[];
  // full_bar[s]: the 128 producer threads wrote stage s's B planes; tma_bar[s]:
  // stage s's A planes landed (its own barrier, so that an exit after a
  // timeout can wait for exactly the TMA loads it issued)
  __shared__ __align__(8) uint64_t full_bar[kStages], tma_bar[kStages], empty_bar[kStages];
  __shared__ __align__(8) uint64_t tfull_bar, tempty_bar, done_bar;
  __shared__ __align__(8) uint64_t tile_full_bar[2], tile_empty_bar[2];
  __shared__ uint32_t tmem_base_sh;
  __shared__ int s_abort;
  __shared__ int s_tile[2];
  __shared__ int s_epi_tile;
  __shared__ int s_epi_abort[2];
  __shared__ double s_sums[32][16];
  __shared__ double s_cscale[2][kN];

  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* sA = smem;
  uint8_t* sB = smem + kStages * kAStageBytes;
  double* sG = (double*)(smem + kStages * (kAStageBytes + kBStageBytes));  // [kN][kRows]

  const TileBatch& tb = args.tb;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full_bar[s], 128);
      mbar_init(&tma_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&tfull_bar, 1);
    mbar_init(&tempty_bar, 128);
    mbar_init(&done_bar, 1);
    for (int i = 0; i < 2; ++i) {
      mbar_init(&tile_full_bar[i], 1);
      mbar_init(&tile_empty_bar[i], kTileReaders);
    }
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == kMmaWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;\n" ::"r"(
                     smem_u32(&tmem_base_sh)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;
  const long long t_start = clock64();
  long long tr0 = 0, tr1 = 0, tr2 = 0;  // per-role trace counters

  // The CTA's i-th tile arrives through slot i & 1 of a two-entry ring: the
  // first producer thread takes the next index of the chunk's tile order from
  // the launch-wide counter, publishes it (-1 when the chunk is exhausted) and
  // every role reads it; a slot is refilled once all kTileReaders readers have
  // released it.  Each role walks the same tile sequence at its own pace.
  //
  // Abort decisions are warp-uniform: a warp takes every decision that leads
  // to a warp-collective instruction (__syncwarp, shuffles, tcgen05 .aligned
  // forms) from one vote, so lanes whose waits end at different moments (a
  // timeout in one lane only) never split around such an instruction.
  auto read_tile = [&](int i) -> int {
    const int slot = i & 1;
    int t = -1;
    if (!mbar_wait(&tile_full_bar[slot], (i >> 1) & 1, args.wait_cycles)) {
      s_abort = 1;
    } else {
      t = s_tile[slot];
    }
    return t;
  };
  // whole-warp form: lane 0 waits, the warp takes its answer
  auto read_tile_warp = [&](int i) -> int {
    int t = -1;
    if (lane == 0) t = read_tile(i);
    return __shfl_sync(0xffffffffu, t, 0);
  };
  auto warp_abort = [&]() -> bool { return __any_sync(0xffffffffu, s_abort != 0); };
  // is stage j (= nu tile * nkb + K block) of tile t active?  (block-sparse D)
  auto stage_on = [&](int t, int j) -> bool {
    return !args.stage_mask ||
           ((__ldg(args.stage_mask + (int64_t)t * args.mask_words + (j >> 5)) >> (j & 31)) & 1u);
  };

  if (warp < 4) {
    // ---------------- producers
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;\n" ::"n"(kProducerRegs));
    // Thread tid owns the 4 mu columns k4 = (tid % 16) * 4 of every stage and the
    // 8 nu rows n = tid / 16 + 8 i of every nu tile; its 32 gathers of D are
    // independent.  Stages are software-pipelined one ahead: the AO indices of
    // stage j + 1 are requested before the wait for stage j's slot, and its
    // gathers right after stage j's shared-memory writes, so the two dependent
    // global latencies overlap the MMAs instead of adding up.
    const int tid = threadIdx.x;
    const int k4 = (tid & 15) * 4, nrow0 = tid >> 4;
    const uint64_t keep = policy_evict_last();
    int it = 0;  // stage counter across tiles
    // thread 0: stage counter of the last TMA issue into each slot (-1: none)
    int last_issue[kStages];
#pragma unroll
    for (int s = 0; s < kStages; ++s) last_issue[s] = -1;
    for (int i = 0;; ++i) {
      if (tid == 0) {
        const int slot = i & 1;
        int next = -1;
        if (!mbar_wait(&tile_empty_bar[slot], ((i >> 1) & 1) ^ 1, args.wait_cycles)) {
          s_abort = 1;
        } else {
          const int c = atomicAdd(args.tile_counter, 1);
          next = c < tb.C ? args.order[c] : -1;
        }
        s_tile[slot] = next;
        mbar_arrive(&tile_full_bar[slot]);
      }
      const int t = read_tile_warp(i);
      if (lane == 0) mbar_arrive(&tile_empty_bar[i & 1]);
      if (t < 0 || warp_abort()) break;
      const int kt = tb.kt[t];
      const int nkb = kt / kBK;
      const int nnt = (kt + kN - 1) / kN;
      const int nst = nnt * nkb;
      const int32_t* am = tb.aomap + (int64_t)t * tb.Kcap;
      auto load_idx = [&](int j, int (&nu)[8], int (&mu)[4]) {
        const int nt = j / nkb, kb = j - nt * nkb;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int nc = nt * kN + nrow0 + 8 * q;
          nu[q] = nc < kt ? am[nc] : -1;
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) mu[q] = am[kb * kBK + k4 + q];
      };
      auto gather = [&](const int (&nu)[8], const int (&mu)[4], uint64_t (&w)[8][4]) {
#pragma unroll
        for (int q = 0; q < 8; ++q)
#pragma unroll
          for (int m = 0; m < 4; ++m)
            w[q][m] = (nu[q] >= 0 && mu[m] >= 0)
                          ? ldg_u64_hint(args.Dp + (int64_t)nu[q] * args.Mpad + mu[m], keep)
                          : 0ull;
      };
      int nu[8], mu[4];
      uint64_t w[8][4];
      // the tile's active stages in order (every stage unless D is block-sparse)
      auto next_on = [&](int j) -> int {
        while (j < nst && !stage_on(t, j)) ++j;
        return j;
      };
      int j = next_on(0);
      if (j < nst) {
        load_idx(j, nu, mu);
        gather(nu, mu, w);
      }
      for (; j < nst; ++it) {
        const int jn = next_on(j + 1);
        const bool more = jn < nst;
        if (more) load_idx(jn, nu, mu);
        const int s = it % kStages;
        const uint32_t ph = (it / kStages) & 1;
        const int k0 = (j % nkb) * kBK;
        const long long tw = clock64();
        if (!__all_sync(0xffffffffu, mbar_wait(&empty_bar[s], ph ^ 1, args.wait_cycles))) {
          s_abort = 1;
          break;
        }
        tr0 += clock64() - tw;
        if (tid == 0) {
          mbar_arrive_expect_tx(&tma_bar[s], kAStageBytes);
          for (int p = 0; p < kPlanesA; ++p)
            tma_load_2d_hint(sA + s * kAStageBytes + p * kAPlaneBytes, &amap, k0,
                             (t * kPlanesA + p) * kRows, &tma_bar[s], keep);
          last_issue[s] = it;
        }
        uint8_t* b = sB + s * kBStageBytes;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          // 4 words of 5 digit bytes -> 5 plane words of 4 consecutive mu:
          // digits 0-3 by a byte transpose of the low halves, digit 4 from
          // byte 4 of each word
          uint32_t pl[4];
          transpose_bytes4x4((uint32_t)w[q][0], (uint32_t)w[q][1], (uint32_t)w[q][2],
                             (uint32_t)w[q][3], pl);
          const uint32_t lo = __byte_perm(__byte_perm((uint32_t)(w[q][0] >> 32), (uint32_t)(w[q][1] >> 32), 0x0040),
                                          __byte_perm((uint32_t)(w[q][2] >> 32), (uint32_t)(w[q][3] >> 32), 0x0040),
                                          0x5410);
          const uint32_t off = sw64_offset(nrow0 + 8 * q, k4);
#pragma unroll
          for (int p = 0; p < 4; ++p) *(uint32_t*)(b + p * kBPlaneBytes + off) = pl[p];
          *(uint32_t*)(b + 4 * kBPlaneBytes + off) = lo;
        }
        fence_proxy_async();
        mbar_arrive(&full_bar[s]);
        if (more) gather(nu, mu, w);
        j = jn;
      }
      if (warp_abort()) break;
    }
    // Before the CTA may exit, every TMA load this thread issued has landed:
    // on the normal path the MMA warp has already seen each of them complete;
    // after a timeout a load can still be writing into shared memory.  The
    // wait uses the full limit, not the launch's (possibly shortened) one.
    if (tid == 0) {
#pragma unroll
      for (int s = 0; s < kStages; ++s)
        if (last_issue[s] >= 0 && !mbar_wait(&tma_bar[s], (last_issue[s] / kStages) & 1))
          atomicExch(args.status, (int32_t)kStatusTimeout);
    }
    if (args.trace && tid == 0) {
      args.trace[(int64_t)blockIdx.x * 8 + 1] = tr0;
      args.trace[(int64_t)blockIdx.x * 8 + 2] = clock64() - t_start - tr0;
    }
  } else if (warp == kMmaWarp) {
    // ---------------- MMA issuer
    // One MMA per A digit plane pa and K step: B is the stage's first D planes
    // read as one operand of 64 * nb rows (the planes are contiguous), so the
    // MMA's column block j is the product a_pa b_j and lands at TMEM column
    // (pa + j) * 64, the accumulator of level L = pa + j.  nb = min(4, 5 - pa)
    // keeps L <= 4.  At the first K step of a nu tile pa = 0 (levels 0-3) and
    // pa = 4 (level 4) initialise the 320 columns; every later MMA
    // accumulates.  Five MMAs of N = 256, 256, 192, 128, 64 plus a_0 b_4
    // (N = 64, level 4) replace the 15 N = 64 products: the same work in
    // fewer, wider instructions.
    const uint32_t idesc0 = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kRows >> 4) << 24);
    int it = 0, gnt = 0;  // stage and nu-tile counters across tiles
    for (int i = 0;; ++i) {
      const int t = read_tile_warp(i);
      if (lane == 0) mbar_arrive(&tile_empty_bar[i & 1]);
      if (t < 0 || warp_abort()) break;
      const int kt = tb.kt[t];
      const int nkb = kt / kBK;
      const int nnt = (kt + kN - 1) / kN;
      bool failed = false;
      for (int nt = 0; nt < nnt && !failed; ++nt, ++gnt) {
        const long long tw = clock64();
        if (!__all_sync(0xffffffffu, mbar_wait(&tempty_bar, (gnt & 1) ^ 1, args.wait_cycles))) {
          s_abort = 1;
          failed = true;
          break;
        }
        tr1 += clock64() - tw;
        tc_fence_after();
        for (int kb = 0; kb < nkb; ++kb) {
          if (!stage_on(t, nt * nkb + kb)) continue;  // zero D block: no data, no MMA
          const int s = it % kStages;
          const uint32_t ph = (it / kStages) & 1;
          const long long tf = clock64();
          const bool ready = mbar_wait(&full_bar[s], ph, args.wait_cycles) &&
                             mbar_wait(&tma_bar[s], ph, args.wait_cycles);
          if (!__all_sync(0xffffffffu, ready)) {
            s_abort = 1;
            failed = true;
            break;
          }
          tr0 += clock64() - tf;
          tc_fence_after();
          if (lane == 0) {
            const uint32_t a0 = smem_u32(sA + s * kAStageBytes);
            const uint32_t b0 = smem_u32(sB + s * kBStageBytes);
#pragma unroll
            for (int ks = 0; ks < kBK / 32; ++ks) {
              const uint64_t bd = umma_desc_sw64(b0 + ks * 32);
              const bool first = kb == 0 && ks == 0;
#pragma unroll
              for (int o = 0; o < kPlanesA; ++o) {
                const int pa = o == 0 ? 0 : (o == 1 ? kPlanesA - 1 : o - 1);  // 0, 4, 1, 2, 3
                const int nb = 4 < kLevels - pa ? 4 : kLevels - pa;  // at most N = 256
                const uint32_t idesc = idesc0 | ((uint32_t)(nb * kN >> 3) << 17);
                const uint64_t ad = umma_desc_sw64(a0 + pa * kAPlaneBytes + ks * 32);
                umma_i8(tmem + pa * kN, ad, bd, idesc, (first && o < 2) ? 0u : 1u);
              }
              // a_0 b_4 (level 4), after level 4 was initialised above
              umma_i8(tmem + 4 * kN, umma_desc_sw64(a0 + ks * 32),
                      umma_desc_sw64(b0 + 4 * kBPlaneBytes + ks * 32),
                      idesc0 | ((uint32_t)(kN >> 3) << 17), 1u);
            }
            umma_commit(&empty_bar[s]);
          }
          __syncwarp();
          ++it;
        }
        if (failed) break;
        if (lane == 0) umma_commit(&tfull_bar);
        __syncwarp();
      }
      if (failed || warp_abort()) break;
    }
    if (args.trace && lane == 0) {
      args.trace[(int64_t)blockIdx.x * 8 + 3] = tr0;
      args.trace[(int64_t)blockIdx.x * 8 + 4] = tr1;
    }
  } else {
    // ---------------- epilogue (warps 4..7 -> TMEM lane quarters 0..3)
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;\n" ::"n"(kEpilogueRegs));
    // Per nu tile: drain the five level accumulators of this warp's TMEM lane
    // quarter into one FP64 value per element, scaled, in the shared-memory
    // copy of G; release TMEM (the MMA warp starts the next nu tile); then
    // contract G with the FP64 AO values while those MMAs run.  A tile's
    // final sums are formed while the MMAs of the next tile run.
    const int quarter = warp & 3;
    const int r = quarter * 32 + lane;        // TMEM lane / G row drained by this thread
    const int role = warp - 4;                // 0..3
    const int etid = role * 32 + lane;        // 0..127
    constexpr int PTS = kRows / NQA;
    const int nq_ao = tb.nq;
    const int64_t ldq = (int64_t)tb.TP * tb.Kcap;
    // point contracted by this thread: NQA = 4 -> lane (all roles share the 32
    // points, each with its own AO quantities); NQA = 1 -> the role's 32 rows
    const int pc = (NQA == 4) ? lane : etid;
    const uint64_t stream = policy_evict_first();
    int gnt = 0;        // nu-tile counter across tiles
    bool stop = false;  // uniform across the four epilogue warps
    for (int i = 0; !stop; ++i) {
      // one reader for the four warps keeps their decisions uniform
      if (etid == 0) {
        s_epi_tile = read_tile(i);
        mbar_arrive(&tile_empty_bar[i & 1]);
      }
      asm volatile("bar.sync 1, 128;\n" ::: "memory");
      const int t = s_epi_tile;
      if (t < 0) break;
      const int kt = tb.kt[t];
      const int nnt = (kt + kN - 1) / kN;
      const int32_t* am = tb.aomap + (int64_t)t * tb.Kcap;
      const double* aop = tb.ao + (int64_t)t * nq_ao * ldq + pc;  // element (q, k) at aop[q*ldq + k*PTS]
      // G = 2^(e_r + f_nu - 76) sum_L acc_L 2^(64 - 8 L); the drain below forms
      // sum_L acc_L 2^(32 - 8 L), so the row factor carries the remaining 2^-44
      const double rowscale = ldexp(1.0, args.eexp[(int64_t)t * kRows + r] - 44);
      double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
      for (int nt = 0; nt < nnt; ++nt, ++gnt) {
        const int n0 = nt * kN;
        double* cs = s_cscale[gnt & 1];
        if (etid < kN) {
          const int nc = n0 + etid;
          const int nu = nc < kt ? am[nc] : -1;
          cs[etid] = nu >= 0 ? ldexp(1.0, args.fexp[nu]) : 0.0;
        }
        // (A) column scales written; every role has finished reading sG
        asm volatile("bar.sync 1, 128;\n" ::: "memory");
        // uniform stop decision: the flag slot read here was written before (B)
        // of the previous nu tile
        if (gnt > 0 && s_epi_abort[(gnt - 1) & 1]) { stop = true; break; }
        const long long te = clock64();
        if (!mbar_wait(&tfull_bar, gnt & 1, args.wait_cycles)) s_abort = 1;
        __syncwarp();  // converged for the .aligned TMEM loads below
        const long long td = clock64();
        tr0 += td - te;
        tc_fence_after();
#pragma unroll 1
        for (int c = 0; c < kN / 16; ++c) {
          int32_t v[kLevels][16];
#pragma unroll
          for (int L = 0; L < kLevels; ++L)
            tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + L * kN + c * 16, v[L]);
          tmem_ld_wait();
#pragma unroll
          for (int L = 0; L < kLevels; ++L) after_wait16(v[L]);
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            // sum_L acc_L 2^(32 - 8 L), smallest terms first
            double g = i32_times_pow2<0>(v[4][j]);
            g += i32_times_pow2<8>(v[3][j]);
            g += i32_times_pow2<16>(v[2][j]);
            g += i32_times_pow2<24>(v[1][j]);
            g += i32_times_pow2<32>(v[0][j]);
            sG[(c * 16 + j) * kRows + r] = g * rowscale * cs[c * 16 + j];
          }
        }
        tc_fence_before();
        mbar_arrive(&tempty_bar);
        const long long tc0 = clock64();
        tr1 += tc0 - td;
        if (etid == 0) s_epi_abort[gnt & 1] = s_abort;
        // (B) G of this nu tile complete in shared memory
        asm volatile("bar.sync 1, 128;\n" ::: "memory");
        const double* ao_nt = aop + (int64_t)n0 * PTS;
        if (NQA == 4) {
          switch (role) {
            case 0: contract_role<0, kEpiGroup>(ao_nt, ldq, sG, lane, nq_ao, stream, acc); break;
            case 1: contract_role<1, kEpiGroup>(ao_nt, ldq, sG, lane, nq_ao, stream, acc); break;
            case 2: contract_role<2, kEpiGroup>(ao_nt, ldq, sG, lane, nq_ao, stream, acc); break;
            default: contract_role<3, kEpiGroup>(ao_nt, ldq, sG, lane, nq_ao, stream, acc); break;
          }
        } else {
          // rows are points: sums over the nq_ao (1 or 4) quantities of this point
          if (nq_ao == 1) contract_rows<1, 4>(ao_nt, ldq, sG, etid, stream, acc);
          else contract_rows<4, 2>(ao_nt, ldq, sG, etid, stream, acc);
        }
        if (args.trace) {
          // results of the contraction are complete when they are used
          double chk = acc[0] + acc[1] + acc[2] + acc[3] + acc[4];
          asm volatile("" : "+d"(chk));
          tr2 += clock64() - tc0;
        }
      }
      // (C) gather the per-point sums and finalise
      asm volatile("bar.sync 1, 128;\n" ::: "memory");
      const bool aborted = stop || s_abort != 0;
      if (NQA == 4) {
        switch (role) {
          case 0: store_role<0>(s_sums, lane, acc); break;
          case 1: store_role<1>(s_sums, lane, acc); break;
          case 2: store_role<2>(s_sums, lane, acc); break;
          default: store_role<3>(s_sums, lane, acc); break;
        }
        asm volatile("bar.sync 1, 128;\n" ::: "memory");
        if (role == 0 && !aborted) {
          const int64_t pi = (int64_t)t * tb.TP + lane;
          const int64_t oidx = tb.out[pi];
          if (oidx >= 0) {
            if (finite_point(tb.xyz + 3 * pi)) finalize_point(s_sums[lane], 4, nq_ao, args.out, oidx, args.prm);
            else nan_point(args.out, oidx);
          }
        }
      } else if (!aborted) {
        const int64_t pi = (int64_t)t * tb.TP + etid;
        const int64_t oidx = tb.out[pi];
        double s16[16];
        for (int q = 0; q < 16; ++q) s16[q] = q < 4 ? acc[q] : 0.0;
        if (oidx >= 0) {
          if (finite_point(tb.xyz + 3 * pi)) finalize_point(s16, 1, nq_ao, args.out, oidx, args.prm);
          else nan_point(args.out, oidx);
        }
      }
    }
    if (args.trace && etid == 0) {
      args.trace[(int64_t)blockIdx.x * 8 + 5] = tr0;
      args.trace[(int64_t)blockIdx.x * 8 + 6] = tr1;
      args.trace[(int64_t)blockIdx.x * 8 + 7] = tr2;
    }
  }
  __syncthreads();
  if (args.trace && threadIdx.x == 0) args.trace[(int64_t)blockIdx.x * 8] = clock64() - t_start;
  if (s_abort && threadIdx.x == 0) atomicExch(args.status, (int32_t)kStatusTimeout);
  if (warp == kMmaWarp) {
    // every MMA this thread issued has completed before TMEM is released
    if (lane == 0) umma_commit(&done_bar);
    __syncwarp();
    if (!mbar_wait(&done_bar, 0) && lane == 0) atomicExch(args.status, (int32_t)kStatusTimeout);
    __syncwarp();  // converged for the .aligned dealloc
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;\n" ::"r"(tmem));
  }
}

PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

}  // namespace

int prepare_tc(ctc_molecule* mol, cudaStream_t st) {
  if (mol->dsl_valid) return CTC_OK;
  int dev = 0, major = 0;
  CTC_CUDA_TRY(cudaGetDevice(&dev));
  CTC_CUDA_TRY(cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev));
  if (major != 10) return fail(CTC_ERR_UNSUPPORTED, "tensor-core split path needs an sm_100 GPU");
  const size_t MM = (size_t)mol->Mpad * mol->Mpad;
  if (!mol->d_Dsl) CTC_CUDA_TRY(cudaMalloc((void**)&mol->d_Dsl, sizeof(uint64_t) * MM));
  if (!mol->d_Dscale) CTC_CUDA_TRY(cudaMalloc((void**)&mol->d_Dscale, sizeof(int32_t) * mol->Mpad));
  slice_d_kernel<<<mol->Mpad, 256, 0, st>>>(mol->d_D, mol->Mpad, (uint64_t*)mol->d_Dsl,
                                            (int32_t*)mol->d_Dscale);
  CTC_CUDA_TRY(cudaGetLastError());
  // atom-pair map of D's non-zero blocks, kept only if some block is zero
  // (every AO on an atom, at most 4096 atoms: a map of 16 MB at most)
  cudaFree(mol->d_nzpair);
  mol->d_nzpair = nullptr;
  const int na = mol->natom;
  bool atoms_ok = na > 0 && na <= 4096;
  for (int a : mol->ao_atom) atoms_ok = atoms_ok && a >= 0 && a < na;
  if (atoms_ok) {
    const size_t nn = (size_t)na * na;
    CTC_CUDA_TRY(cudaMalloc((void**)&mol->d_nzpair, nn));
    CTC_CUDA_TRY(cudaMemsetAsync(mol->d_nzpair, 0, nn, st));
    const int64_t MM2 = (int64_t)mol->M * mol->M;
    atom_pair_nonzero_kernel<<<(unsigned)((MM2 + 255) / 256), 256, 0, st>>>(
        mol->d_D, mol->M, mol->Mpad, mol->d_ao_atom, na, mol->d_nzpair);
    CTC_CUDA_TRY(cudaGetLastError());
    std::vector<uint8_t> h(nn);
    CTC_CUDA_TRY(cudaMemcpyAsync(h.data(), mol->d_nzpair, nn, cudaMemcpyDeviceToHost, st));
    CTC_CUDA_TRY(cudaStreamSynchronize(st));
    if (std::find(h.begin(), h.end(), (uint8_t)0) == h.end()) {  // dense: nothing to skip
      cudaFree(mol->d_nzpair);
      mol->d_nzpair = nullptr;
    }
  }
  mol->dsl_valid = true;
  return CTC_OK;
}

// Chunk workspace of the tensor-core path, one layout for both users (the AO
// kernel that writes the digit planes and the contraction), for tiles of
// `rows` operand rows (ctc_split.cuh):
//   planes [C][rows / 128][5][128][Kcap] int8 | eexp [C][rows] | tile order:
//   keys in/out, ids in, order [C] | tile counter | radix-sort temporary storage
struct TcWorkspace {
  int8_t* planes;
  int32_t* eexp;
  uint32_t* mask;  // active K stages per tile (mask_words each), block-sparse D only
  int mask_words;
  uint32_t* keys_in;
  uint32_t* keys_out;
  int32_t* ids;
  int32_t* order;
  int32_t* counter;
  void* sort_tmp;
  size_t sort_bytes;
};

int tc_workspace(ctc_molecule* mol, const TileBatch& tb, int rows, cudaStream_t st, TcWorkspace* w) {
  size_t sort_bytes = 0;
  CTC_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (uint32_t*)nullptr,
                                               (uint32_t*)nullptr, (int32_t*)nullptr,
                                               (int32_t*)nullptr, tb.C, 0, 15, st));
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = (off + bytes + 255) / 256 * 256;
    return o;
  };
  const size_t o_planes = take((size_t)tb.C * kPlanesA * rows * tb.Kcap);
  const size_t o_eexp = take(sizeof(int32_t) * (size_t)tb.C * rows);
  const int nbmax = tb.Kcap / kBK;
  const int mask_words = mol->d_nzpair ? (nbmax * nbmax + 31) / 32 : 0;
  const size_t o_mask = take(sizeof(uint32_t) * (size_t)tb.C * mask_words);
  const size_t o_kin = take(sizeof(uint32_t) * tb.C);
  const size_t o_kout = take(sizeof(uint32_t) * tb.C);
  const size_t o_ids = take(sizeof(int32_t) * tb.C);
  const size_t o_order = take(sizeof(int32_t) * tb.C);
  const size_t o_counter = take(sizeof(int32_t));
  const size_t o_tmp = take(sort_bytes);
  int rc = mol->ws_sl.ensure(off, st);
  if (rc != CTC_OK) return rc;
  char* base = (char*)mol->ws_sl.p;
  w->planes = (int8_t*)(base + o_planes);
  w->eexp = (int32_t*)(base + o_eexp);
  w->mask = mask_words ? (uint32_t*)(base + o_mask) : nullptr;
  w->mask_words = mask_words;
  w->keys_in = (uint32_t*)(base + o_kin);
  w->keys_out = (uint32_t*)(base + o_kout);
  w->ids = (int32_t*)(base + o_ids);
  w->order = (int32_t*)(base + o_order);
  w->counter = (int32_t*)(base + o_counter);
  w->sort_tmp = base + o_tmp;
  w->sort_bytes = sort_bytes;
  return CTC_OK;
}

namespace {
// sort keys: largest compact K first (ascending kMaxKt - kt), ids = tile index
__global__ void tile_order_keys_kernel(const int32_t* __restrict__ kt, int C, uint32_t* keys,
                                       int32_t* ids, int32_t* counter) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i == 0) *counter = 0;
  if (i < C) {
    keys[i] = (uint32_t)(kMaxKt - min(kt[i], kMaxKt));
    ids[i] = i;
  }
}
}  // namespace

int tc_slice_workspace(ctc_molecule* mol, const TileBatch& tb, int nqa, cudaStream_t st,
                       int8_t** planes, int32_t** eexp, const int32_t** order) {
  TcWorkspace w;
  const int rc = tc_workspace(mol, tb, split_tile_rows(tb.TP, nqa), st, &w);
  if (rc != CTC_OK) return rc;
  // the chunk's tile order, largest compact K first: the AO kernel's CTAs and
  // the contraction's persistent CTAs both take the tiles in this order, so
  // the last tiles of either launch are the cheapest ones
  tile_order_keys_kernel<<<(tb.C + 255) / 256, 256, 0, st>>>(tb.kt, tb.C, w.keys_in, w.ids, w.counter);
  CTC_CUDA_TRY(cudaGetLastError());
  CTC_CUDA_TRY(cub::DeviceRadixSort::SortPairs(w.sort_tmp, w.sort_bytes, w.keys_in, w.keys_out, w.ids,
                                               w.order, tb.C, 0, 15, st));
  *planes = w.planes;
  *eexp = w.eexp;
  *order = w.order;
  return CTC_OK;
}

int tc_local_tiles(ctc_molecule* mol, const LocalPlan& plan, const TileBatch& tb,
                   const ctc_params* prm, const ctc_outputs* out, cudaStream_t st) {
  if (tb.C <= 0) return CTC_OK;
  if (tb.Kcap > kMaxKt)
    return fail(CTC_ERR_UNSUPPORTED, "tensor-core split path: more than 16384 functions per tile");
  int rc = prepare_tc(mol, st);
  if (rc != CTC_OK) return rc;
  // int8 planes of the tile rows, row exponents and the tile order (largest
  // compact K first, zeroed tile counter), written for this chunk by
  // tc_slice_workspace and the AO kernel (launch_ao_tiles_sliced)
  if (!((plan.nqa == 4 && tb.TP == 32) || (plan.nqa == 1 && tb.TP == 128)))
    return fail(CTC_ERR_INVALID, "tensor-core split path: unsupported tile layout");
  const int rows = split_tile_rows(tb.TP, plan.nqa);
  TcWorkspace w;
  if ((rc = tc_workspace(mol, tb, rows, st, &w)) != CTC_OK) return rc;
  // tensor map over the planes: 2-D, rows = C * rows * 5, inner = Kcap bytes;
  // boxes of 64 bytes (64-byte swizzle) by 128 rows
  PFN_cuTensorMapEncodeTiled_v12000 enc = get_encode();
  if (!enc) return fail(CTC_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
  CUtensorMap amap;
  cuuint64_t gdim[2] = {(cuuint64_t)tb.Kcap, (cuuint64_t)tb.C * kPlanesA * rows};
  cuuint64_t gstride[1] = {(cuuint64_t)tb.Kcap};
  cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)kRows};
  cuuint32_t estr[2] = {1, 1};
  CUresult cr = enc(&amap, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, w.planes, gdim, gstride, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (cr != CUDA_SUCCESS) return fail(CTC_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)cr));
  int num_sms = 0;
  if ((rc = device_sm_count(&num_sms)) != CTC_OK) return rc;
  const int grid = std::min(tb.C, num_sms);
  TcArgs a;
  a.tb = tb;
  a.nqa = plan.nqa;
  a.Dp = (const uint64_t*)mol->d_Dsl;
  a.fexp = (const int32_t*)mol->d_Dscale;
  a.eexp = w.eexp;
  a.Mpad = mol->Mpad;
  a.out = *out;
  a.prm = *prm;
  a.status = mol->d_status;
  a.order = w.order;
  a.tile_counter = w.counter;
  a.trace = nullptr;
  a.wait_cycles = mol->wait_cycles > 0 ? (long long)mol->wait_cycles : kWaitCycles;
  a.stage_mask = w.mask;
  a.mask_words = w.mask_words;
  if (w.mask) {
    stage_mask_kernel<<<tb.C, 256, 0, st>>>(tb, mol->d_ao_atom, mol->d_nzpair, mol->natom, w.mask,
                                           w.mask_words);
    CTC_CUDA_TRY(cudaGetLastError());
    mol->host_launches += 1;
  }
  // CTC_TC_TRACE=1: per-CTA cycle counters of the kernel's roles, summarised
  // on stderr after each launch (synchronises the stream; diagnostics only)
  static const bool trace_on = std::getenv("CTC_TC_TRACE") != nullptr;
  if (trace_on) CTC_CUDA_TRY(cudaMallocAsync((void**)&a.trace, sizeof(long long) * 8 * grid, st));
  if ((rc = ensure_smem_attr(plan.nqa == 4 ? (const void*)tc_tile_kernel<4> : (const void*)tc_tile_kernel<1>,
                             kSmemTc)) != CTC_OK)
    return rc;
  ProfScope ps(mol, 0, st);
  if (plan.nqa == 4) tc_tile_kernel<4><<<grid, kThreadsTc, kSmemTc, st>>>(amap, a);
  else tc_tile_kernel<1><<<grid, kThreadsTc, kSmemTc, st>>>(amap, a);
  CTC_CUDA_TRY(cudaGetLastError());
  if (trace_on) {
    std::vector<long long> tr((size_t)8 * grid);
    std::vector<int32_t> kt(tb.C);
    CTC_CUDA_TRY(cudaMemcpyAsync(tr.data(), a.trace, sizeof(long long) * tr.size(), cudaMemcpyDeviceToHost, st));
    CTC_CUDA_TRY(cudaMemcpyAsync(kt.data(), tb.kt, sizeof(int32_t) * tb.C, cudaMemcpyDeviceToHost, st));
    CTC_CUDA_TRY(cudaStreamSynchronize(st));
    CTC_CUDA_TRY(cudaFreeAsync(a.trace, st));
    double sum[8] = {0}, stages = 0, ktmax = 0, ktsum = 0, totmax = 0;
    for (int i = 0; i < grid; ++i) {
      for (int k = 0; k < 8; ++k) sum[k] += (double)tr[(size_t)8 * i + k];
      totmax = std::max(totmax, (double)tr[(size_t)8 * i]);
    }
    for (int i = 0; i < tb.C; ++i) {
      stages += (kt[i] / (double)kBK) * std::ceil(kt[i] / (double)kN);
      ktsum += kt[i];
      ktmax = std::max(ktmax, (double)kt[i]);
    }
    std::fprintf(stderr,
                 "[ctc tc trace] tiles %d CTAs %d mean kt %.0f max kt %.0f | CTA cycles mean %.0f max %.0f | "
                 "per stage: total %.0f prod_wait_empty %.0f prod_work %.0f mma_wait_full %.0f "
                 "mma_wait_tempty %.0f epi_wait_tfull %.0f epi_drain %.0f epi_contract %.0f\n",
                 tb.C, grid, ktsum / tb.C, ktmax, sum[0] / grid, totmax, sum[0] / stages,
                 sum[1] / stages, sum[2] / stages, sum[3] / stages, sum[4] / stages, sum[5] / stages,
                 sum[6] / stages, sum[7] / stages);
  }
  return CTC_OK;
}

}  // namespace ctc
