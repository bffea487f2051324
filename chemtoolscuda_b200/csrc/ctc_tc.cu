// ctc_tc.cu -- tensor-core split-precision contraction (tcgen05, INT8, sm_100a).
//
// G_t = A_t D[S_t, S_t] of the screened tile pipeline (ctc_local.cu) on the
// 5th-generation tensor cores with results equal to the FP64 contraction to
// ~2e-9 relative (measured on the 200-atom benchmark molecule against the
// FP64 oracle; 1e-8 is the target).
//
// Split (an Ozaki-type scheme with exact integer accumulation):
//   * every A row r is scaled by 2^-e_r (e_r from the row's largest |value|),
//     every D row nu by 2^-f_nu, and rounded to a 31-bit fixed-point integer
//     I = rint(x 2^30);
//   * I is written in balanced base-256 digits d_0..d_3 (|d_i| <= 128,
//     I = sum_i d_i 256^(3-i)), one int8 plane per digit;
//   * the 13 digit products with i + j <= 4 are accumulated on INT8 tensor
//     cores (tcgen05.mma kind::i8, int32 accumulators in TMEM), one TMEM
//     accumulator per level L = i + j;  int32 accumulation is exact as long
//     as the compact K of a tile stays below 16 384;
//   * the epilogue forms G = 2^(e_r + f_nu - 60) sum_L acc_L 2^(48 - 8 L) in
//     FP64 and reduces it against the FP64 AO values (same epilogue sums as
//     the FP64 path).
// The dropped products (i + j >= 5) are below 2^-40 of the row/column scale.
//
// Kernel roles (288 threads): warps 0-3 produce the operands of each K block
// (one thread issues the TMA loads of the four A planes; all 128 threads
// gather the four D planes by compact index from the packed copy of D and
// write them in the 64-byte-swizzled K-major layout), warp 4 issues the MMAs
// from one thread and commits them to mbarriers, warps 5-8 read the TMEM
// accumulators (one 32-lane quarter each) and run the FP64 epilogue.  Every
// mbarrier wait is bounded: on timeout the kernel records a status code,
// stops issuing work, and the allocating warp still frees its TMEM.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "ctc_internal.h"

namespace ctc {

namespace {

constexpr int kN = 64;          // nu columns per TMEM accumulator
constexpr int kBK = 64;         // K bytes per pipeline stage
constexpr int kStages = 4;
constexpr int kRows = 128;      // tile rows (MMA M)
constexpr int kLevels = 5;
constexpr int kPlanes = 4;
constexpr int kAPlaneBytes = kRows * kBK;       // 8 KB
constexpr int kBPlaneBytes = kN * kBK;          // 4 KB
constexpr int kAStageBytes = kPlanes * kAPlaneBytes;
constexpr int kBStageBytes = kPlanes * kBPlaneBytes;
constexpr int kSmemTc = kStages * (kAStageBytes + kBStageBytes) + 1024;  // + alignment slack
constexpr int kThreadsTc = 288;
constexpr int kMaxKt = 16384;
constexpr uint32_t kStatusTimeout = 0x7101;

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

// Bounded wait on an mbarrier phase: false after ~2 s of GPU time.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  const long long t0 = clock64();
  for (uint32_t it = 0;; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 255) == 255 && clock64() - t0 > 4000000000LL) return false;
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

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int c0, int c1,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
          smem_u32(dst)),
      "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
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

// balanced base-256 digits of |I| <= 2^30, most significant first, packed in a word
__device__ __forceinline__ uint32_t pack_digits(int32_t I) {
  uint32_t w = 0;
#pragma unroll
  for (int p = 3; p >= 1; --p) {
    const int32_t d = ((I + 128) & 255) - 128;
    w |= (uint32_t)(d & 255) << (8 * p);
    I = (I - d) >> 8;
  }
  w |= (uint32_t)(I & 255);
  return w;
}

__device__ __forceinline__ int32_t to_fixed(double x, int e) {
  // |x| < 2^e  ->  |rint(x 2^(30-e))| <= 2^30
  return (int32_t)llrint(ldexp(x, 30 - e));
}

__device__ __forceinline__ int scale_exponent(double amax) {
  if (!(amax > 0.0)) return 0;
  int e;
  frexp(amax, &e);  // amax = m 2^e, m in [0.5, 1)
  return e;
}

// ------------------------------------------------------------------ preparation kernels
// D (Mpad x Mpad, symmetric) -> packed digit words per element, exponent per row.
__global__ void slice_d_kernel(const double* __restrict__ D, int Mpad, uint32_t* __restrict__ Dp,
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
  for (int k = threadIdx.x; k < Mpad; k += blockDim.x)
    Dp[(int64_t)row * Mpad + k] = pack_digits(to_fixed(d[k], e));
}

// Tile A rows (FP64, compact K, block layout [q][k][point]) -> four int8
// planes [t][plane][row][Kcap] (row = q * PTS + point, K contiguous) and row
// exponents.  Each lane owns one row: the row maximum reads consecutive points
// across lanes, and every lane then writes 32 bytes per plane per step.
__global__ void slice_a_kernel(TileBatch tb, int nqa, int8_t* __restrict__ planes,
                               int32_t* __restrict__ eexp) {
  const int t = blockIdx.x;
  const int kt = tb.kt[t];
  const int PTS = kRows / nqa;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t ldq = (int64_t)PTS * tb.Kcap;
  const double* A = tb.ao + (int64_t)t * tb.nq * ldq;
  int8_t* P = planes + (int64_t)t * kPlanes * kRows * tb.Kcap;
  for (int r = warp * 32 + lane; r < kRows; r += blockDim.x) {
    const int q = r / PTS, pl = r % PTS;
    const double* col = A + q * ldq + pl;  // element k at col[k * PTS]
    double m = 0.0;
    for (int k = 0; k < kt; ++k) m = fmax(m, fabs(col[(int64_t)k * PTS]));
    const int e = scale_exponent(m);
    eexp[(int64_t)t * kRows + r] = e;
    for (int k0 = 0; k0 < kt; k0 += 32) {
      uint32_t pw[kPlanes][8];
#pragma unroll
      for (int g = 0; g < 8; ++g) {
        uint32_t w[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) w[i] = pack_digits(to_fixed(col[(int64_t)(k0 + 4 * g + i) * PTS], e));
#pragma unroll
        for (int p = 0; p < kPlanes; ++p)
          pw[p][g] = ((w[0] >> (8 * p)) & 255) | (((w[1] >> (8 * p)) & 255) << 8) |
                     (((w[2] >> (8 * p)) & 255) << 16) | (((w[3] >> (8 * p)) & 255) << 24);
      }
#pragma unroll
      for (int p = 0; p < kPlanes; ++p) {
        uint4* dst = reinterpret_cast<uint4*>(P + ((int64_t)p * kRows + r) * tb.Kcap + k0);
        dst[0] = make_uint4(pw[p][0], pw[p][1], pw[p][2], pw[p][3]);
        dst[1] = make_uint4(pw[p][4], pw[p][5], pw[p][6], pw[p][7]);
      }
    }
  }
}

// ------------------------------------------------------------------ main kernel
struct TcArgs {
  TileBatch tb;
  int nqa;
  const uint32_t* Dp;    // packed D digits, Mpad x Mpad
  const int32_t* fexp;   // D row exponents
  const int32_t* eexp;   // A row exponents [C][128]
  int Mpad;
  ctc_outputs out;
  ctc_params prm;
  int32_t* status;
};

__device__ __forceinline__ void finalize_point_tc(const double* s, int nqa, int nq_ao,
                                                  const ctc_outputs& o, int64_t idx,
                                                  const ctc_params& prm);

template <int NQA>
__global__ void __launch_bounds__(kThreadsTc, 1)
    tc_tile_kernel(const __grid_constant__ CUtensorMap amap, TcArgs args) {
  extern __shared__ uint8_t smem_raw[];
  __shared__ __align__(8) uint64_t full_bar[kStages], empty_bar[kStages];
  __shared__ __align__(8) uint64_t tfull_bar, tempty_bar, done_bar;
  __shared__ uint32_t tmem_base_sh;
  __shared__ int s_abort;
  __shared__ double s_sums[32][16];
  __shared__ double s_cscale[2][kN];

  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* sA = smem;
  uint8_t* sB = smem + kStages * kAStageBytes;

  const TileBatch& tb = args.tb;
  const int t = blockIdx.x;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int kt = tb.kt[t];
  const int nkb = kt / kBK;
  const int nnt = (kt + kN - 1) / kN;
  const int32_t* am = tb.aomap + (int64_t)t * tb.Kcap;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full_bar[s], 129);
      mbar_init(&empty_bar[s], 1);
    }
    mbar_init(&tfull_bar, 1);
    mbar_init(&tempty_bar, 128);
    mbar_init(&done_bar, 1);
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 4) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;\n" ::"r"(
                     smem_u32(&tmem_base_sh)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_base_sh;

  if (warp < 4) {
    // ---------------- producers
    // Thread tid owns the 4 mu columns k4 = (tid % 16) * 4 of every stage and the
    // 8 nu rows n = tid / 16 + 8 i of every nu tile, so its AO indices are
    // loaded once per stage / tile and its 32 gathers of D are independent.
    const int tid = threadIdx.x;
    const int k4 = (tid & 15) * 4, nrow0 = tid >> 4;
    int it = 0;
    for (int nt = 0; nt < nnt && !s_abort; ++nt) {
      const int n0 = nt * kN;
      int nu[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int nc = n0 + nrow0 + 8 * i;
        nu[i] = nc < kt ? am[nc] : -1;
      }
      for (int kb = 0; kb < nkb; ++kb, ++it) {
        const int s = it % kStages;
        const uint32_t ph = (it / kStages) & 1;
        const int k0 = kb * kBK;
        int mu[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) mu[j] = am[k0 + k4 + j];
        uint32_t w[8][4];
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j)
            w[i][j] = (nu[i] >= 0 && mu[j] >= 0) ? __ldg(args.Dp + (int64_t)nu[i] * args.Mpad + mu[j]) : 0u;
        if (!mbar_wait(&empty_bar[s], ph ^ 1)) { s_abort = 1; break; }
        if (tid == 0) {
          mbar_arrive_expect_tx(&full_bar[s], kAStageBytes);
          for (int p = 0; p < kPlanes; ++p)
            tma_load_2d(sA + s * kAStageBytes + p * kAPlaneBytes, &amap, k0, (t * kPlanes + p) * kRows,
                        &full_bar[s]);
        }
        uint8_t* b = sB + s * kBStageBytes;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const uint32_t off = sw64_offset(nrow0 + 8 * i, k4);
#pragma unroll
          for (int p = 0; p < kPlanes; ++p) {
            const uint32_t v = ((w[i][0] >> (8 * p)) & 255) | (((w[i][1] >> (8 * p)) & 255) << 8) |
                               (((w[i][2] >> (8 * p)) & 255) << 16) | (((w[i][3] >> (8 * p)) & 255) << 24);
            *(uint32_t*)(b + p * kBPlaneBytes + off) = v;
          }
        }
        fence_proxy_async();
        mbar_arrive(&full_bar[s]);
      }
    }
  } else if (warp == 4) {
    // ---------------- MMA issuer
    const uint32_t idesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kN >> 3) << 17) |
                           ((uint32_t)(kRows >> 4) << 24);
    int it = 0;
    for (int nt = 0; nt < nnt && !s_abort; ++nt) {
      if (!mbar_wait(&tempty_bar, (nt & 1) ^ 1)) { s_abort = 1; break; }
      tc_fence_after();
      uint32_t started = 0;  // bit L: level L accumulator initialised
      for (int kb = 0; kb < nkb; ++kb, ++it) {
        const int s = it % kStages;
        const uint32_t ph = (it / kStages) & 1;
        if (!mbar_wait(&full_bar[s], ph)) { s_abort = 1; break; }
        tc_fence_after();
        if (lane == 0) {
          const uint32_t a0 = smem_u32(sA + s * kAStageBytes);
          const uint32_t b0 = smem_u32(sB + s * kBStageBytes);
#pragma unroll
          for (int ks = 0; ks < kBK / 32; ++ks) {
#pragma unroll
            for (int i = 0; i < kPlanes; ++i) {
#pragma unroll
              for (int j = 0; j < kPlanes; ++j) {
                const int L = i + j;
                if (L >= kLevels) continue;
                const uint64_t ad = umma_desc_sw64(a0 + i * kAPlaneBytes + ks * 32);
                const uint64_t bd = umma_desc_sw64(b0 + j * kBPlaneBytes + ks * 32);
                const uint32_t acc = (started >> L) & 1u;
                umma_i8(tmem + L * kN, ad, bd, idesc, acc);
                started |= 1u << L;
              }
            }
          }
          umma_commit(&empty_bar[s]);
        }
        __syncwarp();
      }
      if (s_abort) break;
      if (lane == 0) umma_commit(&tfull_bar);
      __syncwarp();
    }
  } else {
    // ---------------- epilogue (warps 5..8 -> TMEM lane quarters 1,2,3,0)
    const int quarter = warp & 3;
    const int r = quarter * 32 + lane;
    const int etid = (warp - 5) * 32 + lane;  // 0..127
    constexpr int PTS = kRows / NQA;
    const int q = r / PTS, pl = r % PTS;
    const int nq_ao = tb.nq;
    const int64_t ldq = (int64_t)tb.TP * tb.Kcap;
    const double* aop = tb.ao + (int64_t)t * nq_ao * ldq + pl;  // element (q, k) at aop[q*ldq + k*PTS]
    const double rowscale = ldexp(1.0, args.eexp[(int64_t)t * kRows + r] - 60);
    // quantities this row is reduced against: q = 0 -> phi, d phi, d2 phi; q = k -> d_j phi, j >= k
    const int qa = (q == 0) ? 0 : q;
    const int qb = (q == 0) ? nq_ao : 4;
    double sums[10];
#pragma unroll
    for (int i = 0; i < 10; ++i) sums[i] = 0.0;
    for (int nt = 0; nt < nnt && !s_abort; ++nt) {
      const int n0 = nt * kN;
      double* cs = s_cscale[nt & 1];
      if (etid < kN) {
        const int nc = n0 + etid;
        const int nu = nc < kt ? am[nc] : -1;
        cs[etid] = nu >= 0 ? ldexp(1.0, args.fexp[nu]) : 0.0;
      }
      asm volatile("bar.sync 1, 128;\n" ::: "memory");
      if (!mbar_wait(&tfull_bar, nt & 1)) { s_abort = 1; break; }
      tc_fence_after();
#pragma unroll 1
      for (int c = 0; c < kN / 16; ++c) {
        double g[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) g[j] = 0.0;
#pragma unroll
        for (int L = 0; L < kLevels; ++L) {
          int32_t v[16];
          tmem_ld16(tmem + ((uint32_t)(quarter * 32) << 16) + L * kN + c * 16, v);
          tmem_ld_wait();
          const double w = ldexp(1.0, 48 - 8 * L);
#pragma unroll
          for (int j = 0; j < 16; ++j) g[j] += (double)v[j] * w;
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) g[j] *= rowscale * cs[c * 16 + j];
        const int col = n0 + c * 16;
        for (int qq = qa; qq < qb; ++qq) {
          const double* src = aop + qq * ldq + (int64_t)col * PTS;
          double v[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) v[j] = __ldg(src + j * PTS);
          double acc = 0.0;
#pragma unroll
          for (int j = 0; j < 16; ++j) acc += g[j] * v[j];
          sums[qq - qa] += acc;
        }
      }
      tc_fence_before();
      mbar_arrive(&tempty_bar);
    }
    // gather the per-row sums of each point and finalise
    asm volatile("bar.sync 1, 128;\n" ::: "memory");
    if (NQA == 4) {
      if (q == 0) {
        for (int i = 0; i < 10; ++i) s_sums[pl][i] = sums[i];
      } else if (q == 1) {
        s_sums[pl][10] = sums[0]; s_sums[pl][11] = sums[1]; s_sums[pl][12] = sums[2];
      } else if (q == 2) {
        s_sums[pl][13] = sums[0]; s_sums[pl][14] = sums[1];
      } else {
        s_sums[pl][15] = sums[0];
      }
      asm volatile("bar.sync 1, 128;\n" ::: "memory");
      if (q == 0 && !s_abort) {
        const int64_t oidx = tb.out[(int64_t)t * tb.TP + pl];
        if (oidx >= 0) finalize_point_tc(s_sums[pl], 4, nq_ao, args.out, oidx, args.prm);
      }
    } else if (!s_abort) {
      const int64_t oidx = tb.out[(int64_t)t * tb.TP + pl];
      double s16[16];
      for (int i = 0; i < 16; ++i) s16[i] = i < 4 ? sums[i] : 0.0;
      if (oidx >= 0) finalize_point_tc(s16, 1, nq_ao, args.out, oidx, args.prm);
    }
  }
  __syncthreads();
  if (s_abort && threadIdx.x == 0) atomicExch(args.status, (int32_t)kStatusTimeout);
  if (warp == 4) {
    // every MMA this thread issued has completed before TMEM is released
    if (lane == 0) umma_commit(&done_bar);
    __syncwarp();
    if (!mbar_wait(&done_bar, 0) && lane == 0) atomicExch(args.status, (int32_t)kStatusTimeout);
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;\n" ::"r"(tmem));
  }
}

constexpr double kPi = 3.14159265358979323846;

__device__ __forceinline__ void finalize_point_tc(const double* s, int nqa, int nq_ao,
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
    const double pref = 0.5 / cbrt(3.0 * kPi * kPi);
    const double d43 = pow(rho, 4.0 / 3.0);
    o.rdg[idx] = pref * (d43 > 1e-20 ? sqrt(gsq) / d43 : 1e-20);
  }
  if (o.shannon) o.shannon[idx] = rho * log(rho);
  double w = 0.0, tf = 0.0;
  if (o.weizsacker || o.gge) w = 8.0 * rho > 1e-20 ? gsq / (8.0 * rho) : 1e-20;
  if (o.thomas_fermi || o.gge) tf = 0.3 * pow(3.0 * kPi * kPi, 2.0 / 3.0) * pow(rho, 5.0 / 3.0);
  if (o.weizsacker) o.weizsacker[idx] = w;
  if (o.thomas_fermi) o.thomas_fermi[idx] = tf;
  if (o.gge) o.gge[idx] = tf + prm.gge_a * w + prm.gge_b * lap;
  if (o.general_ked) o.general_ked[idx] = tau + 0.25 * (prm.ked_a - 1.0) * lap;
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
  if (!mol->d_Dsl) CTC_CUDA_TRY(cudaMalloc((void**)&mol->d_Dsl, sizeof(uint32_t) * MM));
  if (!mol->d_Dscale) CTC_CUDA_TRY(cudaMalloc((void**)&mol->d_Dscale, sizeof(int32_t) * mol->Mpad));
  slice_d_kernel<<<mol->Mpad, 256, 0, st>>>(mol->d_D, mol->Mpad, (uint32_t*)mol->d_Dsl,
                                            (int32_t*)mol->d_Dscale);
  CTC_CUDA_TRY(cudaGetLastError());
  mol->dsl_valid = true;
  return CTC_OK;
}

int tc_local_tiles(ctc_molecule* mol, const LocalPlan& plan, const TileBatch& tb,
                   const ctc_params* prm, const ctc_outputs* out, cudaStream_t st) {
  if (tb.C <= 0) return CTC_OK;
  if (tb.Kcap > kMaxKt)
    return fail(CTC_ERR_UNSUPPORTED, "tensor-core split path: more than 16384 functions per tile");
  int rc = prepare_tc(mol, st);
  if (rc != CTC_OK) return rc;
  // int8 planes of the tile rows + row exponents
  const size_t plane_bytes = (size_t)tb.C * kPlanes * kRows * tb.Kcap;
  const size_t need = plane_bytes + 256 + sizeof(int32_t) * (size_t)tb.C * kRows;
  if ((rc = mol->ws_sl.ensure(need, st)) != CTC_OK) return rc;
  int8_t* planes = (int8_t*)mol->ws_sl.p;
  int32_t* eexp = (int32_t*)((char*)mol->ws_sl.p + (plane_bytes + 255) / 256 * 256);
  slice_a_kernel<<<tb.C, 256, 0, st>>>(tb, plan.nqa, planes, eexp);
  CTC_CUDA_TRY(cudaGetLastError());
  // tensor map over the planes: 2-D, rows = C*4*128, inner = Kcap bytes
  PFN_cuTensorMapEncodeTiled_v12000 enc = get_encode();
  if (!enc) return fail(CTC_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled unavailable");
  CUtensorMap amap;
  cuuint64_t gdim[2] = {(cuuint64_t)tb.Kcap, (cuuint64_t)tb.C * kPlanes * kRows};
  cuuint64_t gstride[1] = {(cuuint64_t)tb.Kcap};
  cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)kRows};
  cuuint32_t estr[2] = {1, 1};
  CUresult cr = enc(&amap, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, planes, gdim, gstride, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (cr != CUDA_SUCCESS) return fail(CTC_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)cr));
  TcArgs a;
  a.tb = tb;
  a.nqa = plan.nqa;
  a.Dp = (const uint32_t*)mol->d_Dsl;
  a.fexp = (const int32_t*)mol->d_Dscale;
  a.eexp = eexp;
  a.Mpad = mol->Mpad;
  a.out = *out;
  a.prm = *prm;
  a.status = mol->d_status;
  static bool attr[2] = {false, false};
  ProfScope ps(mol, 0, st);
  if (plan.nqa == 4) {
    if (!attr[1]) {
      CTC_CUDA_TRY(cudaFuncSetAttribute(tc_tile_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemTc));
      attr[1] = true;
    }
    tc_tile_kernel<4><<<tb.C, kThreadsTc, kSmemTc, st>>>(amap, a);
  } else {
    if (!attr[0]) {
      CTC_CUDA_TRY(cudaFuncSetAttribute(tc_tile_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemTc));
      attr[0] = true;
    }
    tc_tile_kernel<1><<<tb.C, kThreadsTc, kSmemTc, st>>>(amap, a);
  }
  CTC_CUDA_TRY(cudaGetLastError());
  return CTC_OK;
}

}  // namespace ctc
