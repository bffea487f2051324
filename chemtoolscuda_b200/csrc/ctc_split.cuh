// ctc_split.cuh -- the INT8 digit split shared by the operand producers
// (D in ctc_tc.cu, the tile rows in the AO kernel of ctc_ao.cu).
//
// A row of values x_k is scaled by 2^-e, e the exponent of its largest |x|
// (|x| < 2^e), and rounded to a fixed-point integer written in balanced
// base-256 digits (|d| <= 128), one int8 plane per digit, most significant
// first:
//   * D rows (B operand): I = rint(x 2^(38-e)), |I| <= 2^38, five digits;
//   * tile rows of phi and grad phi (A operand): I = rint(x 2^(38-e)),
//     |I| <= 2^38, five digits.
// 31 bits (four digits) are not enough on either side.  An AO row's error is
// set by its largest entry: a row with one steep function (a tight g shell
// near its centre) and many small ones loses relative precision on the
// small ones (2e-8 of the sum of absolute terms with 31 bits).  A D row
// whose largest entry is a core element loses the small valence entries of
// the same row: near nuclei the Hessian and gradient reached 1.8e-8 (Kr and
// C atoms of the reference's fixtures) and 2.8e-8 (the 200-atom benchmark
// molecule, 0.004 bohr from a nucleus) with 31-bit D rows, 1e-9 and 2.5e-9
// with 39 bits (CPU emulation of this split).
#pragma once

#include <cstdint>

namespace ctc {

constexpr int kSplitPlanesD = 5;  // digit planes of D (B operand)
constexpr int kSplitPlanesA = 5;  // digit planes of the tile rows (A operand)
constexpr int kSplitRows = 128;   // rows of one block of a tile operand (MMA M)

// A tile of TP points with nqa row quantities (nqa = 4: phi and grad phi;
// nqa = 1: phi) has nqa * TP operand rows, stored in blocks of 128 rows:
// digit planes [tile][block][5][128][Kcap], row exponents [tile][rows].
// With nqa = 4 point p's quantity q is row (p / 32) * 128 + q * 32 + p % 32,
// so every block holds 32 points x 4 quantities; with nqa = 1 row = point.
__host__ __device__ constexpr int split_tile_rows(int TP, int nqa) { return TP * nqa; }
constexpr int kFixedBitsD = 38;   // |I| <= 2^38
constexpr int kFixedBitsA = 38;   // |I| <= 2^38

// Lowest row exponent used: rows whose largest |x| is below 2^-980 are
// scaled as if it were 2^-980 (their digits are then zero), so that the row
// factors 2^(bits - e) stay normal doubles.
constexpr int kMinScaleExponent = -980;

// balanced base-256 digits of |I| <= 2^30, packed in a word: byte p holds the
// digit of weight 256^(3-p) (byte 0 = the most significant digit).  Adding
// 128 (256^2 + 256 + 1) turns the three low balanced digits d into unsigned
// bytes d + 128 and leaves the top digit in the high byte; flipping bit 7 of
// the low bytes gives d as int8, and a byte reversal puts the most
// significant digit first.
__device__ __forceinline__ uint32_t pack_digits(int32_t I) {
  const uint32_t u = (uint32_t)(I + 0x808080) ^ 0x808080u;
  return __byte_perm(u, 0u, 0x0123);
}

// The five balanced digits of |I| <= 2^38 in one 64-bit word: bytes 0-3 the
// four most significant (pack_digits of the upper part), byte 4 the lowest
// digit d4 (balanced, as int8); bytes 5-7 zero.
__device__ __forceinline__ uint64_t pack_digits5(long long I) {
  const int32_t d4 = (int32_t)(((I + 128) & 255) - 128);
  return (uint64_t)pack_digits((int32_t)((I - d4) >> 8)) | ((uint64_t)(uint32_t)(d4 & 255) << 32);
}

// rint(y) for |y| < 2^31 (round half to even) with one FP64 add: the sum
// y + 1.5 * 2^52 has unit spacing, so its low word is rint(y) mod 2^32.
__device__ __forceinline__ int32_t rint_i32(double y) {
  return __double2loint(y + 6755399441055744.0);
}

// rint(y) for |y| < 2^51 as int64 (round half to even): the low 52 bits of
// y + 1.5 * 2^52 hold 2^51 + rint(y).
__device__ __forceinline__ long long rint_i64(double y) {
  return __double_as_longlong(y + 6755399441055744.0) - 0x4338000000000000LL;
}

// 2^(bits - e): the factor that maps a row with |x| < 2^e onto |I| <= 2^bits
__device__ __forceinline__ double split_row_factor(int e, int bits) {
  return __longlong_as_double((long long)(bits - e + 1023) << 52);
}

__device__ __forceinline__ int scale_exponent(double amax) {
  if (!(amax > 0.0)) return 0;
  int e;
  frexp(amax, &e);  // amax = m 2^e, m in [0.5, 1)
  return e < kMinScaleExponent ? kMinScaleExponent : e;
}

// 4 x 4 byte transpose: out[p] byte j = byte p of input j
__device__ __forceinline__ void transpose_bytes4x4(uint32_t a, uint32_t b, uint32_t c, uint32_t d,
                                                   uint32_t* out) {
  const uint32_t t0 = __byte_perm(a, b, 0x5140);  // a0 b0 a1 b1
  const uint32_t t1 = __byte_perm(c, d, 0x5140);  // c0 d0 c1 d1
  const uint32_t t2 = __byte_perm(a, b, 0x7362);  // a2 b2 a3 b3
  const uint32_t t3 = __byte_perm(c, d, 0x7362);  // c2 d2 c3 d3
  out[0] = __byte_perm(t0, t1, 0x5410);           // a0 b0 c0 d0
  out[1] = __byte_perm(t0, t1, 0x7632);           // a1 b1 c1 d1
  out[2] = __byte_perm(t2, t3, 0x5410);           // a2 b2 c2 d2
  out[3] = __byte_perm(t2, t3, 0x7632);           // a3 b3 c3 d3
}

// Writes 32 consecutive K entries of one tile row into the five A planes
// [plane][row][Kcap] (32 bytes per plane): x(i) returns the row's value at
// K index k0 + i, f = split_row_factor(e, kFixedBitsA) of the row.  The four
// most significant digits go through pack_digits, the fifth is the balanced
// low byte.
template <class F>
__device__ __forceinline__ void write_row_digits32(F x, double f, int8_t* __restrict__ P, int row,
                                                   int64_t Kcap, int k0) {
  uint32_t pw[kSplitPlanesA][8];
#pragma unroll
  for (int g = 0; g < 8; ++g) {
    uint32_t w[4], lo = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const long long I = rint_i64(x(4 * g + i) * f);
      const int32_t d4 = (int32_t)(((I + 128) & 255) - 128);
      w[i] = pack_digits((int32_t)((I - d4) >> 8));
      lo |= (uint32_t)(d4 & 255) << (8 * i);
    }
    uint32_t pl[4];
    transpose_bytes4x4(w[0], w[1], w[2], w[3], pl);
#pragma unroll
    for (int p = 0; p < 4; ++p) pw[p][g] = pl[p];
    pw[4][g] = lo;
  }
#pragma unroll
  for (int p = 0; p < kSplitPlanesA; ++p) {
    uint4* dst = reinterpret_cast<uint4*>(P + ((int64_t)p * kSplitRows + row) * Kcap + k0);
    dst[0] = make_uint4(pw[p][0], pw[p][1], pw[p][2], pw[p][3]);
    dst[1] = make_uint4(pw[p][4], pw[p][5], pw[p][6], pw[p][7]);
  }
}

}  // namespace ctc
