// final_common.cuh — value of one final aggregate output for one group, and
// the order-preserving key image of ORDER BY parts. Shared by the finalize
// kernel, the key encoder and the fused aggregate top-K.
#pragma once
#include "kern_common.cuh"
#include "kernels.h"

namespace mtl {

// AVG of a 128-bit integer sum as DuckDB computes it on x86-64
// (IntegerAverageOperationHugeint): the quotient is formed in x87 extended
// precision (64-bit significand, round to nearest even) and then stored as
// a double (a second rounding to 53 bits). Emulated exactly with integer
// arithmetic; the sum is assumed below 2^64 in magnitude (the long double
// image of larger sums is rounded, and this emulation rounds it the same
// way only when the discarded bits are not a tie).
static __device__ __noinline__ double avg_extended(__int128 sum, unsigned long long count) {
  if (sum == 0 || count == 0) return 0.0;
  const bool neg = sum < 0;
  unsigned __int128 S = neg ? (unsigned __int128)(-sum) : (unsigned __int128)sum;
  const unsigned __int128 C = count;
  int lenS = 0;
  {
    uint64_t hi = (uint64_t)(S >> 64), lo = (uint64_t)S;
    lenS = hi ? 128 - __clzll((long long)hi) : 64 - __clzll((long long)lo);
  }
  // Round S itself to a 64-bit significand if it is wider.
  int sexp = 0;
  if (lenS > 64) {
    int drop = lenS - 64;
    unsigned __int128 q = S >> drop, rem = S & ((((unsigned __int128)1) << drop) - 1);
    unsigned __int128 half = ((unsigned __int128)1) << (drop - 1);
    if (rem > half || (rem == half && (q & 1))) q += 1;
    if (q >> 64) { q >>= 1; drop += 1; }
    S = q;
    sexp = drop;
    lenS = 64;
  }
  const int lenC = 64 - __clzll((long long)count);
  // Quotient with a 64-bit significand: Q = floor(S * 2^k / C).
  int k = 64 - (lenS - lenC);
  unsigned __int128 Q, R, D;
  for (int attempt = 0; attempt < 3; ++attempt) {
    if (k >= 0) {
      unsigned __int128 N = S << k;
      D = C;
      Q = N / D;
      R = N % D;
    } else {
      D = C << (-k);
      Q = S / D;
      R = S % D;
    }
    if (Q >> 64) { --k; continue; }
    if (!(Q >> 63)) { ++k; continue; }
    break;
  }
  // Round to 64 bits (nearest even) on the exact remainder.
  unsigned __int128 twoR = R << 1;
  if (twoR > D || (twoR == D && (Q & 1))) Q += 1;
  if (Q >> 64) { Q >>= 1; --k; }
  // Second rounding, 64 -> 53 bits, on the 11 dropped bits alone.
  uint64_t q64 = (uint64_t)Q;
  uint64_t low = q64 & 0x7FFULL, m = q64 >> 11;
  if (low > 0x400ULL || (low == 0x400ULL && (m & 1))) m += 1;
  int e = 11 - k + sexp;
  if (m >> 53) { m >>= 1; e += 1; }
  double r = ldexp((double)m, e);
  return neg ? -r : r;
}

// Bits of output `f` for group g as they are stored (i128: lo/hi; 4-byte
// types in the low 32 bits of lo).
__device__ __forceinline__ void final_value(const FinalOut& f, uint64_t g, uint64_t& lo, uint64_t& hi) {
  hi = 0;
  if (f.kind != F_GATHER_COL && f.stride > 1) g *= (uint64_t)f.stride;
  switch (f.kind) {
    case F_COPY_I32:
    case F_COPY_F32: lo = (uint32_t)f.a[g]; break;
    case F_COPY_I64:
    case F_COPY_F64: lo = f.a[g]; break;
    case F_SUM_I128: lo = f.a[g]; hi = (uint64_t)f.a_hi[g]; break;
    case F_SUM_I64_AS_I128: lo = f.a[g]; hi = ((long long)lo < 0) ? ~0ULL : 0ULL; break;
    case F_MINMAX_F32: lo = __float_as_uint((float)unord_f64(f.a[g])); break;
    case F_MINMAX_F64: lo = (uint64_t)__double_as_longlong(unord_f64(f.a[g])); break;
    case F_AVG_I128_LD:
    case F_AVG_DEC: {
      __int128 s = f.a_hi ? (__int128)(((unsigned __int128)(uint64_t)f.a_hi[g] << 64) | f.a[g])
                          : (__int128)(long long)f.a[g];
      const unsigned long long c = f.kind == F_AVG_DEC ? f.cnt[g] * (unsigned long long)f.scale : f.cnt[g];
      lo = (uint64_t)__double_as_longlong(avg_extended(s, c));
      break;
    }
    case F_AVG_I64_D:
      lo = (uint64_t)__double_as_longlong(__ddiv_rn(__ll2double_rn((long long)f.a[g]), __ull2double_rn(f.cnt[g])));
      break;
    case F_AVG_F64:
      lo = (uint64_t)__double_as_longlong(
          __ddiv_rn(__longlong_as_double((long long)f.a[g]), __ull2double_rn(f.cnt[g])));
      break;
    case F_GATHER_COL: {
      const uint32_t r = f.rid ? f.rid[g] : (uint32_t)g;  // null: g is the row itself
      lo = f.width == 4 ? (uint64_t)((const uint32_t*)f.col)[r] : ((const uint64_t*)f.col)[r];
      break;
    }
    default: lo = 0; break;
  }
}

// ------------------------------------------------------------ key images
struct U256 {
  uint64_t w[4];  // w[0] most significant
};

__device__ __forceinline__ void shl_or(U256& k, int bits, uint64_t lo, uint64_t hi) {
  // k = (k << bits) | value, value given as (hi, lo) with `bits` significant bits.
  while (bits > 0) {
    int b = bits > 64 ? 64 : bits;
    uint64_t part = bits > 64 ? hi : lo;
    if (bits > 64) bits -= 64; else bits = 0;
    if (b == 64) {
      k.w[0] = k.w[1]; k.w[1] = k.w[2]; k.w[2] = k.w[3]; k.w[3] = part;
    } else {
      k.w[0] = (k.w[0] << b) | (k.w[1] >> (64 - b));
      k.w[1] = (k.w[1] << b) | (k.w[2] >> (64 - b));
      k.w[2] = (k.w[2] << b) | (k.w[3] >> (64 - b));
      k.w[3] = (k.w[3] << b) | (part & ((1ULL << b) - 1));
    }
  }
}

// Appends the order-preserving image of one ORDER BY part (value bits as
// stored for physical type pt) to the key; DESC parts are complemented.
__device__ __forceinline__ void key_part(U256& k, int32_t pt, bool desc, uint64_t lo, uint64_t hi) {
  int bits = 64;
  switch (pt) {
    case P_I32: lo = (uint64_t)((uint32_t)lo ^ 0x80000000u); hi = 0; bits = 32; break;
    case P_F32: {
      const uint32_t b = (uint32_t)lo;
      lo = (b & 0x80000000u) ? (uint64_t)(~b & 0xFFFFFFFFu) : (uint64_t)(b | 0x80000000u);
      hi = 0;
      bits = 32;
      break;
    }
    case P_I64: lo = ord_i64((int64_t)lo); hi = 0; break;
    case P_F64: lo = ord_f64_bits(lo); hi = 0; break;
    case P_I128: hi ^= 0x8000000000000000ULL; bits = 128; break;
    default: lo = hi = 0; break;
  }
  if (desc) {
    lo = ~lo;
    hi = ~hi;
    if (bits == 32) lo &= 0xFFFFFFFFULL;
  }
  shl_or(k, bits, lo, hi);
}

// Writes output f of group g into result row i (the stores of k_finalize).
__device__ __forceinline__ void finalize_row(const FinalOut& f, uint64_t g, uint64_t i) {
  uint64_t lo, hi;
  final_value(f, g, lo, hi);
  switch (f.kind) {
    case F_SUM_I128:
    case F_SUM_I64_AS_I128: ((longlong2*)f.out)[i] = make_longlong2((long long)lo, (long long)hi); break;
    case F_COPY_I32:
    case F_COPY_F32:
    case F_MINMAX_F32: ((uint32_t*)f.out)[i] = (uint32_t)lo; break;
    case F_GATHER_COL:
      if (f.width == 4) ((uint32_t*)f.out)[i] = (uint32_t)lo;
      else ((uint64_t*)f.out)[i] = lo;
      break;
    default: ((uint64_t*)f.out)[i] = lo; break;
  }
}

}  // namespace mtl
