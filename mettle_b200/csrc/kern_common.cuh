// kern_common.cuh — device helpers shared by the sm_100a kernels: typed
// column loads, predicate compares, the expression VM, order-preserving
// key images, and the decoupled look-back primitives used for
// order-preserving stream compaction.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "dev_types.h"

namespace mtl {

// Bounded spin: every wait in this library gives up after this many polls
// and reports ST_SPIN_LIMIT instead of hanging the GPU.
constexpr uint32_t kSpinLimit = 1u << 22;

struct Val {
  int64_t lo;
  int64_t hi;
};

__device__ __forceinline__ double as_f64(int64_t b) { return __longlong_as_double(b); }
__device__ __forceinline__ int64_t f64_bits(double d) { return __double_as_longlong(d); }
__device__ __forceinline__ float as_f32(int64_t b) { return __int_as_float((int)(uint32_t)b); }
__device__ __forceinline__ int64_t f32_bits(float f) { return (int64_t)(uint32_t)__float_as_int(f); }

// Read-only streaming load of one column value as 64-bit bits (I32 sign
// extended; F32 kept as its 32 bits in the low word).
__device__ __forceinline__ int64_t load_bits(const void* p, int32_t ptype, uint64_t row) {
  switch (ptype) {
    case P_I32: return (int64_t)__ldg((const int*)p + row);
    case P_F32: return (int64_t)(uint32_t)__float_as_int(__ldg((const float*)p + row));
    default: return (int64_t)__ldg((const long long*)p + row);
  }
}

__device__ __forceinline__ bool cmp_i(int64_t x, int32_t op, int64_t k) {
  switch (op) {
    case C_EQ: return x == k;
    case C_LT: return x < k;
    case C_LE: return x <= k;
    case C_GT: return x > k;
    case C_GE: return x >= k;
    case C_NE: return x != k;
    case C_TRUE: return true;
    default: return false;
  }
}
template <typename F>
__device__ __forceinline__ bool cmp_f(F x, int32_t op, F k) {
  switch (op) {
    case C_EQ: return x == k;
    case C_LT: return x < k;
    case C_LE: return x <= k;
    case C_GT: return x > k;
    case C_GE: return x >= k;
    case C_NE: return x != k;
    case C_TRUE: return true;
    default: return false;
  }
}

__device__ __forceinline__ bool eval_pred_bits(int64_t bits, int32_t ptype, const DPred& p) {
  switch (ptype) {
    case P_I32:
    case P_I64: return cmp_i(bits, p.op, p.ilit);
    case P_F32: return cmp_f<float>(as_f32(bits), p.op, (float)p.flit);
    default: return cmp_f<double>(as_f64(bits), p.op, p.flit);
  }
}

// ------------------------------------------------------------ 128-bit helpers
__device__ __forceinline__ __int128 to_i128(const Val& v) {
  return (__int128)(((unsigned __int128)(uint64_t)v.hi << 64) | (unsigned __int128)(uint64_t)v.lo);
}
__device__ __forceinline__ Val from_i128(__int128 x) {
  Val v;
  v.lo = (int64_t)(uint64_t)x;
  v.hi = (int64_t)(x >> 64);
  return v;
}

// Signed 64-bit overflow-checked ops (DuckDB raises on overflow).
__device__ __forceinline__ int64_t add64(int64_t a, int64_t b, uint32_t& st) {
  int64_t r = (int64_t)((uint64_t)a + (uint64_t)b);
  if (((a ^ r) & (b ^ r)) < 0) st |= ST_OVERFLOW;
  return r;
}
__device__ __forceinline__ int64_t sub64(int64_t a, int64_t b, uint32_t& st) {
  int64_t r = (int64_t)((uint64_t)a - (uint64_t)b);
  if (((a ^ b) & (a ^ r)) < 0) st |= ST_OVERFLOW;
  return r;
}
__device__ __forceinline__ int64_t mul64(int64_t a, int64_t b, uint32_t& st) {
  int64_t lo = (int64_t)((uint64_t)a * (uint64_t)b);
  int64_t hi = __mul64hi(a, b);
  if (hi != (lo >> 63)) st |= ST_OVERFLOW;
  return lo;
}
__device__ __forceinline__ int64_t fit32(int64_t r, uint32_t& st) {
  if (r > 2147483647LL || r < -2147483648LL) st |= ST_OVERFLOW;
  return r;
}

// ------------------------------------------------------------ expression VM
// A postfix program over typed 128-bit stack slots. Each arithmetic op is
// rounded separately (no contraction), matching a row-at-a-time evaluator.
__device__ __forceinline__ Val vm_cast(Val v, int32_t from, int32_t to, int64_t mul, int64_t div,
                                       uint32_t& st) {
  Val r{0, 0};
  if (from == to && mul == 1) return v;
  switch (to) {
    case P_I32:
      r.lo = fit32(mul64(v.lo, mul, st), st);
      break;
    case P_I64:
      r.lo = (from == P_I128) ? (int64_t)(uint64_t)to_i128(v) : mul64(v.lo, mul, st);
      break;
    case P_I128: {
      __int128 x = (from == P_I128) ? to_i128(v) : (__int128)v.lo;
      r = from_i128(x * (__int128)mul);
      break;
    }
    case P_F32: {
      float f;
      if (from == P_F64) f = __double2float_rn(as_f64(v.lo));
      else if (from == P_F32) f = as_f32(v.lo);
      else if (from == P_I128) f = __double2float_rn((double)to_i128(v));
      else f = __ll2float_rn(v.lo);
      if (div > 1) f = __fdiv_rn(f, (float)div);
      r.lo = f32_bits(f);
      break;
    }
    case P_F64: {
      double d;
      if (from == P_F32) d = (double)as_f32(v.lo);
      else if (from == P_F64) d = as_f64(v.lo);
      else if (from == P_I128) d = (double)to_i128(v);
      else d = __ll2double_rn(v.lo);
      if (div > 1) d = __ddiv_rn(d, (double)div);
      r.lo = f64_bits(d);
      break;
    }
    default: break;
  }
  return r;
}

__device__ __forceinline__ Val vm_arith(int16_t op, int16_t type, Val a, Val b, uint32_t& st) {
  Val r{0, 0};
  switch (type) {
    case P_I32:
      r.lo = fit32(op == VM_ADD ? a.lo + b.lo : op == VM_SUB ? a.lo - b.lo : a.lo * b.lo, st);
      break;
    case P_I64:
      r.lo = op == VM_ADD ? add64(a.lo, b.lo, st) : op == VM_SUB ? sub64(a.lo, b.lo, st) : mul64(a.lo, b.lo, st);
      break;
    case P_I128: {
      __int128 x = to_i128(a), y = to_i128(b);
      r = from_i128(op == VM_ADD ? x + y : op == VM_SUB ? x - y : x * y);
      break;
    }
    case P_F32: {
      float x = as_f32(a.lo), y = as_f32(b.lo);
      r.lo = f32_bits(op == VM_ADD ? __fadd_rn(x, y) : op == VM_SUB ? __fsub_rn(x, y) : __fmul_rn(x, y));
      break;
    }
    default: {
      double x = as_f64(a.lo), y = as_f64(b.lo);
      r.lo = f64_bits(op == VM_ADD ? __dadd_rn(x, y) : op == VM_SUB ? __dsub_rn(x, y) : __dmul_rn(x, y));
      break;
    }
  }
  return r;
}

// Register-resident selects: rid[]/slots[] are indexed with runtime source
// numbers, which would otherwise demote the arrays to local memory.
__device__ __forceinline__ uint32_t pick(const uint32_t* r, int s) {
  uint32_t v = r[0];
#pragma unroll
  for (int i = 1; i < kMaxSrc; ++i) v = (s == i) ? r[i] : v;
  return v;
}
__device__ __forceinline__ uint32_t pick5(const uint32_t* r, int s) {
  uint32_t v = r[0];
#pragma unroll
  for (int i = 1; i < kMaxProbes; ++i) v = (s == i) ? r[i] : v;
  return v;
}

// Evaluates program `p`; `rid` holds the current tuple's row id per source,
// `slots` the slot of each probe (for VM_SLOT).
__device__ __forceinline__ Val vm_eval(const VmProg& p, const DCol* cols, const uint32_t* rid,
                                       const uint32_t* slots, uint32_t& st) {
  Val stack[6];
  int sp = 0;
  for (int i = 0; i < p.n; ++i) {
    const VmIns& in = p.ins[i];
    switch (in.op) {
      case VM_COL: {
        const DCol& c = cols[in.arg];
        Val v;
        v.lo = load_bits(c.ptr, c.ptype, pick(rid, c.src));
        v.hi = (c.ptype == P_I32 || c.ptype == P_I64) ? (v.lo >> 63) : 0;
        stack[sp++] = v;
        break;
      }
      case VM_CONST:
        stack[sp].lo = in.k;
        stack[sp].hi = in.k2;
        ++sp;
        break;
      case VM_SLOT:
        stack[sp].lo = (int64_t)pick5(slots, in.arg);
        stack[sp].hi = 0;
        ++sp;
        break;
      case VM_CAST:
        stack[sp - 1] = vm_cast(stack[sp - 1], in.arg, in.type, in.k, in.k2, st);
        break;
      case VM_NEG: {
        Val z{0, 0};
        if (in.type == P_F32) z.lo = f32_bits(-0.0f);
        if (in.type == P_F64) z.lo = f64_bits(-0.0);
        if (in.type == P_F32 || in.type == P_F64) {
          // IEEE negation flips the sign bit only.
          stack[sp - 1].lo ^= (in.type == P_F32) ? (int64_t)0x80000000LL : (int64_t)0x8000000000000000ULL;
        } else {
          stack[sp - 1] = vm_arith(VM_SUB, in.type, z, stack[sp - 1], st);
        }
        break;
      }
      default: {  // binary arithmetic
        Val b = stack[--sp];
        Val a = stack[sp - 1];
        stack[sp - 1] = vm_arith(in.op, in.type, a, b, st);
        break;
      }
    }
  }
  return stack[0];
}

// vm_eval with column values prefetched in registers: cv[j] holds the value
// of column sink_cols[j] for the current tuple (j < n_sink); columns outside
// that set are loaded on demand.
template <int NC>
__device__ __forceinline__ Val vm_eval_c(const VmProg& p, const DCol* cols, const uint32_t* rid,
                                         const int32_t* sink_cols, int n_sink, const int64_t* cv, uint32_t& st) {
  Val stack[6];
  int sp = 0;
  for (int i = 0; i < p.n; ++i) {
    const VmIns& in = p.ins[i];
    switch (in.op) {
      case VM_COL: {
        const DCol& c = cols[in.arg];
        int64_t bits = 0;
        bool found = false;
#pragma unroll
        for (int j = 0; j < NC; ++j)
          if (j < n_sink && sink_cols[j] == in.arg) {
            bits = cv[j];
            found = true;
          }
        if (!found) bits = load_bits(c.ptr, c.ptype, pick(rid, c.src));
        Val v;
        v.lo = bits;
        v.hi = (c.ptype == P_I32 || c.ptype == P_I64) ? (bits >> 63) : 0;
        stack[sp++] = v;
        break;
      }
      case VM_CONST:
        stack[sp].lo = in.k;
        stack[sp].hi = in.k2;
        ++sp;
        break;
      case VM_CAST:
        stack[sp - 1] = vm_cast(stack[sp - 1], in.arg, in.type, in.k, in.k2, st);
        break;
      case VM_NEG: {
        Val z{0, 0};
        if (in.type == P_F32 || in.type == P_F64) {
          stack[sp - 1].lo ^= (in.type == P_F32) ? (int64_t)0x80000000LL : (int64_t)0x8000000000000000ULL;
        } else {
          stack[sp - 1] = vm_arith(VM_SUB, in.type, z, stack[sp - 1], st);
        }
        break;
      }
      case VM_SLOT:
        stack[sp].lo = 0;
        stack[sp].hi = 0;
        ++sp;
        break;
      default: {
        Val b = stack[--sp];
        Val a = stack[sp - 1];
        stack[sp - 1] = vm_arith(in.op, in.type, a, b, st);
        break;
      }
    }
  }
  return stack[0];
}

// Stores a VM result into a typed output array at index i.
__device__ __forceinline__ void store_val(void* out, int32_t ptype, uint64_t i, Val v) {
  switch (ptype) {
    case P_I32: ((int32_t*)out)[i] = (int32_t)v.lo; break;
    case P_F32: ((uint32_t*)out)[i] = (uint32_t)v.lo; break;
    case P_I128: ((longlong2*)out)[i] = make_longlong2(v.lo, v.hi); break;
    default: ((int64_t*)out)[i] = v.lo; break;
  }
}

// ------------------------------------------------------------ ordered images
// Order-preserving unsigned images: a < b  <=>  img(a) < img(b).
__device__ __forceinline__ uint64_t ord_i64(int64_t x) { return (uint64_t)x ^ 0x8000000000000000ULL; }
__device__ __forceinline__ uint64_t ord_f64_bits(uint64_t b) {
  return (b & 0x8000000000000000ULL) ? ~b : (b | 0x8000000000000000ULL);
}
__device__ __forceinline__ uint64_t ord_f64(double d) { return ord_f64_bits((uint64_t)__double_as_longlong(d)); }
__device__ __forceinline__ double unord_f64(uint64_t u) {
  uint64_t b = (u & 0x8000000000000000ULL) ? (u & 0x7FFFFFFFFFFFFFFFULL) : ~u;
  return __longlong_as_double((long long)b);
}

// ------------------------------------------------------------ memory order
__device__ __forceinline__ uint64_t ld_acquire(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(uint64_t* p, uint64_t v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_acquire32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release32(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ------------------------------------------------------------ look-back
// Tile status word: [63:48] epoch, [47:46] flag (1 aggregate, 2 prefix),
// [45:0] value. A word from another epoch reads as "not yet published", so
// the status array needs no clearing between launches.
constexpr uint64_t kLbAgg = 1ULL, kLbPre = 2ULL;
__device__ __forceinline__ uint64_t lb_word(uint32_t epoch, uint64_t flag, uint64_t v) {
  return ((uint64_t)(epoch & 0xFFFFu) << 48) | (flag << 46) | (v & ((1ULL << 46) - 1));
}

// Called by one thread: publishes tile t's count c and returns the exclusive
// prefix of all tiles before t (decoupled look-back).
__device__ __forceinline__ uint64_t lb_exclusive(uint64_t* status, uint64_t t, uint64_t c, uint32_t epoch,
                                                 uint32_t* st_flags) {
  if (t == 0) {
    st_release(status, lb_word(epoch, kLbPre, c));
    return 0;
  }
  st_release(status + t, lb_word(epoch, kLbAgg, c));
  uint64_t excl = 0;
  int64_t j = (int64_t)t - 1;
  uint32_t spins = 0;
  while (j >= 0) {
    uint64_t w = ld_acquire(status + j);
    uint32_t ep = (uint32_t)(w >> 48);
    uint64_t flag = (w >> 46) & 3ULL;
    if (ep != (epoch & 0xFFFFu) || flag == 0) {
      if (++spins > kSpinLimit) {
        atomicOr(st_flags, ST_SPIN_LIMIT);
        break;
      }
      continue;
    }
    excl += w & ((1ULL << 46) - 1);
    if (flag == kLbPre) break;
    --j;
  }
  st_release(status + t, lb_word(epoch, kLbPre, excl + c));
  return excl;
}

// Warp-parallel look-back, called by all 32 lanes of one warp: lane i
// inspects predecessor t-1-i, so one round trip covers 32 tiles. Sums the
// aggregates back to the nearest published prefix, publishes this tile's
// inclusive prefix and returns its exclusive prefix (in every lane).
// spin_limit bounds the polls of unpublished predecessors; publish_first =
// false (failure injection only) keeps tile 0 from publishing, so that the
// waits behind it run out.
__device__ __forceinline__ uint64_t lb_exclusive_warp(uint64_t* status, uint64_t t, uint64_t c, uint32_t epoch,
                                                      uint32_t* st_flags, uint32_t spin_limit = kSpinLimit,
                                                      bool publish_first = true) {
  const int lane = threadIdx.x & 31;
  const uint64_t ep = (uint64_t)(epoch & 0xFFFFu);
  const uint64_t vmask = (1ULL << 46) - 1;
  if (t == 0) {
    if (lane == 0 && publish_first) st_release(status, lb_word(epoch, kLbPre, c));
    return 0;
  }
  if (lane == 0) st_release(status + t, lb_word(epoch, kLbAgg, c));
  uint64_t excl = 0;
  int64_t j = (int64_t)t - 1;
  uint32_t spins = 0;
  for (;;) {
    const int64_t idx = j - lane;
    uint64_t flag, val;
    if (idx < 0) {
      flag = kLbPre;  // before the first tile: a prefix of zero
      val = 0;
    } else {
      const uint64_t w = ld_acquire(status + idx);
      flag = ((w >> 48) == ep) ? ((w >> 46) & 3ULL) : 0ULL;
      val = w & vmask;
    }
    const uint32_t pre = __ballot_sync(0xFFFFFFFFu, flag == kLbPre);
    const uint32_t none = __ballot_sync(0xFFFFFFFFu, flag == 0);
    const int limit = pre ? __ffs(pre) - 1 : 31;  // lanes 0..limit are summed
    const uint32_t upto = limit == 31 ? 0xFFFFFFFFu : ((1u << (limit + 1)) - 1u);
    if (none & upto) {
      if (++spins > spin_limit) {
        if (lane == 0) atomicOr(st_flags, ST_SPIN_LIMIT);
        break;
      }
      continue;  // a nearer predecessor has not published yet
    }
    uint64_t v = lane <= limit ? val : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    excl += v;
    if (pre) break;
    j -= 32;
  }
  if (lane == 0) st_release(status + t, lb_word(epoch, kLbPre, excl + c));
  return excl;
}

// ------------------------------------------------------------ block scan
// Exclusive block-wide sum of one u32 per thread; returns the thread's
// exclusive prefix, *total gets the block total. Needs THREADS/32 words of
// shared scratch.
template <int THREADS>
__device__ __forceinline__ uint32_t block_excl_sum(uint32_t x, uint32_t* s_warp, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) s_warp[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < THREADS / 32 ? s_warp[lane] : 0;
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < THREADS / 32) s_warp[lane] = wi - w;
    if (lane == THREADS / 32 - 1) s_warp[THREADS / 32] = wi;
  }
  __syncthreads();
  uint32_t r = s_warp[warp] + inc - x;
  *total = s_warp[THREADS / 32];
  __syncthreads();
  return r;
}

// ------------------------------------------------------------ bulk copies (TMA)
// 1-D bulk global->shared copies completed on an mbarrier (no tensor map,
// no multicast). Sizes and both addresses are multiples of 16 bytes.
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait on an mbarrier phase; false when the limit is reached.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  for (uint32_t i = 0; i < (1u << 20); ++i)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// Multiplicative hash of a 64-bit word.
__device__ __forceinline__ uint64_t hash64(uint64_t x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdULL;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ULL;
  x ^= x >> 33;
  return x;
}
// Maps a hash onto [0, cap) without a power-of-two capacity.
__device__ __forceinline__ uint64_t hash_slot(uint64_t h, uint64_t cap) { return __umul64hi(h, cap); }

// Blocked Bloom filter of a hash-join build (one 32-bit word per key, two
// bits in it), from the key's 64-bit hash h: the word from the low bits (the
// table slot uses the high ones), the bits from the middle.
__device__ __forceinline__ uint32_t bloom_word(uint64_t h, uint64_t words) { return (uint32_t)(h & (words - 1)); }
__device__ __forceinline__ uint32_t bloom_mask(uint64_t h) {
  return (1u << ((h >> 32) & 31)) | (1u << ((h >> 37) & 31));
}
// false: the key is certainly not in the build (true also when there is no filter)
__device__ __forceinline__ bool bloom_maybe(const DBuild& b, uint64_t h) {
  if (!b.bloom) return true;
  const uint32_t m = bloom_mask(h);
  return (__ldg(b.bloom + bloom_word(h, b.bloom_words)) & m) == m;
}

}  // namespace mtl
