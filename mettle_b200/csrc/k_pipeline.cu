// k_pipeline.cu — the fused scan pipeline (sm_100a).
//
// One launch scans one input and runs, per tuple: every filter predicate and
// join probe in planned order (short-circuit), then the pipeline's sink. It
// replaces the reference's chain of one-dispatch-per-op kernels
// (compare_*_scalar, and_masks, filter_to_indices, gather_*, hash_join_*,
// dense_lookup_*, compact_matches, reindex, grouped_aggregate_*,
// src/metal/shaders/kernels.metal:70-1160) with a single pass over HBM:
//   * the first predicate column is streamed with 128-bit vector loads for
//     every tuple; other columns are loaded only for tuples still alive;
//   * compaction is order preserving: a block scan plus a decoupled
//     look-back across tiles gives every tile its output offset in one pass
//     (the reference's filter_to_indices uses one global atomic per row and
//     produces an unordered result);
//   * joins probe unique-key builds (dense direct-mapped or open addressing),
//     so a probe yields at most one match and the pipeline never expands;
//   * aggregates update per-group states with native 64-bit atomics, from
//     shared-memory tables when the group count is small.
#include <cooperative_groups.h>

#include <map>
#include <mutex>

#include "kern_common.cuh"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace mtl {

// ------------------------------------------------------------ join build/probe
__device__ __forceinline__ bool build_lookup(const DBuild& b, int64_t key, uint32_t& slot, uint32_t& st) {
  if (b.kind == B_DENSE) {
    uint64_t k = (uint64_t)(key - b.key_min);
    if (k >= b.capacity) return false;
    if (!((b.dense_bits[k >> 5] >> (k & 31)) & 1u)) return false;
    slot = b.dense_map[k] - 1;
    return true;
  }
  if (key == kEmptyKey) {
    uint32_t v = *b.hash_special;
    if (v == 0) return false;
    slot = v - 1;
    return true;
  }
  uint64_t h = hash_slot(hash64((uint64_t)key), b.capacity);
  for (uint64_t i = 0; i < b.capacity; ++i) {
    int64_t k = b.hash_keys[h];
    if (k == key) {
      slot = b.hash_slot[h] - 1;
      return true;
    }
    if (k == kEmptyKey) return false;
    if (++h == b.capacity) h = 0;
  }
  st |= ST_TABLE_FULL;
  return false;
}

__device__ __forceinline__ void build_insert(const DBuild& b, int64_t key, uint32_t slot, uint32_t& st) {
  if (b.kind == B_DENSE) {
    uint64_t k = (uint64_t)(key - b.key_min);
    if (k >= b.capacity) {
      st |= ST_CAPACITY;
      return;
    }
    // The map entry is written before its presence bit; probes run in a later
    // launch, so the plain store is visible to them.
    b.dense_map[k] = slot + 1;
    const uint32_t bit = 1u << (k & 31);
    if (b.unique_keys) atomicOr(b.dense_bits + (k >> 5), bit);  // no reply needed
    else if (atomicOr(b.dense_bits + (k >> 5), bit) & bit) st |= ST_DUP_BUILD_KEY;
    return;
  }
  if (b.bloom) {
    const uint64_t hh = hash64((uint64_t)key);
    atomicOr(b.bloom + bloom_word(hh, b.bloom_words), bloom_mask(hh));  // no reply needed
  }
  if (key == kEmptyKey) {
    if (atomicCAS(b.hash_special, 0u, slot + 1) != 0u) st |= ST_DUP_BUILD_KEY;
    return;
  }
  uint64_t h = hash_slot(hash64((uint64_t)key), b.capacity);
  for (uint64_t i = 0; i < b.capacity; ++i) {
    unsigned long long prev = atomicCAS((unsigned long long*)(b.hash_keys + h),
                                        (unsigned long long)kEmptyKey, (unsigned long long)key);
    if (prev == (unsigned long long)kEmptyKey) {
      b.hash_slot[h] = slot + 1;
      return;
    }
    if ((int64_t)prev == key) {
      st |= ST_DUP_BUILD_KEY;
      return;
    }
    if (++h == b.capacity) h = 0;
  }
  st |= ST_TABLE_FULL;
}

// ------------------------------------------------------------ aggregate states
__device__ __forceinline__ void agg_init_global(const DAgg& a, uint64_t g) {
  switch (a.fn) {
    case A_MIN_I: a.lo[g] = (uint64_t)0x7FFFFFFFFFFFFFFFULL; break;
    case A_MAX_I: a.lo[g] = (uint64_t)0x8000000000000000ULL; break;
    case A_MIN_F: a.lo[g] = ~0ULL; break;
    case A_MAX_F: a.lo[g] = 0ULL; break;
    case A_SUM_I128: a.lo[g] = 0; a.hi[g] = 0; break;
    default: a.lo[g] = 0; break;
  }
}

// Value as the aggregate's input domain.
__device__ __forceinline__ double val_as_f64(Val v, int32_t ptype) {
  return ptype == P_F32 ? (double)as_f32(v.lo) : ptype == P_F64 ? as_f64(v.lo) : (double)v.lo;
}

// Applies one input value to a state word pair (global or shared memory).
__device__ __forceinline__ void agg_apply(int32_t fn, unsigned long long* lo, long long* hi, Val v,
                                          int32_t vtype) {
  switch (fn) {
    case A_COUNT: atomicAdd(lo, 1ULL); break;
    case A_SUM_I: atomicAdd(lo, (unsigned long long)v.lo); break;
    case A_SUM_I128: {
      unsigned long long add = (unsigned long long)v.lo;
      unsigned long long old = atomicAdd(lo, add);
      long long carry = (old + add) < old ? 1 : 0;
      long long hadd = (vtype == P_I128 ? v.hi : (v.lo >> 63)) + carry;
      if (hadd != 0) atomicAdd((unsigned long long*)hi, (unsigned long long)hadd);
      break;
    }
    case A_SUM_F: atomicAdd((double*)lo, val_as_f64(v, vtype)); break;
    case A_MIN_I:
      if ((long long)v.lo < *(volatile long long*)lo) atomicMin((long long*)lo, (long long)v.lo);
      break;
    case A_MAX_I:
      if ((long long)v.lo > *(volatile long long*)lo) atomicMax((long long*)lo, (long long)v.lo);
      break;
    case A_MIN_F: {
      unsigned long long u = ord_f64(val_as_f64(v, vtype));
      if (u < *(volatile unsigned long long*)lo) atomicMin(lo, u);
      break;
    }
    case A_MAX_F: {
      unsigned long long u = ord_f64(val_as_f64(v, vtype));
      if (u > *(volatile unsigned long long*)lo) atomicMax(lo, u);
      break;
    }
    default: break;
  }
}

// agg_apply for states in global memory: the MIN/MAX pre-checks read L2
// directly (a stale value only costs an extra atomic), so the reads of
// several rows can be in flight together.
__device__ __forceinline__ void agg_apply_g(int32_t fn, unsigned long long* lo, long long* hi, Val v,
                                            int32_t vtype) {
  switch (fn) {
    case A_MIN_I:
      if ((long long)v.lo < __ldcg((const long long*)lo)) atomicMin((long long*)lo, (long long)v.lo);
      break;
    case A_MAX_I:
      if ((long long)v.lo > __ldcg((const long long*)lo)) atomicMax((long long*)lo, (long long)v.lo);
      break;
    case A_MIN_F: {
      unsigned long long u = ord_f64(val_as_f64(v, vtype));
      if (u < __ldcg(lo)) atomicMin(lo, u);
      break;
    }
    case A_MAX_F: {
      unsigned long long u = ord_f64(val_as_f64(v, vtype));
      if (u > __ldcg(lo)) atomicMax(lo, u);
      break;
    }
    default: agg_apply(fn, lo, hi, v, vtype); break;
  }
}

// Merges a partial state (lo, hi) into a state word pair.
__device__ __forceinline__ void agg_merge(int32_t fn, unsigned long long* lo, long long* hi, uint64_t plo,
                                          int64_t phi) {
  switch (fn) {
    case A_COUNT:
    case A_SUM_I: atomicAdd(lo, (unsigned long long)plo); break;
    case A_SUM_I128: {
      unsigned long long old = atomicAdd(lo, (unsigned long long)plo);
      long long carry = (old + plo) < old ? 1 : 0;
      long long hadd = phi + carry;
      if (hadd != 0) atomicAdd((unsigned long long*)hi, (unsigned long long)hadd);
      break;
    }
    case A_SUM_F: atomicAdd((double*)lo, __longlong_as_double((long long)plo)); break;
    case A_MIN_I: atomicMin((long long*)lo, (long long)plo); break;
    case A_MAX_I: atomicMax((long long*)lo, (long long)plo); break;
    case A_MIN_F: atomicMin(lo, (unsigned long long)plo); break;
    case A_MAX_F: atomicMax(lo, (unsigned long long)plo); break;
    default: break;
  }
}

__device__ __forceinline__ uint64_t key_hash(const uint64_t* kw, int nk) {
  uint64_t h = 0x9E3779B97F4A7C15ULL;
  for (int i = 0; i < nk; ++i) h = hash64(h ^ kw[i]) + (uint64_t)i;
  return h;
}

constexpr uint64_t kNoGroup = ~0ULL;

__device__ __forceinline__ uint64_t key_hash1(uint64_t k) { return hash64(0x9E3779B97F4A7C15ULL ^ k); }

// Group of a single 64-bit key in a CAS-claimed table (DAggTable::cas),
// starting at slot idx. kNoGroup when the table is full.
__device__ __noinline__ uint64_t agg_find_cas(const DAggTable& t, uint64_t key, uint64_t idx, uint32_t& st) {
  if ((int64_t)key == kEmptyKey) {
    if (t.state[t.capacity] != 2u) t.state[t.capacity] = 2u;
    return t.capacity;
  }
  const uint64_t stride = t.stride > 1 ? (uint64_t)t.stride : 1;
  for (uint64_t probe = 0; probe < t.capacity; ++probe) {
    uint64_t* const kp = t.keys[0] + idx * stride;
    const uint64_t k = __ldcg(kp);
    if (k == key) return idx;
    if ((int64_t)k == kEmptyKey) {
      const unsigned long long prev =
          atomicCAS((unsigned long long*)kp, (unsigned long long)kEmptyKey, (unsigned long long)key);
      if (prev == (unsigned long long)kEmptyKey) {
        t.state[idx] = 2u;  // read only after the pipeline (compaction, top-K)
        return idx;
      }
      if (prev == key) return idx;
    }
    if (++idx == t.capacity) idx = 0;
  }
  st |= ST_TABLE_FULL;
  return kNoGroup;
}

// Finds or claims the group of key words kw in a global table. Returns
// kNoGroup on failure (table full or wait limit), with status set.
__device__ uint64_t agg_find_global(const PipeDesc& d, const uint64_t* kw, uint32_t& st) {
  const DAggTable& t = d.table;
  if (t.cas) return agg_find_cas(t, kw[0], hash_slot(key_hash1(kw[0]), t.capacity), st);
  uint64_t idx = hash_slot(key_hash(kw, t.n_keys), t.capacity);
  for (uint64_t probe = 0; probe < t.capacity; ++probe) {
    uint32_t s = ld_acquire32(t.state + idx);
    if (s == 0) {
      if (atomicCAS(t.state + idx, 0u, 1u) == 0u) {
        for (int i = 0; i < t.n_keys; ++i) t.keys[i][idx] = kw[i];
        for (int a = 0; a < d.n_aggs; ++a) agg_init_global(d.aggs[a], idx);
        __threadfence();
        st_release32(t.state + idx, 2u);
        return idx;
      }
      s = 1;
    }
    uint32_t spins = 0;
    while (s == 1) {
      if (++spins > kSpinLimit) {
        st |= ST_SPIN_LIMIT;
        return kNoGroup;
      }
      s = ld_acquire32(t.state + idx);
    }
    bool eq = true;
    for (int i = 0; i < t.n_keys; ++i) eq &= (t.keys[i][idx] == kw[i]);
    if (eq) return idx;
    if (++idx == t.capacity) idx = 0;
  }
  st |= ST_TABLE_FULL;
  return kNoGroup;
}

// Shared-memory group table of one CTA (AGG_SMEM). Layout, cap slots:
// state u32[cap] | keys u64[nk][cap] | lo u64[na][cap] | hi i64[n128][cap].
struct SmemAgg {
  uint32_t* state;
  uint64_t* keys;
  uint64_t* lo;
  int64_t* hi;
  int32_t cap;
  int32_t hi_index[kMaxAggs];
};

__device__ __forceinline__ void smem_agg_init(const PipeDesc& d, SmemAgg& s, uint8_t* base) {
  const int cap = d.smem_capacity, nk = d.table.n_keys;
  s.cap = cap;
  s.keys = (uint64_t*)base;
  s.lo = s.keys + (size_t)nk * cap;
  s.hi = (int64_t*)(s.lo + (size_t)d.n_aggs * cap);
  int n128 = 0;
  for (int a = 0; a < kMaxAggs; ++a) s.hi_index[a] = (a < d.n_aggs && d.aggs[a].fn == A_SUM_I128) ? n128++ : -1;
  s.state = (uint32_t*)(s.hi + (size_t)n128 * cap);
  for (int i = threadIdx.x; i < cap; i += blockDim.x) {
    s.state[i] = 0;
    for (int a = 0; a < d.n_aggs; ++a) {
      uint64_t init = 0;
      switch (d.aggs[a].fn) {
        case A_MIN_I: init = 0x7FFFFFFFFFFFFFFFULL; break;
        case A_MAX_I: init = 0x8000000000000000ULL; break;
        case A_MIN_F: init = ~0ULL; break;
        default: init = 0; break;
      }
      s.lo[(size_t)a * cap + i] = init;
      if (s.hi_index[a] >= 0) s.hi[(size_t)s.hi_index[a] * cap + i] = 0;
    }
  }
}

// Finds or claims kw in the CTA table; -1 when the table is full (the
// caller then uses the global table).
__device__ __forceinline__ int smem_agg_find(const PipeDesc& d, SmemAgg& s, const uint64_t* kw, uint32_t& st) {
  const int nk = d.table.n_keys;
  int idx = (int)hash_slot(key_hash(kw, nk), (uint64_t)s.cap);
  for (int probe = 0; probe < s.cap; ++probe) {
    volatile uint32_t* sp = s.state + idx;
    uint32_t v = *sp;
    if (v == 0) {
      if (atomicCAS(s.state + idx, 0u, 1u) == 0u) {
        for (int i = 0; i < nk; ++i) s.keys[(size_t)i * s.cap + idx] = kw[i];
        __threadfence_block();
        *sp = 2u;
        return idx;
      }
      v = 1;
    }
    uint32_t spins = 0;
    while (v == 1) {
      if (++spins > kSpinLimit) {
        st |= ST_SPIN_LIMIT;
        return -1;
      }
      v = *sp;
    }
    __threadfence_block();
    bool eq = true;
    for (int i = 0; i < nk; ++i) eq &= (((volatile uint64_t*)s.keys)[(size_t)i * s.cap + idx] == kw[i]);
    if (eq) return idx;
    if (++idx == s.cap) idx = 0;
  }
  return -1;
}

// Aggregate inputs in one record of the partitioned aggregation: a record
// is the key and up to three inputs, padded to 1, 2 or 4 words.
constexpr int kPartMaxVals = 3;

// Words between entries of a CTA's one-key shared-memory table: the entry's
// words (key, states, high words of 128-bit sums) rounded up to an odd
// count, so that the same state of 16 consecutive entries sits in 16
// different bank pairs and a warp's updates to random groups rarely collide
// on a bank (the global table's 32-byte rounding would put every entry's
// state on the same few banks).
__host__ __device__ inline uint32_t smem_cas_stride(const PipeDesc& d) {
  uint32_t words = 1u + (uint32_t)d.n_aggs;
  for (int a = 0; a < d.n_aggs; ++a) words += d.aggs[a].fn == A_SUM_I128;
  return words | 1u;
}

// One-key shared-memory table of a CTA (AGG_SMEM with DAggTable::cas): the
// global table's word order within an entry (word 0 the key, word 1 + a
// state a, then the high words of 128-bit sums) at the odd stride above,
// keys claimed by CAS, states started at their identities, updates by
// shared-memory reductions.
struct SmemCas {
  uint64_t* e;
  uint32_t cap;
  uint32_t stride;
};

__device__ __forceinline__ void smem_cas_init(const PipeDesc& d, SmemCas& s, uint8_t* base) {
  s.e = (uint64_t*)base;
  s.cap = (uint32_t)d.smem_capacity;
  s.stride = smem_cas_stride(d);
  const uint32_t words = s.cap * s.stride;
  for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) {
    const uint32_t w = i % s.stride;
    uint64_t v = 0;
    if (w == 0) {
      v = (uint64_t)kEmptyKey;
    } else if ((int)w <= d.n_aggs) {
      switch (d.aggs[w - 1].fn) {
        case A_MIN_I: v = 0x7FFFFFFFFFFFFFFFULL; break;
        case A_MAX_I: v = 0x8000000000000000ULL; break;
        case A_MIN_F: v = ~0ULL; break;
        default: v = 0; break;
      }
    }
    s.e[i] = v;
  }
}

// Entry of key in the table, probing at most `limit` slots; -1 when it is
// not there and cannot be claimed (or the key is the empty sentinel).
// hshift drops the hash bits that the keys in the table share (their
// partition), so that those keys still spread over the whole table.
__device__ __forceinline__ int smem_cas_find(const SmemCas& s, uint64_t key, uint32_t limit, int hshift = 0) {
  if ((int64_t)key == kEmptyKey) return -1;
  uint32_t idx = (uint32_t)hash_slot(key_hash1(key) << hshift, (uint64_t)s.cap);
  for (uint32_t probe = 0; probe < limit; ++probe) {
    uint64_t* kp = s.e + (size_t)idx * s.stride;
    const uint64_t k = *(volatile uint64_t*)kp;
    if (k == key) return (int)idx;
    if ((int64_t)k == kEmptyKey) {
      const unsigned long long prev =
          atomicCAS((unsigned long long*)kp, (unsigned long long)kEmptyKey, (unsigned long long)key);
      if (prev == (unsigned long long)kEmptyKey || prev == key) return (int)idx;
    }
    if (++idx == s.cap) idx = 0;
  }
  return -1;
}

__device__ __forceinline__ int64_t lds_s64(uint32_t a) {
  int64_t x;
  asm volatile("ld.volatile.shared.s64 %0, [%1];" : "=l"(x) : "r"(a));
  return x;
}

// Adds x to the 64-bit word at shared address a as two 32-bit atomics: the
// low half's add returns the old value, from which the carry into the high
// half follows, so the word ends as the exact 64-bit sum modulo 2^64 however
// the adds interleave (each carry is counted by the add that wrapped).
__device__ __forceinline__ void smem_add64_split(uint32_t a, uint64_t x) {
  const uint32_t lo = (uint32_t)x;
  uint32_t old;
  asm volatile("atom.shared.add.u32 %0, [%1], %2;" : "=r"(old) : "r"(a), "r"(lo));
  const uint32_t hi = (uint32_t)(x >> 32) + ((uint32_t)(old + lo) < old ? 1u : 0u);
  if (hi) asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(a + 4), "r"(hi));
}

// Applies one value to a state word in shared memory (address `a` in the
// shared window), without waiting for the result where the op allows.
// These asm statements carry no memory clobber: the table is read back as
// plain memory only after a CTA barrier, and without the clobber the
// compiler keeps the global loads of later rows in flight across updates.
// COUNT and 64-bit SUM use 32-bit atomics; MIN and MAX read the state first
// and update only when the value improves on it (a stale read only costs
// an update that changes nothing).
__device__ __forceinline__ void smem_apply(int32_t fn, uint32_t a, uint32_t a_hi, Val v, int32_t vt) {
  switch (fn) {
    case A_COUNT: smem_add64_split(a, 1ULL); break;
    case A_SUM_I: smem_add64_split(a, (uint64_t)v.lo); break;
    case A_SUM_I128: {
      uint64_t old;
      const uint64_t add = (uint64_t)v.lo;
      asm volatile("atom.shared.add.u64 %0, [%1], %2;" : "=l"(old) : "r"(a), "l"(add));
      const int64_t hadd = (vt == P_I128 ? v.hi : (v.lo >> 63)) + ((old + add) < old ? 1 : 0);
      if (hadd) asm volatile("red.shared.add.u64 [%0], %1;" ::"r"(a_hi), "l"((uint64_t)hadd));
      break;
    }
    case A_SUM_F:
      asm volatile("red.shared.add.f64 [%0], %1;" ::"r"(a), "d"(val_as_f64(v, vt)));
      break;
    case A_MIN_I:
      if ((int64_t)v.lo < lds_s64(a)) asm volatile("red.shared.min.s64 [%0], %1;" ::"r"(a), "l"(v.lo));
      break;
    case A_MAX_I:
      if ((int64_t)v.lo > lds_s64(a)) asm volatile("red.shared.max.s64 [%0], %1;" ::"r"(a), "l"(v.lo));
      break;
    case A_MIN_F: {
      const uint64_t u = ord_f64(val_as_f64(v, vt));
      if (u < (uint64_t)lds_s64(a)) asm volatile("red.shared.min.u64 [%0], %1;" ::"r"(a), "l"(u));
      break;
    }
    case A_MAX_F: {
      const uint64_t u = ord_f64(val_as_f64(v, vt));
      if (u > (uint64_t)lds_s64(a)) asm volatile("red.shared.max.u64 [%0], %1;" ::"r"(a), "l"(u));
      break;
    }
    default: break;
  }
}

// Calls f(FnC<fn>{}) with the aggregate function as a compile-time constant,
// so that a loop over rows inside f is compiled once per function.
template <int N>
struct FnC {
  static constexpr int value = N;
};

template <class F>
__device__ __forceinline__ void dispatch_fn(int32_t fn, F& f) {
  switch (fn) {
    case A_COUNT: f(FnC<A_COUNT>{}); break;
    case A_SUM_I: f(FnC<A_SUM_I>{}); break;
    case A_SUM_I128: f(FnC<A_SUM_I128>{}); break;
    case A_SUM_F: f(FnC<A_SUM_F>{}); break;
    case A_MIN_I: f(FnC<A_MIN_I>{}); break;
    case A_MAX_I: f(FnC<A_MAX_I>{}); break;
    case A_MIN_F: f(FnC<A_MIN_F>{}); break;
    case A_MAX_F: f(FnC<A_MAX_F>{}); break;
    default: break;
  }
}

// ------------------------------------------------------------ the kernel
constexpr int kWarps = 8;                 // warps per CTA, each an independent tile processor
constexpr int kThreads = kWarps * 32;
constexpr int kTile = 256;                // rows per warp-tile

struct StreamLayout {
  int n;
  int col[kMaxStream];
  int width[kMaxStream];
  uint32_t off[kMaxStream];
  uint32_t bytes;  // per buffer
};

__host__ __device__ inline uint32_t stream_bytes_per_row(const PipeDesc& d) {
  uint32_t w = 0;
  for (int i = 0; i < d.n_stream && i < kMaxStream; ++i) w += (uint32_t)ptype_width(d.cols[d.stream_cols[i]].ptype);
  return w;
}

// Row ids of sources other than the driving one, per tile row, live in shared
// arrays filled by the probes; `slot_of_src` packs each source's array index
// (4 bits, 0xF = none).
struct TileCtx {
  const PipeDesc* d;
  const StreamLayout* S;
  const uint8_t* buf;  // streamed columns of this tile
  uint64_t base;       // first row of the tile
  uint32_t* srid;      // [nq][kTile] row ids of probed sources
  uint32_t slot_of_src;
};

__device__ __forceinline__ uint32_t tc_rid(const TileCtx& t, int src, uint32_t r) {
  if (src == t.d->drive_src) return (uint32_t)(t.base + r);
  const uint32_t q = (t.slot_of_src >> (4 * src)) & 0xFu;
  return t.srid[(size_t)q * kTile + r];
}

__device__ __forceinline__ int stream_index(const StreamLayout& S, int col) {
  int k = -1;
#pragma unroll
  for (int i = 0; i < kMaxStream; ++i)
    if (i < S.n && S.col[i] == col) k = i;
  return k;
}

__device__ __forceinline__ int64_t stream_value(const StreamLayout& S, const uint8_t* buf, int k, int32_t ptype,
                                                uint32_t r) {
  if (S.width[k] == 4)
    return ptype == P_I32 ? (int64_t)((const int32_t*)(buf + S.off[k]))[r]
                          : (int64_t)((const uint32_t*)(buf + S.off[k]))[r];
  return ((const int64_t*)(buf + S.off[k]))[r];
}

// Where one column's values come from in this tile, resolved once per op:
// the streamed tile buffer, or the column in HBM through the row id of its
// source.
struct ColAcc {
  const uint8_t* sm;  // streamed tile buffer of the column, or null
  const void* g;
  int32_t ptype;
  int32_t src;
  int32_t width;
};

__device__ __forceinline__ ColAcc col_acc(const TileCtx& t, int col) {
  const DCol& c = t.d->cols[col];
  ColAcc a{nullptr, c.ptr, c.ptype, c.src, ptype_width(c.ptype)};
  if (c.src == t.d->drive_src) {
    const int k = stream_index(*t.S, col);
    if (k >= 0) a.sm = t.buf + t.S->off[k];
  }
  return a;
}

__device__ __forceinline__ int64_t acc_get(const ColAcc& a, const TileCtx& t, uint32_t r) {
  if (a.sm) {
    if (a.width == 4)
      return a.ptype == P_I32 ? (int64_t)((const int32_t*)a.sm)[r] : (int64_t)((const uint32_t*)a.sm)[r];
    return ((const int64_t*)a.sm)[r];
  }
  return load_bits(a.g, a.ptype, tc_rid(t, a.src, r));
}

__device__ __forceinline__ int64_t tc_get(const TileCtx& t, int col, uint32_t r) {
  return acc_get(col_acc(t, col), t, r);
}

// ---- typed write phase of the order-preserving compaction
// One output column over the compacted rows with its value source and
// conversion fixed: TIn is how the column is held (int32_t sign-extends,
// uint32_t zero-extends, as acc_get does), TOut how the output stores it
// (the width store_val picks), G whether the column is read from HBM at the
// driving source's rows rather than from the streamed tile. f maps the
// loaded value (widened to int64, as the VM holds it) to the stored one.
// Four rows per lane are loaded before any is stored.
template <typename TIn, typename TOut, bool G, class F>
__device__ __forceinline__ void write_rows(const TIn* __restrict__ src, TOut* __restrict__ dst, uint32_t lim,
                                           bool ident, const uint16_t* sel, int lane, F f) {
  constexpr int B = 4;
  auto ld = [&](uint32_t q) -> int64_t {
    const uint32_t r = ident ? q : (uint32_t)sel[q];
    if (G) return (int64_t)__ldg(src + r);
    return (int64_t)src[r];
  };
  uint32_t p = (uint32_t)lane;
  for (; p + 32 * (B - 1) < lim; p += 32 * B) {
    int64_t v[B];
#pragma unroll
    for (int j = 0; j < B; ++j) v[j] = ld(p + 32 * j);
#pragma unroll
    for (int j = 0; j < B; ++j) dst[p + 32 * j] = (TOut)f(v[j]);
  }
  for (; p < lim; p += 32) dst[p] = (TOut)f(ld(p));
}

// Column value sources the typed writer covers: the streamed tile, or the
// driving source's column in HBM.
struct WriteSrc {
  const uint8_t* p;  // first row of the tile
  bool g;
  int width;
  int32_t ptype;
};

__device__ __forceinline__ bool write_src(const TileCtx& t, int col, WriteSrc& w) {
  const ColAcc a = col_acc(t, col);
  w.width = a.width;
  w.ptype = a.ptype;
  if (a.width != 4 && a.width != 8) return false;
  if (a.sm) {
    w.p = a.sm;
    w.g = false;
    return true;
  }
  if (a.src != t.d->drive_src) return false;
  w.p = (const uint8_t*)a.g + t.base * (uint64_t)a.width;
  w.g = true;
  return true;
}

// Dispatches one typed loop over the (source kind, held type) of a column
// for a fixed output type.
template <typename TOut, class F>
__device__ __forceinline__ void write_any(const WriteSrc& w, void* out, uint64_t base, uint32_t lim, bool ident,
                                          const uint16_t* sel, int lane, F f) {
  TOut* const dst = (TOut*)out + base;
  if (w.width == 8) {
    if (w.g) write_rows<int64_t, TOut, true>((const int64_t*)w.p, dst, lim, ident, sel, lane, f);
    else write_rows<int64_t, TOut, false>((const int64_t*)w.p, dst, lim, ident, sel, lane, f);
  } else if (w.ptype == P_I32) {
    if (w.g) write_rows<int32_t, TOut, true>((const int32_t*)w.p, dst, lim, ident, sel, lane, f);
    else write_rows<int32_t, TOut, false>((const int32_t*)w.p, dst, lim, ident, sel, lane, f);
  } else {
    if (w.g) write_rows<uint32_t, TOut, true>((const uint32_t*)w.p, dst, lim, ident, sel, lane, f);
    else write_rows<uint32_t, TOut, false>((const uint32_t*)w.p, dst, lim, ident, sel, lane, f);
  }
}

// Writes output column `pg` over the compacted rows when it is a column of
// the driving source, plain or combined with a constant by + - * in a
// non-128-bit type, into a 4- or 8-byte output; returns false for every
// other program (the caller evaluates those with the VM). The arithmetic
// is vm_arith's, with the same overflow rules.
__device__ __forceinline__ bool write_col_typed(const VmProg& pg, const TileCtx& t, void* out, uint64_t base,
                                                uint32_t lim, bool ident, const uint16_t* sel, int lane,
                                                uint32_t& st) {
  const int32_t ot = pg.out_type;
  if (ot == P_I128) return false;
  const bool o4 = ot == P_I32 || ot == P_F32;
  WriteSrc w;
  if (pg.n == 1 && pg.ins[0].op == VM_COL) {
    if (!write_src(t, pg.ins[0].arg, w)) return false;
    auto id = [](int64_t x) { return x; };
    if (o4) write_any<uint32_t>(w, out, base, lim, ident, sel, lane, id);
    else write_any<int64_t>(w, out, base, lim, ident, sel, lane, id);
    return true;
  }
  if (!(pg.n == 3 && pg.ins[0].op == VM_COL && pg.ins[1].op == VM_CONST && pg.ins[2].op >= VM_ADD &&
        pg.ins[2].op <= VM_MUL && pg.ins[2].type != P_I128))
    return false;
  if (!write_src(t, pg.ins[0].arg, w)) return false;
  const int64_t k = pg.ins[1].k;
  const int16_t op = pg.ins[2].op;
  uint32_t s2 = 0;
  switch (pg.ins[2].type) {
    case P_I32: {
      auto f = [&](int64_t x) {
        return fit32(op == VM_ADD ? x + k : op == VM_SUB ? x - k : x * k, s2);
      };
      if (o4) write_any<uint32_t>(w, out, base, lim, ident, sel, lane, f);
      else write_any<int64_t>(w, out, base, lim, ident, sel, lane, f);
      break;
    }
    case P_I64: {
      auto f = [&](int64_t x) {
        return op == VM_ADD ? add64(x, k, s2) : op == VM_SUB ? sub64(x, k, s2) : mul64(x, k, s2);
      };
      if (o4) write_any<uint32_t>(w, out, base, lim, ident, sel, lane, f);
      else write_any<int64_t>(w, out, base, lim, ident, sel, lane, f);
      break;
    }
    case P_F32: {
      const float y = as_f32(k);
      auto f = [&](int64_t x) {
        const float a = as_f32(x);
        return f32_bits(op == VM_ADD ? __fadd_rn(a, y) : op == VM_SUB ? __fsub_rn(a, y) : __fmul_rn(a, y));
      };
      if (o4) write_any<uint32_t>(w, out, base, lim, ident, sel, lane, f);
      else write_any<int64_t>(w, out, base, lim, ident, sel, lane, f);
      break;
    }
    default: {
      const double y = as_f64(k);
      auto f = [&](int64_t x) {
        const double a = as_f64(x);
        return f64_bits(op == VM_ADD ? __dadd_rn(a, y) : op == VM_SUB ? __dsub_rn(a, y) : __dmul_rn(a, y));
      };
      if (o4) write_any<uint32_t>(w, out, base, lim, ident, sel, lane, f);
      else write_any<int64_t>(w, out, base, lim, ident, sel, lane, f);
      break;
    }
  }
  st |= s2;
  return true;
}

// Stack slots of the expression VM held in registers. Every instruction's
// stack position depends on the program only, so it is the same in all
// lanes and the slot selects below are uniform branches.
struct RegStack {
  Val s0, s1, s2, s3;
  __device__ __forceinline__ Val get(int i) const { return i == 0 ? s0 : i == 1 ? s1 : i == 2 ? s2 : s3; }
  __device__ __forceinline__ void put(int i, const Val& v) {
    if (i == 0) s0 = v;
    else if (i == 1) s1 = v;
    else if (i == 2) s2 = v;
    else s3 = v;
  }
};

// Programs deeper than the register stack.
__device__ __forceinline__ Val vm_eval_deep(const VmProg& p, const TileCtx& t, uint32_t r, uint32_t& st) {
  Val stack[kMaxIns];
  int sp = 0;
  for (int i = 0; i < p.n; ++i) {
    const VmIns& in = p.ins[i];
    switch (in.op) {
      case VM_COL: {
        const int32_t pt = t.d->cols[in.arg].ptype;
        Val v;
        v.lo = tc_get(t, in.arg, r);
        v.hi = (pt == P_I32 || pt == P_I64) ? (v.lo >> 63) : 0;
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
        if (in.type == P_F32 || in.type == P_F64)
          stack[sp - 1].lo ^= (in.type == P_F32) ? (int64_t)0x80000000LL : (int64_t)0x8000000000000000ULL;
        else
          stack[sp - 1] = vm_arith(VM_SUB, in.type, z, stack[sp - 1], st);
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

__device__ __forceinline__ Val fast_leaf(const VmIns& in, const VmCast& c, const TileCtx& t, uint32_t r,
                                        uint32_t& st) {
  Val v;
  if (in.op == VM_COL) {
    v.lo = tc_get(t, in.arg, r);
    v.hi = (in.type == P_I32 || in.type == P_I64) ? (v.lo >> 63) : 0;
  } else {
    v.lo = in.k;
    v.hi = in.k2;
  }
  if (c.on) v = vm_cast(v, c.from, c.to, c.mul, c.div, st);
  return v;
}

__device__ __forceinline__ Val fast_op(const VmIns& op, const VmCast& c, Val a, Val b, uint32_t& st) {
  Val x = vm_arith(op.op, op.type, a, b, st);
  if (c.on) x = vm_cast(x, c.from, c.to, c.mul, c.div, st);
  return x;
}

// A program recast as a fixed tree (VmFast): leaves load together, then at
// most two ops; no stack, no per-instruction dispatch.
__device__ __forceinline__ Val vm_eval_fast(const VmFast& f, const TileCtx& t, uint32_t r, uint32_t& st) {
  const Val a = fast_leaf(f.leaf[0], f.leaf_cast[0], t, r, st);
  if (f.shape == 1) return a;
  const Val b = fast_leaf(f.leaf[1], f.leaf_cast[1], t, r, st);
  if (f.shape == 2) return fast_op(f.op[0], f.op_cast[0], a, b, st);
  const Val c = fast_leaf(f.leaf[2], f.leaf_cast[2], t, r, st);
  if (f.shape == 3) return fast_op(f.op[1], f.op_cast[1], a, fast_op(f.op[0], f.op_cast[0], b, c, st), st);
  return fast_op(f.op[1], f.op_cast[1], fast_op(f.op[0], f.op_cast[0], a, b, st), c, st);
}

// Expression VM over one tile row, all forms.
__device__ __forceinline__ Val vm_eval_full(const VmProg& p, const TileCtx& t, uint32_t r, uint32_t& st) {
  if (p.fast.shape) return vm_eval_fast(p.fast, t, r, st);
  if (p.depth > 4) return vm_eval_deep(p, t, r, st);
  RegStack S;
  S.s0 = S.s1 = S.s2 = S.s3 = Val{0, 0};
  int sp = 0;
  for (int i = 0; i < p.n; ++i) {
    const VmIns& in = p.ins[i];
    switch (in.op) {
      case VM_COL: {
        const int32_t pt = t.d->cols[in.arg].ptype;
        Val v;
        v.lo = tc_get(t, in.arg, r);
        v.hi = (pt == P_I32 || pt == P_I64) ? (v.lo >> 63) : 0;
        S.put(sp++, v);
        break;
      }
      case VM_CONST:
        S.put(sp++, Val{in.k, in.k2});
        break;
      case VM_CAST:
        S.put(sp - 1, vm_cast(S.get(sp - 1), in.arg, in.type, in.k, in.k2, st));
        break;
      case VM_NEG: {
        Val v = S.get(sp - 1);
        if (in.type == P_F32 || in.type == P_F64)
          v.lo ^= (in.type == P_F32) ? (int64_t)0x80000000LL : (int64_t)0x8000000000000000ULL;
        else
          v = vm_arith(VM_SUB, in.type, Val{0, 0}, v, st);
        S.put(sp - 1, v);
        break;
      }
      case VM_SLOT:
        S.put(sp++, Val{0, 0});
        break;
      default: {
        const Val b = S.get(sp - 1);
        const Val a = S.get(sp - 2);
        --sp;
        S.put(sp - 1, vm_arith(in.op, in.type, a, b, st));
        break;
      }
    }
  }
  return S.s0;
}

// Expression VM over one tile row.
__device__ __forceinline__ Val vm_eval_t(const VmProg& p, const TileCtx& t, uint32_t r, uint32_t& st) {
  return vm_eval_full(p, t, r, st);
}

// Integer predicates are evaluated as a closed interval [lo, hi] (negated for
// <>), so the row loop carries no op dispatch.
struct IntRange {
  int64_t lo, hi;
  bool neg, none;
};
__device__ __forceinline__ IntRange to_range(const DPred& p) {
  IntRange r{INT64_MIN, INT64_MAX, false, false};
  switch (p.op) {
    case C_EQ: r.lo = r.hi = p.ilit; break;
    case C_NE: r.lo = r.hi = p.ilit; r.neg = true; break;
    case C_LT: if (p.ilit == INT64_MIN) r.none = true; else r.hi = p.ilit - 1; break;
    case C_LE: r.hi = p.ilit; break;
    case C_GT: if (p.ilit == INT64_MAX) r.none = true; else r.lo = p.ilit + 1; break;
    case C_GE: r.lo = p.ilit; break;
    case C_FALSE: r.none = true; break;
    default: break;
  }
  return r;
}

// Filter op over a warp's selection: one loop per (column type, source),
// chosen once per op. A lane evaluates all of its (at most kTile / 32)
// entries before the first ballot, so their loads are in flight together;
// kept rows are compacted in order with ballots. Returns the new count.
template <typename GET>
__device__ __forceinline__ uint32_t filter_w(uint32_t n_sel, bool ident, const uint16_t* in, uint16_t* out,
                                             GET get_keep) {
  constexpr int U = kTile / 32;
  const int lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  uint32_t km = 0;  // bit j: entry j * 32 + lane is kept
#pragma unroll
  for (int j = 0; j < U; ++j) {
    const uint32_t i = (uint32_t)j * 32 + lane;
    if (i < n_sel && get_keep(ident ? i : (uint32_t)in[i])) km |= 1u << j;
  }
  uint32_t base = 0;
#pragma unroll
  for (int j = 0; j < U; ++j) {
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, (km >> j) & 1u);
    if ((km >> j) & 1u) {
      const uint32_t i = (uint32_t)j * 32 + lane;
      out[base + __popc(m & lt)] = (uint16_t)(ident ? i : (uint32_t)in[i]);
    }
    base += __popc(m);
  }
  return base;
}

// First filter of a warp-tile on a streamed integer column: lane l owns the
// kTile / 32 consecutive rows from l * (kTile / 32), reads them with 128-bit
// shared-memory loads, and writes the rows it keeps after a warp prefix sum,
// so the selection stays sorted. Returns the new count.
template <typename T>
__device__ __forceinline__ uint32_t filter_ident_blocked(const T* col, uint32_t nrow, const IntRange& rg,
                                                         uint16_t* out) {
  constexpr int U = kTile / 32;
  static_assert(U * sizeof(T) % 16 == 0, "rows per lane must fill whole 16-byte vectors");
  const int lane = threadIdx.x & 31;
  const uint32_t b0 = (uint32_t)lane * U;
  T v[U];
  const uint4* src = (const uint4*)(col + b0);
#pragma unroll
  for (int q = 0; q < (int)(U * sizeof(T) / 16); ++q) ((uint4*)v)[q] = src[q];
  // bounds of a 32-bit column narrowed to its range; an empty range keeps
  // nothing (or everything when negated)
  T lo, hi;
  bool empty = rg.none || rg.lo > rg.hi;
  if (sizeof(T) == 4) {
    empty = empty || rg.lo > (int64_t)INT32_MAX || rg.hi < (int64_t)INT32_MIN;
    lo = (T)(rg.lo < (int64_t)INT32_MIN ? (int64_t)INT32_MIN : rg.lo);
    hi = (T)(rg.hi > (int64_t)INT32_MAX ? (int64_t)INT32_MAX : rg.hi);
  } else {
    lo = (T)rg.lo;
    hi = (T)rg.hi;
  }
  uint32_t km = 0;
#pragma unroll
  for (int j = 0; j < U; ++j) {
    const bool in_range = !empty && v[j] >= lo && v[j] <= hi;
    if ((in_range != rg.neg) && b0 + j < nrow) km |= 1u << j;
  }
  const uint32_t c = __popc(km);
  uint32_t incl = c;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += y;
  }
  uint32_t pos = incl - c;
#pragma unroll
  for (int j = 0; j < U; ++j)
    if ((km >> j) & 1u) out[pos++] = (uint16_t)(b0 + j);
  return __shfl_sync(0xFFFFFFFFu, incl, 31);
}

// Join probe over the current selection, kProbeBatch rows per lane at a
// time: keys, then the presence words and map entries (dense) or first
// probed slots (hash) of the whole batch are loaded before any is used.
constexpr int kProbeBatch = 4;
constexpr int kAggBatch = 4;  // rows per lane in flight in the single-key hash sink
constexpr int kTileFetch = 1;  // warp-tiles taken per fetch of the dynamic tile counter

// Bytes of the CTA-wide shared-memory sink area (the AGG_SMEM table),
// rounded to 128.
__host__ __device__ inline uint32_t sink_area_bytes(const PipeDesc& d) {
  if (d.sink == SK_PART_COUNT || d.sink == SK_PART_SCATTER) return ((4u << d.part_bits) + 127) & ~127u;
  if (d.sink != SK_AGG_SMEM) return 0;
  if (d.table.cas) return ((uint32_t)d.smem_capacity * smem_cas_stride(d) * 8 + 127) & ~127u;
  uint32_t n128 = 0;
  for (int a = 0; a < d.n_aggs; ++a) n128 += d.aggs[a].fn == A_SUM_I128;
  const uint32_t b = (uint32_t)d.smem_capacity * (4 + 8 * (uint32_t)d.table.n_keys + 8 * (uint32_t)d.n_aggs + 8 * n128);
  return (b + 127) & ~127u;
}

// Bytes of one warp's shared-memory region, rounded to 128: two stream
// buffers (row_bytes streamed per row), two selection vectors, probe slots,
// probed row ids.
__host__ __device__ inline uint32_t warp_area_bytes(uint32_t row_bytes, int nq) {
  const uint32_t b = 2 * (uint32_t)kTile * row_bytes + 2 * kTile * 2 + kTile * 4 + (uint32_t)nq * kTile * 4;
  return (b + 127) & ~127u;
}

__host__ __device__ inline int probed_source_count(const PipeDesc& d) {
  int nq = 0;
  for (int s = 0; s < kMaxSrc; ++s) {
    if (s == d.drive_src) continue;
    bool used = false;
    for (int p = 0; p < d.n_probes; ++p) used |= ((d.probes[p].fill_mask >> s) & 1u) != 0;
    nq += used;
  }
  return nq;
}

// Decoded fused opening of a pipeline (see the kernel).
struct FusedOpen {
  int32_t on, empty, neg, want_slot;
  uint32_t foff, koff;
  int32_t lo, hi;
  int64_t kmin;
  uint64_t cap;
  const uint32_t* bits;
  const uint32_t* map;
};

// One CTA of kWarps warps; every warp is an independent tile processor. A
// warp streams its own kTile-row tiles into its own double buffer (one TMA
// bulk copy per streamed column, its own mbarriers), runs the ops and the
// sink over them with warp-level compaction, and never waits for the other
// warps of the CTA inside the tile loop: a slow tile (a long sink chain, a
// look-back) stalls only its warp while the others keep the SM busy.
template <int SINK>
__global__ void __launch_bounds__(kThreads, (SINK == SK_AGG_SCALAR || SINK == SK_AGG_SMEM || SINK == SK_PART_SCATTER) ? 2 : 3)
    k_pipeline(const __grid_constant__ PipeDesc d) {
  constexpr int TILE = kTile;
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t s_mbar[kWarps][2];
  __shared__ FusedOpen s_fz;
  __shared__ uint64_t s_red[SINK == SK_AGG_SCALAR ? kMaxAggs : 1][kWarps];
  __shared__ int64_t s_redhi[SINK == SK_AGG_SCALAR ? kMaxAggs : 1][kWarps];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  const uint64_t n = d.in_count ? *d.in_count : d.n;
  const uint64_t n_tiles = (n + TILE - 1) / TILE;
  uint32_t st = 0;

  StreamLayout S;
  S.n = d.n_stream < kMaxStream ? d.n_stream : kMaxStream;
  {
    uint32_t off = 0;
#pragma unroll
    for (int i = 0; i < kMaxStream; ++i) {
      S.col[i] = i < S.n ? d.stream_cols[i] : -1;
      S.width[i] = i < S.n ? ptype_width(d.cols[S.col[i]].ptype) : 0;
      S.off[i] = off;
      off += (uint32_t)TILE * (uint32_t)S.width[i];
    }
    S.bytes = off;
  }
  // probed sources whose row ids are kept per tile row
  uint32_t slot_of_src = 0xFFFFFFFFu;
  int nq = 0;
  for (int s = 0; s < kMaxSrc; ++s) {
    if (s == d.drive_src) continue;
    bool used = false;
    for (int p = 0; p < d.n_probes; ++p) used |= ((d.probes[p].fill_mask >> s) & 1u) != 0;
    if (used) {
      slot_of_src = (slot_of_src & ~(0xFu << (4 * s))) | ((uint32_t)nq << (4 * s));
      ++nq;
    }
  }
  // shared layout: sink area | warp 0 | warp 1 | ...; a warp's region holds
  // stream buffers x2 | sel A | sel B | slots | probed row ids
  uint8_t* const wreg = smem + sink_area_bytes(d) + (size_t)warp * warp_area_bytes(S.bytes / TILE, nq);
  uint8_t* const sbuf0 = wreg;
  uint8_t* const sbuf1 = wreg + S.bytes;
  uint16_t* const selA = (uint16_t*)(wreg + 2 * S.bytes);
  uint16_t* const selB = selA + TILE;
  uint32_t* const s_slot = (uint32_t*)(selB + TILE);
  uint32_t* const s_srid = s_slot + TILE;

  SmemAgg sagg;
  SmemCas scas;
  if (SINK == SK_AGG_SMEM) {
    if (d.table.cas) smem_cas_init(d, scas, smem);
    else smem_agg_init(d, sagg, smem);
  }
  // key partitions: per-CTA counters, or this CTA's write cursors
  if (SINK == SK_PART_COUNT || SINK == SK_PART_SCATTER) {
    uint32_t* const s_part = (uint32_t*)smem;
    const uint32_t np = 1u << d.part_bits;
    for (uint32_t p = tid; p < np; p += kThreads)
      s_part[p] = SINK == SK_PART_COUNT ? 0u : d.part_start[p] + d.part_offsets[(size_t)blockIdx.x * np + p];
  }
  uint64_t plo[SINK == SK_AGG_SCALAR ? kMaxAggs : 1];
  int64_t phi[SINK == SK_AGG_SCALAR ? kMaxAggs : 1];
  if (SINK == SK_AGG_SCALAR) {
#pragma unroll
    for (int a = 0; a < kMaxAggs; ++a) {
      uint64_t init = 0;
      if (a < d.n_aggs) {
        switch (d.aggs[a].fn) {
          case A_MIN_I: init = 0x7FFFFFFFFFFFFFFFULL; break;
          case A_MAX_I: init = 0x8000000000000000ULL; break;
          case A_MIN_F: init = ~0ULL; break;
          default: init = 0; break;
        }
      }
      plo[a] = init;
      phi[a] = 0;
    }
  }
  if (lane == 0 && S.n) {
    mbar_init(&s_mbar[warp][0], 1);
    mbar_init(&s_mbar[warp][1], 1);
    mbar_fence_init();
  }
  __syncthreads();

  // Tile order: order-preserving compaction takes tiles from a counter in
  // increasing order (kTileFetch at a time), so every tile's predecessors
  // are held by running warps; other sinks stride over the tiles.
  const bool dynamic_tiles = SINK == SK_MATERIALIZE;
  const uint64_t n_warps = (uint64_t)gridDim.x * kWarps;
  uint64_t chunk_next = 0, chunk_end = 0;
  auto fetch = [&](uint64_t prev, bool first) -> uint64_t {
    if (!dynamic_tiles) {
      // groups of G consecutive tiles per warp, groups strided over the warps
      const uint64_t G = d.tile_group > 1 ? (uint64_t)d.tile_group : 1;
      if (first) return ((uint64_t)blockIdx.x * kWarps + warp) * G;
      return (prev + 1) % G ? prev + 1 : prev + 1 + (n_warps - 1) * G;
    }
    if (chunk_next < chunk_end) return chunk_next++;
    uint32_t t = 0;
    if (lane == 0) t = atomicAdd(d.tile_counter, (uint32_t)kTileFetch);
    t = __shfl_sync(0xFFFFFFFFu, t, 0);
    chunk_next = (uint64_t)t + 1;
    chunk_end = (uint64_t)t + kTileFetch;
    return (uint64_t)t;
  };
  // Lane 0 stages the streamed columns of a full tile into buffer `b`.
  auto issue = [&](uint64_t tile, int b) {
    const uint64_t base = tile * (uint64_t)TILE;
    if (base + TILE > n) return;  // the tail tile is loaded directly
    uint8_t* dst = b ? sbuf1 : sbuf0;
    fence_proxy_async();
    mbar_arrive_expect_tx(&s_mbar[warp][b], S.bytes);
    for (int i = 0; i < S.n; ++i)
      bulk_g2s(dst + S.off[i], (const uint8_t*)d.cols[S.col[i]].ptr + base * (uint64_t)S.width[i],
               (uint32_t)TILE * (uint32_t)S.width[i], &s_mbar[warp][b]);
  };

  // The common opening of a join pipeline — a range filter on a streamed
  // INTEGER/DATE column, then a dense-join probe keyed by a streamed INTEGER
  // column — runs fused per lane over its own rows: no selection vector
  // between the two, and the probe loads of all of a lane's rows in flight
  // together. Decoded once per CTA into shared memory (s_fz).
  if (tid == 0) {
    s_fz.on = 0;
    if (d.n_ops >= 2 && d.ops[0].kind == OPK_FILTER && d.ops[1].kind == OPK_PROBE) {
      const DPred& p = d.preds[d.ops[0].idx];
      const DCol& c = d.cols[p.col];
      const int si = c.src == d.drive_src ? stream_index(S, p.col) : -1;
      const DProbe& pr = d.probes[d.ops[1].idx];
      const DBuild& bd = d.builds[pr.build];
      const DCol& kc = d.cols[pr.key_col];
      const int sk = kc.src == d.drive_src ? stream_index(S, pr.key_col) : -1;
      const uint32_t fill = pr.fill_mask & ~(1u << d.drive_src);
      if (si >= 0 && c.ptype == P_I32 && S.width[si] == 4 && sk >= 0 && kc.ptype == P_I32 && S.width[sk] == 4 &&
          bd.kind == B_DENSE && fill == 0) {
        const IntRange rg = to_range(p);
        s_fz.on = 1;
        s_fz.foff = S.off[si];
        s_fz.koff = S.off[sk];
        s_fz.empty = (rg.none || rg.lo > rg.hi || rg.lo > (int64_t)INT32_MAX || rg.hi < (int64_t)INT32_MIN) ? 1 : 0;
        s_fz.lo = (int32_t)(rg.lo < (int64_t)INT32_MIN ? (int64_t)INT32_MIN : rg.lo);
        s_fz.hi = (int32_t)(rg.hi > (int64_t)INT32_MAX ? (int64_t)INT32_MAX : rg.hi);
        s_fz.neg = rg.neg ? 1 : 0;
        s_fz.kmin = bd.key_min;
        s_fz.cap = bd.capacity;
        s_fz.bits = bd.dense_bits;
        s_fz.map = bd.dense_map;
        s_fz.want_slot = d.ops[1].idx == d.slot_probe ? 1 : 0;
      }
    }
  }
  __syncthreads();
  const bool fz = s_fz.on != 0;

  uint64_t cur = fetch(0, true);
  if (lane == 0 && S.n && cur < n_tiles) issue(cur, 0);
  uint32_t parity = 0;
  int b = 0;
  while (cur < n_tiles) {
    const uint64_t nx = fetch(cur, false);
    if (lane == 0 && S.n && nx < n_tiles) issue(nx, b ^ 1);
    const uint64_t tile = cur;
    const uint64_t tile_base = tile * (uint64_t)TILE;
    const uint32_t nrow = (uint32_t)(n - tile_base < (uint64_t)TILE ? n - tile_base : (uint64_t)TILE);
    uint8_t* const buf = b ? sbuf1 : sbuf0;
    if (S.n) {
      bool ok = true;
      if (nrow == TILE) {
        ok = mbar_wait(&s_mbar[warp][b], (parity >> b) & 1u);
        parity ^= 1u << b;
      } else {
        for (int i = 0; i < S.n; ++i) {
          const DCol& c = d.cols[S.col[i]];
          for (int r = lane; r < TILE; r += 32) {
            int64_t v = (uint32_t)r < nrow ? load_bits(c.ptr, c.ptype, tile_base + r) : 0;
            if (S.width[i] == 4) ((uint32_t*)(buf + S.off[i]))[r] = (uint32_t)v;
            else ((int64_t*)(buf + S.off[i]))[r] = v;
          }
        }
        __syncwarp();
      }
      if (__any_sync(0xFFFFFFFFu, !ok)) {
        st |= ST_SPIN_LIMIT;
        // give the copy still in flight a bounded chance to land, then stop
        if (nx < n_tiles) mbar_wait(&s_mbar[warp][b ^ 1], (parity >> (b ^ 1)) & 1u);
        break;
      }
    }
    TileCtx tc{&d, &S, buf, tile_base, s_srid, slot_of_src};

    // ---- ops over the warp's selection vector
    uint32_t n_sel = nrow;
    bool ident = true;
    uint16_t* sel_in = selA;
    uint16_t* sel_out = selB;
    int o0 = 0;
    if (fz) {
      constexpr int U = TILE / 32;
      const uint32_t b0 = (uint32_t)lane * U;
      int32_t fv[U], kv[U];
#pragma unroll
      for (int q = 0; q < U / 4; ++q) {
        ((uint4*)fv)[q] = ((const uint4*)(buf + s_fz.foff))[lane * (U / 4) + q];
        ((uint4*)kv)[q] = ((const uint4*)(buf + s_fz.koff))[lane * (U / 4) + q];
      }
      uint32_t w[U], mv[U];
      uint64_t kk[U];
      const bool fz_empty = s_fz.empty != 0, fz_neg = s_fz.neg != 0;
      const int32_t fz_lo = s_fz.lo, fz_hi = s_fz.hi;
      const int64_t fz_kmin = s_fz.kmin;
      const uint64_t fz_cap = s_fz.cap;
      const uint32_t* const fz_bits = s_fz.bits;
      const uint32_t* const fz_map = s_fz.map;
      const bool fz_want_slot = s_fz.want_slot != 0;
#pragma unroll
      for (int j = 0; j < U; ++j) {
        const bool pass = ((!fz_empty && fv[j] >= fz_lo && fv[j] <= fz_hi) != fz_neg) && b0 + j < nrow;
        kk[j] = (uint64_t)((int64_t)kv[j] - fz_kmin);
        const bool inb = pass && kk[j] < fz_cap;
        w[j] = inb ? __ldg(fz_bits + (kk[j] >> 5)) : 0u;
        // the slot only when grouping by it (always loaded by the slot sink,
        // whose code then stays that of the common case)
        mv[j] = inb && (SINK == SK_AGG_SLOT || fz_want_slot) ? __ldg(fz_map + kk[j]) : 0u;
      }
      uint32_t km = 0;
#pragma unroll
      for (int j = 0; j < U; ++j) {
        if ((w[j] >> (kk[j] & 31)) & 1u) {
          km |= 1u << j;
          if (fz_want_slot) s_slot[b0 + j] = mv[j] - 1u;
        }
      }
      const uint32_t c = __popc(km);
      uint32_t incl = c;
#pragma unroll
      for (int q = 1; q < 32; q <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, q);
        if (lane >= q) incl += y;
      }
      uint32_t pos = incl - c;
#pragma unroll
      for (int j = 0; j < U; ++j)
        if ((km >> j) & 1u) sel_out[pos++] = (uint16_t)(b0 + j);
      n_sel = __shfl_sync(0xFFFFFFFFu, incl, 31);
      __syncwarp();
      ident = false;
      sel_in = sel_out;
      sel_out = selA;
      o0 = 2;
    }
    for (int o = o0; o < d.n_ops && n_sel > 0; ++o) {
      const PipeOp op = d.ops[o];
      uint32_t kept = 0;
      if (op.kind == OPK_FILTER) {
        const DPred& p = d.preds[op.idx];
        const DCol& c = d.cols[p.col];
        const int si = (c.src == d.drive_src) ? stream_index(S, p.col) : -1;
        if (c.ptype == P_I32 || c.ptype == P_I64) {
          const IntRange rg = to_range(p);
          if (rg.none) {
            kept = 0;
          } else if (si >= 0 && ident && S.width[si] == 4 && c.ptype == P_I32) {
            kept = filter_ident_blocked<int32_t>((const int32_t*)(buf + S.off[si]), n_sel, rg, sel_out);
          } else if (si >= 0 && ident && S.width[si] == 8) {
            kept = filter_ident_blocked<int64_t>((const int64_t*)(buf + S.off[si]), n_sel, rg, sel_out);
          } else if (si >= 0 && S.width[si] == 4) {
            const int32_t* col = (const int32_t*)(buf + S.off[si]);
            kept = filter_w(n_sel, ident, sel_in, sel_out, [&](uint32_t r) {
              const int64_t x = col[r];
              return (x >= rg.lo && x <= rg.hi) != rg.neg;
            });
          } else if (si >= 0) {
            const int64_t* col = (const int64_t*)(buf + S.off[si]);
            kept = filter_w(n_sel, ident, sel_in, sel_out, [&](uint32_t r) {
              const int64_t x = col[r];
              return (x >= rg.lo && x <= rg.hi) != rg.neg;
            });
          } else {
            kept = filter_w(n_sel, ident, sel_in, sel_out, [&](uint32_t r) {
              const int64_t x = load_bits(c.ptr, c.ptype, tc_rid(tc, c.src, r));
              return (x >= rg.lo && x <= rg.hi) != rg.neg;
            });
          }
        } else {
          kept = filter_w(n_sel, ident, sel_in, sel_out, [&](uint32_t r) {
            return eval_pred_bits(tc_get(tc, p.col, r), c.ptype, p);
          });
        }
      } else {
        const DProbe& pr = d.probes[op.idx];
        const DBuild& bd = d.builds[pr.build];
        const bool want_slot = op.idx == d.slot_probe;
        const uint32_t fill = pr.fill_mask & ~(1u << d.drive_src);
        const ColAcc ka = col_acc(tc, pr.key_col);
        const bool k32 = ka.sm && ka.width == 4 && ka.ptype == P_I32;  // streamed INTEGER key
        // Descriptor fields used per row, read once: the loop's shared-memory
        // stores would otherwise force reloads through the descriptor.
        const int64_t b_kmin = bd.key_min;
        const uint64_t b_cap = bd.capacity;
        const uint32_t* const b_bits = bd.dense_bits;
        const uint32_t* const b_map = bd.dense_map;
        const bool b_dense = bd.kind == B_DENSE;
        for (uint32_t i0 = 0; i0 < n_sel; i0 += 32 * kProbeBatch) {
          uint32_t r[kProbeBatch], slot[kProbeBatch];
          bool act[kProbeBatch], keep[kProbeBatch];
          int64_t key[kProbeBatch];
#pragma unroll
          for (int j = 0; j < kProbeBatch; ++j) {
            const uint32_t i = i0 + (uint32_t)j * 32 + lane;
            act[j] = i < n_sel;
            r[j] = act[j] ? (ident ? i : (uint32_t)sel_in[i]) : 0u;
            key[j] = !act[j] ? 0 : k32 ? (int64_t)((const int32_t*)ka.sm)[r[j]] : acc_get(ka, tc, r[j]);
          }
          if (b_dense) {
            uint32_t w[kProbeBatch], mv[kProbeBatch];
            uint64_t kk[kProbeBatch];
#pragma unroll
            for (int j = 0; j < kProbeBatch; ++j) {
              kk[j] = (uint64_t)(key[j] - b_kmin);
              const bool inb = act[j] && kk[j] < b_cap;
              // The map entry is read beside its presence word; it is only
              // used when the presence bit is set.
              w[j] = inb ? __ldg(b_bits + (kk[j] >> 5)) : 0u;
              mv[j] = inb ? __ldg(b_map + kk[j]) : 0u;
            }
#pragma unroll
            for (int j = 0; j < kProbeBatch; ++j) {
              keep[j] = ((w[j] >> (kk[j] & 31)) & 1u) != 0;
              slot[j] = mv[j] - 1u;
            }
          } else {
            uint64_t h[kProbeBatch];
            int64_t k0[kProbeBatch];
            bool maybe[kProbeBatch];
            // the build's Bloom filter (L2-resident) first: keys it rules
            // out never touch the table in HBM
#pragma unroll
            for (int j = 0; j < kProbeBatch; ++j) {
              h[j] = hash64((uint64_t)key[j]);
              maybe[j] = act[j] && bloom_maybe(bd, h[j]);
            }
#pragma unroll
            for (int j = 0; j < kProbeBatch; ++j) {
              h[j] = hash_slot(h[j], bd.capacity);
              k0[j] = (maybe[j] && key[j] != kEmptyKey) ? bd.hash_keys[h[j]] : kEmptyKey;
            }
#pragma unroll
            for (int j = 0; j < kProbeBatch; ++j) {
              keep[j] = false;
              slot[j] = 0;
              if (!maybe[j]) continue;
              if (k0[j] == key[j] && key[j] != kEmptyKey) {
                keep[j] = true;
                slot[j] = bd.hash_slot[h[j]] - 1u;
              } else if (k0[j] != kEmptyKey || key[j] == kEmptyKey) {
                keep[j] = build_lookup(bd, key[j], slot[j], st);
              }
            }
          }
#pragma unroll
          for (int j = 0; j < kProbeBatch; ++j) {
            if (keep[j]) {
              if (want_slot) s_slot[r[j]] = slot[j];
              if (fill)
                for (int s = 0; s < kMaxSrc; ++s)
                  if ((fill >> s) & 1u)
                    s_srid[(size_t)((slot_of_src >> (4 * s)) & 0xFu) * TILE + r[j]] =
                        bd.payload[s] ? bd.payload[s][slot[j]] : slot[j];  // no array: the build's own row
            }
            const uint32_t m = __ballot_sync(0xFFFFFFFFu, keep[j]);
            if (keep[j]) sel_out[kept + __popc(m & lt)] = (uint16_t)r[j];
            kept += __popc(m);
          }
        }
      }
      __syncwarp();
      n_sel = kept;
      ident = false;
      uint16_t* t_ = sel_in;
      sel_in = sel_out;
      sel_out = t_;
    }

    // ---- sink over the surviving rows (sorted: ballots keep row order)
    if (SINK == SK_MAT_COUNT) {
      // first pass of the two-pass compaction: the tile's survivors
      if (lane == 0) d.tile_pos[tile] = n_sel;
      if (d.tile_mask) {
        // and their 256-bit mask, built in the free selection buffer
        uint32_t* const m = (uint32_t*)sel_out;
        if (lane < 8) m[lane] = 0u;
        __syncwarp();
        for (uint32_t p = lane; p < n_sel; p += 32) {
          const uint32_t r = ident ? p : (uint32_t)sel_in[p];
          atomicOr(&m[r >> 5], 1u << (r & 31));
        }
        __syncwarp();
        if (lane < 8) d.tile_mask[tile * 8 + lane] = m[lane];
      }
    } else if (SINK == SK_MATERIALIZE || SINK == SK_MAT_WRITE) {
      const uint32_t total = n_sel;
      uint64_t base;
      if (SINK == SK_MAT_WRITE) {
        // second pass: the tile's offset from the scan of the first pass's counts
        base = (uint64_t)d.tile_pos[tile] + d.chunk_pos[tile / kMatScanTiles];
      } else {
        base = lb_exclusive_warp(d.tile_status, tile, total, d.epoch, d.status,
                                 d.lb_spin_limit ? d.lb_spin_limit : kSpinLimit, !d.lb_stall_first);
        if (lane == 0 && tile == n_tiles - 1) *d.out_count = base + total;
      }
      // write phase: one output column at a time over the compacted rows
      const uint32_t lim = base >= d.out_capacity ? 0u
                           : (uint32_t)(d.out_capacity - base < (uint64_t)total ? d.out_capacity - base : total);
      if (lim < total) st |= ST_CAPACITY;
      for (int q = 0; q < d.n_out; ++q) {
        const VmProg& pg = d.progs[d.out_prog[q]];
        void* out = d.out_ptr[q];
        const int32_t ot = pg.out_type;
        if (write_col_typed(pg, tc, out, base, lim, ident, sel_in, lane, st)) {
          // typed loop over the column
        } else if (pg.n == 1 && pg.ins[0].op == VM_COL) {
          // plain column: typed copy
          const ColAcc ca = col_acc(tc, pg.ins[0].arg);
#pragma unroll 4
          for (uint32_t p = lane; p < lim; p += 32) {
            Val v;
            v.lo = acc_get(ca, tc, ident ? p : (uint32_t)sel_in[p]);
            v.hi = v.lo >> 63;
            store_val(out, ot, base + p, v);
          }
        } else if (pg.n == 3 && pg.ins[0].op == VM_COL && pg.ins[1].op == VM_CONST && pg.ins[2].op >= VM_ADD &&
                   pg.ins[2].op <= VM_MUL && pg.ins[2].type != P_I128) {
          // column op constant, evaluated inline
          const ColAcc ca = col_acc(tc, pg.ins[0].arg);
          const Val kc{pg.ins[1].k, pg.ins[1].k2};
          const int16_t aop = pg.ins[2].op, aty = pg.ins[2].type;
#pragma unroll 4
          for (uint32_t p = lane; p < lim; p += 32) {
            Val v;
            v.lo = acc_get(ca, tc, ident ? p : (uint32_t)sel_in[p]);
            v.hi = v.lo >> 63;
            store_val(out, ot, base + p, vm_arith(aop, aty, v, kc, st));
          }
        } else {
          for (uint32_t p = lane; p < lim; p += 32)
            store_val(out, ot, base + p, vm_eval_t(pg, tc, ident ? p : (uint32_t)sel_in[p], st));
        }
      }
      for (int s = 0; s < kMaxSrc; ++s)
        if ((d.out_rid_mask >> s) & 1u)
          for (uint32_t p = lane; p < lim; p += 32)
            d.out_rids[s][base + p] = tc_rid(tc, s, ident ? p : (uint32_t)sel_in[p]);
    } else if (SINK == SK_PART_COUNT || SINK == SK_PART_SCATTER) {
      // The key's partition is the top part_bits of its hash. With few
      // partitions, a warp's rows of one partition reserve their positions
      // with one shared-memory atomic (their leader's).
      uint32_t* const s_part = (uint32_t*)smem;
      const VmProg& kp = d.progs[d.key_prog[0]];
      const int shift = 64 - d.part_bits;
      const int nv = d.part_nvals;
      const bool grouped = d.part_bits <= 8;
      auto plain = [](const VmProg& pg) {
        return pg.fast.shape == 1 && pg.fast.leaf[0].op == VM_COL && !pg.fast.leaf_cast[0].on;
      };
      const bool kcol = plain(kp);
      const ColAcc kca = col_acc(tc, kcol ? kp.fast.leaf[0].arg : 0);
      const VmProg* vp[kPartMaxVals];
      bool vcol[kPartMaxVals];
      ColAcc vca[kPartMaxVals];
#pragma unroll
      for (int v = 0; v < kPartMaxVals; ++v) {
        vp[v] = (SINK == SK_PART_SCATTER && v < nv) ? &d.progs[d.aggs[d.part_src[v]].prog] : nullptr;
        vcol[v] = vp[v] && plain(*vp[v]);
        vca[v] = col_acc(tc, vcol[v] ? vp[v]->fast.leaf[0].arg : 0);
      }
      for (uint32_t i0 = 0; i0 < n_sel; i0 += 32) {
        const uint32_t i = i0 + lane;
        const bool act = i < n_sel;
        const uint32_t r = act ? (ident ? i : (uint32_t)sel_in[i]) : 0u;
        uint64_t key = 0;
        if (act) key = kcol ? (uint64_t)acc_get(kca, tc, r) : (uint64_t)vm_eval_t(kp, tc, r, st).lo;
        const uint32_t p = act ? (uint32_t)(key_hash1(key) >> shift) : 0xFFFFFFFFu;
        uint32_t pos = 0;
        if (grouped) {
          // all lanes vote; lanes without a row form their own group, whose leader adds nothing
          const unsigned peers = __match_any_sync(0xFFFFFFFFu, p);
          const int leader = __ffs(peers) - 1;
          uint32_t base = 0;
          if (act && (int)lane == leader) base = atomicAdd(&s_part[p], (uint32_t)__popc(peers));
          if (SINK == SK_PART_SCATTER) {
            base = __shfl_sync(0xFFFFFFFFu, base, leader);
            pos = base + (uint32_t)__popc(peers & ((1u << lane) - 1u));
          }
        } else if (act) {
          if (SINK == SK_PART_COUNT) atomicAdd(&s_part[p], 1u);
          else pos = atomicAdd(&s_part[p], 1u);
        }
        if (SINK == SK_PART_COUNT || !act) continue;
        // 1, 2 or 4 words: the key, then the inputs (zero padded), written
        // with one 16- or 32-byte store
        uint64_t wv[kPartMaxVals + 1];
        wv[0] = key;
#pragma unroll
        for (int v = 0; v < kPartMaxVals; ++v)
          wv[1 + v] = !vp[v] ? 0 : vcol[v] ? (uint64_t)acc_get(vca[v], tc, r) : (uint64_t)vm_eval_t(*vp[v], tc, r, st).lo;
        uint64_t* const rec = d.part_records + (uint64_t)pos * (uint64_t)d.part_words;
        if (d.part_words == 1) {
          rec[0] = key;
        } else {
          if (d.part_words == 4)  // one 32-byte store (records are 32-byte aligned)
            asm volatile("st.global.v4.u64 [%0], {%1, %2, %3, %4};" ::"l"(rec), "l"(wv[0]), "l"(wv[1]), "l"(wv[2]),
                         "l"(wv[3])
                         : "memory");
          else
            *(ulonglong2*)rec = make_ulonglong2(wv[0], wv[1]);
        }
      }
    } else if (SINK == SK_BUILD) {
      const DBuild& bd = d.builds[d.sink_build];
      // A build row's slot is its row number in the build table: no shared
      // counter to contend on, and the build's own row ids need no payload
      // array (payload[drive_src] stays null).
      for (uint32_t i = lane; i < n_sel; i += 32) {
        const uint32_t r = ident ? i : (uint32_t)sel_in[i];
        const uint32_t slot = (uint32_t)(tile_base + r);
        const int64_t key = tc_get(tc, d.build_key_col, r);
        for (int s = 0; s < kMaxSrc; ++s)
          if (s != d.drive_src && ((d.build_payload_mask >> s) & 1u)) bd.payload[s][slot] = tc_rid(tc, s, r);
        // A representative-row aggregate downstream keeps its states by
        // this slot: initialize them here, so the (build-table sized)
        // state arrays need no clearing per query.
        for (int a = 0; a < d.n_aggs; ++a) agg_init_global(d.aggs[a], slot);
        build_insert(bd, key, slot, st);
      }
    } else if ((SINK == SK_AGG_HASH || SINK == SK_AGG_SMEM) && d.table.cas) {
      // One 64-bit group key. Phase 1 finds every surviving row's group
      // (kAggBatch rows per lane in flight; keys held in the CTA's
      // shared-memory table stay there) and parks it in s_slot; phase 2
      // applies one aggregate at a time over the rows, with the column
      // access resolved once per aggregate, and updates global states with
      // atomics whose results are not waited for.
      constexpr int B = kAggBatch;
      const DAggTable& tb = d.table;
      const VmProg& kp = d.progs[d.key_prog[0]];
      const uint64_t gstride = tb.stride > 1 ? (uint64_t)tb.stride : 1;
      const uint64_t* const gkeys = tb.keys[0];
      const uint64_t gcap = tb.capacity;
      const bool key_col = kp.fast.shape == 1 && kp.fast.leaf[0].op == VM_COL && !kp.fast.leaf_cast[0].on;
      const ColAcc kca = col_acc(tc, key_col ? kp.fast.leaf[0].arg : 0);
      for (uint32_t i0 = 0; i0 < n_sel; i0 += 32 * B) {
        uint32_t r[B];
        bool act[B];
        int sidx[B];
        uint64_t key[B], h[B], k0[B], g[B];
#pragma unroll
        for (int b = 0; b < B; ++b) {
          const uint32_t i = i0 + (uint32_t)b * 32 + lane;
          act[b] = i < n_sel;
          r[b] = act[b] ? (ident ? i : (uint32_t)sel_in[i]) : 0u;
          key[b] = !act[b] ? 0 : key_col ? (uint64_t)acc_get(kca, tc, r[b]) : (uint64_t)vm_eval_t(kp, tc, r[b], st).lo;
        }
#pragma unroll
        for (int b = 0; b < B; ++b) {
          sidx[b] = -1;
          if (SINK == SK_AGG_SMEM && act[b]) sidx[b] = smem_cas_find(scas, key[b], (uint32_t)d.smem_probes);
        }
#pragma unroll
        for (int b = 0; b < B; ++b) {
          h[b] = hash_slot(key_hash1(key[b]), gcap);
          k0[b] = (act[b] && sidx[b] < 0 && (int64_t)key[b] != kEmptyKey) ? __ldcg(gkeys + h[b] * gstride) : 0;
        }
#pragma unroll
        for (int b = 0; b < B; ++b) {
          g[b] = kNoGroup;
          if (act[b] && sidx[b] < 0)
            g[b] = ((int64_t)key[b] != kEmptyKey && k0[b] == key[b]) ? h[b] : agg_find_cas(tb, key[b], h[b], st);
          if (act[b])
            s_slot[i0 + (uint32_t)b * 32 + lane] =
                sidx[b] >= 0 ? (0x80000000u | (uint32_t)sidx[b]) : (g[b] == kNoGroup ? 0xFFFFFFFFu : (uint32_t)g[b]);
        }
      }
      __syncwarp();
      for (int a = 0; a < d.n_aggs; ++a) {
        const DAgg& ag = d.aggs[a];
        const int32_t fn = ag.fn;
        unsigned long long* const alo = (unsigned long long*)ag.lo;
        long long* const ahi = (long long*)ag.hi;
        const VmProg* const pg = ag.prog >= 0 ? &d.progs[ag.prog] : nullptr;
        const int32_t vt = pg ? pg->out_type : P_I64;
        const bool vcol = pg && pg->fast.shape == 1 && pg->fast.leaf[0].op == VM_COL && !pg->fast.leaf_cast[0].on;
        const ColAcc vca = col_acc(tc, vcol ? pg->fast.leaf[0].arg : 0);
        const bool vsigned = vcol && (pg->fast.leaf[0].type == P_I32 || pg->fast.leaf[0].type == P_I64);
        // shared-window addresses of this state's words in entry 0
        uint32_t s_lo = 0, s_hi = 0;
        if (SINK == SK_AGG_SMEM) {
          int hw = 0;
          for (int q = 0; q < a; ++q) hw += d.aggs[q].fn == A_SUM_I128;
          s_lo = smem_u32(scas.e + 1 + a);
          s_hi = smem_u32(scas.e + 1 + d.n_aggs + hw);
        }
#pragma unroll 4
        for (uint32_t p = lane; p < n_sel; p += 32) {
          const uint32_t code = s_slot[p];
          if (code == 0xFFFFFFFFu) continue;
          const uint32_t rr = ident ? p : (uint32_t)sel_in[p];
          Val v{0, 0};
          if (vcol) {
            v.lo = acc_get(vca, tc, rr);
            v.hi = vsigned ? (v.lo >> 63) : 0;
          } else if (pg) {
            v = vm_eval_t(*pg, tc, rr, st);
          }
          if (SINK == SK_AGG_SMEM && (code & 0x80000000u)) {
            const uint32_t eo = (code & 0x7FFFFFFFu) * scas.stride * 8;
            smem_apply(fn, s_lo + eo, s_hi + eo, v, vt);
          } else {
            const uint64_t o = (uint64_t)code * gstride;
            agg_apply_g(fn, alo + o, ahi ? ahi + o : nullptr, v, vt);
          }
        }
      }
    } else {
      uint8_t* const slot_hit = d.slot_hit;
      for (uint32_t i = lane; i < n_sel; i += 32) {
        const uint32_t r = ident ? i : (uint32_t)sel_in[i];
        if (SINK == SK_AGG_SLOT) {
          const uint32_t g = s_slot[r];
          slot_hit[g] = 1;
          for (int a = 0; a < d.n_aggs; ++a) {
            const DAgg& ag = d.aggs[a];
            Val v{0, 0};
            int32_t vt = P_I64;
            if (ag.prog >= 0) {
              v = vm_eval_t(d.progs[ag.prog], tc, r, st);
              vt = d.progs[ag.prog].out_type;
            }
            agg_apply(ag.fn, (unsigned long long*)(ag.lo + g), (long long*)(ag.hi ? ag.hi + g : nullptr), v, vt);
          }
        } else if (SINK == SK_AGG_HASH || SINK == SK_AGG_SMEM) {
          uint64_t kw[kMaxKeys];
#pragma unroll
          for (int q = 0; q < kMaxKeys; ++q)
            kw[q] = q < d.table.n_keys ? (uint64_t)vm_eval_t(d.progs[d.key_prog[q]], tc, r, st).lo : 0;
          int sidx = -1;
          if (SINK == SK_AGG_SMEM) sidx = smem_agg_find(d, sagg, kw, st);
          uint64_t g = kNoGroup;
          if (sidx < 0) g = agg_find_global(d, kw, st);
          if (sidx < 0 && g == kNoGroup) continue;
          for (int a = 0; a < d.n_aggs; ++a) {
            const DAgg& ag = d.aggs[a];
            Val v{0, 0};
            int32_t vt = P_I64;
            if (ag.prog >= 0) {
              v = vm_eval_t(d.progs[ag.prog], tc, r, st);
              vt = d.progs[ag.prog].out_type;
            }
            if (sidx >= 0) {
              long long* hp = sagg.hi_index[a] >= 0
                                  ? (long long*)(sagg.hi + (size_t)sagg.hi_index[a] * sagg.cap + sidx)
                                  : nullptr;
              agg_apply(ag.fn, (unsigned long long*)(sagg.lo + (size_t)a * sagg.cap + sidx), hp, v, vt);
            } else {
              agg_apply(ag.fn, (unsigned long long*)(ag.lo + g), (long long*)(ag.hi ? ag.hi + g : nullptr), v,
                        vt);
            }
          }
        } else if (SINK == SK_AGG_SCALAR) {
#pragma unroll
          for (int a = 0; a < kMaxAggs; ++a) {
            if (a >= d.n_aggs) break;
            const DAgg& ag = d.aggs[a];
            Val v{0, 0};
            int32_t vt = P_I64;
            if (ag.prog >= 0) {
              v = vm_eval_t(d.progs[ag.prog], tc, r, st);
              vt = d.progs[ag.prog].out_type;
            }
            switch (ag.fn) {
              case A_COUNT: plo[a] += 1; break;
              case A_SUM_I: plo[a] += (uint64_t)v.lo; break;
              case A_SUM_I128: {
                uint64_t o = plo[a];
                plo[a] += (uint64_t)v.lo;
                phi[a] += (vt == P_I128 ? v.hi : (v.lo >> 63)) + (plo[a] < o ? 1 : 0);
                break;
              }
              case A_SUM_F:
                plo[a] = (uint64_t)__double_as_longlong(
                    __dadd_rn(__longlong_as_double((long long)plo[a]), val_as_f64(v, vt)));
                break;
              case A_MIN_I: if ((int64_t)v.lo < (int64_t)plo[a]) plo[a] = (uint64_t)v.lo; break;
              case A_MAX_I: if ((int64_t)v.lo > (int64_t)plo[a]) plo[a] = (uint64_t)v.lo; break;
              case A_MIN_F: { uint64_t u = ord_f64(val_as_f64(v, vt)); if (u < plo[a]) plo[a] = u; break; }
              case A_MAX_F: { uint64_t u = ord_f64(val_as_f64(v, vt)); if (u > plo[a]) plo[a] = u; break; }
              default: break;
            }
          }
        }
      }
    }
    // Every lane is done with `buf` and the selection before they are reused.
    __syncwarp();
    cur = nx;
    b ^= 1;
  }

  // End-of-kernel work.
  if (SINK == SK_PART_COUNT) {
    __syncthreads();
    const uint32_t np = 1u << d.part_bits;
    const uint32_t* const s_part = (const uint32_t*)smem;
    for (uint32_t p = tid; p < np; p += kThreads) d.part_counts[(size_t)blockIdx.x * np + p] = s_part[p];
  } else if (SINK == SK_MATERIALIZE) {
    __syncthreads();
    if (tid == 0) {
      if (n == 0 && blockIdx.x == 0) *d.out_count = 0;
      // The last CTA to finish resets the dynamic tile counter for the next launch.
      __threadfence();
      uint32_t done = atomicAdd(d.tile_counter + 1, 1u);
      if (done == gridDim.x - 1) {
        d.tile_counter[0] = 0;
        d.tile_counter[1] = 0;
      }
    }
  } else if (SINK == SK_AGG_SMEM && d.table.cas) {
    __syncthreads();
    const uint64_t gstride = d.table.stride > 1 ? (uint64_t)d.table.stride : 1;
    for (uint32_t i = tid; i < scas.cap; i += kThreads) {
      const uint64_t* ent = scas.e + (size_t)i * scas.stride;
      const uint64_t key = ent[0];
      if ((int64_t)key == kEmptyKey) continue;
      const uint64_t g = agg_find_cas(d.table, key, hash_slot(key_hash1(key), d.table.capacity), st);
      if (g == kNoGroup) continue;
      const uint64_t o = g * gstride;
      int hw = 0;
      for (int a = 0; a < d.n_aggs; ++a) {
        const DAgg& ag = d.aggs[a];
        const int64_t hv = ag.fn == A_SUM_I128 ? (int64_t)ent[1 + d.n_aggs + hw++] : 0;
        agg_merge(ag.fn, (unsigned long long*)(ag.lo + o), (long long*)(ag.hi ? ag.hi + o : nullptr), ent[1 + a], hv);
      }
    }
  } else if (SINK == SK_AGG_SMEM) {
    __syncthreads();
    for (int i = tid; i < sagg.cap; i += kThreads) {
      if (sagg.state[i] != 2u) continue;
      uint64_t kw[kMaxKeys];
#pragma unroll
      for (int q = 0; q < kMaxKeys; ++q) kw[q] = q < d.table.n_keys ? sagg.keys[(size_t)q * sagg.cap + i] : 0;
      uint64_t g = agg_find_global(d, kw, st);
      if (g == kNoGroup) continue;
      const uint64_t o = g * (d.table.stride > 1 ? (uint64_t)d.table.stride : 1);
      for (int a = 0; a < d.n_aggs; ++a) {
        const DAgg& ag = d.aggs[a];
        int64_t hv = sagg.hi_index[a] >= 0 ? sagg.hi[(size_t)sagg.hi_index[a] * sagg.cap + i] : 0;
        agg_merge(ag.fn, (unsigned long long*)(ag.lo + o), (long long*)(ag.hi ? ag.hi + o : nullptr),
                  sagg.lo[(size_t)a * sagg.cap + i], hv);
      }
    }
  } else if (SINK == SK_AGG_SCALAR) {
    // Block reduction of the register partials, then one atomic per CTA.
#pragma unroll
    for (int a = 0; a < kMaxAggs; ++a) {
      if (a >= d.n_aggs) break;
      const int32_t fn = d.aggs[a].fn;
      uint64_t x = plo[a];
      int64_t h = phi[a];
      for (int o = 16; o > 0; o >>= 1) {
        uint64_t y = __shfl_down_sync(0xFFFFFFFFu, x, o);
        int64_t yh = __shfl_down_sync(0xFFFFFFFFu, h, o);
        switch (fn) {
          case A_COUNT: case A_SUM_I: x += y; break;
          case A_SUM_I128: { uint64_t o2 = x; x += y; h += yh + (x < o2 ? 1 : 0); break; }
          case A_SUM_F: x = (uint64_t)__double_as_longlong(__dadd_rn(__longlong_as_double((long long)x), __longlong_as_double((long long)y))); break;
          case A_MIN_I: if ((int64_t)y < (int64_t)x) x = y; break;
          case A_MAX_I: if ((int64_t)y > (int64_t)x) x = y; break;
          case A_MIN_F: if (y < x) x = y; break;
          case A_MAX_F: if (y > x) x = y; break;
          default: break;
        }
      }
      if (lane == 0) {
        s_red[a][warp] = x;
        s_redhi[a][warp] = h;
      }
    }
    __syncthreads();
    if (tid < d.n_aggs) {
      const DAgg& ag = d.aggs[tid];
      for (int w = 0; w < kWarps; ++w)
        agg_merge(ag.fn, (unsigned long long*)ag.lo, (long long*)ag.hi, s_red[tid][w], s_redhi[tid][w]);
    }
  }
  if (st) atomicOr(d.status, st);
}

// ------------------------------------------------- partitioned aggregation
// A one-key aggregate over many groups runs in three passes instead of
// updating a global table per row: the pipeline counts each CTA's surviving
// rows per key partition (SK_PART_COUNT), k_part_scan turns the counts into
// write positions, the pipeline writes each row's key and aggregate inputs
// into its partition (SK_PART_SCATTER, the same tiles per CTA), and
// k_part_agg aggregates one partition per CTA in a shared-memory table
// before merging its groups into the global table. A partition is the top
// part_bits of the key's hash, so a partition's groups also occupy one
// contiguous stretch of the global table.

// One CTA. counts and offsets are [CTA][partition]; offsets become each
// CTA's first position within the partition, start[p] the partition's first
// record (start[P] = all records), and chunk_start[p] the first of the
// partition's ceil(records / chunk) chunks (chunk_start[P] = all chunks).
constexpr int kScanThreads = 1024;
constexpr int kMaxPartBits = 13;

// Exclusive scan of s_vals[0, np) into out[0, np], out[np] = the total.
__device__ void block_scan_excl(const uint32_t* s_vals, uint32_t np, uint32_t* out, uint32_t* s_warp) {
  const uint32_t per = (np + kScanThreads - 1) / kScanThreads;
  const uint32_t b = threadIdx.x * per;
  uint32_t sum = 0;
  for (uint32_t i = 0; i < per; ++i)
    if (b + i < np) sum += s_vals[b + i];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t incl = sum;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_warp[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = s_warp[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
      if (lane >= o) w += y;
    }
    s_warp[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  uint32_t run = (warp ? s_warp[warp - 1] : 0u) + incl - sum;
  for (uint32_t i = 0; i < per; ++i)
    if (b + i < np) {
      out[b + i] = run;
      run += s_vals[b + i];
    }
  if (threadIdx.x == 0) out[np] = s_warp[kScanThreads / 32 - 1];
  __syncthreads();  // s_warp and s_vals may be reused
}

__global__ void __launch_bounds__(kScanThreads) k_part_scan(const uint32_t* __restrict__ counts,
                                                             uint32_t* __restrict__ offsets,
                                                             uint32_t* __restrict__ start,
                                                             uint32_t* __restrict__ chunk_start, int n_ctas,
                                                             int part_bits, uint32_t chunk) {
  __shared__ uint32_t s_tot[1 << kMaxPartBits];
  __shared__ uint32_t s_warp[kScanThreads / 32];
  const uint32_t np = 1u << part_bits;
  for (uint32_t p = threadIdx.x; p < np; p += kScanThreads) {
    uint32_t run = 0;
#pragma unroll 8
    for (int c = 0; c < n_ctas; ++c) {
      const size_t i = (size_t)c * np + p;
      const uint32_t v = counts[i];
      offsets[i] = run;
      run += v;
    }
    s_tot[p] = run;
  }
  __syncthreads();
  block_scan_excl(s_tot, np, start, s_warp);
  for (uint32_t p = threadIdx.x; p < np; p += kScanThreads) s_tot[p] = (s_tot[p] + chunk - 1) / chunk;
  __syncthreads();
  block_scan_excl(s_tot, np, chunk_start, s_warp);
}

// A row's value in its state's domain (COUNT 1, SUM_F a double's bits,
// MIN_F/MAX_F the order-preserving image): the one-word states (all but
// A_SUM_I128) combine these with state_combine and merge them once.
__device__ __forceinline__ uint64_t lane_state_value(int32_t fn, Val v, int32_t vt) {
  switch (fn) {
    case A_COUNT: return 1;
    case A_SUM_F: return (uint64_t)__double_as_longlong(val_as_f64(v, vt));
    case A_MIN_F:
    case A_MAX_F: return ord_f64(val_as_f64(v, vt));
    default: return (uint64_t)v.lo;
  }
}

__device__ __forceinline__ uint64_t state_combine(int32_t fn, uint64_t x, uint64_t y) {
  switch (fn) {
    case A_SUM_F:
      return (uint64_t)__double_as_longlong(
          __dadd_rn(__longlong_as_double((long long)x), __longlong_as_double((long long)y)));
    case A_MIN_I: return (int64_t)y < (int64_t)x ? y : x;
    case A_MAX_I: return (int64_t)y > (int64_t)x ? y : x;
    case A_MIN_F: return y < x ? y : x;
    case A_MAX_F: return y > x ? y : x;
    default: return x + y;  // COUNT, SUM_I (mod 2^64)
  }
}

// Combines x over each group of lanes that share a key (`peers`: the lanes
// of this lane's group, this lane included; 0 for a lane outside every
// group); the group's lowest lane ends with the group's total. Each round
// every lane still collecting adds the value of the next higher lane of its
// group that is still collecting, and the lanes at odd ranks within their
// group drop out, so a group of n lanes takes ceil(log2 n) rounds.
__device__ __forceinline__ uint64_t peer_combine(int32_t fn, unsigned peers, uint64_t x, uint32_t lane) {
  // one key across the whole warp: a butterfly leaves the total in every lane
  if (__all_sync(0xFFFFFFFFu, peers == 0xFFFFFFFFu)) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = state_combine(fn, x, __shfl_xor_sync(0xFFFFFFFFu, x, o));
    return x;
  }
  unsigned rank = __popc(peers & ((1u << lane) - 1u));  // lanes of the group below this one
  unsigned rest = peers & ~((2u << lane) - 1u);          // lanes of the group above this one
  while (__any_sync(0xFFFFFFFFu, rest != 0)) {
    const int next = __ffs(rest) - 1;
    const uint64_t y = __shfl_sync(0xFFFFFFFFu, x, next < 0 ? (int)lane : next);
    if (next >= 0) x = state_combine(fn, x, y);
    const unsigned done = __ballot_sync(0xFFFFFFFFu, (rank & 1u) != 0);
    rest &= ~done;
    rank >>= 1;
  }
  return x;
}

// Merges a one-word partial state into a shared-memory state word.
__device__ __forceinline__ void smem_merge(int32_t fn, uint32_t a, uint64_t x) {
  switch (fn) {
    case A_COUNT:
    case A_SUM_I: smem_add64_split(a, x); break;
    case A_SUM_F: asm volatile("red.shared.add.f64 [%0], %1;" ::"r"(a), "d"(__longlong_as_double((long long)x))); break;
    case A_MIN_I:
      if ((int64_t)x < lds_s64(a)) asm volatile("red.shared.min.s64 [%0], %1;" ::"r"(a), "l"(x));
      break;
    case A_MAX_I:
      if ((int64_t)x > lds_s64(a)) asm volatile("red.shared.max.s64 [%0], %1;" ::"r"(a), "l"(x));
      break;
    case A_MIN_F:
      if (x < (uint64_t)lds_s64(a)) asm volatile("red.shared.min.u64 [%0], %1;" ::"r"(a), "l"(x));
      break;
    case A_MAX_F:
      if (x > (uint64_t)lds_s64(a)) asm volatile("red.shared.max.u64 [%0], %1;" ::"r"(a), "l"(x));
      break;
    default: break;
  }
}

constexpr int kPartAggThreads = 512;
constexpr int kPartBatch = 2;  // records per thread with loads in flight together

// One CTA per chunk: a partition's records split into pieces of at most
// d.part_chunk, so that a large partition (a skewed key's) is shared by
// several CTAs while a CTA sees one partition's keys only. The records go
// into a shared-memory table (the layout of SmemCas, capacity
// d.smem_capacity); a record whose key finds no entry within d.smem_probes
// (at most kPartProbes) slots of its home slot goes to the global table
// directly (a key is claimed only within that window, so its records always
// take the same route). Then every entry is merged into the global table.
//
// Partitions holding more groups than a table (beyond the partition limit)
// are sub-partitioned by the CTA itself: with d.part_split = s > 0 it counts
// its chunk's records per sub-partition (the 2^s hash bits below the
// partition's), places them by sub-partition into d.part_sub (a counting
// sort, at the chunk's own positions), and then aggregates one
// sub-partition at a time, merging and clearing the table after each, so
// that each round's groups fit the table.
constexpr uint32_t kPartProbes = 64;
constexpr int kMaxPartSplit = 5;  // sub-partitions per chunk: up to 32, one per lane

__global__ void __launch_bounds__(kPartAggThreads, 2) k_part_agg(const __grid_constant__ PipeDesc d) {
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ uint32_t s_sub[1 << kMaxPartSplit];       // records per sub-partition, then write cursors
  __shared__ uint32_t s_subpos[(1 << kMaxPartSplit) + 1];  // first record of each sub-partition
  const uint32_t np = 1u << d.part_bits;
  const uint32_t split = (uint32_t)d.part_split;
  const uint32_t cb = blockIdx.x;
  if (cb >= d.part_chunk_start[np]) return;  // the whole CTA leaves, before any barrier
  // the chunk's partition: chunk_start[lo] <= cb < chunk_start[hi]
  uint32_t lo = 0, hi = np;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (d.part_chunk_start[mid] <= cb) lo = mid;
    else hi = mid;
  }
  const uint32_t pend = d.part_start[lo + 1];
  const uint32_t psize = pend - d.part_start[lo];
  const uint32_t rb = d.part_start[lo] + (cb - d.part_chunk_start[lo]) * d.part_chunk;
  const uint32_t re = pend - rb < d.part_chunk ? pend : rb + d.part_chunk;
  SmemCas s;
  smem_cas_init(d, s, smem);
  uint32_t st = 0;
  const int W = d.part_words;
  const int na = d.n_aggs;
  const DAggTable& tb = d.table;
  const uint64_t gstride = tb.stride > 1 ? (uint64_t)tb.stride : 1;
  const uint32_t estride = s.stride * 8;
  const uint32_t probes = d.smem_probes > 0 && (uint32_t)d.smem_probes < kPartProbes ? (uint32_t)d.smem_probes
                                                                                     : kPartProbes;
  constexpr int B = kPartBatch;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  // Records of one key are combined within a warp before updating where a
  // warp often holds several of them: in a partition over twice the average
  // size (a skewed key's), or when partitions have few keys. Every state must
  // be one word.
  bool warp_ok = d.part_combine != 0 || psize > 2 * (d.part_start[np] >> d.part_bits) + 1024;
  for (int a = 0; a < na; ++a) warp_ok &= d.aggs[a].fn != A_SUM_I128;
  const int hshift = d.part_bits + (int)split;

  // Aggregates the records [b, e) of `recs` into the table (keys it cannot
  // hold into the global table). Each record is read once (evict first).
  auto agg_range = [&](const uint64_t* recs, uint32_t b, uint32_t e) {
    for (uint32_t i0 = b; i0 < e; i0 += kPartAggThreads * B) {
      uint64_t key[B];
      uint64_t val[B][kPartMaxVals];
      bool act[B];
#pragma unroll
      for (int q = 0; q < B; ++q) {
        const uint32_t i = i0 + (uint32_t)q * kPartAggThreads + threadIdx.x;
        act[q] = i < e;
        const uint64_t* rec = recs + (uint64_t)(act[q] ? i : b) * (uint64_t)W;
        key[q] = 0;
#pragma unroll
        for (int v = 0; v < kPartMaxVals; ++v) val[q][v] = 0;
        if (act[q]) {
          if (W == 1) {
            key[q] = __ldcs(rec);
          } else if (W == 4) {  // one 32-byte load
            asm volatile("ld.global.cs.v4.u64 {%0, %1, %2, %3}, [%4];"
                         : "=l"(key[q]), "=l"(val[q][0]), "=l"(val[q][1]), "=l"(val[q][2])
                         : "l"(rec));
          } else {
            const ulonglong2 x = __ldcs((const ulonglong2*)rec);
            key[q] = x.x;
            val[q][0] = x.y;
          }
        }
      }
      // Records of one key in the same warp (a skewed key's) are combined in
      // registers first: only the lowest lane of each key's group updates.
      bool upd[B];      // this lane's record updates an entry
      bool comb[B];     // (warp-uniform) batch q combines records of a key first
      unsigned peers[B];
#pragma unroll
      for (int q = 0; q < B; ++q) {
        upd[q] = act[q];
        comb[q] = false;
        peers[q] = 0;
        if (warp_ok) {
          // every lane takes part in the warp votes (key[q] is 0 where the lane has no record)
          const unsigned am = __ballot_sync(0xFFFFFFFFu, act[q]);
          const unsigned same = __match_any_sync(0xFFFFFFFFu, key[q]);
          peers[q] = act[q] ? (same & am) : 0u;
          // combining pays for itself once some key holds four lanes
          comb[q] = __any_sync(0xFFFFFFFFu, __popc(peers[q]) >= 4);
          // when combining, only the lowest lane of each key's group updates
          if (comb[q]) upd[q] = act[q] && (peers[q] & lt) == 0;
        }
      }
      // the updating records' entries: shared-memory index, else the global group
      int idx[B];
      uint64_t g[B];
#pragma unroll
      for (int q = 0; q < B; ++q) {
        idx[q] = -1;
        g[q] = kNoGroup;
        if (upd[q]) {
          // the default window as a constant: the loop then compiles as in
          // the common case it is (a short window only for overfull tables)
          idx[q] = probes == kPartProbes ? smem_cas_find(s, key[q], kPartProbes, hshift)
                                         : smem_cas_find(s, key[q], probes, hshift);
          if (idx[q] < 0) g[q] = agg_find_cas(tb, key[q], hash_slot(key_hash1(key[q]), tb.capacity), st);
        }
      }
      // one aggregate at a time over the batch, compiled per function
      int hw = 0;
      for (int a = 0; a < na; ++a) {
        const DAgg& ag = d.aggs[a];
        const int vs = d.part_val[a];
        const int32_t vt = vs >= 0 ? d.progs[ag.prog].out_type : P_I64;
        Val v[B];
#pragma unroll
        for (int q = 0; q < B; ++q) {
          const uint64_t x = vs == 0 ? val[q][0] : vs == 1 ? val[q][1] : vs == 2 ? val[q][2] : 0;
          v[q].lo = (int64_t)x;
          v[q].hi = v[q].lo >> 63;
        }
        const uint32_t sa = smem_u32(s.e + 1 + a), sh = smem_u32(s.e + 1 + na + hw);
        unsigned long long* const glo = (unsigned long long*)ag.lo;
        long long* const ghi = (long long*)ag.hi;
        auto apply = [&](auto fnc) {
          constexpr int FN = decltype(fnc)::value;
#pragma unroll
          for (int q = 0; q < B; ++q) {
            if (comb[q]) {  // warp-uniform; only when every state is one word
              if (FN != A_SUM_I128) {
                const uint64_t x = peer_combine(FN, peers[q], lane_state_value(FN, v[q], vt), lane);
                if (idx[q] >= 0) smem_merge(FN, sa + (uint32_t)idx[q] * estride, x);
                else if (g[q] != kNoGroup) agg_merge(FN, glo + g[q] * gstride, nullptr, x, 0);
              }
              continue;
            }
            if (idx[q] >= 0) {
              const uint32_t eo = (uint32_t)idx[q] * estride;
              smem_apply(FN, sa + eo, sh + eo, v[q], vt);
            } else if (g[q] != kNoGroup) {
              const uint64_t o = g[q] * gstride;
              agg_apply_g(FN, glo + o, ghi ? ghi + o : nullptr, v[q], vt);
            }
          }
        };
        dispatch_fn(ag.fn, apply);
        hw += ag.fn == A_SUM_I128;
      }
    }
  };

  // Merges every entry of the table into the global table.
  auto merge_table = [&]() {
    for (uint32_t i = threadIdx.x; i < s.cap; i += kPartAggThreads) {
      const uint64_t* ent = s.e + (size_t)i * s.stride;
      const uint64_t key = ent[0];
      if ((int64_t)key == kEmptyKey) continue;
      const uint64_t gg = agg_find_cas(tb, key, hash_slot(key_hash1(key), tb.capacity), st);
      if (gg == kNoGroup) continue;
      const uint64_t o = gg * gstride;
      int hw2 = 0;
      for (int a = 0; a < na; ++a) {
        const DAgg& ag = d.aggs[a];
        const int64_t hv = ag.fn == A_SUM_I128 ? (int64_t)ent[1 + na + hw2++] : 0;
        agg_merge(ag.fn, (unsigned long long*)(ag.lo + o), (long long*)(ag.hi ? ag.hi + o : nullptr), ent[1 + a],
                  hv);
      }
    }
  };

  if (split == 0) {
    __syncthreads();
    agg_range(d.part_records, rb, re);
    __syncthreads();
    merge_table();
    if (st) atomicOr(d.status, st);
    return;
  }

  // ---- sub-partitioned chunk: count, place, then one round per sub-partition
  const uint32_t S = 1u << split;
  const int sub_shift = 64 - d.part_bits - (int)split;
  if (threadIdx.x < S) s_sub[threadIdx.x] = 0;
  __syncthreads();
  // This lane's sub-partition (S: no record), the lanes of the warp that share
  // it, and (in lane j < S) how many lanes hold sub-partition j: S ballots.
  auto sub_masks = [&](uint32_t sb, unsigned& mine, uint32_t& cnt_j) {
    mine = 0;
    cnt_j = 0;
    for (uint32_t j = 0; j < S; ++j) {
      const unsigned m = __ballot_sync(0xFFFFFFFFu, sb == j);
      if (sb == j) mine = m;
      if (lane == j) cnt_j = (uint32_t)__popc(m);
    }
  };
  // the loops below run whole warps over the chunk, so every lane votes
  const uint32_t span = (re - rb + 31) & ~31u;
  for (uint32_t i0 = 0; i0 < span; i0 += kPartAggThreads) {
    const uint32_t i = rb + i0 + threadIdx.x;
    if (i0 + (threadIdx.x & ~31u) >= span) break;  // warp-uniform
    uint32_t sb = S;
    if (i < re) sb = (uint32_t)(key_hash1(__ldcg(d.part_records + (uint64_t)i * (uint64_t)W)) >> sub_shift) & (S - 1u);
    unsigned mine;
    uint32_t cnt_j;
    sub_masks(sb, mine, cnt_j);
    if (lane < S && cnt_j) atomicAdd(&s_sub[lane], cnt_j);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t run = 0;
    for (uint32_t j = 0; j < S; ++j) {
      s_subpos[j] = run;
      run += s_sub[j];
      s_sub[j] = s_subpos[j];  // write cursor
    }
    s_subpos[S] = run;
  }
  __syncthreads();
  for (uint32_t i0 = 0; i0 < span; i0 += kPartAggThreads) {
    const uint32_t i = rb + i0 + threadIdx.x;
    if (i0 + (threadIdx.x & ~31u) >= span) break;  // warp-uniform
    const bool act = i < re;
    const uint64_t* rec = d.part_records + (uint64_t)(act ? i : rb) * (uint64_t)W;
    uint64_t w[4] = {0, 0, 0, 0};
    if (act) {
      if (W == 4)
        asm volatile("ld.global.cs.v4.u64 {%0, %1, %2, %3}, [%4];"
                     : "=l"(w[0]), "=l"(w[1]), "=l"(w[2]), "=l"(w[3])
                     : "l"(rec));
      else if (W == 2) {
        const ulonglong2 x = __ldcs((const ulonglong2*)rec);
        w[0] = x.x;
        w[1] = x.y;
      } else {
        w[0] = __ldcs(rec);
      }
    }
    const uint32_t sb = act ? (uint32_t)(key_hash1(w[0]) >> sub_shift) & (S - 1u) : S;
    unsigned mine;
    uint32_t cnt_j;
    sub_masks(sb, mine, cnt_j);
    uint32_t base_j = 0;
    if (lane < S && cnt_j) base_j = atomicAdd(&s_sub[lane], cnt_j);
    const uint32_t base = __shfl_sync(0xFFFFFFFFu, base_j, sb < S ? sb : 0);
    if (act) {
      uint64_t* dst = d.part_sub + ((uint64_t)rb + base + (uint32_t)__popc(mine & lt)) * (uint64_t)W;
      if (W == 4) {  // one 32-byte store
        asm volatile("st.global.v4.u64 [%0], {%1, %2, %3, %4};" ::"l"(dst), "l"(w[0]), "l"(w[1]), "l"(w[2]),
                     "l"(w[3])
                     : "memory");
      } else if (W == 2) {
        *(ulonglong2*)dst = make_ulonglong2(w[0], w[1]);
      } else {
        dst[0] = w[0];
      }
    }
  }
  __syncthreads();
  for (uint32_t j = 0; j < S; ++j) {
    agg_range(d.part_sub, rb + s_subpos[j], rb + s_subpos[j + 1]);
    __syncthreads();
    merge_table();
    __syncthreads();
    if (j + 1 < S) {
      smem_cas_init(d, s, smem);
      __syncthreads();
    }
  }
  if (st) atomicOr(d.status, st);
}

// ------------------------------------------------------------ launch
static int g_sm_count = 0;
static int sm_count() {
  if (!g_sm_count) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (g_sm_count <= 0) g_sm_count = 148;
  }
  return g_sm_count;
}


size_t pipeline_smem_bytes(const PipeDesc& d) {
  return (size_t)sink_area_bytes(d) +
         (size_t)kWarps * warp_area_bytes(stream_bytes_per_row(d), probed_source_count(d));
}

// Occupancy per (sink, dynamic smem) is computed once and cached: these
// queries cost host time on every launch otherwise.
static std::mutex g_occ_mu;
static std::map<std::pair<int, size_t>, int> g_occ;
static size_t g_smem_set[16];  // indexed by sink

template <int SINK>
static cudaError_t launch_sink(const PipeDesc& d, uint64_t n_hint, cudaStream_t s) {
  auto kern = k_pipeline<SINK>;
  const size_t smem = pipeline_smem_bytes(d);
  int blocks_per_sm = 0;
  {
    std::lock_guard<std::mutex> g(g_occ_mu);
    // static shared memory counts against the same 48 KB default, so the
    // opt-in limit is raised for any dynamic size not set before
    if (smem > g_smem_set[SINK]) {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      g_smem_set[SINK] = smem;
    }
    auto it = g_occ.find({SINK, smem});
    if (it != g_occ.end()) {
      blocks_per_sm = it->second;
    } else {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, kern, kThreads, smem) != cudaSuccess ||
          blocks_per_sm < 1) {
        cudaGetLastError();
        blocks_per_sm = 1;
      }
      g_occ[{SINK, smem}] = blocks_per_sm;
    }
  }
  // Grid = resident CTAs per SM x SM count (a persistent grid-stride
  // grid); the autotuner may ask for fewer CTAs per SM and for groups of
  // consecutive tiles per warp.
  const uint64_t G = d.tile_group > 1 ? (uint64_t)d.tile_group : 1;
  uint64_t tiles = (n_hint + (uint64_t)kTile * kWarps * G - 1) / ((uint64_t)kTile * kWarps * G);
  if (d.grid_per_sm > 0 && d.grid_per_sm < blocks_per_sm) blocks_per_sm = d.grid_per_sm;
  uint64_t max_grid = (uint64_t)sm_count() * (uint64_t)blocks_per_sm;
  uint64_t grid = tiles < max_grid ? tiles : max_grid;
  if (grid == 0) grid = 1;
  // both partition passes must give every CTA the same tiles
  if (SINK == SK_PART_COUNT || SINK == SK_PART_SCATTER) grid = (uint64_t)d.part_ctas;
  kern<<<(unsigned)grid, kThreads, smem, s>>>(d);
  return cudaGetLastError();
}

int part_max_bits() { return kMaxPartBits; }
int part_max_split() { return kMaxPartSplit; }
size_t pipeline_warp_tile_rows() { return kTile; }
int part_max_values() { return kPartMaxVals; }

// Both partition passes run this many CTAs (they must cover the same tiles):
// two per SM, which the scatter pass's shared memory allows.
int pipeline_part_ctas() { return 2 * sm_count(); }

cudaError_t launch_part_scan(const PipeDesc& d, cudaStream_t s) {
  if (d.part_bits < 1 || d.part_bits > kMaxPartBits) return cudaErrorInvalidValue;
  if (d.part_chunk == 0) return cudaErrorInvalidValue;
  k_part_scan<<<1, kScanThreads, 0, s>>>(d.part_counts, d.part_offsets, d.part_start, d.part_chunk_start, d.part_ctas,
                                         d.part_bits, d.part_chunk);
  return cudaGetLastError();
}

// ------------------------------------------------- two-pass compaction scan
// Between the two passes of the order-preserving compaction: the tiles'
// survivor counts (tile_pos) become offsets within their chunk of
// kMatScanTiles tiles, in place, and chunk_pos the rows before each chunk;
// out_count gets the total. Two launches, no waits between CTAs.
constexpr int kMatScanThreads = kMatScanTiles / 4;

__global__ void __launch_bounds__(kMatScanThreads) k_mat_scan_local(uint32_t* __restrict__ pos, uint64_t n_tiles,
                                                                     uint64_t* __restrict__ chunk_pos) {
  __shared__ uint32_t s_warp[kMatScanThreads / 32 + 1];
  const uint64_t base = (uint64_t)blockIdx.x * kMatScanTiles + (uint64_t)threadIdx.x * 4;
  uint32_t v[4], sum = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    v[i] = base + i < n_tiles ? pos[base + i] : 0u;
    sum += v[i];
  }
  uint32_t total;
  uint32_t run = block_excl_sum<kMatScanThreads>(sum, s_warp, &total);
#pragma unroll
  for (int i = 0; i < 4; ++i)
    if (base + i < n_tiles) {
      pos[base + i] = run;
      run += v[i];
    }
  if (threadIdx.x == 0) chunk_pos[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kMatScanThreads) k_mat_scan_chunks(uint64_t* __restrict__ chunk_pos,
                                                                      uint32_t n_chunks, uint64_t* out_count) {
  __shared__ uint64_t s_w[kMatScanThreads / 32];
  const uint32_t b = threadIdx.x * 4;
  uint64_t v[4], sum = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    v[i] = b + i < n_chunks ? chunk_pos[b + i] : 0ull;
    sum += v[i];
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) s_w[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint64_t w = s_w[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
      if (lane >= o) w += y;
    }
    s_w[lane] = w;  // inclusive over warps
  }
  __syncthreads();
  uint64_t run = (warp ? s_w[warp - 1] : 0ull) + incl - sum;
#pragma unroll
  for (int i = 0; i < 4; ++i)
    if (b + i < n_chunks) {
      chunk_pos[b + i] = run;
      run += v[i];
    }
  if (threadIdx.x == 0) *out_count = s_w[kMatScanThreads / 32 - 1];
}

// Survivor masks into row ids: one warp per tile at a time; for each of the
// tile's 8 mask words every lane writes its own row when its bit is set, at
// the word's offset plus the set bits below it, so each store instruction
// covers consecutive positions.
__global__ void __launch_bounds__(256) k_mat_expand(const uint32_t* __restrict__ mask,
                                                    const uint32_t* __restrict__ pos,
                                                    const uint64_t* __restrict__ chunk_pos, uint64_t n_tiles,
                                                    uint32_t* __restrict__ rid) {
  const uint32_t lane = threadIdx.x & 31, lt = (1u << lane) - 1u;
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  for (uint64_t tile = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); tile < n_tiles;
       tile += warps) {
    const uint32_t mw = lane < 8 ? mask[tile * 8 + lane] : 0u;
    uint64_t at = (uint64_t)pos[tile] + chunk_pos[tile / kMatScanTiles];
    const uint32_t row0 = (uint32_t)(tile * kTile);
#pragma unroll
    for (int w = 0; w < 8; ++w) {
      const uint32_t bits = __shfl_sync(0xFFFFFFFFu, mw, w);
      if ((bits >> lane) & 1u) rid[at + (uint64_t)__popc(bits & lt)] = row0 + (uint32_t)w * 32 + lane;
      at += (uint64_t)__popc(bits);
    }
  }
}

cudaError_t launch_mat_scan(const PipeDesc& d, uint64_t n_rows, cudaStream_t s) {
  const uint64_t n_tiles = (n_rows + kTile - 1) / kTile;
  const uint64_t n_chunks = (n_tiles + kMatScanTiles - 1) / kMatScanTiles;
  if (n_chunks > (uint64_t)kMatScanTiles) return cudaErrorInvalidValue;  // beyond 2^32 rows
  if (n_tiles) k_mat_scan_local<<<(unsigned)n_chunks, kMatScanThreads, 0, s>>>(d.tile_pos, n_tiles, d.chunk_pos);
  k_mat_scan_chunks<<<1, kMatScanThreads, 0, s>>>(d.chunk_pos, (uint32_t)n_chunks, d.out_count);
  if (d.tile_mask && n_tiles) {
    uint64_t blocks = (n_tiles + 7) / 8;
    if (blocks > (uint64_t)sm_count() * 8) blocks = (uint64_t)sm_count() * 8;
    k_mat_expand<<<(unsigned)blocks, 256, 0, s>>>(d.tile_mask, d.tile_pos, d.chunk_pos, n_tiles,
                                                  d.out_rids[d.drive_src]);
  }
  return cudaGetLastError();
}

size_t part_agg_smem_bytes(const PipeDesc& d) { return (size_t)d.smem_capacity * smem_cas_stride(d) * 8; }

cudaError_t launch_part_agg(const PipeDesc& d, uint64_t n_hint, cudaStream_t s) {
  if (d.part_chunk == 0) return cudaErrorInvalidValue;
  static std::mutex mu;
  static size_t smem_set = 0;
  const size_t smem = part_agg_smem_bytes(d);
  {
    std::lock_guard<std::mutex> g(mu);
    if (smem > smem_set) {
      cudaError_t e = cudaFuncSetAttribute(k_part_agg, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      smem_set = smem;
    }
  }
  if (d.part_split < 0 || d.part_split > kMaxPartSplit || (d.part_split > 0 && !d.part_sub))
    return cudaErrorInvalidValue;
  // at most records / chunk + one partial chunk per partition
  const uint64_t grid = n_hint / d.part_chunk + (1ull << d.part_bits);
  k_part_agg<<<(unsigned)grid, kPartAggThreads, smem, s>>>(d);
  return cudaGetLastError();
}

// ------------------------------------------------- one-pass few-group aggregation
// A one-key aggregate over few groups (all of them fit one CTA's
// shared-memory table) read straight from its columns in a single pass, with
// no intermediate records: a grouped aggregate over one table without
// filters or joins whose key and inputs are plain columns. Each thread reads
// kFewRows rows per step, one row per CTA-wide stripe so that every warp
// load is 32 consecutive rows, with all of a step's loads issued before any
// is used. A row finds its group in the CTA table (keys claimed by CAS;
// states in one array per aggregate, indexed like the keys); a warp's rows of
// one group are combined in registers first (match.any, log-step shuffles),
// so a group takes one shared-memory update per warp and step. The CTA's
// table is merged into the global table at the end.
constexpr int kFewThreads = 512;
constexpr int kFewRows = 4;
constexpr int kFewCols = 4;  // distinct input columns

__host__ __device__ inline uint32_t few_words(const PipeDesc& d) {
  uint32_t w = 1u + (uint32_t)d.n_aggs;
  for (int a = 0; a < d.n_aggs; ++a) w += d.aggs[a].fn == A_SUM_I128;
  return w;
}

__device__ __forceinline__ int few_find(uint64_t* keys, uint32_t cap, uint64_t key) {
  if ((int64_t)key == kEmptyKey) return -1;
  uint32_t idx = (uint32_t)hash_slot(key_hash1(key), (uint64_t)cap);
  for (uint32_t probe = 0; probe < cap; ++probe) {
    const uint64_t k = *(volatile uint64_t*)(keys + idx);
    if (k == key) return (int)idx;
    if ((int64_t)k == kEmptyKey) {
      const unsigned long long prev =
          atomicCAS((unsigned long long*)(keys + idx), (unsigned long long)kEmptyKey, (unsigned long long)key);
      if (prev == (unsigned long long)kEmptyKey || prev == key) return (int)idx;
    }
    if (++idx == cap) idx = 0;
  }
  return -1;
}

__global__ void __launch_bounds__(kFewThreads, 2) k_agg_few(const __grid_constant__ PipeDesc d) {
  extern __shared__ __align__(16) uint64_t fsm[];
  const uint32_t cap = (uint32_t)d.smem_capacity;
  const int na = d.n_aggs;
  uint64_t* const skey = fsm;
  uint64_t* const sst = fsm + cap;               // [aggregate][cap]
  uint64_t* const shi = sst + (size_t)na * cap;  // [128-bit sum][cap] high words
  // per aggregate: the row of its high words and its input column (-1: none)
  __shared__ int hidx[kMaxAggs], acol[kMaxAggs], vcol[kFewCols];
  __shared__ int s_ncol;
  int n128 = 0;
  for (int a = 0; a < na; ++a) n128 += d.aggs[a].fn == A_SUM_I128;
  if (threadIdx.x == 0) {
    int h = 0, nc = 0;
    for (int a = 0; a < kMaxAggs; ++a) {
      hidx[a] = (a < na && d.aggs[a].fn == A_SUM_I128) ? h++ : -1;
      acol[a] = -1;
      if (a >= na || d.aggs[a].prog < 0) continue;
      const int c = d.progs[d.aggs[a].prog].fast.leaf[0].arg;
      int f = -1;
      for (int j = 0; j < nc; ++j)
        if (vcol[j] == c) f = j;
      if (f < 0 && nc < kFewCols) {
        f = nc;
        vcol[nc++] = c;
      }
      acol[a] = f;
    }
    for (int j = nc; j < kFewCols; ++j) vcol[j] = 0;
    s_ncol = nc;
  }
  for (uint32_t i = threadIdx.x; i < cap; i += kFewThreads) {
    skey[i] = (uint64_t)kEmptyKey;
    for (int a = 0; a < na; ++a) {
      uint64_t v = 0;
      switch (d.aggs[a].fn) {
        case A_MIN_I: v = 0x7FFFFFFFFFFFFFFFULL; break;
        case A_MAX_I: v = 0x8000000000000000ULL; break;
        case A_MIN_F: v = ~0ULL; break;
        default: v = 0; break;
      }
      sst[(size_t)a * cap + i] = v;
    }
    for (int h = 0; h < n128; ++h) shi[(size_t)h * cap + i] = 0;
  }
  __syncthreads();
  const int ncol = s_ncol;
  const DCol kc = d.cols[d.progs[d.key_prog[0]].fast.leaf[0].arg];
  const uint64_t n = d.n;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  const DAggTable& tb = d.table;
  const uint64_t gstride = tb.stride > 1 ? (uint64_t)tb.stride : 1;
  uint32_t st = 0;
  const bool combinable = n128 == 0;
  const uint64_t step = (uint64_t)kFewThreads * kFewRows;
  for (uint64_t base = (uint64_t)blockIdx.x * step; base < n; base += (uint64_t)gridDim.x * step) {
    uint64_t key[kFewRows];
    int64_t val[kFewCols][kFewRows];
    bool act[kFewRows];
#pragma unroll
    for (int r = 0; r < kFewRows; ++r) {
      const uint64_t row = base + (uint64_t)r * kFewThreads + threadIdx.x;
      act[r] = row < n;
      const uint64_t rr = act[r] ? row : 0;
      key[r] = (uint64_t)load_bits(kc.ptr, kc.ptype, rr);
#pragma unroll
      for (int c = 0; c < kFewCols; ++c)
        val[c][r] = c < ncol ? load_bits(d.cols[vcol[c]].ptr, d.cols[vcol[c]].ptype, rr) : 0;
    }
#pragma unroll
    for (int r = 0; r < kFewRows; ++r) {
      const int slot = act[r] ? few_find(skey, cap, key[r]) : -1;
      // rows whose key has no CTA entry (the empty-slot sentinel key, or a
      // table fuller than planned) update the global table directly
      uint64_t g = kNoGroup;
      if (act[r] && slot < 0) g = agg_find_cas(tb, key[r], hash_slot(key_hash1(key[r]), tb.capacity), st);
      const uint32_t code = slot >= 0 ? (uint32_t)slot : 0xFFFFFFFFu;
      const unsigned peers = __match_any_sync(0xFFFFFFFFu, code);
      const bool comb = combinable && __any_sync(0xFFFFFFFFu, slot >= 0 && __popc(peers) >= 3);
      const bool lead = (peers & lt) == 0;
      for (int a = 0; a < na; ++a) {
        const DAgg& ag = d.aggs[a];
        const int c = acol[a];
        const int32_t vt = c >= 0 ? d.cols[vcol[c]].ptype : P_I64;
        Val v;
        v.lo = c == 0 ? val[0][r] : c == 1 ? val[1][r] : c == 2 ? val[2][r] : c == 3 ? val[3][r] : 0;
        v.hi = v.lo >> 63;
        const uint32_t sa = smem_u32(sst + (size_t)a * cap + (slot >= 0 ? slot : 0));
        const uint32_t sh = hidx[a] >= 0 ? smem_u32(shi + (size_t)hidx[a] * cap + (slot >= 0 ? slot : 0)) : 0;
        auto apply = [&](auto fnc) {
          constexpr int FN = decltype(fnc)::value;
          if (comb) {  // warp-uniform; every state is one word
            if (FN != A_SUM_I128) {
              const uint64_t x = peer_combine(FN, slot >= 0 ? peers : 0u, lane_state_value(FN, v, vt), lane);
              if (slot >= 0 && lead) smem_merge(FN, sa, x);
            }
          } else if (slot >= 0) {
            smem_apply(FN, sa, sh, v, vt);
          }
          if (slot < 0 && g != kNoGroup) {
            const uint64_t o = g * gstride;
            agg_apply_g(FN, (unsigned long long*)ag.lo + o, ag.hi ? (long long*)ag.hi + o : nullptr, v, vt);
          }
        };
        dispatch_fn(ag.fn, apply);
      }
    }
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < cap; i += kFewThreads) {
    const uint64_t key = skey[i];
    if ((int64_t)key == kEmptyKey) continue;
    const uint64_t g = agg_find_cas(tb, key, hash_slot(key_hash1(key), tb.capacity), st);
    if (g == kNoGroup) continue;
    const uint64_t o = g * gstride;
    for (int a = 0; a < na; ++a) {
      const DAgg& ag = d.aggs[a];
      const int64_t hv = hidx[a] >= 0 ? (int64_t)shi[(size_t)hidx[a] * cap + i] : 0;
      agg_merge(ag.fn, (unsigned long long*)(ag.lo + o), (long long*)(ag.hi ? ag.hi + o : nullptr),
                sst[(size_t)a * cap + i], hv);
    }
  }
  if (st) atomicOr(d.status, st);
}

size_t agg_few_smem_bytes(const PipeDesc& d) { return (size_t)d.smem_capacity * few_words(d) * 8; }

int agg_few_max_cols() { return kFewCols; }

cudaError_t launch_agg_few(const PipeDesc& d, uint64_t n_hint, cudaStream_t s) {
  if (d.smem_capacity <= 0) return cudaErrorInvalidValue;
  static std::mutex mu;
  static size_t smem_set = 0;
  static std::map<size_t, int> occ;
  const size_t smem = agg_few_smem_bytes(d);
  int per_sm = 1;
  {
    std::lock_guard<std::mutex> g(mu);
    if (smem > smem_set) {
      cudaError_t e = cudaFuncSetAttribute(k_agg_few, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      smem_set = smem;
    }
    auto it = occ.find(smem);
    if (it != occ.end()) {
      per_sm = it->second;
    } else {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_agg_few, kFewThreads, smem) != cudaSuccess ||
          per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
      }
      occ[smem] = per_sm;
    }
  }
  if (d.grid_per_sm > 0 && d.grid_per_sm < per_sm) per_sm = d.grid_per_sm;
  const uint64_t steps = (n_hint + (uint64_t)kFewThreads * kFewRows - 1) / ((uint64_t)kFewThreads * kFewRows);
  uint64_t grid = (uint64_t)sm_count() * (uint64_t)per_sm;
  if (steps < grid) grid = steps ? steps : 1;
  k_agg_few<<<(unsigned)grid, kFewThreads, smem, s>>>(d);
  return cudaGetLastError();
}

cudaError_t launch_pipeline(const PipeDesc& d, uint64_t n_hint, cudaStream_t s) {
  if (d.tuple_input) return cudaErrorInvalidValue;  // every pipeline scans a base table
  switch (d.sink) {
    case SK_BUILD: return launch_sink<SK_BUILD>(d, n_hint, s);
    case SK_MATERIALIZE:
      return d.mat_warp_tiles ? launch_sink<SK_MATERIALIZE>(d, n_hint, s) : launch_pipeline_materialize(d, n_hint, s);
    case SK_MAT_COUNT: return launch_sink<SK_MAT_COUNT>(d, n_hint, s);
    case SK_MAT_WRITE: return launch_sink<SK_MAT_WRITE>(d, n_hint, s);
    case SK_AGG_HASH: return launch_sink<SK_AGG_HASH>(d, n_hint, s);
    case SK_AGG_SMEM: return launch_sink<SK_AGG_SMEM>(d, n_hint, s);
    case SK_AGG_SLOT: return launch_sink<SK_AGG_SLOT>(d, n_hint, s);
    case SK_AGG_SCALAR: return launch_sink<SK_AGG_SCALAR>(d, n_hint, s);
    case SK_PART_COUNT: return launch_sink<SK_PART_COUNT>(d, n_hint, s);
    case SK_PART_SCATTER: return launch_sink<SK_PART_SCATTER>(d, n_hint, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace mtl
