// k_pipeline_cta.cu — the fused scan pipeline with CTA-wide tiles (sm_100a),
// used for order-preserving compaction (SK_MATERIALIZE): a 1024-row tile per
// CTA keeps the decoupled look-back to one step per 1024 rows. The other
// sinks run the warp-autonomous kernel of k_pipeline.cu.
//
// Original notes:
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
namespace cta {

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

// Finds or claims kw in the CTA table; -1 when it is not among the first
// kSmemProbes slots of its chain (the caller then uses the global table), so
// a full table costs a bounded number of probes per row.
constexpr int kSmemProbes = 4;
__device__ __forceinline__ int smem_agg_find(const PipeDesc& d, SmemAgg& s, const uint64_t* kw, uint32_t& st) {
  const int nk = d.table.n_keys;
  int idx = (int)hash_slot(key_hash(kw, nk), (uint64_t)s.cap);
  const int probes = s.cap < kSmemProbes ? s.cap : kSmemProbes;
  for (int probe = 0; probe < probes; ++probe) {
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

// ------------------------------------------------------------ the kernel
constexpr int kThreads = 128;
constexpr int kTile = 1024;  // tuples per tile

struct StreamLayout {
  int n;
  int col[4];
  int width[4];
  uint32_t off[4];
  uint32_t bytes;  // per buffer
};

__host__ __device__ inline uint32_t stream_bytes_per_row(const PipeDesc& d) {
  uint32_t w = 0;
  for (int i = 0; i < d.n_stream && i < 4; ++i) w += (uint32_t)ptype_width(d.cols[d.stream_cols[i]].ptype);
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
  for (int i = 0; i < 4; ++i)
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

// Expression VM over one tile row.
__device__ __forceinline__ Val vm_eval_t(const VmProg& p, const TileCtx& t, uint32_t r, uint32_t& st) {
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

// Warp-aggregated append of tile row r to a shared selection list. Every
// lane of the warp must call it (keep may be false).
__device__ __forceinline__ void sel_push(bool keep, uint32_t r, uint16_t* out, uint32_t* cnt) {
  const uint32_t m = __ballot_sync(0xFFFFFFFFu, keep);
  const int lane = threadIdx.x & 31;
  uint32_t base = 0;
  if (lane == 0 && m) base = atomicAdd(cnt, (uint32_t)__popc(m));
  base = __shfl_sync(0xFFFFFFFFu, base, 0);
  if (keep) out[base + __popc(m & ((1u << lane) - 1u))] = (uint16_t)r;
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

// Filter op over the current selection: one loop per (column type, source),
// chosen once per tile. A thread evaluates all of its (at most kTile /
// kThreads) rows before the first ballot, so their loads are in flight
// together, and each warp reserves its output range with one atomic.
template <typename GET>
__device__ __forceinline__ void filter_loop(uint32_t n_sel, bool ident, const uint16_t* in, uint16_t* out,
                                            uint32_t* cnt, GET get_keep) {
  constexpr int U = kTile / kThreads;
  const int lane = threadIdx.x & 31;
  uint32_t km = 0;  // bit j: row j of this thread is kept
#pragma unroll
  for (int j = 0; j < U; ++j) {
    const uint32_t i = (uint32_t)j * kThreads + threadIdx.x;
    if (i < n_sel && get_keep(ident ? i : (uint32_t)in[i])) km |= 1u << j;
  }
  uint32_t tot = 0;
#pragma unroll
  for (int j = 0; j < U; ++j) tot += __popc(__ballot_sync(0xFFFFFFFFu, (km >> j) & 1u));
  uint32_t base = 0;
  if (lane == 0 && tot) base = atomicAdd(cnt, tot);
  base = __shfl_sync(0xFFFFFFFFu, base, 0);
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int j = 0; j < U; ++j) {
    const uint32_t m = __ballot_sync(0xFFFFFFFFu, (km >> j) & 1u);
    if ((km >> j) & 1u) {
      const uint32_t i = (uint32_t)j * kThreads + threadIdx.x;
      out[base + __popc(m & lt)] = (uint16_t)(ident ? i : (uint32_t)in[i]);
    }
    base += __popc(m);
  }
}

// First filter of a tile on a streamed integer column: thread t owns the
// kTile / kThreads consecutive rows starting at t * (kTile / kThreads),
// reads them with 128-bit shared-memory loads, and writes the rows it keeps
// in order after a warp prefix sum, so the selection comes out sorted within
// each warp's range.
template <typename T>
__device__ __forceinline__ void filter_ident_blocked(const T* col, uint32_t nrow, const IntRange& rg, uint16_t* out,
                                                     uint32_t* cnt) {
  constexpr int U = kTile / kThreads;
  static_assert(U * sizeof(T) % 16 == 0, "rows per thread must fill whole 16-byte vectors");
  const int lane = threadIdx.x & 31;
  const uint32_t b0 = threadIdx.x * U;
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
  const uint32_t tot = __shfl_sync(0xFFFFFFFFu, incl, 31);
  uint32_t base = 0;
  if (lane == 0 && tot) base = atomicAdd(cnt, tot);
  uint32_t pos = __shfl_sync(0xFFFFFFFFu, base, 0) + incl - c;
#pragma unroll
  for (int j = 0; j < U; ++j)
    if ((km >> j) & 1u) out[pos++] = (uint16_t)(b0 + j);
}

// Join probe over the current selection, kProbeBatch rows per thread at a
// time: keys, then the presence words and map entries (dense) or first
// probed slots (hash) of the whole batch are loaded before any is used.
constexpr int kProbeBatch = 4;
constexpr int kAggBatch = 4;  // rows per thread in flight in the single-key hash sink

template <int SINK>
__global__ void __launch_bounds__(kThreads) k_pipeline(const __grid_constant__ PipeDesc d) {
  constexpr int THREADS = kThreads, TILE = kTile;
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t s_mbar[2];
  __shared__ uint32_t s_warp[THREADS / 32 + 1];
  __shared__ uint64_t s_base;
  __shared__ uint64_t s_tile[2];
  __shared__ uint32_t s_cnt[3];
  __shared__ uint64_t s_red[SINK == SK_AGG_SCALAR ? kMaxAggs : 1][THREADS / 32];
  __shared__ int64_t s_redhi[SINK == SK_AGG_SCALAR ? kMaxAggs : 1][THREADS / 32];

  const int tid = threadIdx.x;
  const uint64_t n = d.in_count ? *d.in_count : d.n;
  const uint64_t n_tiles = (n + TILE - 1) / TILE;
  uint32_t st = 0;

  StreamLayout S;
  S.n = d.n_stream < 4 ? d.n_stream : 4;
  {
    uint32_t off = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
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
  // shared layout: stream buffers x2 | sel A | sel B | slot | rid arrays | sink
  uint8_t* const sbuf0 = smem;
  uint8_t* const sbuf1 = smem + S.bytes;
  uint16_t* const selA = (uint16_t*)(smem + 2 * S.bytes);
  uint16_t* const selB = selA + TILE;
  uint32_t* const s_slot = (uint32_t*)(selB + TILE);
  uint32_t* const s_srid = s_slot + TILE;
  uint8_t* const sink_smem = (uint8_t*)(s_srid + (size_t)nq * TILE);
  uint8_t* s_keep = sink_smem;                       // MATERIALIZE
  uint16_t* s_list = (uint16_t*)(sink_smem + TILE);  // MATERIALIZE

  SmemAgg sagg;
  if (SINK == SK_AGG_SMEM) smem_agg_init(d, sagg, sink_smem);
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
  if (tid == 0) {
    if (S.n) {
      mbar_init(&s_mbar[0], 1);
      mbar_init(&s_mbar[1], 1);
      mbar_fence_init();
    }
    s_cnt[0] = s_cnt[1] = s_cnt[2] = 0;
  }

  const bool dynamic_tiles = SINK == SK_MATERIALIZE;
  // Thread 0 stages the streamed columns of a full tile into buffer `b`.
  auto issue = [&](uint64_t tile, int b) {
    const uint64_t base = tile * (uint64_t)TILE;
    if (base + TILE > n) return;  // the tail tile is loaded directly
    uint8_t* dst = b ? sbuf1 : sbuf0;
    fence_proxy_async();
    mbar_arrive_expect_tx(&s_mbar[b], S.bytes);
    for (int i = 0; i < S.n; ++i)
      bulk_g2s(dst + S.off[i], (const uint8_t*)d.cols[S.col[i]].ptr + base * (uint64_t)S.width[i],
               (uint32_t)TILE * (uint32_t)S.width[i], &s_mbar[b]);
  };

  if (tid == 0) s_tile[0] = dynamic_tiles ? (uint64_t)atomicAdd(d.tile_counter, 1u) : (uint64_t)blockIdx.x;
  __syncthreads();
  uint64_t cur = s_tile[0];
  if (tid == 0 && S.n && cur < n_tiles) issue(cur, 0);
  uint32_t parity = 0;
  int b = 0;
  uint32_t k = 0;
  uint32_t cq = 0;  // selection-counter rotation
  while (cur < n_tiles) {
    if (tid == 0) {
      const uint64_t nx = dynamic_tiles ? (uint64_t)atomicAdd(d.tile_counter, 1u) : cur + gridDim.x;
      s_tile[(k + 1) & 1] = nx;
      if (S.n && nx < n_tiles) issue(nx, b ^ 1);
    }
    const uint64_t tile = cur;
    const uint64_t tile_base = tile * (uint64_t)TILE;
    const uint32_t nrow = (uint32_t)(n - tile_base < (uint64_t)TILE ? n - tile_base : (uint64_t)TILE);
    uint8_t* const buf = b ? sbuf1 : sbuf0;
    if (S.n) {
      bool ok = true;
      if (nrow == TILE) {
        ok = mbar_wait(&s_mbar[b], (parity >> b) & 1u);
        parity ^= 1u << b;
      } else {
        for (int i = 0; i < S.n; ++i) {
          const DCol& c = d.cols[S.col[i]];
          for (int r = tid; r < TILE; r += THREADS) {
            int64_t v = (uint32_t)r < nrow ? load_bits(c.ptr, c.ptype, tile_base + r) : 0;
            if (S.width[i] == 4) ((uint32_t*)(buf + S.off[i]))[r] = (uint32_t)v;
            else ((int64_t*)(buf + S.off[i]))[r] = v;
          }
        }
      }
      if (__syncthreads_or(!ok)) {
        st |= ST_SPIN_LIMIT;
        // give the copy still in flight a bounded chance to land, then stop
        mbar_wait(&s_mbar[b ^ 1], (parity >> (b ^ 1)) & 1u);
        break;
      }
    }
    TileCtx tc{&d, &S, buf, tile_base, s_srid, slot_of_src};

    // ---- ops over the selection vector
    uint32_t n_sel = nrow;
    bool ident = true;
    uint16_t* sel_in = selA;
    uint16_t* sel_out = selB;
    for (int o = 0; o < d.n_ops && n_sel > 0; ++o) {
      uint32_t* cnt = &s_cnt[cq];
      if (tid == 0) s_cnt[(cq + 1) % 3] = 0;  // next op's counter (last read two barriers ago)
      const PipeOp op = d.ops[o];
      if (op.kind == OPK_FILTER) {
        const DPred& p = d.preds[op.idx];
        const DCol& c = d.cols[p.col];
        const int si = (c.src == d.drive_src) ? stream_index(S, p.col) : -1;
        if (c.ptype == P_I32 || c.ptype == P_I64) {
          const IntRange rg = to_range(p);
          if (rg.none) {
            filter_loop(n_sel, ident, sel_in, sel_out, cnt, [&](uint32_t) { return false; });
          } else if (si >= 0 && ident && S.width[si] == 4 && c.ptype == P_I32) {
            filter_ident_blocked<int32_t>((const int32_t*)(buf + S.off[si]), n_sel, rg, sel_out, cnt);
          } else if (si >= 0 && ident && S.width[si] == 8) {
            filter_ident_blocked<int64_t>((const int64_t*)(buf + S.off[si]), n_sel, rg, sel_out, cnt);
          } else if (si >= 0 && S.width[si] == 4) {
            const int32_t* col = (const int32_t*)(buf + S.off[si]);
            filter_loop(n_sel, ident, sel_in, sel_out, cnt, [&](uint32_t r) {
              const int64_t x = col[r];
              return (x >= rg.lo && x <= rg.hi) != rg.neg;
            });
          } else if (si >= 0) {
            const int64_t* col = (const int64_t*)(buf + S.off[si]);
            filter_loop(n_sel, ident, sel_in, sel_out, cnt, [&](uint32_t r) {
              const int64_t x = col[r];
              return (x >= rg.lo && x <= rg.hi) != rg.neg;
            });
          } else {
            filter_loop(n_sel, ident, sel_in, sel_out, cnt, [&](uint32_t r) {
              const int64_t x = load_bits(c.ptr, c.ptype, tc_rid(tc, c.src, r));
              return (x >= rg.lo && x <= rg.hi) != rg.neg;
            });
          }
        } else {
          filter_loop(n_sel, ident, sel_in, sel_out, cnt, [&](uint32_t r) {
            return eval_pred_bits(tc_get(tc, p.col, r), c.ptype, p);
          });
        }
      } else {
        const DProbe& pr = d.probes[op.idx];
        const DCol& c = d.cols[pr.key_col];
        const DBuild& bd = d.builds[pr.build];
        const bool want_slot = op.idx == d.slot_probe;
        const uint32_t fill = pr.fill_mask & ~(1u << d.drive_src);
        const int lane = tid & 31;
        const uint32_t lt = (1u << lane) - 1u;
        const ColAcc ka = col_acc(tc, pr.key_col);
        const bool k32 = ka.sm && ka.width == 4 && ka.ptype == P_I32;  // streamed INTEGER key
        // Descriptor fields used per row, read once: the loop's shared-memory
        // stores would otherwise force reloads through the descriptor.
        const int64_t b_kmin = bd.key_min;
        const uint64_t b_cap = bd.capacity;
        const uint32_t* const b_bits = bd.dense_bits;
        const uint32_t* const b_map = bd.dense_map;
        const bool b_dense = bd.kind == B_DENSE;
        (void)c;
        for (uint32_t i0 = 0; i0 < n_sel; i0 += THREADS * kProbeBatch) {
          uint32_t r[kProbeBatch], slot[kProbeBatch];
          bool act[kProbeBatch], keep[kProbeBatch];
          int64_t key[kProbeBatch];
#pragma unroll
          for (int j = 0; j < kProbeBatch; ++j) {
            const uint32_t i = i0 + (uint32_t)j * THREADS + tid;
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
          uint32_t m[kProbeBatch];
          uint32_t tot = 0;
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
            m[j] = __ballot_sync(0xFFFFFFFFu, keep[j]);
            tot += __popc(m[j]);
          }
          uint32_t obase = 0;
          if (lane == 0 && tot) obase = atomicAdd(cnt, tot);
          obase = __shfl_sync(0xFFFFFFFFu, obase, 0);
#pragma unroll
          for (int j = 0; j < kProbeBatch; ++j) {
            if (keep[j]) sel_out[obase + __popc(m[j] & lt)] = (uint16_t)r[j];
            obase += __popc(m[j]);
          }
        }
      }
      __syncthreads();
      n_sel = *cnt;
      ident = false;
      uint16_t* t_ = sel_in;
      sel_in = sel_out;
      sel_out = t_;
      cq = (cq + 1) % 3;
    }

    // ---- sink over the surviving tile rows
    if (SINK == SK_MATERIALIZE) {
      for (int r = tid; r < TILE; r += THREADS) s_keep[r] = 0;
      __syncthreads();
      for (uint32_t i = tid; i < n_sel; i += THREADS) s_keep[ident ? i : sel_in[i]] = 1;
      __syncthreads();
      // Blocked arrangement for the scan: thread t owns tile rows [t*8, (t+1)*8).
      constexpr int PER = TILE / THREADS;
      uint32_t cntk = 0;
#pragma unroll
      for (int i = 0; i < PER; ++i) cntk += s_keep[tid * PER + i];
      uint32_t total;
      uint32_t pos = block_excl_sum<THREADS>(cntk, s_warp, &total);
#pragma unroll
      for (int i = 0; i < PER; ++i)
        if (s_keep[tid * PER + i]) s_list[pos++] = (uint16_t)(tid * PER + i);
      if (tid < 32) {
        const uint64_t excl = lb_exclusive_warp(d.tile_status, tile, total, d.epoch, d.status,
                                                d.lb_spin_limit ? d.lb_spin_limit : kSpinLimit, !d.lb_stall_first);
        if (tid == 0) {
          s_base = excl;
          if (tile == n_tiles - 1) *d.out_count = excl + total;
        }
      }
      __syncthreads();
      const uint64_t base = s_base;
      // write phase: one output column at a time over the compacted rows
      const uint32_t lim = base >= d.out_capacity ? 0u
                           : (uint32_t)(d.out_capacity - base < (uint64_t)total ? d.out_capacity - base : total);
      if (lim < total) st |= ST_CAPACITY;
      for (int q = 0; q < d.n_out; ++q) {
        const VmProg& pg = d.progs[d.out_prog[q]];
        void* out = d.out_ptr[q];
        const int32_t ot = pg.out_type;
        if (pg.n == 1 && pg.ins[0].op == VM_COL) {
          // plain column: typed copy
          const ColAcc ca = col_acc(tc, pg.ins[0].arg);
#pragma unroll 4
          for (uint32_t p = tid; p < lim; p += THREADS) {
            Val v;
            v.lo = acc_get(ca, tc, s_list[p]);
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
          for (uint32_t p = tid; p < lim; p += THREADS) {
            Val v;
            v.lo = acc_get(ca, tc, s_list[p]);
            v.hi = v.lo >> 63;
            store_val(out, ot, base + p, vm_arith(aop, aty, v, kc, st));
          }
        } else {
          for (uint32_t p = tid; p < lim; p += THREADS) store_val(out, ot, base + p, vm_eval_t(pg, tc, s_list[p], st));
        }
      }
      for (int s = 0; s < kMaxSrc; ++s)
        if ((d.out_rid_mask >> s) & 1u)
          for (uint32_t p = tid; p < lim; p += THREADS) d.out_rids[s][base + p] = tc_rid(tc, s, s_list[p]);
    } else if (SINK == SK_BUILD) {
      const DBuild& bd = d.builds[d.sink_build];
      // A build row's slot is its row number in the build table.
      for (uint32_t i = tid; i < n_sel; i += THREADS) {
        const uint32_t r = ident ? i : (uint32_t)sel_in[i];
        const uint32_t slot = (uint32_t)(tc.base + r);
        const int64_t key = tc_get(tc, d.build_key_col, r);
        for (int s = 0; s < kMaxSrc; ++s)
          if (s != d.drive_src && ((d.build_payload_mask >> s) & 1u)) bd.payload[s][slot] = tc_rid(tc, s, r);
        for (int a = 0; a < d.n_aggs; ++a) agg_init_global(d.aggs[a], slot);
        build_insert(bd, key, slot, st);
      }
    } else if ((SINK == SK_AGG_HASH || SINK == SK_AGG_SMEM) && d.table.cas) {
      // One 64-bit group key: kAggBatch rows per thread at a time. Keys held
      // in the CTA's shared-memory table are updated there; for the others
      // the first probed global key words are read together, and states are
      // updated with atomics whose results are not waited for.
      constexpr int B = kAggBatch;
      const DAggTable& tb = d.table;
      const VmProg& kp = d.progs[d.key_prog[0]];
      const uint64_t gstride = tb.stride > 1 ? (uint64_t)tb.stride : 1;
      const uint64_t* const gkeys = tb.keys[0];
      const uint64_t gcap = tb.capacity;
      for (uint32_t i0 = 0; i0 < n_sel; i0 += THREADS * B) {
        uint32_t r[B];
        bool act[B];
        int sidx[B];
        uint64_t key[B], h[B], k0[B], g[B];
#pragma unroll
        for (int b = 0; b < B; ++b) {
          const uint32_t i = i0 + (uint32_t)b * THREADS + tid;
          act[b] = i < n_sel;
          r[b] = act[b] ? (ident ? i : (uint32_t)sel_in[i]) : 0u;
          key[b] = act[b] ? (uint64_t)vm_eval_t(kp, tc, r[b], st).lo : 0;
        }
#pragma unroll
        for (int b = 0; b < B; ++b) {
          sidx[b] = -1;
          if (SINK == SK_AGG_SMEM && act[b]) {
            const uint64_t kw[kMaxKeys] = {key[b], 0, 0, 0};
            sidx[b] = smem_agg_find(d, sagg, kw, st);
          }
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
        }
        for (int a = 0; a < d.n_aggs; ++a) {
          const DAgg& ag = d.aggs[a];
          const int32_t vt = ag.prog >= 0 ? d.progs[ag.prog].out_type : P_I64;
          Val v[B];
#pragma unroll
          for (int b = 0; b < B; ++b) {
            v[b] = Val{0, 0};
            if (ag.prog >= 0 && (sidx[b] >= 0 || g[b] != kNoGroup)) v[b] = vm_eval_t(d.progs[ag.prog], tc, r[b], st);
          }
#pragma unroll
          for (int b = 0; b < B; ++b) {
            if (SINK == SK_AGG_SMEM && sidx[b] >= 0) {
              long long* hp = sagg.hi_index[a] >= 0
                                  ? (long long*)(sagg.hi + (size_t)sagg.hi_index[a] * sagg.cap + sidx[b])
                                  : nullptr;
              agg_apply(ag.fn, (unsigned long long*)(sagg.lo + (size_t)a * sagg.cap + sidx[b]), hp, v[b], vt);
            } else if (g[b] != kNoGroup) {
              const uint64_t o = g[b] * gstride;
              agg_apply_g(ag.fn, (unsigned long long*)(ag.lo + o), (long long*)(ag.hi ? ag.hi + o : nullptr), v[b],
                          vt);
            }
          }
        }
      }
    } else {
      uint8_t* const slot_hit = d.slot_hit;
      for (uint32_t i = tid; i < n_sel; i += THREADS) {
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
    // Every thread is done with `buf`, the selection and the sink scratch.
    __syncthreads();
    cur = s_tile[(k + 1) & 1];
    ++k;
    b ^= 1;
  }

  // End-of-kernel work.
  if (SINK == SK_MATERIALIZE) {
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
  } else if (SINK == SK_AGG_SMEM) {
    __syncthreads();
    for (int i = tid; i < sagg.cap; i += THREADS) {
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
    const int lane = tid & 31, warp = tid >> 5;
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
      for (int w = 0; w < THREADS / 32; ++w)
        agg_merge(ag.fn, (unsigned long long*)ag.lo, (long long*)ag.hi, s_red[tid][w], s_redhi[tid][w]);
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



static int probed_sources(const PipeDesc& d) {
  int nq = 0;
  for (int s = 0; s < kMaxSrc; ++s) {
    if (s == d.drive_src) continue;
    bool used = false;
    for (int p = 0; p < d.n_probes; ++p) used |= ((d.probes[p].fill_mask >> s) & 1u) != 0;
    nq += used;
  }
  return nq;
}

size_t cta_smem_bytes(const PipeDesc& d) {
  constexpr size_t TILE = kTile;
  size_t s = 2ull * TILE * stream_bytes_per_row(d);  // stream buffers
  s += 2 * TILE * 2;                                  // selection vectors
  s += TILE * 4;                                      // probe slots
  s += (size_t)probed_sources(d) * TILE * 4;          // probed row ids
  if (d.sink == SK_MATERIALIZE) s += TILE + 2 * TILE;  // keep flags + compacted list
  if (d.sink == SK_AGG_SMEM) {
    size_t n128 = 0;
    for (int a = 0; a < d.n_aggs; ++a) n128 += d.aggs[a].fn == A_SUM_I128;
    s += (size_t)d.smem_capacity * (4 + 8 * d.table.n_keys + 8 * d.n_aggs + 8 * n128);
  }
  return s;
}

// Occupancy per (sink, dynamic smem) is computed once and cached: these
// queries cost host time on every launch otherwise.
static std::mutex g_occ_mu;
static std::map<std::pair<int, size_t>, int> g_occ;
static size_t g_smem_set[8];

template <int SINK>
static cudaError_t launch_sink(const PipeDesc& d, uint64_t n_hint, cudaStream_t s) {
  auto kern = k_pipeline<SINK>;
  const size_t smem = cta_smem_bytes(d);
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
  // Grid = resident CTAs per SM x SM count (a persistent grid-stride grid);
  // the autotuner may ask for fewer CTAs per SM.
  if (d.grid_per_sm > 0 && d.grid_per_sm < blocks_per_sm) blocks_per_sm = d.grid_per_sm;
  uint64_t tiles = (n_hint + kTile - 1) / kTile;
  uint64_t max_grid = (uint64_t)sm_count() * (uint64_t)blocks_per_sm;
  uint64_t grid = tiles < max_grid ? tiles : max_grid;
  if (grid == 0) grid = 1;
  kern<<<(unsigned)grid, kThreads, smem, s>>>(d);
  return cudaGetLastError();
}

}  // namespace cta

size_t pipeline_tile_rows() { return cta::kTile; }
cudaError_t launch_pipeline_materialize(const PipeDesc& d, uint64_t n_hint, cudaStream_t s) {
  return cta::launch_sink<SK_MATERIALIZE>(d, n_hint, s);
}

}  // namespace mtl
