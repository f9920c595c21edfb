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

#include "kern_common.cuh"
#include "kernels.h"

namespace cg = cooperative_groups;

namespace mtl {

// ------------------------------------------------------------ join build/probe
__device__ __forceinline__ bool build_lookup(const DBuild& b, int64_t key, uint32_t& slot, uint32_t& st) {
  if (b.kind == B_DENSE) {
    uint64_t k = (uint64_t)(key - b.key_min);
    if (k >= b.capacity) return false;
    uint32_t v = b.dense_map[k];
    if (v == 0) return false;
    slot = v - 1;
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
    if (atomicCAS(b.dense_map + k, 0u, slot + 1) != 0u) st |= ST_DUP_BUILD_KEY;
    return;
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

// Finds or claims the group of key words kw in a global table. Returns
// capacity on failure (table full or wait limit), with status set.
__device__ uint64_t agg_find_global(const PipeDesc& d, const uint64_t* kw, uint32_t& st) {
  const DAggTable& t = d.table;
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
        return t.capacity;
      }
      s = ld_acquire32(t.state + idx);
    }
    bool eq = true;
    for (int i = 0; i < t.n_keys; ++i) eq &= (t.keys[i][idx] == kw[i]);
    if (eq) return idx;
    if (++idx == t.capacity) idx = 0;
  }
  st |= ST_TABLE_FULL;
  return t.capacity;
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

// Finds or claims kw in the CTA table; -1 when the table is full.
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

// ------------------------------------------------------------ the kernel
constexpr int kThreads = 256;
constexpr int kItems = 8;
constexpr int kTile = kThreads * kItems;  // tuples per tile
constexpr int kBatch = 4;                 // tuples a thread advances through the ops together
constexpr int kAggCols = 4;               // sink columns fetched ahead in phase A
constexpr int kOutCols = 6;               // output columns fetched ahead in the write phase

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

// SINK is a compile-time constant so each instantiation carries only its own
// sink code. Tiles: tuple ti of a tile is handled by thread ti % 256 (striped),
// which keeps shared-memory reads conflict free. The streamed columns of the
// next tile are copied into the idle shared buffer by one thread with bulk
// (TMA) copies while the CTA works on the current tile. Other columns are
// read for a batch of kBatch tuples at once so their loads overlap.
template <int SINK>
__global__ void __launch_bounds__(kThreads) k_pipeline(const __grid_constant__ PipeDesc d) {
  constexpr int THREADS = kThreads, ITEMS = kItems, TILE = kTile;
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ __align__(8) uint64_t s_mbar[2];
  __shared__ uint32_t s_warp[THREADS / 32 + 1];
  __shared__ uint64_t s_base;
  __shared__ uint64_t s_tile[2];
  __shared__ uint64_t s_red[SINK == SK_AGG_SCALAR ? kMaxAggs : 1][THREADS / 32];
  __shared__ int64_t s_redhi[SINK == SK_AGG_SCALAR ? kMaxAggs : 1][THREADS / 32];

  const int tid = threadIdx.x;
  const uint64_t n = d.in_count ? *d.in_count : d.n;
  const uint64_t n_tiles = (n + TILE - 1) / TILE;
  uint32_t st = 0;

  StreamLayout S;
  S.n = d.tuple_input ? 0 : (d.n_stream < 4 ? d.n_stream : 4);
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
  uint8_t* const sbuf0 = smem;
  uint8_t* const sbuf1 = smem + S.bytes;
  uint8_t* const sink_smem = smem + 2 * S.bytes;

  // MATERIALIZE shared memory: keep flags | compacted tile list | row ids
  uint8_t* s_keep = sink_smem;
  uint16_t* s_list = (uint16_t*)(sink_smem + TILE);
  uint32_t* s_rid = (uint32_t*)(sink_smem + 3 * TILE);
  int rid_slot[kMaxSrc];
  {
    int q = 0;
#pragma unroll
    for (int s = 0; s < kMaxSrc; ++s) {
      bool implicit = !d.tuple_input && s == d.drive_src;
      rid_slot[s] = ((d.mat_src_mask >> s) & 1u) && !implicit ? q++ : -1;
    }
  }
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
  if (tid == 0 && S.n) {
    mbar_init(&s_mbar[0], 1);
    mbar_init(&s_mbar[1], 1);
    mbar_fence_init();
  }

  const bool dynamic_tiles = SINK == SK_MATERIALIZE;
  // Thread 0 stages the streamed columns of a full tile into buffer `b`.
  auto issue = [&](uint64_t tile, int b) {
    const uint64_t base = tile * (uint64_t)TILE;
    if (base + TILE > n) return;  // the tail tile is loaded directly
    uint8_t* dst = b ? sbuf1 : sbuf0;
    fence_proxy_async();
    mbar_arrive_expect_tx(&s_mbar[b], S.bytes);
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if (i < S.n)
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
  while (cur < n_tiles) {
    // Claim the next tile and start its copies before waiting on this one.
    uint64_t nxt_static = cur + gridDim.x;
    if (tid == 0) {
      uint64_t nx = dynamic_tiles ? (uint64_t)atomicAdd(d.tile_counter, 1u) : nxt_static;
      s_tile[(k + 1) & 1] = nx;
      if (S.n && nx < n_tiles) issue(nx, b ^ 1);
    }
    const uint64_t tile = cur;
    const uint64_t tile_base = tile * (uint64_t)TILE;
    uint8_t* const buf = b ? sbuf1 : sbuf0;
    if (S.n) {
      bool ok = true;
      if (tile_base + TILE <= n) {
        ok = mbar_wait(&s_mbar[b], (parity >> b) & 1u);
        parity ^= 1u << b;
      } else {
        for (int i = 0; i < S.n; ++i) {
          const DCol& c = d.cols[S.col[i]];
          for (int r = tid; r < TILE; r += THREADS) {
            const uint64_t g = tile_base + r;
            int64_t v = g < n ? load_bits(c.ptr, c.ptype, g) : 0;
            if (S.width[i] == 4) ((uint32_t*)(buf + S.off[i]))[r] = (uint32_t)v;
            else ((int64_t*)(buf + S.off[i]))[r] = v;
          }
        }
      }
      if (__syncthreads_or(!ok)) {
        st |= ST_SPIN_LIMIT;
        // give the copies still in flight a bounded chance to land, then stop
        mbar_wait(&s_mbar[b ^ 1], (parity >> (b ^ 1)) & 1u);
        break;
      }
    }

    // Value of column `col` for a tuple: shared memory when it is a streamed
    // column of the driving table, else a global load.
    auto fetch = [&](int col, uint32_t rowid, uint32_t ti) -> int64_t {
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (i < S.n && S.col[i] == col) {
          if (S.width[i] == 4)
            return d.cols[col].ptype == P_I32 ? (int64_t)((const int32_t*)(buf + S.off[i]))[ti]
                                              : (int64_t)((const uint32_t*)(buf + S.off[i]))[ti];
          return ((const int64_t*)(buf + S.off[i]))[ti];
        }
      const DCol& c = d.cols[col];
      return load_bits(c.ptr, c.ptype, rowid);
    };

    uint32_t alive = 0;
#pragma unroll
    for (int it = 0; it < ITEMS; ++it) alive |= (tile_base + (uint64_t)it * THREADS + tid < n ? 1u : 0u) << it;

    // Phase A: ops and sink, kBatch tuples at a time.
#pragma unroll 1
    for (int h = 0; h < ITEMS / kBatch; ++h) {
      uint32_t am = (alive >> (h * kBatch)) & ((1u << kBatch) - 1u);
      uint32_t rid[kBatch][kMaxSrc];
      uint32_t gslot[kBatch];
      uint32_t ti[kBatch];
#pragma unroll
      for (int bb = 0; bb < kBatch; ++bb) {
        ti[bb] = (uint32_t)((h * kBatch + bb) * THREADS + tid);
        gslot[bb] = 0;
#pragma unroll
        for (int s = 0; s < kMaxSrc; ++s)
          rid[bb][s] = (!d.tuple_input && s == d.drive_src) ? (uint32_t)(tile_base + ti[bb]) : 0u;
      }
      if (d.tuple_input) {
#pragma unroll
        for (int s = 0; s < kMaxSrc; ++s)
          if ((d.src_mask >> s) & 1u) {
#pragma unroll
            for (int bb = 0; bb < kBatch; ++bb)
              if ((am >> bb) & 1u) rid[bb][s] = d.in_rids[s][tile_base + ti[bb]];
          }
      }
      for (int o = 0; o < d.n_ops && am; ++o) {
        const PipeOp op = d.ops[o];
        if (op.kind == OPK_FILTER) {
          const DPred& p = d.preds[op.idx];
          const DCol& c = d.cols[p.col];
          int64_t v[kBatch];
#pragma unroll
          for (int bb = 0; bb < kBatch; ++bb)
            v[bb] = ((am >> bb) & 1u) ? fetch(p.col, pick(rid[bb], c.src), ti[bb]) : 0;
#pragma unroll
          for (int bb = 0; bb < kBatch; ++bb)
            if (((am >> bb) & 1u) && !eval_pred_bits(v[bb], c.ptype, p)) am &= ~(1u << bb);
        } else {
          const DProbe& pr = d.probes[op.idx];
          const DCol& c = d.cols[pr.key_col];
          const DBuild& bd = d.builds[pr.build];
          int64_t key[kBatch];
          uint32_t sl[kBatch];
#pragma unroll
          for (int bb = 0; bb < kBatch; ++bb)
            key[bb] = ((am >> bb) & 1u) ? fetch(pr.key_col, pick(rid[bb], c.src), ti[bb]) : 0;
          if (bd.kind == B_DENSE) {
            uint32_t m[kBatch];
#pragma unroll
            for (int bb = 0; bb < kBatch; ++bb) {
              const uint64_t kk = (uint64_t)(key[bb] - bd.key_min);
              m[bb] = (((am >> bb) & 1u) && kk < bd.capacity) ? bd.dense_map[kk] : 0u;
            }
#pragma unroll
            for (int bb = 0; bb < kBatch; ++bb) {
              if (m[bb] == 0u) am &= ~(1u << bb);
              sl[bb] = m[bb] - 1u;
            }
          } else {
#pragma unroll
            for (int bb = 0; bb < kBatch; ++bb) {
              uint32_t s_ = 0;
              if (((am >> bb) & 1u) && !build_lookup(bd, key[bb], s_, st)) am &= ~(1u << bb);
              sl[bb] = s_;
            }
          }
          if (op.idx == d.slot_probe) {
#pragma unroll
            for (int bb = 0; bb < kBatch; ++bb) gslot[bb] = sl[bb];
          }
#pragma unroll
          for (int s = 0; s < kMaxSrc; ++s)
            if ((pr.fill_mask >> s) & 1u) {
#pragma unroll
              for (int bb = 0; bb < kBatch; ++bb)
                if ((am >> bb) & 1u) rid[bb][s] = bd.payload[s][sl[bb]];
            }
        }
      }

      if (SINK == SK_MATERIALIZE) {
#pragma unroll
        for (int bb = 0; bb < kBatch; ++bb) {
          const bool keep = (am >> bb) & 1u;
          s_keep[ti[bb]] = keep ? 1 : 0;
          if (keep) {
#pragma unroll
            for (int s = 0; s < kMaxSrc; ++s)
              if (rid_slot[s] >= 0) s_rid[(size_t)rid_slot[s] * TILE + ti[bb]] = rid[bb][s];
          }
        }
        continue;
      }
      if (!am) continue;

      // Fetch the sink's columns for the whole batch, then run the sink.
      int64_t cv[kBatch][kAggCols];
#pragma unroll
      for (int jc = 0; jc < kAggCols; ++jc) {
        const bool use = jc < d.n_sink_cols;
        const int col = use ? d.sink_cols[jc] : 0;
        const int src = d.cols[col].src;
#pragma unroll
        for (int bb = 0; bb < kBatch; ++bb)
          cv[bb][jc] = (use && ((am >> bb) & 1u)) ? fetch(col, pick(rid[bb], src), ti[bb]) : 0;
      }
#pragma unroll
      for (int bb = 0; bb < kBatch; ++bb) {
        if (!((am >> bb) & 1u)) continue;
        switch (SINK) {
          case SK_BUILD: {
            const DBuild& bd = d.builds[d.sink_build];
            cg::coalesced_group g = cg::coalesced_threads();
            uint32_t base = 0;
            if (g.thread_rank() == 0) base = atomicAdd(bd.n_slots, g.size());
            base = g.shfl(base, 0);
            const uint32_t slot = base + g.thread_rank();
            const int64_t key = (d.n_sink_cols > 0 && d.sink_cols[0] == d.build_key_col)
                                    ? cv[bb][0]
                                    : fetch(d.build_key_col, pick(rid[bb], d.cols[d.build_key_col].src), ti[bb]);
#pragma unroll
            for (int s = 0; s < kMaxSrc; ++s)
              if ((d.build_payload_mask >> s) & 1u) bd.payload[s][slot] = rid[bb][s];
            // A representative-row aggregate downstream keeps its states by
            // this slot: initialize them here so no memset of the (build
            // table sized) state arrays is needed per query.
            for (int a = 0; a < d.n_aggs; ++a) agg_init_global(d.aggs[a], slot);
            if (d.slot_hit) d.slot_hit[slot] = 0;
            build_insert(bd, key, slot, st);
            break;
          }
          case SK_AGG_SLOT: {
            const uint32_t g = gslot[bb];
            d.slot_hit[g] = 1;
            for (int a = 0; a < d.n_aggs; ++a) {
              const DAgg& ag = d.aggs[a];
              Val v{0, 0};
              int32_t vt = P_I64;
              if (ag.prog >= 0) {
                v = vm_eval_c<kAggCols>(d.progs[ag.prog], d.cols, rid[bb], d.sink_cols, d.n_sink_cols, cv[bb], st);
                vt = d.progs[ag.prog].out_type;
              }
              agg_apply(ag.fn, (unsigned long long*)(ag.lo + g), (long long*)(ag.hi ? ag.hi + g : nullptr), v, vt);
            }
            break;
          }
          case SK_AGG_HASH:
          case SK_AGG_SMEM: {
            uint64_t kw[kMaxKeys];
#pragma unroll
            for (int i = 0; i < kMaxKeys; ++i)
              kw[i] = i < d.table.n_keys
                          ? (uint64_t)vm_eval_c<kAggCols>(d.progs[d.key_prog[i]], d.cols, rid[bb], d.sink_cols,
                                                          d.n_sink_cols, cv[bb], st).lo
                          : 0;
            int sidx = -1;
            if (SINK == SK_AGG_SMEM) sidx = smem_agg_find(d, sagg, kw, st);
            uint64_t g = d.table.capacity;
            if (sidx < 0) g = agg_find_global(d, kw, st);
            if (sidx < 0 && g >= d.table.capacity) break;
            for (int a = 0; a < d.n_aggs; ++a) {
              const DAgg& ag = d.aggs[a];
              Val v{0, 0};
              int32_t vt = P_I64;
              if (ag.prog >= 0) {
                v = vm_eval_c<kAggCols>(d.progs[ag.prog], d.cols, rid[bb], d.sink_cols, d.n_sink_cols, cv[bb], st);
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
            break;
          }
          case SK_AGG_SCALAR: {
#pragma unroll
            for (int a = 0; a < kMaxAggs; ++a) {
              if (a >= d.n_aggs) break;
              const DAgg& ag = d.aggs[a];
              Val v{0, 0};
              int32_t vt = P_I64;
              if (ag.prog >= 0) {
                v = vm_eval_c<kAggCols>(d.progs[ag.prog], d.cols, rid[bb], d.sink_cols, d.n_sink_cols, cv[bb], st);
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
            break;
          }
          default: break;
        }
      }
    }

    if (SINK == SK_MATERIALIZE) {
      __syncthreads();
      // Blocked arrangement for the scan: thread t owns tile rows [t*ITEMS, (t+1)*ITEMS).
      uint32_t cnt = 0;
#pragma unroll
      for (int i = 0; i < ITEMS; ++i) cnt += s_keep[tid * ITEMS + i];
      uint32_t total;
      uint32_t pos = block_excl_sum<THREADS>(cnt, s_warp, &total);
#pragma unroll
      for (int i = 0; i < ITEMS; ++i)
        if (s_keep[tid * ITEMS + i]) s_list[pos++] = (uint16_t)(tid * ITEMS + i);
      if (tid == 0) {
        uint64_t excl = lb_exclusive(d.tile_status, tile, total, d.epoch, d.status);
        s_base = excl;
        if (tile == n_tiles - 1) *d.out_count = excl + total;
      }
      __syncthreads();
      const uint64_t base = s_base;
      // Write phase: kBatch compacted rows per thread, columns fetched first.
      for (uint32_t p0 = tid; p0 < total; p0 += THREADS * kBatch) {
        uint32_t rr[kBatch][kMaxSrc];
        uint32_t tx[kBatch];
        uint32_t okm = 0;
#pragma unroll
        for (int bb = 0; bb < kBatch; ++bb) {
          const uint32_t p = p0 + bb * THREADS;
          const bool ok = p < total;
          okm |= (ok ? 1u : 0u) << bb;
          tx[bb] = ok ? s_list[p] : 0u;
#pragma unroll
          for (int s = 0; s < kMaxSrc; ++s) {
            uint32_t r = (rid_slot[s] >= 0 && ok) ? s_rid[(size_t)rid_slot[s] * TILE + tx[bb]] : 0u;
            if (!d.tuple_input && s == d.drive_src) r = (uint32_t)(tile_base + tx[bb]);
            rr[bb][s] = r;
          }
        }
        int64_t cv[kBatch][kOutCols];
#pragma unroll
        for (int jc = 0; jc < kOutCols; ++jc) {
          const bool use = jc < d.n_sink_cols;
          const int col = use ? d.sink_cols[jc] : 0;
          const int src = d.cols[col].src;
#pragma unroll
          for (int bb = 0; bb < kBatch; ++bb)
            cv[bb][jc] = (use && ((okm >> bb) & 1u)) ? fetch(col, pick(rr[bb], src), tx[bb]) : 0;
        }
#pragma unroll
        for (int bb = 0; bb < kBatch; ++bb) {
          if (!((okm >> bb) & 1u)) continue;
          const uint64_t o = base + p0 + bb * THREADS;
          if (o >= d.out_capacity) {
            st |= ST_CAPACITY;
            continue;
          }
          for (int q = 0; q < d.n_out; ++q) {
            const VmProg& pg = d.progs[d.out_prog[q]];
            Val v = vm_eval_c<kOutCols>(pg, d.cols, rr[bb], d.sink_cols, d.n_sink_cols, cv[bb], st);
            store_val(d.out_ptr[q], pg.out_type, o, v);
          }
#pragma unroll
          for (int s = 0; s < kMaxSrc; ++s)
            if ((d.out_rid_mask >> s) & 1u) d.out_rids[s][o] = rr[bb][s];
        }
      }
    }
    // Every thread is done with `buf` (and the sink scratch) before reuse.
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
      if (g >= d.table.capacity) continue;
      for (int a = 0; a < d.n_aggs; ++a) {
        const DAgg& ag = d.aggs[a];
        int64_t hv = sagg.hi_index[a] >= 0 ? sagg.hi[(size_t)sagg.hi_index[a] * sagg.cap + i] : 0;
        agg_merge(ag.fn, (unsigned long long*)(ag.lo + g), (long long*)(ag.hi ? ag.hi + g : nullptr),
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

size_t pipeline_tile_rows() { return kTile; }

size_t pipeline_stream_bytes(const PipeDesc& d) {
  return d.tuple_input ? 0 : 2ull * kTile * stream_bytes_per_row(d);
}

size_t pipeline_smem_bytes(const PipeDesc& d) {
  constexpr size_t TILE = kTile;
  size_t s = pipeline_stream_bytes(d);
  if (d.sink == SK_MATERIALIZE) {
    size_t q = 0;
    for (int i = 0; i < kMaxSrc; ++i) {
      bool implicit = !d.tuple_input && i == d.drive_src;
      if (((d.mat_src_mask >> i) & 1u) && !implicit) ++q;
    }
    s += TILE + 2 * TILE + 4 * TILE * q;
  }
  if (d.sink == SK_AGG_SMEM) {
    size_t n128 = 0;
    for (int a = 0; a < d.n_aggs; ++a) n128 += d.aggs[a].fn == A_SUM_I128;
    s += (size_t)d.smem_capacity * (4 + 8 * d.table.n_keys + 8 * d.n_aggs + 8 * n128);
  }
  return s;
}

template <int SINK>
static cudaError_t launch_sink(const PipeDesc& d, uint64_t n_hint, cudaStream_t s) {
  auto kern = k_pipeline<SINK>;
  const size_t smem = pipeline_smem_bytes(d);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  // Grid = resident CTAs per SM x SM count (a persistent grid-stride grid).
  int blocks_per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, kern, kThreads, smem) != cudaSuccess ||
      blocks_per_sm < 1) {
    cudaGetLastError();
    blocks_per_sm = 1;
  }
  uint64_t tiles = (n_hint + kTile - 1) / kTile;
  uint64_t max_grid = (uint64_t)sm_count() * (uint64_t)blocks_per_sm;
  uint64_t grid = tiles < max_grid ? tiles : max_grid;
  if (grid == 0) grid = 1;
  kern<<<(unsigned)grid, kThreads, smem, s>>>(d);
  return cudaGetLastError();
}

cudaError_t launch_pipeline(const PipeDesc& d, uint64_t n_hint, cudaStream_t s) {
  switch (d.sink) {
    case SK_BUILD: return launch_sink<SK_BUILD>(d, n_hint, s);
    case SK_MATERIALIZE: return launch_sink<SK_MATERIALIZE>(d, n_hint, s);
    case SK_AGG_HASH: return launch_sink<SK_AGG_HASH>(d, n_hint, s);
    case SK_AGG_SMEM: return launch_sink<SK_AGG_SMEM>(d, n_hint, s);
    case SK_AGG_SLOT: return launch_sink<SK_AGG_SLOT>(d, n_hint, s);
    case SK_AGG_SCALAR: return launch_sink<SK_AGG_SCALAR>(d, n_hint, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace mtl
