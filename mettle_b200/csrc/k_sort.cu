// k_sort.cu — ORDER BY on sm_100a: order-preserving key encoding, a stable
// LSD radix sort (8-bit digits, warp match-based stable ranking), and a
// block-local top-K with threshold pruning and bitonic merges in shared
// memory. The reference sorts the final batch on the CPU
// (src/plan/helpers.rs:627-667) and runs its grouped top-K with a single
// thread for K > 20 (topk_dense_grouped_rows, kernels.metal:1162) or one
// 128-thread group with a serial merge (kernels.metal:1249); its tie order
// (sum DESC, secondary ASC, row id ASC, kernels.metal:1102-1118) is kept by
// encoding every ORDER BY part, then the tie-break parts, into one key.
#include "final_common.cuh"
#include "kern_common.cuh"
#include "kernels.h"
#include <mutex>

namespace mtl {

namespace {
int sms() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n <= 0) n = 148;
  }
  return n;
}
}  // namespace

// ------------------------------------------------------------ key encoding
__global__ void k_encode(const __grid_constant__ SortKeySpec spec, const uint64_t* count, uint64_t n_max,
                         SortItem* __restrict__ keys, uint32_t* __restrict__ idx) {
  const uint64_t n = count ? *count : n_max;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    U256 k{{0, 0, 0, 0}};
    for (int p = 0; p < spec.n_parts; ++p) {
      const int pt = spec.ptype[p];
      uint64_t lo = 0, hi = 0;
      switch (pt) {
        case P_I32:
        case P_F32: lo = ((const uint32_t*)spec.col[p])[i]; break;
        case P_I64:
        case P_F64: lo = ((const uint64_t*)spec.col[p])[i]; break;
        case P_I128: {
          const longlong2 v = ((const longlong2*)spec.col[p])[i];
          lo = (uint64_t)v.x;
          hi = (uint64_t)v.y;
          break;
        }
        default: break;
      }
      key_part(k, pt, spec.desc[p] != 0, lo, hi);
    }
    SortItem it;
    it.w[0] = k.w[0]; it.w[1] = k.w[1]; it.w[2] = k.w[2]; it.w[3] = k.w[3];
    keys[i] = it;
    idx[i] = (uint32_t)i;
  }
}

cudaError_t launch_encode_keys(const SortKeySpec& spec, const uint64_t* count, uint64_t n_max, SortItem* keys,
                               uint32_t* idx, cudaStream_t s) {
  uint64_t b = (n_max + 255) / 256;
  uint64_t cap = (uint64_t)sms() * 8;
  if (b > cap) b = cap;
  if (!b) b = 1;
  k_encode<<<(unsigned)b, 256, 0, s>>>(spec, count, n_max, keys, idx);
  return cudaGetLastError();
}

// ------------------------------------------------------------ radix sort
constexpr int kRThreads = 256;
constexpr int kRItems = 16;
constexpr int kRTile = kRThreads * kRItems;
constexpr int kRWarps = kRThreads / 32;

__device__ __forceinline__ uint32_t digit_of(const SortItem& k, int byte) {
  return (uint32_t)(k.w[3 - (byte >> 3)] >> ((byte & 7) * 8)) & 0xFFu;
}

__global__ void __launch_bounds__(kRThreads) k_radix_hist(const SortItem* __restrict__ keys, const uint64_t* count,
                                                          uint64_t n_tiles_max, int byte, uint32_t* __restrict__ hist) {
  __shared__ uint32_t s_h[256];
  const uint64_t n = *count;
  for (uint64_t tile = blockIdx.x; tile < n_tiles_max; tile += gridDim.x) {
    for (int i = threadIdx.x; i < 256; i += kRThreads) s_h[i] = 0;
    __syncthreads();
    const uint64_t base = tile * kRTile;
    for (int r = 0; r < kRItems; ++r) {
      uint64_t g = base + (uint64_t)r * kRThreads + threadIdx.x;
      if (g < n) atomicAdd(&s_h[digit_of(keys[g], byte)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 256; i += kRThreads) hist[(uint64_t)i * n_tiles_max + tile] = s_h[i];
    __syncthreads();
  }
}

// In-place exclusive scan of a u32 array in chunks: chunk sums first.
constexpr int kSChunk = 4096;
__global__ void k_scan_chunks(uint32_t* __restrict__ a, uint64_t n, uint32_t* __restrict__ sums) {
  __shared__ uint32_t s_warp[kRThreads / 32 + 1];
  const uint64_t base = (uint64_t)blockIdx.x * kSChunk;
  constexpr int per = kSChunk / kRThreads;
  uint32_t v[per];
  uint32_t tot = 0;
#pragma unroll
  for (int i = 0; i < per; ++i) {
    uint64_t g = base + (uint64_t)threadIdx.x * per + i;
    v[i] = g < n ? a[g] : 0;
    tot += v[i];
  }
  uint32_t total;
  uint32_t pre = block_excl_sum<kRThreads>(tot, s_warp, &total);
#pragma unroll
  for (int i = 0; i < per; ++i) {
    uint64_t g = base + (uint64_t)threadIdx.x * per + i;
    if (g < n) a[g] = pre;
    pre += v[i];
  }
  if (threadIdx.x == 0) sums[blockIdx.x] = total;
}
__global__ void k_scan_small(uint32_t* __restrict__ a, uint64_t n) {
  // One CTA: exclusive scan of up to a few hundred thousand entries.
  __shared__ uint32_t s_warp[kRThreads / 32 + 1];
  uint32_t carry = 0;
  for (uint64_t base = 0; base < n; base += kRThreads) {
    uint64_t g = base + threadIdx.x;
    uint32_t v = g < n ? a[g] : 0;
    uint32_t total;
    uint32_t pre = block_excl_sum<kRThreads>(v, s_warp, &total);
    if (g < n) a[g] = carry + pre;
    carry += total;
  }
}
__global__ void k_scan_add(uint32_t* __restrict__ a, uint64_t n, const uint32_t* __restrict__ sums) {
  const uint64_t base = (uint64_t)blockIdx.x * kSChunk;
  const uint32_t add = sums[blockIdx.x];
  for (int i = threadIdx.x; i < kSChunk; i += kRThreads) {
    uint64_t g = base + i;
    if (g < n) a[g] += add;
  }
}

// Stable scatter: elements are ranked in index order within the tile using
// warp match masks and per-warp digit counts in shared memory.
__global__ void __launch_bounds__(kRThreads) k_radix_scatter(const SortItem* __restrict__ keys,
                                                             const uint32_t* __restrict__ idx, const uint64_t* count,
                                                             uint64_t n_tiles_max, int byte,
                                                             const uint32_t* __restrict__ hist,
                                                             SortItem* __restrict__ okeys, uint32_t* __restrict__ oidx) {
  __shared__ uint32_t s_base[256];
  __shared__ uint16_t s_wc[kRWarps][256];
  const uint64_t n = *count;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  for (uint64_t tile = blockIdx.x; tile < n_tiles_max; tile += gridDim.x) {
    const uint64_t base = tile * kRTile;
    if (base >= n) break;
    for (int i = threadIdx.x; i < 256; i += kRThreads) s_base[i] = hist[(uint64_t)i * n_tiles_max + tile];
    __syncthreads();
    for (int r = 0; r < kRItems; ++r) {
      const uint64_t g = base + (uint64_t)r * kRThreads + threadIdx.x;
      const bool valid = g < n;
      SortItem k;
      uint32_t ix = 0, d = 256;
      if (valid) {
        k = keys[g];
        ix = idx[g];
        d = digit_of(k, byte);
      }
      for (int i = threadIdx.x; i < kRWarps * 256; i += kRThreads) (&s_wc[0][0])[i] = 0;
      __syncthreads();
      const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
      const uint32_t rank = __popc(peers & lt);
      if (valid && rank == 0) s_wc[warp][d] = (uint16_t)__popc(peers);
      __syncthreads();
      uint32_t off = 0;
      if (valid) {
        off = s_base[d];
        for (int w = 0; w < warp; ++w) off += s_wc[w][d];
        off += rank;
        okeys[off] = k;
        oidx[off] = ix;
      }
      __syncthreads();
      // advance the running per-digit base by this round's counts
      for (int dd = threadIdx.x; dd < 256; dd += kRThreads) {
        uint32_t t = 0;
        for (int w = 0; w < kRWarps; ++w) t += s_wc[w][dd];
        s_base[dd] += t;
      }
      __syncthreads();
    }
  }
}

size_t radix_sort_temp_bytes(uint64_t n_max) {
  uint64_t tiles = (n_max + kRTile - 1) / kRTile;
  if (!tiles) tiles = 1;
  uint64_t hist = tiles * 256;
  uint64_t chunks = (hist + kSChunk - 1) / kSChunk;
  return (hist + chunks + 64) * sizeof(uint32_t);
}

cudaError_t launch_radix_sort(SortItem* keys, uint32_t* idx, SortItem* keys_tmp, uint32_t* idx_tmp,
                              const uint64_t* count, uint64_t n_max, int key_bytes, void* temp, cudaStream_t s,
                              int* result_in_tmp) {
  uint64_t tiles = (n_max + kRTile - 1) / kRTile;
  if (!tiles) tiles = 1;
  const uint64_t hn = tiles * 256;
  uint32_t* hist = (uint32_t*)temp;
  uint32_t* sums = hist + hn;
  const uint64_t chunks = (hn + kSChunk - 1) / kSChunk;
  unsigned grid = (unsigned)(tiles < (uint64_t)sms() * 4 ? tiles : (uint64_t)sms() * 4);
  SortItem* src_k = keys;
  uint32_t* src_i = idx;
  SortItem* dst_k = keys_tmp;
  uint32_t* dst_i = idx_tmp;
  for (int b = 0; b < key_bytes; ++b) {
    k_radix_hist<<<grid, kRThreads, 0, s>>>(src_k, count, tiles, b, hist);
    if (chunks == 1) {
      k_scan_small<<<1, kRThreads, 0, s>>>(hist, hn);
    } else {
      k_scan_chunks<<<(unsigned)chunks, kRThreads, 0, s>>>(hist, hn, sums);
      k_scan_small<<<1, kRThreads, 0, s>>>(sums, chunks);
      k_scan_add<<<(unsigned)chunks, kRThreads, 0, s>>>(hist, hn, sums);
    }
    k_radix_scatter<<<grid, kRThreads, 0, s>>>(src_k, src_i, count, tiles, b, hist, dst_k, dst_i);
    SortItem* tk = src_k; src_k = dst_k; dst_k = tk;
    uint32_t* ti = src_i; src_i = dst_i; dst_i = ti;
  }
  *result_in_tmp = (key_bytes & 1) ? 1 : 0;
  return cudaGetLastError();
}

// ------------------------------------------------------------ top-K
__device__ __forceinline__ bool item_less(const SortItem& a, uint32_t ia, const SortItem& b, uint32_t ib) {
#pragma unroll
  for (int w = 0; w < 4; ++w)
    if (a.w[w] != b.w[w]) return a.w[w] < b.w[w];
  return ia < ib;
}

// Bitonic sort of B (SortItem, idx) pairs in shared memory, ascending.
template <int B, int THREADS>
__device__ void bitonic_sort(SortItem* sk, uint32_t* si) {
  for (int size = 2; size <= B; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = threadIdx.x; t < B / 2; t += THREADS) {
        int lo = 2 * t - (t & (stride - 1));
        int hi = lo + stride;
        bool up = ((lo & size) == 0);
        SortItem a = sk[lo], b = sk[hi];
        uint32_t ia = si[lo], ib = si[hi];
        bool sw = up ? item_less(b, ib, a, ia) : item_less(a, ia, b, ib);
        if (sw) {
          sk[lo] = b; sk[hi] = a;
          si[lo] = ib; si[hi] = ia;
        }
      }
      __syncthreads();
    }
  }
}

constexpr int kTopkRows = 8;  // rows per thread loaded together in k_topk

// Per-CTA top-K. Rows are taken in rounds of THREADS; a row enters the
// candidate buffer only if it beats the current K-th best, and the buffer is
// merged (bitonic sort of best-K + candidates) whenever it could overflow.
template <int B, int THREADS>
__global__ void __launch_bounds__(THREADS) k_topk(const SortItem* __restrict__ keys, const uint32_t* __restrict__ idx,
                                                  const uint64_t* count, uint64_t n_max, int K,
                                                  SortItem* __restrict__ out_keys, uint32_t* __restrict__ out_idx,
                                                  uint64_t* out_count, int final_pass) {
  extern __shared__ __align__(16) uint8_t smem[];
  SortItem* sk = (SortItem*)smem;
  uint32_t* si = (uint32_t*)(sk + B);
  __shared__ int s_n;         // entries in [0, B): [0, K) best so far, then candidates
  __shared__ int s_have;      // best entries valid (<= K)
  const uint64_t n = count ? *count : n_max;
  const SortItem inf{{~0ULL, ~0ULL, ~0ULL, ~0ULL}};
  if (threadIdx.x == 0) {
    s_n = 0;
    s_have = 0;
  }
  __syncthreads();
  // Rows handled by this CTA: a contiguous range.
  const uint64_t per = (n + gridDim.x - 1) / gridDim.x;
  const uint64_t lo = (uint64_t)blockIdx.x * per;
  uint64_t hi = lo + per;
  if (hi > n) hi = n;
  auto merge = [&]() {
    // pad, sort, keep the first K
    for (int i = s_n + threadIdx.x; i < B; i += THREADS) {
      sk[i] = inf;
      si[i] = 0xFFFFFFFFu;
    }
    __syncthreads();
    bitonic_sort<B, THREADS>(sk, si);
    if (threadIdx.x == 0) {
      int valid = s_n < K ? s_n : K;
      s_have = valid;
      s_n = valid;
    }
    __syncthreads();
  };
  // Rows are loaded kTopkRows per thread at a time (all loads in flight
  // together), then offered one THREADS-row step at a time.
  for (uint64_t base = lo; base < hi; base += (uint64_t)THREADS * kTopkRows) {
    SortItem kr[kTopkRows];
    uint32_t ir[kTopkRows];
#pragma unroll
    for (int r = 0; r < kTopkRows; ++r) {
      const uint64_t g = base + (uint64_t)r * THREADS + threadIdx.x;
      ir[r] = 0xFFFFFFFFu;
      if (g < hi) {
        kr[r] = keys[g];
        ir[r] = idx ? idx[g] : (uint32_t)g;
      }
    }
#pragma unroll
    for (int r = 0; r < kTopkRows; ++r) {
      if (base + (uint64_t)r * THREADS >= hi) break;  // CTA-uniform
      // 0xFFFFFFFF marks padding from the per-CTA pass (and rows past the end).
      const bool take = ir[r] != 0xFFFFFFFFu && (s_have < K || item_less(kr[r], ir[r], sk[K - 1], si[K - 1]));
      if (take) {
        const int p = atomicAdd(&s_n, 1);
        sk[p] = kr[r];
        si[p] = ir[r];
      }
      __syncthreads();
      if (s_n > B - THREADS) merge();
    }
  }
  if (s_n > s_have || s_have < K) merge();
  const int m = s_have;
  if (final_pass) {
    for (int i = threadIdx.x; i < m; i += THREADS) out_idx[i] = si[i];
    if (threadIdx.x == 0) *out_count = (uint64_t)m;
  } else {
    for (int i = threadIdx.x; i < K; i += THREADS) {
      out_keys[(uint64_t)blockIdx.x * K + i] = i < m ? sk[i] : inf;
      out_idx[(uint64_t)blockIdx.x * K + i] = i < m ? si[i] : 0xFFFFFFFFu;
    }
  }
}

// The leading 64 bits of a key of `bits` significant bits (right aligned in
// w[0..3], w[0] most significant); shorter keys are returned whole.
__device__ __forceinline__ uint64_t key_top64(const uint64_t* w, int bits) {
  if (bits <= 64) return w[3];
  const int s = bits - 64;  // lowest bit of the leading 64
  const int wi = 3 - (s >> 6), sh = s & 63;
  uint64_t x = w[wi] >> sh;
  if (sh) x |= w[wi - 1] << (64 - sh);
  return x;
}

// Bits 0-3: which bytes of w are nonzero.
__device__ __forceinline__ uint32_t nz_bytes(uint32_t w) {
  return ((w & 0xFFu) ? 1u : 0u) | ((w & 0xFF00u) ? 2u : 0u) | ((w & 0xFF0000u) ? 4u : 0u) |
         ((w & 0xFF000000u) ? 8u : 0u);
}

// ------------------------------------------------------------ warp top-K
// K <= 32: each warp keeps its best K as a sorted list in registers (lane i
// holds rank i). A row enters only if it beats the warp's current K-th best
// (one ballot per 32 rows); an insertion is one ballot plus a one-lane shift.
// No block-wide barrier runs in the scan loop.
struct Cand {
  uint64_t w[4];
  uint32_t ix;
};

__device__ __forceinline__ bool cand_less(const Cand& a, const Cand& b) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
    if (a.w[i] != b.w[i]) return a.w[i] < b.w[i];
  return a.ix < b.ix;
}
__device__ __forceinline__ Cand cand_shfl(const Cand& c, int src) {
  Cand r;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.w[i] = __shfl_sync(0xFFFFFFFFu, c.w[i], src);
  r.ix = __shfl_sync(0xFFFFFFFFu, c.ix, src);
  return r;
}
__device__ __forceinline__ Cand cand_shfl_up(const Cand& c) {
  Cand r;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.w[i] = __shfl_up_sync(0xFFFFFFFFu, c.w[i], 1);
  r.ix = __shfl_up_sync(0xFFFFFFFFu, c.ix, 1);
  return r;
}
__device__ __forceinline__ Cand cand_inf() {
  Cand c;
  c.w[0] = c.w[1] = c.w[2] = c.w[3] = ~0ULL;
  c.ix = 0xFFFFFFFFu;
  return c;
}

// Offers each lane's candidate (when `valid`) to the warp list L.
__device__ __forceinline__ void warp_offer(Cand& L, const Cand& c, bool valid, int K, int lane) {
  Cand thr = cand_shfl(L, K - 1);
  uint32_t m = __ballot_sync(0xFFFFFFFFu, valid && cand_less(c, thr));
  while (m) {
    const int src = __ffs(m) - 1;
    m &= m - 1;
    const Cand x = cand_shfl(c, src);
    const uint32_t less = __ballot_sync(0xFFFFFFFFu, lane < K && cand_less(L, x));
    const int pos = __popc(less);
    if (pos < K) {
      const Cand up = cand_shfl_up(L);
      if (lane == pos) L = x;
      else if (lane > pos && lane < K) L = up;
      thr = cand_shfl(L, K - 1);
      m &= __ballot_sync(0xFFFFFFFFu, valid && cand_less(c, thr));
    }
  }
}

__device__ __forceinline__ Cand cand_shfl_xor(const Cand& c, int m) {
  Cand r;
#pragma unroll
  for (int i = 0; i < 4; ++i) r.w[i] = __shfl_xor_sync(0xFFFFFFFFu, c.w[i], m);
  r.ix = __shfl_xor_sync(0xFFFFFFFFu, c.ix, m);
  return r;
}

// Bitonic sort of one candidate per lane, ascending across the warp.
__device__ __forceinline__ void warp_sort32(Cand& c, int lane) {
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      const Cand p = cand_shfl_xor(c, j);
      const bool take_min = ((lane & j) == 0) == ((lane & k) == 0);
      if (take_min ? cand_less(p, c) : cand_less(c, p)) c = p;
    }
  }
}

// L and M are ascending across the warp; L becomes the 32 smallest of both,
// ascending. Elementwise min against M reversed leaves a bitonic sequence
// holding the 32 smallest, which five half-cleaner steps sort.
__device__ __forceinline__ void warp_merge32(Cand& L, const Cand& M, int lane) {
  const Cand r = cand_shfl(M, 31 - lane);
  if (cand_less(r, L)) L = r;
#pragma unroll
  for (int j = 16; j > 0; j >>= 1) {
    const Cand p = cand_shfl_xor(L, j);
    if (((lane & j) == 0) ? cand_less(p, L) : cand_less(L, p)) L = p;
  }
}

// Offers one candidate per lane to the warp's ascending list L (whose first
// K lanes are the best so far): a few winners are inserted one at a time,
// more are sorted as a batch and merged.
__device__ __forceinline__ void warp_offer_batch(Cand& L, const Cand& c, bool valid, int K, int lane) {
  const Cand thr = cand_shfl(L, K - 1);
  const bool beat = valid && cand_less(c, thr);
  const uint32_t m = __ballot_sync(0xFFFFFFFFu, beat);
  if (!m) return;
  if (__popc(m) <= 2) {
    warp_offer(L, c, beat, K, lane);
    return;
  }
  Cand s = beat ? c : cand_inf();
  warp_sort32(s, lane);
  warp_merge32(L, s, lane);
}

// Merges the warps' lists of a block into warp 0's L (tree of merges).
template <int WARPS>
__device__ __forceinline__ void block_merge_lists(Cand& L, Cand (*s_l)[32], int warp, int lane) {
  s_l[warp][lane] = L;
#pragma unroll
  for (int s = 1; s < WARPS; s <<= 1) {
    __syncthreads();
    if ((warp & (2 * s - 1)) == 0 && warp + s < WARPS) {
      warp_merge32(L, s_l[warp + s][lane], lane);
      s_l[warp][lane] = L;
    }
  }
  __syncthreads();
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS) k_topk_warp(const SortItem* __restrict__ keys,
                                                       const uint32_t* __restrict__ idx, const uint64_t* count,
                                                       uint64_t n_max, int K, SortItem* __restrict__ out_keys,
                                                       uint32_t* __restrict__ out_idx, uint64_t* out_count,
                                                       int final_pass, const uint32_t* __restrict__ remap = nullptr,
                                                       uint64_t* reset = nullptr, int cut_bits = 0) {
  constexpr int WARPS = THREADS / 32;
  __shared__ Cand s_l[WARPS][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t n = count ? *count : n_max;
  if (n > n_max) n = n_max;
  const uint64_t per = (n + gridDim.x - 1) / gridDim.x;
  const uint64_t lo = (uint64_t)blockIdx.x * per;
  const uint64_t hi = lo + per < n ? lo + per : n;
  // merge of the fused top-K's candidates: the first pass is over, so its
  // cut is final (the smallest leading bits of any warp's K-th key)
  const uint64_t cut = (reset && cut_bits > 0) ? ~*(volatile unsigned long long*)reset : ~0ULL;
  Cand L = cand_inf();
  for (uint64_t base = lo + (uint64_t)warp * 32; base < hi; base += (uint64_t)THREADS) {
    const uint64_t g = base + lane;
    Cand c = cand_inf();
    bool valid = g < hi;
    if (valid) {
      const SortItem k = keys[g];
      c.w[0] = k.w[0]; c.w[1] = k.w[1]; c.w[2] = k.w[2]; c.w[3] = k.w[3];
      c.ix = idx ? idx[g] : (uint32_t)g;
      valid = c.ix != 0xFFFFFFFFu;  // padding of a previous pass
      if (cut_bits > 0 && key_top64(c.w, cut_bits) > cut) valid = false;
    }
    warp_offer_batch(L, c, valid, K, lane);
  }
  block_merge_lists<WARPS>(L, s_l, warp, lane);
  if (warp == 0) {
    if (final_pass) {
      const uint32_t valid = __ballot_sync(0xFFFFFFFFu, lane < K && L.ix != 0xFFFFFFFFu);
      if (lane < K && L.ix != 0xFFFFFFFFu) out_idx[lane] = remap ? remap[L.ix] : L.ix;
      if (lane == 0) *out_count = (uint64_t)__popc(valid);
    } else if (lane < K) {
      SortItem it;
      it.w[0] = L.w[0]; it.w[1] = L.w[1]; it.w[2] = L.w[2]; it.w[3] = L.w[3];
      out_keys[(uint64_t)blockIdx.x * K + lane] = it;
      out_idx[(uint64_t)blockIdx.x * K + lane] = L.ix;
    }
  }
  // Every thread read *count before the block merge's barriers: the
  // cross-CTA state of the first pass can be cleared for the next launch.
  if (reset && threadIdx.x == 0) {
    reset[0] = 0;
    reset[1] = 0;
  }
}

// Fused aggregate top-K (K <= 32): the ORDER BY image of each live group is
// computed from its aggregate states and offered straight to the warp lists,
// so no per-group output columns, key array or compacted group list is
// written. Ties are broken by the group index, which orders groups the same
// way as the order-preserving compaction the unfused path uses. A group
// whose first ORDER BY part alone already places it after the warp's current
// K-th key, or after the grid-wide cut below, is dropped before its other
// parts (often gathers through a representative row) are read.
//
// Grid-wide cut: a warp whose list holds K groups knows that the K best keys
// of the whole input start with at most the leading 64 key bits of its own
// K-th entry, so every warp publishes that value (an atomic max of its
// complement, so that a zero word means "no cut yet") and prunes against the
// smallest one published. Each CTA then appends only the candidates that
// can still win to one list (an atomic counter), and the merge pass reads
// that list alone: its work no longer grows with the number of CTAs.
__device__ __forceinline__ bool u256_gt(const U256& a, const Cand& b) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
    if (a.w[i] != b.w[i]) return a.w[i] > b.w[i];
  return false;
}

// Cross-CTA state of one fused top-K launch, at the start of its temp area;
// it must be zero when the launch starts (the merge pass clears it again).
struct TopkFinalState {
  unsigned long long cut_inv;  // ~(smallest published cut); 0: none yet
  unsigned long long unused;   // (cleared with the cut)
};

template <int THREADS>
__global__ void __launch_bounds__(THREADS) k_topk_final(const __grid_constant__ TopkFinalSpec spec, int K,
                                                        TopkFinalState* __restrict__ gst,
                                                        SortItem* __restrict__ out_keys,
                                                        uint32_t* __restrict__ out_idx) {
  constexpr int WARPS = THREADS / 32;
  __shared__ Cand s_l[WARPS][32];
  __shared__ uint32_t s_live[WARPS][64];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t n = spec.n_dev ? (*spec.n_dev < spec.n_max ? *spec.n_dev : spec.n_max) : spec.n_max;
  // CTA ranges start on multiples of 512 groups (16-byte aligned flag loads)
  const uint64_t per = ((n + gridDim.x - 1) / gridDim.x + 511) & ~511ULL;
  const uint64_t lo = (uint64_t)blockIdx.x * per < n ? (uint64_t)blockIdx.x * per : n;
  const uint64_t hi = lo + per < n ? lo + per : n;
  const int tb = spec.total_bits;
  uint32_t* const wb = s_live[warp];
  Cand L = cand_inf();
  uint64_t cut = ~0ULL;  // warp-uniform: no group whose leading bits exceed it can win
  // Offers the live groups wb[0 .. m): the first ORDER BY part alone drops
  // most of them; the others get their full key.
  auto process = [&](uint32_t m) {
    {
      uint64_t g = 0;
      if (lane == 0) g = ~*(volatile unsigned long long*)&gst->cut_inv;
      g = __shfl_sync(0xFFFFFFFFu, g, 0);
      if (g < cut) cut = g;
    }
    const bool in = (uint32_t)lane < m;
    const uint64_t g = in ? wb[lane] : 0;
    bool v = in;
    const Cand thr = cand_shfl(L, K - 1);
    U256 k{{0, 0, 0, 0}};
    if (v) {
      uint64_t vlo, vhi;
      final_value(spec.part[0], g, vlo, vhi);
      key_part(k, spec.ptype[0], spec.desc[0] != 0, vlo, vhi);
      U256 probe = k;
      shl_or(probe, tb - spec.bits0, 0, 0);
      if (u256_gt(probe, thr) || key_top64(probe.w, tb) > cut) v = false;
    }
    Cand c = cand_inf();
    if (v) {
      for (int p = 1; p < spec.n_parts; ++p) {
        uint64_t vlo, vhi;
        final_value(spec.part[p], g, vlo, vhi);
        key_part(k, spec.ptype[p], spec.desc[p] != 0, vlo, vhi);
      }
      c.w[0] = k.w[0]; c.w[1] = k.w[1]; c.w[2] = k.w[2]; c.w[3] = k.w[3];
      c.ix = (uint32_t)g;
    }
    warp_offer_batch(L, c, v, K, lane);
    // publish this warp's K-th key when it tightens the cut
    const Cand kth = cand_shfl(L, K - 1);
    if (kth.ix != 0xFFFFFFFFu) {
      const uint64_t t = key_top64(kth.w, tb);
      if (t < cut) {
        if (lane == 0) atomicMax(&gst->cut_inv, ~t);
        cut = t;
      }
    }
  };
  // Each lane takes 16 consecutive groups per step (one 16-byte load of
  // their flags, or four of their states), so a warp covers 512 groups per
  // step; the live ones are gathered in wb with one ballot per position and
  // offered 32 at a time.
  const bool vec_flag = spec.flag && (((uintptr_t)spec.flag & 15) == 0);
  const bool vec_state = spec.state && (((uintptr_t)spec.state & 15) == 0);
  uint32_t cnt = 0;
  for (uint64_t base = lo + (uint64_t)warp * 512; base < hi; base += (uint64_t)THREADS * 16) {
    const uint64_t g0 = base + (uint64_t)lane * 16;
    uint32_t m16 = 0;  // bit j: group g0 + j is live
    if (g0 < hi) {
      const uint32_t nin = hi - g0 >= 16 ? 16u : (uint32_t)(hi - g0);
      m16 = nin == 16 ? 0xFFFFu : ((1u << nin) - 1u);
      if (spec.flag) {
        uint32_t f = 0;
        if (vec_flag && nin == 16) {
          const uint4 v = *(const uint4*)(spec.flag + g0);
          f = nz_bytes(v.x) | (nz_bytes(v.y) << 4) | (nz_bytes(v.z) << 8) | (nz_bytes(v.w) << 12);
        } else {
          for (uint32_t j = 0; j < nin; ++j) f |= (spec.flag[g0 + j] != 0 ? 1u : 0u) << j;
        }
        m16 &= f;
      }
      if (spec.state) {
        uint32_t f = 0;
        if (vec_state && nin == 16) {
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const uint4 v = *(const uint4*)(spec.state + g0 + 4 * q);
            f |= ((v.x == 2u ? 1u : 0u) | (v.y == 2u ? 2u : 0u) | (v.z == 2u ? 4u : 0u) | (v.w == 2u ? 8u : 0u))
                 << (4 * q);
          }
        } else {
          for (uint32_t j = 0; j < nin; ++j) f |= (spec.state[g0 + j] == 2u ? 1u : 0u) << j;
        }
        m16 &= f;
      }
    }
    // each lane appends its live groups at its prefix position; live groups
    // are sparse, so a lane rarely has more than one
    const uint32_t c = __popc(m16);
    uint32_t incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += y;
    }
    const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    if (total == 0) continue;
    // wb holds logical entries [shift, shift + 64); this step's entries take
    // logical positions [cnt, cnt + total), this lane's from `pos`; every
    // full batch of 32 is offered and the rest moves down
    uint32_t pos = cnt + incl - c;
    uint32_t bits = m16;
    const uint32_t fill = cnt + total;
    uint32_t shift = 0;
    for (;;) {
      while (bits && pos < shift + 64) {
        const int j = __ffs(bits) - 1;
        bits &= bits - 1;
        wb[pos - shift] = (uint32_t)(g0 + (uint64_t)j);
        ++pos;
      }
      __syncwarp();
      const uint32_t have = (fill < shift + 64 ? fill : shift + 64) - shift;  // warp-uniform
      if (have < 32) {
        cnt = have;
        break;
      }
      process(32);
      __syncwarp();
      const uint32_t rest = have - 32;
      const uint32_t x = (uint32_t)lane < rest ? wb[32 + lane] : 0u;
      __syncwarp();
      if ((uint32_t)lane < rest) wb[lane] = x;
      __syncwarp();
      shift += 32;
    }
  }
  if (cnt) process(cnt);
  block_merge_lists<WARPS>(L, s_l, warp, lane);
  if (warp == 0 && lane < K) {
    // the CTA's list in its own K slots, best first: the candidates that can
    // still win (a prefix: the leading bits grow along the list), then
    // padding
    const uint64_t gc = ~*(volatile unsigned long long*)&gst->cut_inv;
    const bool keep = L.ix != 0xFFFFFFFFu && key_top64(L.w, tb) <= gc;
    const uint64_t at = (uint64_t)blockIdx.x * (uint64_t)K + (uint64_t)lane;
    SortItem it;
    it.w[0] = L.w[0]; it.w[1] = L.w[1]; it.w[2] = L.w[2]; it.w[3] = L.w[3];
    out_keys[at] = it;
    out_idx[at] = keep ? L.ix : 0xFFFFFFFFu;
  }
}

// Merge pass of the fused top-K. The first pass leaves each CTA's K best in
// the CTA's own K slots, best first (padding, index 0xFFFFFFFF, after the last
// that can still win). The K-th smallest of the lists' heads, H, bounds the
// result: the K heads at or below H are K candidates, so no candidate above
// H wins, and only the (at most K) lists whose heads are at or below H hold
// candidates at or below it: at most K * K survivors. One CTA ranks the heads
// by counting (each thread one head against all), keeps the candidates at or
// below H, and ranks those by counting again; every step is parallel over
// the CTA, with three barriers. (A serial merge of the lists on one warp, a
// radix select and a bitonic sort of all candidates each measured 35-88 us
// here: one CTA's dependent steps are latency-bound.)
constexpr int kMhThreads = 1024;

__global__ void __launch_bounds__(kMhThreads) k_topk_merge_heads(const SortItem* __restrict__ keys,
                                                                 const uint32_t* __restrict__ idx, uint32_t lists,
                                                                 int K, int cut_bits, uint32_t* __restrict__ out_idx,
                                                                 uint64_t* out_count, uint64_t* reset,
                                                                 const FinalOut* __restrict__ fin, int n_fin) {
  extern __shared__ __align__(16) uint8_t mh_smem[];
  Cand* const s_head = (Cand*)mh_smem;             // [lists]
  Cand* const s_sel = s_head + lists;              // [K * K]
  uint64_t* const s_ht = (uint64_t*)(s_sel + (size_t)K * K);  // [lists] leading 64 key bits of each head
  uint32_t* const s_rank = (uint32_t*)(s_ht + lists);         // [lists]
  __shared__ Cand s_h;
  __shared__ uint32_t s_valid, s_m;
  auto load = [&](uint64_t i) {
    Cand c = cand_inf();
    const uint32_t ix = idx[i];
    if (ix != 0xFFFFFFFFu) {
      const SortItem k = keys[i];
      c.w[0] = k.w[0]; c.w[1] = k.w[1]; c.w[2] = k.w[2]; c.w[3] = k.w[3];
      c.ix = ix;
    }
    return c;
  };
  // a before b in the result's order: leading words first, full keys on ties
  auto before = [&](uint64_t ta, const Cand& a, uint64_t tb, const Cand& b) {
    return ta < tb || (ta == tb && cand_less(a, b));
  };
  if (threadIdx.x == 0) {
    s_valid = 0;
    s_m = 0;
    s_h = cand_inf();
  }
  for (uint32_t l = threadIdx.x; l < lists; l += kMhThreads) {
    const Cand h = load((uint64_t)l * K);
    s_head[l] = h;
    s_ht[l] = h.ix == 0xFFFFFFFFu ? ~0ULL : key_top64(h.w, cut_bits);
    s_rank[l] = 0;
  }
  __syncthreads();
  // Rank of every valid head among the heads: P threads per head, each
  // counting the heads before it in one share of the list.
  const uint32_t P = lists >= kMhThreads ? 1u : (kMhThreads / lists < 32 ? kMhThreads / lists : 32);
  for (uint32_t t = threadIdx.x; t < lists * P; t += kMhThreads) {
    const uint32_t l = t / P, part = t % P;
    const Cand h = s_head[l];
    if (h.ix == 0xFFFFFFFFu) continue;
    const uint64_t th = s_ht[l];
    if (part == 0) atomicAdd(&s_valid, 1u);
    uint32_t r = 0;
    for (uint32_t j = part; j < lists; j += P) {
      const uint64_t tj = s_ht[j];
      if (tj < th) ++r;
      else if (tj == th && j != l && cand_less(s_head[j], h)) ++r;
    }
    atomicAdd(&s_rank[l], r);
  }
  __syncthreads();
  for (uint32_t l = threadIdx.x; l < lists; l += kMhThreads)
    if (s_head[l].ix != 0xFFFFFFFFu && s_rank[l] == (uint32_t)K - 1) s_h = s_head[l];
  __syncthreads();
  // fewer valid heads than K: every valid candidate survives
  const Cand H = s_valid >= (uint32_t)K ? s_h : cand_inf();
  const uint64_t tH = H.ix == 0xFFFFFFFFu ? ~0ULL : key_top64(H.w, cut_bits);
  const uint32_t n = lists * (uint32_t)K;
  for (uint32_t i = threadIdx.x; i < n; i += kMhThreads) {
    const Cand c = load(i);
    if (c.ix == 0xFFFFFFFFu) continue;
    const uint64_t tc = key_top64(c.w, cut_bits);
    if (tc < tH || (tc == tH && !cand_less(H, c))) s_sel[atomicAdd(&s_m, 1u)] = c;
  }
  __syncthreads();
  const uint32_t m = s_m;
  for (uint32_t p = threadIdx.x; p < m; p += kMhThreads) {
    const Cand c = s_sel[p];
    const uint64_t tc = key_top64(c.w, cut_bits);
    uint32_t rank = 0;
    for (uint32_t q = 0; q < m; ++q) rank += before(key_top64(s_sel[q].w, cut_bits), s_sel[q], tc, c) ? 1u : 0u;
    if (rank < (uint32_t)K) {
      out_idx[rank] = c.ix;
      // the winner's final outputs, in its result row
      for (int o = 0; o < n_fin; ++o) finalize_row(fin[o], c.ix, rank);
    }
  }
  if (threadIdx.x == 0) {
    *out_count = m < (uint32_t)K ? m : (uint32_t)K;
    if (reset) {
      reset[0] = 0;
      reset[1] = 0;
    }
  }
}

// Dynamic shared memory of the merge: the heads and the survivors.
static size_t merge_heads_smem(unsigned lists, int k) {
  return ((size_t)lists + (size_t)k * k) * sizeof(Cand) + (size_t)lists * (sizeof(uint64_t) + sizeof(uint32_t));
}
constexpr size_t kMhMaxSmem = 200 * 1024;

constexpr int kTfThreads = 256;  // first pass
constexpr int kTfItems = 16;     // groups per lane per step
static unsigned topk_final_ctas(uint64_t n_max, unsigned max_ctas) {
  static int per_sm = 0;
  if (!per_sm) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_topk_final<kTfThreads>, kTfThreads, 0);
    if (per_sm <= 0) per_sm = 1;
  }
  // one wave of CTAs, each covering at least one step of 16 groups per lane
  uint64_t ctas = (uint64_t)sms() * (uint64_t)per_sm;
  const uint64_t want = (n_max + kTfThreads * kTfItems - 1) / (kTfThreads * kTfItems);
  if (want < ctas) ctas = want ? want : 1;
  if (max_ctas && ctas > max_ctas) ctas = max_ctas;
  return (unsigned)ctas;
}

// temp: the cross-CTA state (256 bytes), then the candidate keys and indices.
size_t topk_final_temp_bytes(uint64_t n_max, int k, unsigned max_ctas) {
  return 256 + (size_t)topk_final_ctas(n_max, max_ctas) * (size_t)k * (sizeof(SortItem) + sizeof(uint32_t));
}

unsigned topk_final_max_ctas_for(size_t temp_bytes, int k) {
  if (temp_bytes <= 256 || k <= 0) return 0;
  return (unsigned)((temp_bytes - 256) / ((size_t)k * (sizeof(SortItem) + sizeof(uint32_t))));
}

cudaError_t launch_topk_final(const TopkFinalSpec& spec, int k, uint32_t* out_g, uint64_t* out_count, void* temp,
                              cudaStream_t s, unsigned max_ctas, int phase, const FinalOut* fin, int n_fin) {
  if (k <= 0 || k > 32 || spec.n_parts <= 0 || spec.n_parts > kMaxOrder || spec.total_bits > 256 ||
      spec.bits0 <= 0 || spec.bits0 > spec.total_bits)
    return cudaErrorInvalidValue;
  const unsigned ctas = topk_final_ctas(spec.n_max, max_ctas);
  if (ctas == 0) return cudaErrorInvalidValue;
  TopkFinalState* gst = (TopkFinalState*)temp;
  SortItem* pk = (SortItem*)((uint8_t*)temp + 256);
  uint32_t* pi = (uint32_t*)(pk + (uint64_t)ctas * k);
  if (phase != 2) k_topk_final<kTfThreads><<<ctas, kTfThreads, 0, s>>>(spec, k, gst, pk, pi);
  if (phase != 1) {
    const size_t smem = merge_heads_smem(ctas, k);
    if (smem <= kMhMaxSmem) {
      // the opt-in shared memory limit, raised once for the largest size used here
      static std::once_flag once;
      static cudaError_t attr = cudaSuccess;
      std::call_once(once, [] {
        attr = cudaFuncSetAttribute(k_topk_merge_heads, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMhMaxSmem);
      });
      if (attr != cudaSuccess) return attr;
      k_topk_merge_heads<<<1, kMhThreads, smem, s>>>(pk, pi, ctas, k, spec.total_bits, out_g, out_count,
                                                     (uint64_t*)gst, fin, n_fin);
    } else {
      // the padded lists as one array (padding skipped), then the outputs
      k_topk_warp<1024><<<1, 1024, 0, s>>>(pk, pi, nullptr, (uint64_t)ctas * k, k, nullptr, out_g, out_count, 1,
                                           nullptr, (uint64_t*)gst, spec.total_bits);
      if (n_fin > 0) {
        const cudaError_t e = launch_finalize(fin, n_fin, out_g, out_count, (uint64_t)k, s);
        if (e != cudaSuccess) return e;
      }
    }
  }
  return cudaGetLastError();
}

size_t topk_temp_bytes(uint64_t n_max, int k) {
  uint64_t ctas = (uint64_t)sms();
  const uint64_t want = (n_max + 4095) / 4096;
  if (want < ctas) ctas = want ? want : 1;
  return ctas * (uint64_t)k * (sizeof(SortItem) + sizeof(uint32_t)) + 256;
}

template <int B>
static cudaError_t topk_b(const SortItem* keys, const uint32_t* idx, const uint64_t* count, uint64_t n_max, int k,
                          uint32_t* out_idx, uint64_t* out_count, void* temp, cudaStream_t s) {
  constexpr int T = 256;
  const size_t smem = (size_t)B * (sizeof(SortItem) + sizeof(uint32_t));
  auto k1 = k_topk<B, T>;
  cudaError_t e = cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  unsigned ctas = (unsigned)sms();
  uint64_t want = (n_max + 4095) / 4096;
  if (want < ctas) ctas = (unsigned)(want ? want : 1);
  SortItem* pk = (SortItem*)temp;
  uint32_t* pi = (uint32_t*)(pk + (uint64_t)ctas * k);
  k1<<<ctas, T, smem, s>>>(keys, idx, count, n_max, k, pk, pi, nullptr, 0);
  // Second pass over the per-CTA winners; the padding entries sort last.
  k1<<<1, T, smem, s>>>(pk, pi, nullptr, (uint64_t)ctas * k, k, nullptr, out_idx, out_count, 1);
  return cudaGetLastError();
}

cudaError_t launch_topk(const SortItem* keys, const uint32_t* idx, const uint64_t* count, uint64_t n_max, int k,
                        uint32_t* out_idx, uint64_t* out_count, void* temp, uint32_t* status, cudaStream_t s,
                        const uint32_t* remap) {
  if (k <= 0 || k > 1024 || (remap && k > 32)) return cudaErrorInvalidValue;
  if (k <= 32) {
    unsigned ctas = (unsigned)sms();
    const uint64_t want = (n_max + 4095) / 4096;
    if (want < ctas) ctas = (unsigned)(want ? want : 1);
    SortItem* pk = (SortItem*)temp;
    uint32_t* pi = (uint32_t*)(pk + (uint64_t)ctas * k);
    k_topk_warp<256><<<ctas, 256, 0, s>>>(keys, idx, count, n_max, k, pk, pi, nullptr, 0);
    k_topk_warp<256><<<1, 256, 0, s>>>(pk, pi, nullptr, (uint64_t)ctas * k, k, nullptr, out_idx, out_count, 1, remap);
    return cudaGetLastError();
  }
  if (k <= 128) return topk_b<512>(keys, idx, count, n_max, k, out_idx, out_count, temp, s);
  return topk_b<2048>(keys, idx, count, n_max, k, out_idx, out_count, temp, s);
}

}  // namespace mtl
