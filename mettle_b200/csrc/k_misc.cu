// k_misc.cu — compaction of aggregate tables, final aggregate outputs,
// gathers, the scalar SQL hooks and column statistics (sm_100a).
#include "final_common.cuh"
#include "kern_common.cuh"
#include "kernels.h"

namespace mtl {

namespace {
constexpr int kCThreads = 256;
constexpr int kCItems = 16;
constexpr int kCTile = kCThreads * kCItems;

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
unsigned grid_for(uint64_t n, int threads, int per_sm = 8) {
  uint64_t b = (n + threads - 1) / threads;
  uint64_t cap = (uint64_t)sms() * per_sm;
  if (b > cap) b = cap;
  return b ? (unsigned)b : 1u;
}
}  // namespace

size_t compact_tile_rows() { return kCTile; }

// ------------------------------------------------------------ compaction
// Order-preserving index compaction with decoupled look-back; the reference
// compacts with a global atomic per element (compact_grouped_rows,
// kernels.metal:1120), which loses the order.
template <typename Flag>
__global__ void __launch_bounds__(kCThreads) k_compact(Flag flag, uint64_t n_static, const uint64_t* n_dev,
                                                       uint32_t* out_idx, uint64_t* out_count, uint64_t* tstatus,
                                                       uint32_t* counter, uint32_t epoch, uint32_t* status) {
  __shared__ uint32_t s_warp[kCThreads / 32 + 1];
  __shared__ uint64_t s_tile, s_base;
  const uint64_t n = n_dev ? *n_dev : n_static;
  const uint64_t n_tiles = (n + kCTile - 1) / kCTile;
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) s_tile = atomicAdd(counter, 1u);
    __syncthreads();
    const uint64_t tile = s_tile;
    if (tile >= n_tiles) break;
    const uint64_t base_i = tile * kCTile + (uint64_t)tid * kCItems;
    uint32_t bits = 0;
#pragma unroll
    for (int i = 0; i < kCItems; ++i) {
      uint64_t g = base_i + i;
      bits |= (g < n && flag(g)) ? (1u << i) : 0u;
    }
    uint32_t total;
    uint32_t pos = block_excl_sum<kCThreads>(__popc(bits), s_warp, &total);
    if (tid < 32) {
      const uint64_t excl = lb_exclusive_warp(tstatus, tile, total, epoch, status);
      if (tid == 0) {
        s_base = excl;
        if (tile == n_tiles - 1) *out_count = excl + total;
      }
    }
    __syncthreads();
    const uint64_t base = s_base;
#pragma unroll
    for (int i = 0; i < kCItems; ++i)
      if ((bits >> i) & 1u) out_idx[base + pos++] = (uint32_t)(base_i + i);
    __syncthreads();
  }
  if (tid == 0) {
    if (n == 0 && blockIdx.x == 0) *out_count = 0;
    __threadfence();
    if (atomicAdd(counter + 1, 1u) == gridDim.x - 1) {
      counter[0] = 0;
      counter[1] = 0;
    }
  }
}

struct ReadyFlag {
  const uint32_t* state;
  __device__ bool operator()(uint64_t i) const { return state[i] == 2u; }
};
struct ByteFlag {
  const uint8_t* f;
  __device__ bool operator()(uint64_t i) const { return f[i] != 0; }
};

cudaError_t launch_compact_ready(const uint32_t* state, uint64_t capacity, uint32_t* out_idx, uint64_t* out_count,
                                 uint64_t* tile_status, uint32_t* tile_counter, uint32_t epoch, uint32_t* status,
                                 cudaStream_t s) {
  uint64_t tiles = (capacity + kCTile - 1) / kCTile;
  unsigned grid = (unsigned)(tiles < (uint64_t)sms() * 8 ? (tiles ? tiles : 1) : sms() * 8);
  k_compact<ReadyFlag><<<grid, kCThreads, 0, s>>>(ReadyFlag{state}, capacity, nullptr, out_idx, out_count,
                                                  tile_status, tile_counter, epoch, status);
  return cudaGetLastError();
}

cudaError_t launch_compact_flags(const uint8_t* flag, uint64_t n, const uint64_t* n_dev, uint32_t* out_idx,
                                 uint64_t* out_count, uint64_t* tile_status, uint32_t* tile_counter, uint32_t epoch,
                                 uint32_t* status, cudaStream_t s) {
  uint64_t tiles = (n + kCTile - 1) / kCTile;
  unsigned grid = (unsigned)(tiles < (uint64_t)sms() * 8 ? (tiles ? tiles : 1) : sms() * 8);
  k_compact<ByteFlag><<<grid, kCThreads, 0, s>>>(ByteFlag{flag}, n, n_dev, out_idx, out_count, tile_status,
                                                 tile_counter, epoch, status);
  return cudaGetLastError();
}

// ------------------------------------------------------------ gathers
template <typename T>
__global__ void k_gather(const T* __restrict__ in, const uint32_t* __restrict__ idx, const uint64_t* count,
                         uint64_t n_max, T* __restrict__ out) {
  const uint64_t n = count ? *count : n_max;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[idx[i]];
}

cudaError_t launch_gather_u64(const uint64_t* in, const uint32_t* idx, const uint64_t* count, uint64_t n_max,
                              uint64_t* out, cudaStream_t s) {
  k_gather<uint64_t><<<grid_for(n_max, 256), 256, 0, s>>>(in, idx, count, n_max, out);
  return cudaGetLastError();
}
cudaError_t launch_gather_u32(const uint32_t* in, const uint32_t* idx, const uint64_t* count, uint64_t n_max,
                              uint32_t* out, cudaStream_t s) {
  k_gather<uint32_t><<<grid_for(n_max, 256), 256, 0, s>>>(in, idx, count, n_max, out);
  return cudaGetLastError();
}
cudaError_t launch_gather_width(const void* in, int width, const uint32_t* idx, const uint64_t* count, uint64_t n_max,
                                void* out, cudaStream_t s) {
  unsigned g = grid_for(n_max, 256);
  switch (width) {
    case 4: k_gather<uint32_t><<<g, 256, 0, s>>>((const uint32_t*)in, idx, count, n_max, (uint32_t*)out); break;
    case 8: k_gather<uint64_t><<<g, 256, 0, s>>>((const uint64_t*)in, idx, count, n_max, (uint64_t*)out); break;
    case 16: k_gather<longlong2><<<g, 256, 0, s>>>((const longlong2*)in, idx, count, n_max, (longlong2*)out); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// ------------------------------------------------------------ finalize
__global__ void k_finalize(const FinalOut* __restrict__ outs, int n_outs, const uint32_t* __restrict__ idx,
                           const uint64_t* count, uint64_t n_max) {
  const uint64_t n = count ? *count : n_max;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t g = idx ? idx[i] : i;
    for (int o = 0; o < n_outs; ++o) finalize_row(outs[o], g, i);
  }
}

// ------------------------------------------------------------ late materialization
// Each thread takes kGoRows output rows (one per 256-row stripe of the
// CTA's step, so that every warp access is 32 consecutive rows), reads their
// row ids once, and then writes every output for them with its source loads
// issued before any value is stored.
constexpr int kGoThreads = 256;
constexpr int kGoRows = 4;

__device__ __forceinline__ int64_t gather_apply(const GatherOut& g, int64_t x, uint32_t& st) {
  if (g.op == 0) return x;
  const int64_t k = g.k;
  switch (g.type) {
    case P_I32: return fit32(g.op == VM_ADD ? x + k : g.op == VM_SUB ? x - k : x * k, st);
    case P_I64: return g.op == VM_ADD ? add64(x, k, st) : g.op == VM_SUB ? sub64(x, k, st) : mul64(x, k, st);
    case P_F32: {
      const float a = as_f32(x), y = as_f32(k);
      return f32_bits(g.op == VM_ADD ? __fadd_rn(a, y) : g.op == VM_SUB ? __fsub_rn(a, y) : __fmul_rn(a, y));
    }
    default: {
      const double a = as_f64(x), y = as_f64(k);
      return f64_bits(g.op == VM_ADD ? __dadd_rn(a, y) : g.op == VM_SUB ? __dsub_rn(a, y) : __dmul_rn(a, y));
    }
  }
}

__global__ void __launch_bounds__(kGoThreads) k_gather_outs(const GatherOut* __restrict__ outs, int n_outs,
                                                            const uint32_t* __restrict__ rid, const uint64_t* count,
                                                            uint64_t n_max, uint32_t* status) {
  uint64_t n = count ? *count : n_max;
  if (n > n_max) n = n_max;
  uint32_t st = 0;
  const uint64_t step = (uint64_t)kGoThreads * kGoRows;
  for (uint64_t base = (uint64_t)blockIdx.x * step; base < n; base += (uint64_t)gridDim.x * step) {
    uint32_t r[kGoRows];
#pragma unroll
    for (int j = 0; j < kGoRows; ++j) {
      const uint64_t i = base + (uint64_t)j * kGoThreads + threadIdx.x;
      r[j] = i < n ? __ldg(rid + i) : 0u;
    }
    for (int o = 0; o < n_outs; ++o) {
      const GatherOut g = outs[o];
      int64_t v[kGoRows];
#pragma unroll
      for (int j = 0; j < kGoRows; ++j) {
        const uint64_t i = base + (uint64_t)j * kGoThreads + threadIdx.x;
        v[j] = 0;
        if (i < n) {
          if (g.in_kind == 2) v[j] = __ldg((const long long*)g.src + r[j]);
          else if (g.in_kind == 0) v[j] = (int64_t)__ldg((const int*)g.src + r[j]);
          else v[j] = (int64_t)(uint32_t)__ldg((const unsigned int*)g.src + r[j]);
        }
      }
#pragma unroll
      for (int j = 0; j < kGoRows; ++j) {
        const uint64_t i = base + (uint64_t)j * kGoThreads + threadIdx.x;
        if (i >= n) continue;
        const int64_t y = gather_apply(g, v[j], st);
        if (g.out_width == 4) ((uint32_t*)g.out)[i] = (uint32_t)y;
        else ((int64_t*)g.out)[i] = y;
      }
    }
  }
  if (st && status) atomicOr(status, st);
}

cudaError_t launch_gather_outs(const GatherOut* outs, int n_outs, const uint32_t* rid, const uint64_t* count,
                               uint64_t n_max, uint32_t* status, cudaStream_t s) {
  if (n_outs <= 0) return cudaSuccess;
  k_gather_outs<<<grid_for((n_max + kGoRows - 1) / kGoRows, kGoThreads), kGoThreads, 0, s>>>(outs, n_outs, rid, count,
                                                                                          n_max, status);
  return cudaGetLastError();
}

cudaError_t launch_finalize(const FinalOut* outs, int n_outs, const uint32_t* idx, const uint64_t* count,
                            uint64_t n_max, cudaStream_t s) {
  k_finalize<<<grid_for(n_max, 256), 256, 0, s>>>(outs, n_outs, idx, count, n_max);
  return cudaGetLastError();
}

// ------------------------------------------------------------ scalar hooks
// gpu_add_scalar / gpu_mul_scalar: out = in op k with DuckDB result types
// and overflow errors; the reference's project_*_scalar kernels
// (kernels.metal:4-68) compute the same element-wise op.
__global__ void k_scalar_arith(int op, int ptype, const void* __restrict__ in, uint64_t n, int64_t ilit, double flit,
                               void* __restrict__ out, uint32_t* status) {
  uint32_t st = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    switch (ptype) {
      case P_I32: {
        int64_t x = ((const int32_t*)in)[i];
        int64_t r = op == 0 ? x + ilit : x * ilit;
        ((int32_t*)out)[i] = (int32_t)fit32(r, st);
        break;
      }
      case P_I64: {
        int64_t x = ((const int64_t*)in)[i];
        ((int64_t*)out)[i] = op == 0 ? add64(x, ilit, st) : mul64(x, ilit, st);
        break;
      }
      case P_F32: {
        float x = ((const float*)in)[i], k = (float)flit;
        ((float*)out)[i] = op == 0 ? __fadd_rn(x, k) : __fmul_rn(x, k);
        break;
      }
      default: {
        double x = ((const double*)in)[i];
        ((double*)out)[i] = op == 0 ? __dadd_rn(x, flit) : __dmul_rn(x, flit);
        break;
      }
    }
  }
  if (st) atomicOr(status, st);
}

// gpu_{eq,lt,le,gt,ge}_scalar: u8 mask with the reference's op codes
// (compare_*_scalar, kernels.metal:70-173).
__global__ void k_scalar_compare(int op, int ptype, const void* __restrict__ in, uint64_t n, int64_t ilit, double flit,
                                 uint8_t* __restrict__ out) {
  DPred p;
  p.col = 0;
  p.op = op;
  p.ilit = ilit;
  p.flit = flit;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = eval_pred_bits(load_bits(in, ptype, i), ptype, p) ? 1 : 0;
}

cudaError_t launch_scalar_arith(int op, int ptype, const void* in, uint64_t n, int64_t ilit, double flit, void* out,
                                uint32_t* status, cudaStream_t s) {
  k_scalar_arith<<<grid_for(n, 256), 256, 0, s>>>(op, ptype, in, n, ilit, flit, out, status);
  return cudaGetLastError();
}
cudaError_t launch_scalar_compare(int op, int ptype, const void* in, uint64_t n, int64_t ilit, double flit, uint8_t* out,
                                  cudaStream_t s) {
  k_scalar_compare<<<grid_for(n, 256), 256, 0, s>>>(op, ptype, in, n, ilit, flit, out);
  return cudaGetLastError();
}

// ------------------------------------------------------------ statistics
__global__ void k_minmax(const void* __restrict__ col, int ptype, uint64_t n, int64_t* out) {
  int64_t mn = 0x7FFFFFFFFFFFFFFFLL, mx = (int64_t)0x8000000000000000ULL;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    int64_t v = load_bits(col, ptype, i);
    mn = v < mn ? v : mn;
    mx = v > mx ? v : mx;
  }
  for (int o = 16; o > 0; o >>= 1) {
    int64_t a = __shfl_down_sync(0xFFFFFFFFu, mn, o), b = __shfl_down_sync(0xFFFFFFFFu, mx, o);
    mn = a < mn ? a : mn;
    mx = b > mx ? b : mx;
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin((long long*)out, (long long)mn);
    atomicMax((long long*)out + 1, (long long)mx);
  }
}

cudaError_t launch_minmax_i(const void* col, int ptype, uint64_t n, int64_t* out, cudaStream_t s) {
  k_minmax<<<grid_for(n, 256, 4), 256, 0, s>>>(col, ptype, n, out);
  return cudaGetLastError();
}

__global__ void k_count_dups(const void* __restrict__ col, int ptype, uint64_t n, int64_t* table, uint64_t cap,
                             uint32_t* special, unsigned long long* out) {
  unsigned long long dups = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    int64_t key = load_bits(col, ptype, i);
    if (key == kEmptyKey) {
      if (atomicAdd(special, 1u) != 0u) ++dups;
      continue;
    }
    uint64_t h = hash_slot(hash64((uint64_t)key), cap);
    for (uint64_t p = 0; p < cap; ++p) {
      unsigned long long prev =
          atomicCAS((unsigned long long*)(table + h), (unsigned long long)kEmptyKey, (unsigned long long)key);
      if (prev == (unsigned long long)kEmptyKey) break;
      if ((int64_t)prev == key) {
        ++dups;
        break;
      }
      if (++h == cap) h = 0;
    }
  }
  for (int o = 16; o > 0; o >>= 1) dups += __shfl_down_sync(0xFFFFFFFFu, dups, o);
  if ((threadIdx.x & 31) == 0 && dups) atomicAdd(out, dups);
}

cudaError_t launch_count_dups(const void* col, int ptype, uint64_t n, int64_t* table, uint64_t cap, uint32_t* special,
                              unsigned long long* out, cudaStream_t s) {
  k_count_dups<<<grid_for(n, 256), 256, 0, s>>>(col, ptype, n, table, cap, special, out);
  return cudaGetLastError();
}

// Duplicate count for an integer column whose value range is small: one
// presence bit per value in [vmin, vmin + span).
__global__ void k_count_dups_dense(const void* __restrict__ col, int ptype, uint64_t n, int64_t vmin, uint64_t span,
                                   uint32_t* bits, unsigned long long* out) {
  unsigned long long dups = 0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t k = (uint64_t)(load_bits(col, ptype, i) - vmin);
    if (k >= span) continue;  // cannot happen for a true min/max
    const uint32_t bit = 1u << (k & 31);
    if (atomicOr(bits + (k >> 5), bit) & bit) ++dups;
  }
  for (int o = 16; o > 0; o >>= 1) dups += __shfl_down_sync(0xFFFFFFFFu, dups, o);
  if ((threadIdx.x & 31) == 0 && dups) atomicAdd(out, dups);
}

cudaError_t launch_count_dups_dense(const void* col, int ptype, uint64_t n, int64_t vmin, uint64_t span,
                                    uint32_t* bits, unsigned long long* out, cudaStream_t s) {
  k_count_dups_dense<<<grid_for(n, 256), 256, 0, s>>>(col, ptype, n, vmin, span, bits, out);
  return cudaGetLastError();
}

__global__ void k_fill_u64(uint64_t* p, uint64_t n, uint64_t v) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = v;
}
cudaError_t launch_fill_u64(uint64_t* p, uint64_t n, uint64_t v, cudaStream_t s) {
  k_fill_u64<<<grid_for(n, 256), 256, 0, s>>>(p, n, v);
  return cudaGetLastError();
}

__global__ void k_fill_segments(const FillSeg* __restrict__ segs) {
  const FillSeg sg = segs[blockIdx.y];
  if (sg.stride) {
    const uint64_t n = sg.bytes / sg.stride;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
      *(uint64_t*)((char*)sg.ptr + i * sg.stride) = sg.pattern;
    return;
  }
  const uint64_t n16 = sg.bytes / 16;
  if (sg.entry) {
    const uint64_t h = sg.entry_words / 2;  // 16-byte pieces per entry
    ulonglong2* p = (ulonglong2*)sg.ptr;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n16; i += (uint64_t)gridDim.x * blockDim.x) {
      const uint64_t w = 2 * (i % h);
      p[i] = make_ulonglong2(__ldg(sg.entry + w), __ldg(sg.entry + w + 1));
    }
    return;
  }
  const ulonglong2 v = make_ulonglong2(sg.pattern, sg.pattern);
  ulonglong2* p = (ulonglong2*)sg.ptr;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n16; i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

cudaError_t launch_fill_segments(const FillSeg* segs_dev, int n_segs, uint64_t max_bytes, cudaStream_t s) {
  if (n_segs <= 0) return cudaSuccess;
  dim3 grid(grid_for(max_bytes / 16, 256, 4), (unsigned)n_segs);
  k_fill_segments<<<grid, 256, 0, s>>>(segs_dev);
  return cudaGetLastError();
}

}  // namespace mtl
