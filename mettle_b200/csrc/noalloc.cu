// noalloc.cu — top-K of one device column that allocates nothing.
//
// Some callers cannot allocate device memory at the point where they need a
// top-K. One example is a host that has handed all of the GPU's memory to
// its own pool and may not grow it. Another is code that must not stall the
// device, which cudaMalloc and cudaFree can do by synchronizing it. For
// them, mtl_topk_noalloc runs the fused top-K kernels (k_sort.cu) on buffers
// the caller owns. The kernels' one piece of scratch, the per-CTA candidate
// lists, lives in a fixed array in device memory that the library owns.
//
// * The array holds kScratchBytes (1 MiB) on every GPU that loads the
//   library, for as long as the process lives.
// * All calls share it, and it keeps whatever the last call left in it.
//   Its first 256 bytes (the pruning cut shared by the CTAs of one call)
//   must start at zero, so every call clears them on its stream before the
//   kernels run; the per-CTA candidate slots are all written by every call.
//   Calls whose kernels overlap on the GPU (on different streams, or from
//   different host threads without ordering) race on the array and can
//   return wrong rows; order them on one stream.
// * The first kernel's grid is capped so that its candidate lists fit the
//   array (each CTA then covers more rows), so every n up to 2^32 - 2 runs.
// * The first call on each device looks up the array's device address with
//   that device current. Make that first call before any stream capture
//   begins on the device.
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/mettle_cuda.h"
#include "kernels.h"

namespace mtl {
void set_last_error(const std::string& m);
}

namespace {

constexpr size_t kScratchBytes = 1u << 20;
constexpr int kMaxDevices = 64;

// Device scratch for the per-CTA candidate lists. Host code must not pass
// this symbol to a kernel: on the host it names a stand-in, not device
// memory. Use the address from scratch_for_current_device().
static __device__ __align__(256) unsigned char g_topk_scratch[kScratchBytes];

std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_topk_scratch on the current device, looked up once per
// device (with that device current).
int scratch_for_current_device(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    mtl::set_last_error(std::string("mtl_topk_noalloc: cudaGetDevice failed: ") + cudaGetErrorString(e));
    return MTL_DEVICE_ERROR;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    mtl::set_last_error("mtl_topk_noalloc: device ordinal out of range");
    return MTL_DEVICE_ERROR;
  }
  std::lock_guard<std::mutex> g(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_topk_scratch);
    if (e != cudaSuccess || !p) {
      mtl::set_last_error(std::string("mtl_topk_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
      return MTL_DEVICE_ERROR;
    }
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return MTL_OK;
}

}  // namespace

extern "C" int mtl_topk_noalloc(int32_t type, const void* values, uint64_t n, int32_t k, int32_t descending,
                                uint32_t* out_rows, uint64_t* out_count, void* stream) {
  if (type != MTL_T_BIGINT && type != MTL_T_TIMESTAMP) {
    mtl::set_last_error("mtl_topk_noalloc: only BIGINT and TIMESTAMP (64-bit) columns are supported");
    return MTL_UNSUPPORTED;
  }
  if (k < 1 || k > 32) {
    mtl::set_last_error("mtl_topk_noalloc: k must be between 1 and 32");
    return MTL_INVALID;
  }
  if (n >= 0xFFFFFFFFull) {
    mtl::set_last_error("mtl_topk_noalloc: at most 2^32 - 2 rows (row numbers are 32-bit)");
    return MTL_INVALID;
  }
  if ((n > 0 && !values) || !out_rows || !out_count) {
    mtl::set_last_error("mtl_topk_noalloc: null buffer");
    return MTL_INVALID;
  }
  const unsigned max_ctas = mtl::topk_final_max_ctas_for(kScratchBytes, k);
  const size_t need = mtl::topk_final_temp_bytes(n, k, max_ctas);
  if (max_ctas == 0 || need > kScratchBytes) {
    mtl::set_last_error("mtl_topk_noalloc: needs " + std::to_string(need) + " bytes of scratch; the fixed scratch holds " +
                        std::to_string(kScratchBytes));
    return MTL_INVALID;
  }
  void* scratch = nullptr;
  int rc = scratch_for_current_device(&scratch);
  if (rc != MTL_OK) return rc;

  // One ORDER BY part: the column's 64-bit values, read in place; ties go to
  // the lower row number.
  mtl::TopkFinalSpec spec;
  memset(&spec, 0, sizeof(spec));
  spec.n_parts = 1;
  spec.total_bits = 64;
  spec.bits0 = 64;
  spec.ptype[0] = mtl::P_I64;
  spec.desc[0] = descending ? 1 : 0;
  spec.part[0].kind = mtl::F_COPY_I64;
  spec.part[0].a = (const uint64_t*)values;
  spec.n_max = n;
  // the cross-CTA state starts at zero (a memset, not an allocation)
  cudaError_t e = cudaMemsetAsync(scratch, 0, 256, (cudaStream_t)stream);
  if (e == cudaSuccess)
    e = mtl::launch_topk_final(spec, k, out_rows, out_count, scratch, (cudaStream_t)stream, max_ctas);
  if (e != cudaSuccess) {
    mtl::set_last_error(std::string("mtl_topk_noalloc: launch failed: ") + cudaGetErrorString(e));
    return MTL_DEVICE_ERROR;
  }
  return MTL_OK;
}
