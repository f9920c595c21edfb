// kernels.h — host-callable launchers for the sm_100a kernels. All take a
// stream and enqueue asynchronously; none synchronizes.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "dev_types.h"

namespace mtl {

// ---- pipeline (k_pipeline.cu)
size_t pipeline_tile_rows();
size_t pipeline_warp_tile_rows();  // rows of a warp-tile (k_pipeline.cu)
// Two-pass order-preserving compaction (k_pipeline.cu): an SK_MAT_COUNT
// pipeline writes each 256-row tile's survivors into d.tile_pos,
// launch_mat_scan turns them into offsets (d.tile_pos within chunks of
// kMatScanTiles tiles, d.chunk_pos per chunk, *d.out_count the total), and an
// SK_MAT_WRITE pipeline over the same rows and ops writes the outputs there.
cudaError_t launch_mat_scan(const PipeDesc& d, uint64_t n_rows, cudaStream_t s);
size_t pipeline_smem_bytes(const PipeDesc& d);
// n_hint bounds the tuples (grid sizing when the count lives on the device).
cudaError_t launch_pipeline(const PipeDesc& d, uint64_t n_hint, cudaStream_t s);
// Order-preserving compaction (SK_MATERIALIZE) runs a kernel with CTA-wide
// tiles of pipeline_tile_rows() rows (k_pipeline_cta.cu); launch_pipeline
// dispatches to it.
cudaError_t launch_pipeline_materialize(const PipeDesc& d, uint64_t n_hint, cudaStream_t s);
// Partitioned one-key aggregation (k_pipeline.cu): the SK_PART_COUNT and
// SK_PART_SCATTER pipelines run pipeline_part_ctas() CTAs; between them
// launch_part_scan turns the per-CTA partition counts into write positions;
// launch_part_agg then aggregates the records into d.table: one CTA per
// chunk of at most d.part_chunk records of one partition, with a
// shared-memory table of d.smem_capacity entries; n_hint bounds the records.
int part_max_bits();
int part_max_split();  // log2 of the most sub-partitions k_part_agg takes a chunk in
int part_max_values();
int pipeline_part_ctas();
size_t part_agg_smem_bytes(const PipeDesc& d);
cudaError_t launch_part_scan(const PipeDesc& d, cudaStream_t s);
cudaError_t launch_part_agg(const PipeDesc& d, uint64_t n_hint, cudaStream_t s);
// One-pass few-group aggregation (k_pipeline.cu): d describes one table
// (no filters, probes or tuple input), a one-key CAS table in d.table, a
// plain-column key (d.key_prog[0]) and aggregates whose inputs are plain
// columns (at most agg_few_max_cols() distinct) or none; d.smem_capacity is
// the CTA table's entries (a power of two above the group count).
size_t agg_few_smem_bytes(const PipeDesc& d);
int agg_few_max_cols();
cudaError_t launch_agg_few(const PipeDesc& d, uint64_t n_hint, cudaStream_t s);

// ---- aggregate finalize (k_misc.cu)
// Order-preserving list of READY slots of a hash aggregate table.
cudaError_t launch_compact_ready(const uint32_t* state, uint64_t capacity, uint32_t* out_idx,
                                 uint64_t* out_count, uint64_t* tile_status, uint32_t* tile_counter,
                                 uint32_t epoch, uint32_t* status, cudaStream_t s);
// Order-preserving list of indices i < n with flag[i] != 0 (u8 flags).
cudaError_t launch_compact_flags(const uint8_t* flag, uint64_t n, const uint64_t* n_dev, uint32_t* out_idx,
                                 uint64_t* out_count, uint64_t* tile_status, uint32_t* tile_counter,
                                 uint32_t epoch, uint32_t* status, cudaStream_t s);
size_t compact_tile_rows();

// Gather one u64 state array / key array through an index list into a
// dense array (out[i] = in[idx[i]]), for i < *count.
cudaError_t launch_gather_u64(const uint64_t* in, const uint32_t* idx, const uint64_t* count, uint64_t n_max,
                              uint64_t* out, cudaStream_t s);
cudaError_t launch_gather_u32(const uint32_t* in, const uint32_t* idx, const uint64_t* count, uint64_t n_max,
                              uint32_t* out, cudaStream_t s);

// Final aggregate outputs. kind: see FinalKind in k_misc.cu.
enum FinalKind : int32_t {
  F_COPY_I32 = 1,   // low 32 bits of a u64 state/key word
  F_COPY_I64 = 2,
  F_COPY_F32 = 3,   // key word holding f32 bits
  F_COPY_F64 = 4,
  F_SUM_I128 = 5,   // (lo, hi) -> i128
  F_SUM_I64_AS_I128 = 6,
  F_MINMAX_F32 = 7,  // ordered image -> f32
  F_MINMAX_F64 = 8,  // ordered image -> f64
  F_AVG_I128_LD = 9,  // (long double)sum / count -> double (DuckDB BIGINT AVG)
  F_AVG_I64_D = 10,   // (double)sum / (double)count (DuckDB INTEGER AVG)
  F_AVG_F64 = 11,     // double sum / count
  F_AVG_DEC = 12,     // decimal: (long double)sum / count / 10^scale
  F_GATHER_COL = 13,  // out[i] = col[rid[g]] (group key of a representative row), width 4/8
};
struct FinalOut {
  int32_t kind;
  int32_t width;         // F_GATHER_COL element width
  const uint64_t* a;     // state or key words, indexed by group g
  const int64_t* a_hi;   // high words
  const uint64_t* cnt;   // counts (AVG)
  int32_t stride;        // words between consecutive groups' words in a, a_hi, cnt (0 or 1: dense)
  int32_t pad;
  void* out;
  double scale;          // AVG of DECIMAL: 10^scale
  const void* col;       // F_GATHER_COL column
  const uint32_t* rid;   // F_GATHER_COL row id per group
};
// For i < *count (or n_max): g = idx ? idx[i] : i; writes out[i] per FinalOut.
cudaError_t launch_finalize(const FinalOut* outs, int n_outs, const uint32_t* idx, const uint64_t* count,
                            uint64_t n_max, cudaStream_t s);

// ---- order by / top-K (k_sort.cu)
// Encodes ORDER BY keys of rows [0, *count) into 32-byte order-preserving
// images (most significant word first) plus a row index.
struct SortItem {
  uint64_t w[4];
};
cudaError_t launch_encode_keys(const SortKeySpec& spec, const uint64_t* count, uint64_t n_max, SortItem* keys,
                               uint32_t* idx, cudaStream_t s);
// Stable LSD radix sort of (keys, idx) on the given number of significant
// key bytes (from the least significant), count on the device.
size_t radix_sort_temp_bytes(uint64_t n_max);
cudaError_t launch_radix_sort(SortItem* keys, uint32_t* idx, SortItem* keys_tmp, uint32_t* idx_tmp,
                              const uint64_t* count, uint64_t n_max, int key_bytes, void* temp,
                              cudaStream_t s, int* result_in_tmp);
// Top-K of (keys, idx): smallest K images first. Writes K (or fewer) indices.
size_t topk_temp_bytes(uint64_t n_max, int k);
// remap (K <= 32 only): write remap[i] instead of the winning index i.
cudaError_t launch_topk(const SortItem* keys, const uint32_t* idx, const uint64_t* count, uint64_t n_max, int k,
                        uint32_t* out_idx, uint64_t* out_count, void* temp, uint32_t* status, cudaStream_t s,
                        const uint32_t* remap = nullptr);

// Fused aggregate top-K (K <= 32) straight from the aggregate states: the
// candidates are the groups g < n (n = min(*n_dev, n_max) when n_dev is
// given) whose flag byte is nonzero or whose table state is READY (2), or
// every g < n when both are null. A candidate's key is the order-preserving
// image of the ORDER BY parts (each a FinalOut evaluated at g, of physical
// type ptype), ties broken by g. Writes the K best g, best first, and their
// number.
struct TopkFinalSpec {
  int32_t n_parts;
  int32_t total_bits;  // bits of all parts
  int32_t bits0;       // bits of the first part
  int32_t ptype[kMaxOrder];
  int32_t desc[kMaxOrder];
  FinalOut part[kMaxOrder];
  const uint8_t* flag;
  const uint32_t* state;
  const uint64_t* n_dev;
  uint64_t n_max;
};
// temp starts with 256 bytes of cross-CTA state that must be zero when the
// launch starts (the launch leaves it zero again). max_ctas (0: no limit)
// caps the first pass's grid, and with it the temp size; each CTA then
// covers more groups.
size_t topk_final_temp_bytes(uint64_t n_max, int k, unsigned max_ctas = 0);
// The largest max_ctas whose temp fits in temp_bytes.
unsigned topk_final_max_ctas_for(size_t temp_bytes, int k);
// phase: 0 both kernels, 1 the first pass only, 2 the merge pass only (the
// two phases as separate steps of a program, each timed on its own). With
// `fin` (n_fin outputs) the merge pass also writes the winners' final
// outputs, row i for winner i (as launch_finalize over out_g would).
cudaError_t launch_topk_final(const TopkFinalSpec& spec, int k, uint32_t* out_g, uint64_t* out_count, void* temp,
                              cudaStream_t s, unsigned max_ctas = 0, int phase = 0, const FinalOut* fin = nullptr,
                              int n_fin = 0);

// ---- gathers for final materialization (k_misc.cu)
// out[i] = in[idx[i]] for fixed width elements (4, 8 or 16 bytes).
cudaError_t launch_gather_width(const void* in, int width, const uint32_t* idx, const uint64_t* count,
                                uint64_t n_max, void* out, cudaStream_t s);

// Late materialization of a scan's outputs (k_misc.cu): out[i] = f(src[rid[i]])
// for i < *count, f a plain copy or one + - * with a constant in a
// non-128-bit type (the VM's arithmetic and overflow rules).
struct GatherOut {
  const void* src;    // column, indexed by row id
  void* out;
  int32_t in_kind;    // 0: 32-bit signed (widened by sign), 1: 32-bit other (zero), 2: 64-bit
  int32_t out_width;  // 4 or 8
  int32_t op;         // 0: copy, else VM_ADD, VM_SUB or VM_MUL
  int32_t type;       // arithmetic type of the op (P_I32, P_I64, P_F32, P_F64)
  int64_t k;          // constant (bits)
};
cudaError_t launch_gather_outs(const GatherOut* outs, int n_outs, const uint32_t* rid, const uint64_t* count,
                               uint64_t n_max, uint32_t* status, cudaStream_t s);

// ---- scalar hooks (k_misc.cu): gpu_{add,mul}_scalar, gpu_{eq,lt,le,gt,ge}_scalar
cudaError_t launch_scalar_arith(int op, int ptype, const void* in, uint64_t n, int64_t ilit, double flit, void* out,
                                uint32_t* status, cudaStream_t s);
cudaError_t launch_scalar_compare(int op, int ptype, const void* in, uint64_t n, int64_t ilit, double flit,
                                  uint8_t* out, cudaStream_t s);

// ---- column statistics (k_misc.cu)
// min/max of an integer-like column as i64 (out[0] = min, out[1] = max).
cudaError_t launch_minmax_i(const void* col, int ptype, uint64_t n, int64_t* out, cudaStream_t s);
// Counts keys that occur more than once by inserting into an open-addressing
// table of `cap` i64 slots (all bits set = empty); out[0] = duplicates.
cudaError_t launch_count_dups(const void* col, int ptype, uint64_t n, int64_t* table, uint64_t cap,
                              uint32_t* special, unsigned long long* out, cudaStream_t s);
// Same count with a presence bitmap over [vmin, vmin + span) (span / 8 bytes).
cudaError_t launch_count_dups_dense(const void* col, int ptype, uint64_t n, int64_t vmin, uint64_t span,
                                    uint32_t* bits, unsigned long long* out, cudaStream_t s);

// ---- utility
cudaError_t launch_fill_u64(uint64_t* p, uint64_t n, uint64_t v, cudaStream_t s);
// One launch that fills every segment with a repeated 64-bit pattern
// (scratch initialization of a whole query). Segments are 16-byte aligned
// and their sizes multiples of 16.
struct FillSeg {
  void* ptr;
  uint64_t bytes;
  uint64_t pattern;
  uint64_t stride;  // 0: fill [ptr, ptr + bytes); else one 8-byte word every `stride` bytes
  // non-null (with stride 0): whole entries of entry_words words (even), word
  // w of the segment set to entry[w % entry_words], in 16-byte stores
  const uint64_t* entry;
  uint64_t entry_words;
};
cudaError_t launch_fill_segments(const FillSeg* segs_dev, int n_segs, uint64_t max_bytes, cudaStream_t s);

}  // namespace mtl
