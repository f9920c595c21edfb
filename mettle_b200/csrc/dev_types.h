// dev_types.h — plain-old-data descriptors shared by the host planner and the
// sm_100a kernels. Everything here is passed to kernels by value
// (__grid_constant__) or lives in device memory; no pointers to host memory.
//
// The engine runs a query as a short sequence of "pipelines". A pipeline
// scans one input (a base table, or a list of row-id tuples), applies the
// filters and join probes of that input in order, and ends in one sink:
// a join build, a grouped/ungrouped aggregate, or an order-preserving
// materialization. This replaces the reference's per-op dispatch chain
// (compare -> and_masks -> filter_to_indices -> gather -> join -> compact ->
// reindex, src/plan/executor/fast_path/*.rs) with one launch per pipeline.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mtl {

// ------------------------------------------------------------ limits
constexpr int kMatScanTiles = 4096;  // tiles per chunk of the two-pass compaction's scan
constexpr int kMaxStream = 6;        // columns a warp-tile pipeline stages into shared memory
constexpr int kMaxSrc = 6;       // tables in one query
constexpr int kMaxPreds = 12;    // filter predicates in one pipeline
constexpr int kMaxProbes = 5;    // join probes in one pipeline
constexpr int kMaxCols = 32;     // columns referenced by one pipeline
constexpr int kMaxProgs = 16;    // expression programs in one pipeline
constexpr int kMaxIns = 12;      // instructions per expression program
constexpr int kMaxKeys = 4;      // group-by key words
constexpr int kMaxAggs = 12;     // aggregate states per group
constexpr int kMaxOrder = 8;     // ORDER BY key parts (incl. tie-breaks)

// ------------------------------------------------------------ physical types
enum PType : int32_t { P_NONE = 0, P_I32 = 1, P_I64 = 2, P_F32 = 3, P_F64 = 4, P_I128 = 5 };

__host__ __device__ inline int ptype_width(int32_t p) {
  return p == P_I32 || p == P_F32 ? 4 : (p == P_I128 ? 16 : 8);
}

// Compare op codes; 0..4 match the reference's compare_*_scalar op codes
// (src/metal/shaders/kernels.metal:70-173).
enum CmpOp : int32_t { C_EQ = 0, C_LT = 1, C_LE = 2, C_GT = 3, C_GE = 4, C_NE = 5, C_FALSE = 6, C_TRUE = 7 };

// Device status bits (one u32 per query; the host turns them into errors).
enum DevStatus : uint32_t {
  ST_OVERFLOW = 1u,        // integer overflow (DuckDB raises an error)
  ST_DUP_BUILD_KEY = 2u,   // a build side assumed unique had a duplicate key
  ST_SPIN_LIMIT = 4u,      // a bounded wait gave up
  ST_TABLE_FULL = 8u,      // a hash table ran out of slots
  ST_CAPACITY = 16u,       // an output buffer was too small
};

// ------------------------------------------------------------ columns
struct DCol {
  const void* ptr;   // device column (row-indexed)
  int32_t ptype;     // PType
  int32_t src;       // source (table) index the row id comes from
};

struct DPred {
  int32_t col;       // index into PipeDesc::cols
  int32_t op;        // CmpOp
  int64_t ilit;      // integer literal (I32/I64 columns)
  double flit;       // float literal (F32 compares in binary32)
};

// ------------------------------------------------------------ expressions
enum VmOp : int16_t {
  VM_COL = 1,    // push cols[arg]
  VM_CONST = 2,  // push constant bits k (lo) / k2 (hi for I128)
  VM_ADD = 3,
  VM_SUB = 4,
  VM_MUL = 5,
  VM_CAST = 6,   // convert top of stack from ptype arg to ptype `type`, scaled by k
  VM_NEG = 7,
  VM_SLOT = 8,   // push the slot of probe `arg` (representative-row grouping)
};

struct VmIns {
  int16_t op;
  int16_t type;   // result PType
  int32_t arg;
  int64_t k;      // constant bits / cast multiplier (power of ten, 1 = none)
  int64_t k2;     // constant hi bits (I128) / cast divisor flag
};

// A cast applied to one node of a FastExpr (on = 0: none).
struct VmCast {
  int16_t from, to;
  int32_t on;
  int64_t mul, div;
};

// The same expression as a fixed tree of at most three leaves (column or
// constant) and two binary ops, each node with an optional cast, so the
// device evaluates it without a stack machine. shape 0: not expressible;
// 1: L0; 2: L0 op0 L1; 3: L0 op1 (L1 op0 L2); 4: (L0 op0 L1) op1 L2.
struct VmFast {
  int32_t shape;
  int32_t pad;
  VmIns leaf[3];  // VM_COL or VM_CONST
  VmCast leaf_cast[3];
  VmIns op[2];    // op, type
  VmCast op_cast[2];
};

struct VmProg {
  int32_t n;
  int32_t out_type;
  int32_t depth;  // deepest stack the program reaches
  int32_t pad;
  VmIns ins[kMaxIns];
  VmFast fast;
};

// ------------------------------------------------------------ join builds
enum BuildKind : int32_t { B_NONE = 0, B_DENSE = 1, B_HASH = 2 };

// Hash-table entries start as kEmptyKey (all bits set, so a byte memset
// clears a table); the one key equal to it is kept in a side word.
constexpr int64_t kEmptyKey = -1;

// A build side with unique keys: key -> compact slot -> payload row ids.
struct DBuild {
  int32_t kind;
  int32_t key_ptype;        // P_I32 or P_I64
  int64_t key_min;          // dense: first key
  uint64_t capacity;        // dense: key span; hash: slots
  uint32_t* dense_map;      // dense: slot + 1 (valid only where dense_bits is set)
  uint32_t* dense_bits;     // dense: presence bitmap, one bit per key
  int64_t* hash_keys;       // hash: keys
  uint32_t* hash_slot;      // hash: slot + 1 per table entry
  uint32_t* hash_special;   // hash: slot + 1 of the key equal to kEmptyKey
  // payload[s][slot] = row id of source s; a build's slot is its own row
  // number, so the build's own source has no array (null)
  uint32_t* payload[kMaxSrc];
  int32_t unique_keys;      // the key column holds no duplicates (no check needed)
  int32_t pad;
  // hash: optional blocked Bloom filter of the inserted keys (null: none);
  // bloom_words is a power of two
  uint32_t* bloom;
  uint64_t bloom_words;
};

struct DProbe {
  int32_t key_col;          // index into cols (probe-side key)
  int32_t build;            // index into PipeDesc::builds
  uint32_t fill_mask;       // bit s: rid[s] = payload[s][slot]
  int32_t pad;
};

// ------------------------------------------------------------ pipeline ops
enum PipeOpKind : int32_t { OPK_FILTER = 1, OPK_PROBE = 2 };
struct PipeOp {
  int32_t kind;
  int32_t idx;
};

// ------------------------------------------------------------ aggregates
enum AggFn : int32_t {
  A_COUNT = 1,     // u64 count
  A_SUM_I = 2,     // 64-bit integer sum (exact; bound proven by the planner)
  A_SUM_I128 = 3,  // 128-bit integer sum, lo word + carry into hi word
  A_SUM_F = 4,     // double sum
  A_MIN_I = 5,     // signed 64-bit min
  A_MAX_I = 6,
  A_MIN_F = 7,     // order-preserving u64 image of a double
  A_MAX_F = 8,
};

struct DAgg {
  int32_t fn;
  int32_t prog;          // expression program index (-1 for COUNT)
  uint64_t* lo;          // state words (per group)
  int64_t* hi;           // A_SUM_I128 high word
};

enum SinkKind : int32_t {
  SK_NONE = 0,
  SK_BUILD = 1,        // insert into builds[sink_build]
  SK_MATERIALIZE = 2,  // order-preserving compaction of outputs / row ids
  SK_AGG_HASH = 3,     // global hash table keyed by up to 4 words
  SK_AGG_SMEM = 4,     // per-CTA shared-memory tables merged into AGG_HASH
  SK_AGG_SLOT = 5,     // dense states indexed by a build slot
  SK_AGG_SCALAR = 6,   // one group (no GROUP BY)
  SK_PART_COUNT = 7,   // count the surviving rows per key partition, per CTA
  SK_PART_SCATTER = 8, // write (key, values) records into their partitions
  SK_AGG_FEW = 9,      // one pass into per-CTA tables of every group (k_agg_few, not a pipeline)
  SK_MAT_COUNT = 10,   // two-pass order-preserving compaction: survivors per tile
  SK_MAT_WRITE = 11,   // two-pass order-preserving compaction: outputs at scanned offsets
};

// Hash aggregate table (SoA). State word: 0 empty, 1 claimed, 2 ready.
struct DAggTable {
  uint32_t* state;
  uint64_t* keys[kMaxKeys];
  uint64_t capacity;
  int32_t n_keys;
  // One group key claimed with a CAS on the key word itself: keys[0] starts
  // all ones (kEmptyKey), states start at their identities, entry
  // `capacity` holds the group whose key equals kEmptyKey, and state[g] is
  // set to 2 when group g is first used.
  int32_t cas;
  // Words between consecutive groups in keys[0] and the states (0 or 1:
  // one array per state; larger: all of a group's words in one entry).
  int32_t stride;
  int32_t pad;
};

// ------------------------------------------------------------ pipeline
struct PipeDesc {
  // input
  uint64_t n;                       // tuples when in_count == nullptr
  const uint64_t* in_count;         // device tuple count (tuple-list input)
  int32_t drive_src;                // source whose row id is the scan index
  int32_t tuple_input;              // 1: row ids come from in_rids
  const uint32_t* in_rids[kMaxSrc];
  uint32_t src_mask;                // sources present in the input tuples
  int32_t n_cols, n_preds, n_probes, n_ops, n_progs, n_builds;
  DCol cols[kMaxCols];
  DPred preds[kMaxPreds];
  DProbe probes[kMaxProbes];
  PipeOp ops[kMaxPreds + kMaxProbes];
  VmProg progs[kMaxProgs];
  DBuild builds[kMaxProbes + 1];
  int32_t first_col;                // column prefetched for every tuple (-1 none)
  // Columns the sink reads for every surviving tuple (build key, group keys,
  // aggregate inputs, outputs): fetched for a batch of tuples at once so
  // their loads overlap, then served to the expression VM from registers.
  int32_t n_sink_cols;
  int32_t sink_cols[6];
  // Columns of the driving table read for (nearly) every tuple: each tile of
  // them is staged into shared memory with bulk (TMA) copies, double
  // buffered, so their HBM traffic is in flight independently of registers.
  int32_t n_stream;
  int32_t stream_cols[kMaxStream];

  // sink
  int32_t sink;
  // SK_BUILD
  int32_t sink_build;               // index into builds
  int32_t build_key_col;            // key column index
  uint32_t build_payload_mask;      // sources whose row ids are stored
  // SK_MATERIALIZE
  int32_t n_out;                    // output programs (0: row ids only)
  int32_t out_prog[kMaxProgs];
  void* out_ptr[kMaxProgs];
  uint32_t out_rid_mask;            // sources whose row ids are written
  uint32_t mat_src_mask;            // sources whose row ids the write phase reads
  uint32_t* out_rids[kMaxSrc];
  uint64_t* out_count;              // device count of written tuples
  uint64_t out_capacity;
  uint64_t* tile_status;            // look-back state, one word per tile
  uint32_t* tile_counter;           // dynamic tile ids + finished CTAs
  uint32_t epoch;                   // look-back epoch (no memset per launch)
  uint32_t lb_spin_limit;           // polls before a look-back wait gives up (0: kSpinLimit)
  // two-pass compaction (SK_MAT_COUNT, then SK_MAT_WRITE): per 256-row tile
  // its survivors, then (after the scan) its offset within its chunk of
  // kMatScanTiles tiles; chunk_pos[c] = rows before chunk c
  uint32_t* tile_pos;
  uint64_t* chunk_pos;
  // with it, the count pass also writes each tile's survivors as a 256-bit
  // mask (8 words), and the scan expands the masks into the surviving row
  // ids (out_rids[drive_src]) in place of a write pass
  uint32_t* tile_mask;
  int32_t lb_stall_first;           // failure injection: tile 0 never publishes its prefix
  // aggregates
  int32_t n_aggs;
  DAgg aggs[kMaxAggs];
  int32_t key_prog[kMaxKeys];       // group key programs (AGG_HASH/SMEM)
  DAggTable table;
  int32_t slot_probe;               // AGG_SLOT: probe whose slot is the group
  uint8_t* slot_hit;                // AGG_SLOT: 1 when the group saw a row
  int32_t smem_capacity;            // AGG_SMEM: slots per CTA table
  int32_t smem_probes;              // AGG_SMEM one-key tables: slots probed before the global table

  // PART_COUNT / PART_SCATTER: the key's partition is the top part_bits of
  // its hash; counts/offsets are [CTA][partition] (the grid is fixed to
  // part_ctas CTAs so both launches give every CTA the same tiles); a
  // record is part_words u64 words (1, 2 or 4): the key, then value slot v
  // of each aggregate (part_val[a], -1 when it takes no value), zero padded.
  int32_t part_bits;
  int32_t part_words;
  int32_t part_nvals;               // inputs per record (value slots in use)
  int32_t part_combine;             // few keys per partition: combine a warp's records of one key
  int32_t part_split;               // log2 of the sub-partitions a chunk is aggregated in, one at a time
  int32_t part_ctas;
  uint32_t part_chunk;              // records per CTA of the per-partition aggregation
  int32_t part_val[kMaxAggs];
  int32_t part_src[kMaxAggs];       // aggregate whose program computes value slot v
  uint32_t* part_counts;
  uint32_t* part_offsets;           // per [CTA][partition], relative to part_start
  uint32_t* part_start;             // first record of each partition (P + 1 entries)
  uint32_t* part_chunk_start;       // first chunk of each partition (P + 1 entries)
  uint64_t* part_records;
  uint64_t* part_sub;               // records placed by sub-partition (part_split > 0), same positions

  // launch shape (0: defaults), picked per pipeline by the autotuner:
  // resident CTAs per SM of the grid, and consecutive warp-tiles a warp
  // takes per step of its grid stride (a warp's step covers tile_group x
  // 256 rows)
  int32_t grid_per_sm;
  int32_t tile_group;
  // SK_MATERIALIZE: 0 = 1024-row CTA tiles (k_pipeline_cta.cu), 1 = 256-row
  // warp tiles, each warp with its own look-back (k_pipeline.cu)
  int32_t mat_warp_tiles;

  uint32_t* status;                 // DevStatus bits
};

// Encoded ORDER BY key: up to kMaxOrder parts, each an order-preserving
// unsigned image, most significant part first.
struct SortKeySpec {
  int32_t n_parts;
  int32_t pad;
  int32_t ptype[kMaxOrder];       // P_I32/P_I64/P_F32/P_F64/P_I128
  int32_t desc[kMaxOrder];
  const void* col[kMaxOrder];     // dense arrays over the rows being ordered
  const int64_t* col_hi[kMaxOrder];  // P_I128 high words
};

}  // namespace mtl
