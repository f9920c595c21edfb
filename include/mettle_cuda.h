/*
 * mettle_cuda.h — C ABI of the B200-native execution path for mettle's
 * offloaded SQL subset (libmettle_cuda.so / libmettle_cuda.a).
 *
 * The reference extension (Rust, DuckDB loadable extension) offloads a SQL
 * subset to Apple Metal through ~40 Rust free functions in src/metal/mod.rs.
 * This library replaces that backend and the planner/executor above it
 * (src/plan, src/state.rs, src/pinned.rs, src/source_cache.rs) with
 * hand-written sm_100a CUDA kernels behind plain C entry points: no C++
 * exception and no torch type crosses this boundary, every function returns
 * an int status, and the library owns all device memory.
 *
 * Threading: a context is safe to use from several host threads; queries
 * submitted concurrently are admitted against the processing-region budget
 * and overlap on the device (the serving loop).
 */
#ifndef METTLE_CUDA_H
#define METTLE_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
/* Replaces the reference's MettleError variants (src/error.rs:6-11):
 * InvalidBufferConfig -> MTL_INVALID, MetalUnavailable -> MTL_DEVICE_ERROR,
 * NotInitialized -> MTL_NOT_INITIALIZED, Processing -> the other codes.
 * "Unsupported shape" (the reference's Ok(None) -> DuckDB fallback,
 * src/plan/executor/mod.rs:97-105) is MTL_UNSUPPORTED. */
#define MTL_OK 0
#define MTL_UNSUPPORTED 1
#define MTL_BUDGET_EXCEEDED 2
#define MTL_OOM 3
#define MTL_DEVICE_ERROR 4
#define MTL_TIMEOUT 5
#define MTL_INVALID 6
#define MTL_NOT_INITIALIZED 7
#define MTL_OVERFLOW 8 /* integer overflow, DuckDB's "Overflow in ..." error */

/* --------------------------------------------------------- logical types */
/* The column types the reference pins (PinnedColumn, src/pinned.rs:19-30),
 * plus BIGINT-exact DECIMAL and TIMESTAMP, and the result-only types. */
#define MTL_T_INTEGER 1   /* int32 */
#define MTL_T_BIGINT 2    /* int64 */
#define MTL_T_FLOAT 3     /* binary32 */
#define MTL_T_DOUBLE 4    /* binary64 */
#define MTL_T_DATE 5      /* int32 days since 1970-01-01 */
#define MTL_T_TIMESTAMP 6 /* int64 microseconds since 1970-01-01 */
#define MTL_T_DECIMAL 7   /* int64 scaled by 10^scale (width <= 18) */
#define MTL_T_VARCHAR 8   /* int32 dictionary codes into a sorted dictionary */
#define MTL_T_HUGEINT 9   /* result only: int128 as {uint64 lo, int64 hi} */
#define MTL_T_BOOLEAN 10  /* result only: uint8 */
#define MTL_T_DECIMAL128 11 /* result only: int128 scaled by 10^scale */

/* --------------------------------------------------------------- budgets */
/* gpu_buffer_init(cache, processing, pinned_memory_size := ...)
 * (src/table_functions.rs:30-52, src/config.rs:11-53). */
typedef struct mtl_budgets {
  uint64_t cache_region_bytes;      /* device column / hash-table cache */
  uint64_t processing_region_bytes; /* per-query device scratch, all in flight */
  uint64_t pinned_region_bytes;     /* cudaHostAlloc staging */
} mtl_budgets;

typedef struct mtl_ctx mtl_ctx;
typedef struct mtl_result mtl_result;
typedef struct mtl_request mtl_request;
typedef struct mtl_stmt mtl_stmt;

/* Parses the human sizes of gpu_buffer_init ("64 KB", "1.5 MB", "2gb"; 1024
 * based), defaulting pinned to cache + processing. Replaces
 * BufferConfig::parse / parse_human_bytes (src/config.rs:11-123). `pinned`
 * may be NULL. On error writes a message into errbuf. */
int mtl_parse_buffer_config(const char *cache, const char *processing, const char *pinned, mtl_budgets *out,
                            char *errbuf, size_t errlen);

/* Creates the runtime on `device` (state::initialize + validate_runtime,
 * src/state.rs:23-40, src/metal/runtime/mod.rs:112-151). */
int mtl_ctx_create(const mtl_budgets *budgets, int device, mtl_ctx **out);
void mtl_ctx_destroy(mtl_ctx *ctx);

/* gpu_buffer_init's row: device_name and backend string (MetalDeviceInfo,
 * src/metal/mod.rs:15-20; backend_mode, src/state.rs:30). */
int mtl_device_info(mtl_ctx *ctx, char *name, size_t name_cap, char *backend, size_t backend_cap,
                    uint64_t *total_mem, int32_t *sm_count);

/* Last error message of this context (thread-local to the calling thread). */
const char *mtl_last_error(mtl_ctx *ctx);

/* last_execution_mode() (src/state.rs:91-111): "cuda_generic_plan",
 * "cuda_hot_query_cache", "host_constant", or "" after a reset. */
const char *mtl_last_execution_mode(mtl_ctx *ctx);

/* -------------------------------------------------------- table pinning */
typedef struct mtl_column_desc {
  const char *name;
  int32_t type;  /* MTL_T_* */
  int32_t scale; /* DECIMAL scale */
  const void *data;         /* host rows (VARCHAR: int32 codes) */
  const char *const *dict;  /* VARCHAR dictionary, sorted ascending */
  int32_t dict_size;
  int32_t pad;
} mtl_column_desc;

typedef struct mtl_pin_summary {
  uint64_t row_count;
  uint64_t byte_count;
  char skipped_columns[256];
} mtl_pin_summary;

/* Flags for mtl_table_register. */
#define MTL_PIN_COPY 0u      /* copy rows into library-owned pinned memory */
#define MTL_PIN_BORROW 1u    /* caller keeps the host rows alive and unchanged until drop */
#define MTL_PIN_UPLOAD 2u    /* upload every column to HBM now (default: on first use) */

/* gpu_register_table (src/table_functions.rs:132-159 -> pinned::register_table,
 * src/pinned.rs:187-244): registers a table's columns; they are staged in
 * pinned host memory and uploaded to the device column cache with async
 * copies. DECIMAL stays a scaled int64 (the reference casts it to FLOAT,
 * src/pinned.rs:246-273); BIGINT stays 64-bit (the reference truncates to
 * int32 on upload, src/metal/runtime/mod.rs:424-432). */
int mtl_table_register(mtl_ctx *ctx, const char *table, uint64_t rows, int32_t ncols,
                       const mtl_column_desc *cols, uint32_t flags, mtl_pin_summary *out);
int mtl_table_drop(mtl_ctx *ctx, const char *table);
/* Drops one column's device copy from the HBM cache (it re-uploads on use). */
int mtl_column_evict(mtl_ctx *ctx, const char *table, const char *column);

/* --------------------------------------------------------------- queries */
/* gpu_processing(sql) (src/processing.rs:103-143): parses, plans and runs
 * the query on the GPU; returns MTL_UNSUPPORTED for SQL outside the
 * offloaded subset (the caller then runs it on DuckDB's CPU path) and
 * MTL_NOT_INITIALIZED with "call gpu_buffer_init before gpu_processing"
 * (src/state.rs:42-54). Empty SQL is MTL_INVALID with "gpu_processing
 * requires a non-empty SQL string" (src/processing.rs:104-106). */
int mtl_processing(mtl_ctx *ctx, const char *sql, mtl_result **out);

/* Prepared statements: plan once, run many times without host work per
 * launch. mtl_stmt_launch enqueues the whole query on `stream` (a
 * cudaStream_t, or NULL for the context stream) with no host
 * synchronization; mtl_stmt_fetch waits and returns the result. */
int mtl_stmt_prepare(mtl_ctx *ctx, const char *sql, mtl_stmt **out);
int mtl_stmt_launch(mtl_stmt *stmt, void *stream);
int mtl_stmt_fetch(mtl_stmt *stmt, mtl_result **out);
/* Device milliseconds of the last launch (CUDA events around it). */
double mtl_stmt_device_ms(mtl_stmt *stmt);
/* Number of kernels one launch enqueues. */
int32_t mtl_stmt_kernel_count(mtl_stmt *stmt);
/* Per-step device timing: with profiling on, every launch records CUDA
 * events around each step (memsets, pipelines, compaction, finalize, sort,
 * top-K, gathers); mtl_stmt_step_ms waits for and returns the last launch's
 * time of step i. The reference's METTLE_PROFILE phase timers
 * (src/plan/executor/cache.rs:10-21) are host wall-clock only. */
int mtl_stmt_set_profiling(mtl_stmt *stmt, int32_t on);
int32_t mtl_stmt_step_count(mtl_stmt *stmt);
const char *mtl_stmt_step_name(mtl_stmt *stmt, int32_t i);
double mtl_stmt_step_ms(mtl_stmt *stmt, int32_t i);
void mtl_stmt_free(mtl_stmt *stmt);

/* Serving loop: asynchronous submission with memory-budget admission;
 * requests overlap on the device. */
int mtl_query_submit(mtl_ctx *ctx, const char *sql, mtl_request **out);
/* timeout_ns < 0 waits forever; MTL_TIMEOUT if not finished in time. */
int mtl_request_wait(mtl_request *req, int64_t timeout_ns, mtl_result **out);
/* Host-observed latency of a finished request (submit -> completion). */
double mtl_request_latency_ms(mtl_request *req);
void mtl_request_free(mtl_request *req);

/* --------------------------------------------------------------- results */
int64_t mtl_result_rows(const mtl_result *r);
int32_t mtl_result_columns(const mtl_result *r);
const char *mtl_result_column_name(const mtl_result *r, int32_t col);
/* Type MTL_T_*, with the DECIMAL scale in *scale when non-NULL. */
int32_t mtl_result_column_type(const mtl_result *r, int32_t col, int32_t *scale);
/* Host pointer to the column's rows (fixed width; VARCHAR columns hold
 * int32 dictionary codes, decoded with mtl_result_dict). */
const void *mtl_result_column_data(const mtl_result *r, int32_t col);
/* Validity bytes of a column (1 = value, 0 = NULL), or NULL when every
 * row is valid; only ungrouped aggregates over no rows produce NULLs. */
const uint8_t *mtl_result_column_valid(const mtl_result *r, int32_t col);
/* Dictionary string for a VARCHAR result code. */
const char *mtl_result_dict(const mtl_result *r, int32_t col, int32_t code);
/* Device milliseconds the query spent on the GPU. */
double mtl_result_device_ms(const mtl_result *r);
void mtl_result_free(mtl_result *r);

/* ---------------------------------------------------------------- caches */
/* The 18 numeric columns of gpu_cache_status() in order
 * (src/table_functions.rs:205-230; column 0 is last_execution_mode). */
typedef struct mtl_cache_stats {
  int64_t entries, cached_bytes, hits, misses, evictions, bypasses;
  int64_t input_entries, input_cached_bytes, selection_entries, selection_cached_bytes;
  int64_t join_result_entries, join_result_cached_bytes;
  int64_t source_selection_entries, source_selection_bytes;
  int64_t grouped_topk_entries, grouped_topk_bytes;
  int64_t query_result_entries, query_result_bytes;
} mtl_cache_stats;
int mtl_cache_stats_get(mtl_ctx *ctx, mtl_cache_stats *out);
/* gpu_cache_reset() (src/table_functions.rs:399-433 -> reset_query_caches,
 * src/lib.rs:48-53). */
int mtl_cache_reset(mtl_ctx *ctx);

/* ---------------------------------------------------- rewrite and hooks */
/* gpu_rewrite_query(VARCHAR) -> VARCHAR (README.md:57): the SQL with the
 * supported scalar expressions rewritten to the hook functions. */
int mtl_rewrite_query(mtl_ctx *ctx, const char *sql, char *out, size_t cap);

#define MTL_HOOK_ADD 0
#define MTL_HOOK_MUL 1
/* gpu_add_scalar / gpu_mul_scalar (README.md:57): out[i] = in[i] op k over
 * host rows, DuckDB result type of (type op integer literal). */
int mtl_scalar_arith(mtl_ctx *ctx, int32_t op, int32_t type, const void *in, uint64_t n, int64_t ilit,
                     double flit, void *out);
/* gpu_{eq,lt,le,gt,ge}_scalar (README.md:57): op codes 0..4 as
 * compare_*_scalar (src/metal/shaders/kernels.metal:70-173); out is a
 * uint8 BOOLEAN mask. */
int mtl_scalar_compare(mtl_ctx *ctx, int32_t op, int32_t type, const void *in, uint64_t n, int64_t ilit,
                       double flit, uint8_t *out);

/* ------------------------------------------------- allocation-free top-K */
/* No counterpart in the reference. Top-K rows of one BIGINT or TIMESTAMP
 * column already in device memory, for callers that cannot allocate device
 * memory when they need the result (their device memory is all handed to
 * their own pool, or they must not let cudaMalloc/cudaFree synchronize the
 * device). Nothing is allocated: the kernels' scratch is a fixed 1 MiB array
 * in device memory that the library holds on every GPU that loads it.
 * values: n int64 values on the current device. out_rows: k uint32 row
 * numbers, best first (DESC when descending != 0, else ASC; ties go to the
 * lower row number); out_count: the number written (min(n, k)). Both are
 * device pointers. stream: a cudaStream_t (NULL = the legacy default
 * stream); the call only enqueues work. Limits: 1 <= k <= 32,
 * n <= 2^32 - 2; sizes beyond them are rejected with MTL_INVALID and a
 * message, and every size within them runs (the kernels' grid is capped so
 * that their scratch fits the array). Each call clears the array's first
 * 256 bytes on its stream before its kernels run. The first call on a device looks
 * up the array's address with that device current; make it before any
 * stream capture. All calls share the array: calls whose kernels overlap on
 * the GPU race and can return wrong rows. */
int mtl_topk_noalloc(int32_t type, const void *values, uint64_t n, int32_t k, int32_t descending,
                     uint32_t *out_rows, uint64_t *out_count, void *stream);

/* -------------------------------------------------------------- autotuner */
/* No counterpart in the reference, which fixes its launch shapes (one thread
 * per row, a constant threadgroup size: src/metal/shaders/compiler.rs:69-91)
 * and its hash capacity (src/plan/executor/join_plan.rs:300-303). Runs the
 * query's program once per candidate and keeps, per device, the fastest
 * CTAs per SM and tile size (rows a warp takes per step) of each pipeline,
 * and the hash-table load factor of its join and aggregate tables, keyed by
 * the kind of step and the size class of its input. The table is saved to
 * $METTLE_TUNE_FILE (default ~/.cache/mettle_b200/autotune_<device>.txt) and
 * applied to every query compiled afterwards on that device. `reps` timed
 * runs per candidate; a text report of the choices goes to `report`. */
int mtl_autotune(mtl_ctx *ctx, const char *sql, int32_t reps, char *report, size_t report_cap);

/* ------------------------------------------------- failure injection */
/* Test hook for the failure paths, with no counterpart in the reference
 * (its waits are host-side only). Nothing it does faults, traps or hangs the
 * GPU: every device wait it shortens is bounded and ends in a status the
 * host turns into an error, after which the context stays usable.
 *   MTL_INJECT_NONE: clears any injection.
 *   MTL_INJECT_LOOKBACK_STALL: in queries compiled from now on, the first
 *     tile of every order-preserving compaction never publishes its prefix,
 *     and a look-back wait gives up after `arg` polls (0: the default
 *     limit); the query fails with MTL_DEVICE_ERROR ("a device wait
 *     exceeded its iteration limit").
 *   MTL_INJECT_HOLD_QUEUE: the serving loop starts no queued request until
 *     the injection is cleared (mtl_request_wait then times out). */
#define MTL_INJECT_NONE 0
#define MTL_INJECT_LOOKBACK_STALL 1
#define MTL_INJECT_HOLD_QUEUE 2
int mtl_debug_inject(mtl_ctx *ctx, int32_t what, uint32_t arg);

/* -------------------------------------------------------------- serving */
typedef struct mtl_serve_stats {
  int64_t submitted, completed, rejected, in_flight, queued;
  int64_t admitted_bytes; /* processing-region bytes held by running requests */
  int64_t batched_launches; /* batches that carried several small queries */
  int64_t program_reuses;   /* requests that reused a resident compiled program */
  int64_t cached_programs;  /* compiled programs resident now */
  int64_t graph_updates;    /* parameter updates of resident programs' CUDA graphs */
  int64_t builds_kept;      /* join builds a resident program kept from its previous run */
} mtl_serve_stats;
int mtl_serve_stats_get(mtl_ctx *ctx, mtl_serve_stats *out);
/* Streams (slots) the serving loop may run concurrently (default 4). */
int mtl_serve_set_slots(mtl_ctx *ctx, int32_t slots);

#ifdef __cplusplus
}
#endif
#endif /* METTLE_CUDA_H */
