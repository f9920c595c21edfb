// engine.h — host-side engine: catalog of pinned tables with a device column
// cache, the binder's typed plan, and the compiled device program a
// prepared statement replays.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/mettle_cuda.h"
#include "dev_types.h"
#include "kernels.h"
#include "sql.h"

namespace mtl {

// ------------------------------------------------------------ errors
struct EngineError : std::runtime_error {
  int code;
  EngineError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
[[noreturn]] inline void fail(int code, const std::string& m) { throw EngineError(code, m); }

// ------------------------------------------------------------ types
struct LType {
  int32_t t = 0;      // MTL_T_*
  int32_t width = 0;  // DECIMAL width
  int32_t scale = 0;  // DECIMAL scale
};
inline bool is_int_family(const LType& t) {
  return t.t == MTL_T_INTEGER || t.t == MTL_T_BIGINT || t.t == MTL_T_HUGEINT;
}
inline bool is_float_family(const LType& t) { return t.t == MTL_T_FLOAT || t.t == MTL_T_DOUBLE; }
inline bool is_decimal(const LType& t) { return t.t == MTL_T_DECIMAL || t.t == MTL_T_DECIMAL128; }
int32_t storage_ptype(const LType& t);  // physical type a column/result is stored as
std::string type_name(const LType& t);

// ------------------------------------------------------------ catalog
struct Column {
  std::string name;
  LType type;
  const void* host = nullptr;      // host rows (owned copy or borrowed)
  void* host_owned = nullptr;      // cudaHostAlloc'd copy
  bool host_owned_pinned = false;
  std::vector<std::string> dict;   // VARCHAR dictionary (sorted)
  // device cache
  void* dev = nullptr;
  uint64_t dev_bytes = 0;
  uint64_t last_use = 0;
  int pins = 0;                    // live statements using the device copy
  // statistics (lazy, on the device)
  bool has_minmax = false;
  int64_t vmin = 0, vmax = 0;
  bool has_unique = false;
  bool unique = false;
  bool has_distinct = false;
  uint64_t distinct = 0;
  uint64_t rows = 0;
  uint64_t width() const;
  ~Column();
};

struct Table {
  std::string name;
  uint64_t rows = 0;
  uint64_t version = 0;
  std::vector<std::unique_ptr<Column>> cols;
  Column* find(const std::string& n) const;
};

// ------------------------------------------------------------ bound plan
struct BExpr;
using BExprP = std::shared_ptr<BExpr>;
struct BExpr {
  enum Kind { COL, CONST, ARITH, CAST, NEG, AGG } k = COL;
  LType type;
  int32_t ptype = P_NONE;  // VM representation
  int src = -1;
  Column* col = nullptr;
  int64_t lo = 0, hi = 0;  // CONST bits
  int16_t op = 0;          // ARITH: VM_ADD / VM_SUB / VM_MUL
  int64_t mul = 1, div = 1;  // CAST scaling
  bool bounded = false;    // integer-valued range known
  __int128 bmin = 0, bmax = 0;
  std::vector<BExprP> a;
  std::string text;
  bool is_int_literal = false;
  bool is_dec_literal = false;
  // AGG
  int agg_fn = 0;          // 1 SUM, 2 COUNT, 3 MIN, 4 MAX, 5 AVG
  bool count_star = false;
};

struct Source {
  std::string name, alias;
  std::shared_ptr<Table> table;
};

struct BFilter {
  int src = 0;
  Column* col = nullptr;
  int32_t op = C_TRUE;
  int64_t ilit = 0;
  double flit = 0;
};

struct BJoin {
  int ls = 0, rs = 0;
  Column* lc = nullptr;
  Column* rc = nullptr;
};

enum AggKind { AG_SUM = 1, AG_COUNT = 2, AG_MIN = 3, AG_MAX = 4, AG_AVG = 5 };

struct BAgg {
  int fn = 0;
  BExprP arg;          // null for COUNT(*)
  LType result;
  std::string text;
};

struct BOut {
  std::string name;
  LType type;
  BExprP expr;         // non-aggregate output
  int group_idx = -1;  // aggregate query: group key output
  int agg_idx = -1;    // aggregate query: aggregate output
  bool hidden = false; // only used for ORDER BY
  const std::vector<std::string>* dict = nullptr;  // VARCHAR outputs
};

struct BOrder {
  int out = 0;
  bool desc = false;
};

struct BoundPlan {
  std::vector<Source> sources;
  std::vector<BFilter> filters;
  std::vector<BJoin> joins;
  bool is_agg = false;
  std::vector<BExprP> group_keys;  // COL expressions
  std::vector<BAgg> aggs;
  std::vector<BOut> outputs;
  std::vector<BOrder> order;
  int64_t limit = -1;
  bool constant_only = false;
  bool grouped_topk = false;  // aggregate + ORDER BY + LIMIT (result cache class)
};

struct Ctx;
BoundPlan bind_select(Ctx& ctx, const SelectStmt& st);

// ------------------------------------------------------------ device arena
// First-fit allocator over one cudaMalloc'd processing region; blocks are
// 256-byte aligned. Thread safe.
class Arena {
 public:
  ~Arena();
  void init(uint64_t bytes);
  void* alloc(uint64_t bytes);  // nullptr when no room
  void free(void* p);
  uint64_t capacity() const { return cap_; }
  uint64_t used() const;
  uint64_t largest_free() const;

 private:
  mutable std::mutex mu_;
  char* base_ = nullptr;
  uint64_t cap_ = 0;
  std::map<uint64_t, uint64_t> free_;  // offset -> size
  std::map<uint64_t, uint64_t> used_;  // offset -> size
};

// ------------------------------------------------------------ program
struct Step {
  enum Kind {
    MEMSET, FILL, PIPELINE, COMPACT_FLAGS, COMPACT_READY, FINALIZE, ENCODE, RADIX, TOPK, TOPK_FINAL, GATHER,
    PART_SCAN, PART_AGG,  // partitioned aggregation (descriptor in `pipe`)
    AGG_FEW,              // one-pass few-group aggregation (descriptor in `pipe`)
    MAT_SCAN,             // scan between the two passes of the compaction (descriptor in `pipe`)
    GATHER_OUTS           // a scan's outputs gathered at its compacted row ids (go[0 .. n_go))
  } k;
  std::string name;  // for per-step profiles, e.g. "pipeline:agg_slot:lineitem"
  // MEMSET / FILL (u64 words)
  void* ptr = nullptr;
  int byte = 0;
  uint64_t bytes = 0;
  uint64_t fill = 0;
  // PIPELINE
  PipeDesc pipe;
  uint64_t n_hint = 0;
  std::vector<int> pred_filter;  // BoundPlan filter behind each of pipe.preds
  // build pipelines: the source built, the sources of its subtree, whether
  // its result can be kept across runs, and its row count
  int build_src = -1;
  uint32_t build_src_mask = 0;
  bool build_keepable = false;
  uint64_t orig_n = 0;
  // COMPACT_*
  const void* flag = nullptr;
  uint64_t n = 0;
  const uint64_t* n_dev = nullptr;
  uint32_t* out_idx = nullptr;
  uint64_t* out_count = nullptr;
  uint64_t* tstatus = nullptr;
  uint32_t* tcounter = nullptr;
  // FINALIZE
  FinalOut* fin_dev = nullptr;
  int n_fin = 0;
  GatherOut* go = nullptr;
  int n_go = 0;
  const uint32_t* idx = nullptr;
  const uint64_t* count = nullptr;
  uint64_t n_max = 0;
  // ENCODE / RADIX / TOPK / GATHER
  SortKeySpec spec;
  SortItem* keys = nullptr;
  SortItem* keys_tmp = nullptr;
  uint32_t* kidx = nullptr;
  uint32_t* kidx_tmp = nullptr;
  int key_bytes = 0;
  int topk = 0;
  void* temp = nullptr;
  const void* gin = nullptr;
  int width = 0;
  void* gout = nullptr;
  // TOPK_FINAL
  TopkFinalSpec tfs;
  int topk_phase = 0;  // launch_topk_final's phase
  const uint32_t* remap = nullptr;  // TOPK: write remap[i] for winner i
};

struct OutBuf {
  std::string name;
  LType type;
  void* dev = nullptr;   // final device column
  int width = 0;
  const std::vector<std::string>* dict = nullptr;
  int valid_agg = -1;    // ungrouped aggregates: NULL when the input was empty
};

struct Program {
  std::vector<Step> steps;
  std::vector<OutBuf> outs;
  const uint64_t* out_count = nullptr;  // device count of result rows
  uint64_t fixed_count = UINT64_MAX;    // host-known count (ungrouped aggregate)
  int64_t limit = -1;
  uint64_t n_max = 0;                   // bound on result rows
  const uint64_t* empty_count = nullptr;  // ungrouped aggregate: COUNT(*) state
  uint32_t* status = nullptr;
  std::vector<void*> blocks;            // arena blocks
  uint64_t scratch_bytes = 0;
  int kernels = 0;
  std::vector<Column*> pinned_cols;
  std::vector<std::string> notes;
  // per-step CUDA events (profiling on): ev[2i] before step i, ev[2i+1] after
  bool profile = false;
  std::vector<cudaEvent_t> prof_ev;
  // the whole program captured once as a CUDA graph and replayed
  cudaGraphExec_t graph = nullptr;
  // autotuner keys of the capacities (hash load factors) this compile chose
  std::vector<std::pair<std::string, uint64_t>> load_keys;
  int64_t graph_updates = 0;  // parameter updates of the instantiated graph
  // scratch initialization (host copy), the build each segment belongs to
  // (-1: the query's own state), and its device copy read by the fill step
  std::vector<FillSeg> fills_host, fills_sent;
  std::vector<int> fill_owner;
  FillSeg* fills_dev = nullptr;
  // the filter literals of the last run that completed, for resident builds
  std::vector<std::pair<int64_t, double>> last_lits;
  bool last_ok = false;
  std::string agg_strategy_key;  // autotuner key of a one-key aggregate's strategy ("" none)
  std::string mat_strategy_key;  // autotuner key of the compaction's strategy ("" none)
  ~Program();
};

// ------------------------------------------------------------ results
// Host bytes of a result column. Large buffers are page-locked and come from
// a process-wide pool, so device->host copies run at full PCIe rate and
// repeated queries do not pay cudaHostAlloc.
class HostBuf {
 public:
  HostBuf() = default;
  HostBuf(const HostBuf&) = delete;
  HostBuf& operator=(const HostBuf&) = delete;
  HostBuf(HostBuf&& o) noexcept { swap(o); }
  HostBuf& operator=(HostBuf&& o) noexcept {
    swap(o);
    return *this;
  }
  ~HostBuf();
  void resize(size_t bytes);  // contents are not preserved
  uint8_t* data() { return p_; }
  const uint8_t* data() const { return p_; }
  size_t size() const { return n_; }

 private:
  void swap(HostBuf& o) {
    std::swap(p_, o.p_);
    std::swap(n_, o.n_);
    std::swap(cap_, o.cap_);
    std::swap(pinned_, o.pinned_);
  }
  uint8_t* p_ = nullptr;
  size_t n_ = 0, cap_ = 0;
  bool pinned_ = false;
};

struct ResultCol {
  std::string name;
  LType type;
  int width = 0;
  HostBuf data;
  std::vector<uint8_t> valid;  // empty = all valid
  std::vector<std::string> dict;
};
struct Result {
  std::vector<ResultCol> cols;
  int64_t rows = 0;
  double device_ms = 0;
  uint64_t approx_bytes() const;
};

// ------------------------------------------------------------ context
struct CacheCounters {
  std::atomic<int64_t> hits{0}, misses{0}, evictions{0}, bypasses{0};
};

struct ServeState;

struct Ctx {
  mtl_budgets budgets{};
  int device = 0;
  std::string device_name;
  uint64_t total_mem = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t copy_stream = nullptr;
  std::recursive_mutex mu;  // catalog + caches
  std::map<std::string, std::shared_ptr<Table>> tables;
  uint64_t dev_cache_bytes = 0;
  uint64_t pinned_bytes = 0;
  uint64_t tick = 0;
  uint64_t table_version = 0;
  Arena arena;
  CacheCounters cc;
  // query result cache (LRU by SQL text)
  std::list<std::pair<std::string, std::shared_ptr<Result>>> qcache;
  int64_t grouped_topk_entries = 0;
  std::string last_mode;
  ServeState* serve = nullptr;  // owned; created by the first submit
  // failure injection (mtl_debug_inject): MTL_INJECT_* and its argument
  std::atomic<int> inject_kind{0};
  std::atomic<uint32_t> inject_arg{0};
  // autotuner table (tune.cpp): key -> (choice a, choice b), read from and
  // written to a file per device
  std::map<std::string, std::pair<double, double>> tune;
  bool tune_loaded = false;
  ~Ctx();
};

// device cache + stats (exec.cpp)
void* column_device(Ctx& ctx, Column& c);  // uploads on demand (LRU within cache_region)
void column_minmax(Ctx& ctx, Column& c);
void column_unique(Ctx& ctx, Table& t, Column& c);
void column_distinct(Ctx& ctx, Table& t, Column& c);

// planning / execution (exec.cpp)
std::unique_ptr<Program> compile(Ctx& ctx, const BoundPlan& plan);
void run_program(Ctx& ctx, Program& p, cudaStream_t s);
void run_program_graph(Ctx& ctx, Program& p, cudaStream_t s, bool refresh = false);
// Program reuse across queries of one shape (serving): the plan's shape
// (all but its filter literals) and the literals written into a program
// compiled for that shape.
std::string plan_shape(const BoundPlan& p);
void patch_literals(Program& p, const BoundPlan& plan);
int keep_builds(Program& p, const BoundPlan& plan, cudaStream_t s);
void mark_completed(Program& p, const BoundPlan& plan, bool ok);
std::shared_ptr<Result> fetch_program(Ctx& ctx, Program& p, cudaStream_t s);
void free_program(Ctx& ctx, Program& p);
std::shared_ptr<Result> constant_result(const BoundPlan& plan);
std::shared_ptr<Result> processing(Ctx& ctx, const std::string& sql);

// autotuner (tune.cpp)
std::string tune_key_pipeline(const Step& s);
std::string tune_key_load(const char* what, uint64_t rows);
void tune_apply(Ctx& ctx, Program& p);
double tune_load_factor(Ctx& ctx, const char* what, uint64_t rows);
// One-key aggregate over few groups: 0 planner default, 1 one pass into
// shared-memory tables, 2 partitioned passes.
std::string tune_key_agg(uint64_t groups, uint64_t rows);
int tune_agg_strategy(Ctx& ctx, uint64_t groups, uint64_t rows);
// Order-preserving compaction: 0 default (two passes), 1 one pass with a
// decoupled look-back, 2 two passes.
std::string tune_key_mat(uint64_t rows);
int tune_mat_strategy(Ctx& ctx, uint64_t rows);
std::string tune_file_path(const Ctx& ctx);
std::string autotune(Ctx& ctx, const BoundPlan& plan, int reps);

// serving (serve.cpp)
struct Request;
void serve_init(Ctx& ctx);
void serve_shutdown(Ctx& ctx);
Request* serve_submit(Ctx& ctx, const std::string& sql);

void set_last_error(const std::string& m);
const char* last_error();

}  // namespace mtl
