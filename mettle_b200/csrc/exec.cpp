// exec.cpp — runtime and executor: device column cache bounded by
// cache_region, the processing-region arena, lazy column statistics, the
// compiler from a BoundPlan to a device Program, and result fetch.
//
// The reference keeps pinned tables as host Vecs and uploads columns lazily,
// keyed by host pointer, truncating i64 to i32 and f64 to f32
// (src/metal/runtime/mod.rs:397-469); its executor dispatches one Metal
// kernel per operator and waits on the host between the join batch and the
// aggregate batch (src/plan/executor/fast_path/join_loop.rs:240). Here a
// query compiles to a fixed list of device steps that runs on one stream
// with no host synchronization until the result is fetched.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <set>

#include "engine.h"

namespace mtl {

// ------------------------------------------------------------ errors
static thread_local std::string tl_err;
void set_last_error(const std::string& m) { tl_err = m; }
const char* last_error() { return tl_err.c_str(); }

#define CK(x)                                                                                           \
  do {                                                                                                  \
    cudaError_t e_ = (x);                                                                               \
    if (e_ != cudaSuccess) fail(MTL_DEVICE_ERROR, std::string("CUDA error: ") + cudaGetErrorString(e_) + \
                                                      " (" #x ")");                                   \
  } while (0)

// ------------------------------------------------------------ types
int32_t storage_ptype(const LType& t) {
  switch (t.t) {
    case MTL_T_INTEGER:
    case MTL_T_DATE:
    case MTL_T_VARCHAR: return P_I32;
    case MTL_T_BIGINT:
    case MTL_T_TIMESTAMP:
    case MTL_T_DECIMAL: return P_I64;
    case MTL_T_FLOAT: return P_F32;
    case MTL_T_DOUBLE: return P_F64;
    case MTL_T_HUGEINT:
    case MTL_T_DECIMAL128: return P_I128;
    case MTL_T_BOOLEAN: return P_I32;
    default: return P_NONE;
  }
}

std::string type_name(const LType& t) {
  switch (t.t) {
    case MTL_T_INTEGER: return "INTEGER";
    case MTL_T_BIGINT: return "BIGINT";
    case MTL_T_FLOAT: return "FLOAT";
    case MTL_T_DOUBLE: return "DOUBLE";
    case MTL_T_DATE: return "DATE";
    case MTL_T_TIMESTAMP: return "TIMESTAMP";
    case MTL_T_DECIMAL:
    case MTL_T_DECIMAL128: return "DECIMAL(" + std::to_string(t.width) + "," + std::to_string(t.scale) + ")";
    case MTL_T_VARCHAR: return "VARCHAR";
    case MTL_T_HUGEINT: return "HUGEINT";
    case MTL_T_BOOLEAN: return "BOOLEAN";
    default: return "UNKNOWN";
  }
}

uint64_t Column::width() const { return (uint64_t)ptype_width(storage_ptype(type)); }

Column* Table::find(const std::string& n) const {
  for (auto& c : cols)
    if (c->name == n) return c.get();
  return nullptr;
}

// ------------------------------------------------------------ host buffers
namespace {
std::mutex g_pin_mu;
std::map<size_t, std::vector<void*>> g_pin_free;  // capacity -> free blocks
size_t g_pin_pooled = 0;
constexpr size_t kPinnedFrom = 64 * 1024;        // smaller results stay pageable
constexpr size_t kPinnedPoolMax = 8ull << 30;    // bytes kept for reuse
}  // namespace

void HostBuf::resize(size_t bytes) {
  if (bytes <= cap_) {
    n_ = bytes;
    return;
  }
  this->~HostBuf();
  p_ = nullptr;
  n_ = cap_ = 0;
  pinned_ = false;
  if (bytes >= kPinnedFrom) {
    size_t cap = kPinnedFrom;
    while (cap < bytes) cap <<= 1;
    {
      std::lock_guard<std::mutex> g(g_pin_mu);
      auto it = g_pin_free.find(cap);
      if (it != g_pin_free.end() && !it->second.empty()) {
        p_ = (uint8_t*)it->second.back();
        it->second.pop_back();
        g_pin_pooled -= cap;
      }
    }
    if (!p_ && cudaHostAlloc((void**)&p_, cap, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      p_ = nullptr;
    }
    if (p_) {
      pinned_ = true;
      cap_ = cap;
      n_ = bytes;
      return;
    }
  }
  p_ = (uint8_t*)malloc(bytes ? bytes : 1);
  if (!p_) throw std::bad_alloc();
  cap_ = bytes;
  n_ = bytes;
}

HostBuf::~HostBuf() {
  if (!p_) return;
  if (pinned_) {
    std::lock_guard<std::mutex> g(g_pin_mu);
    if (g_pin_pooled + cap_ <= kPinnedPoolMax) {
      g_pin_free[cap_].push_back(p_);
      g_pin_pooled += cap_;
    } else {
      cudaFreeHost(p_);
    }
  } else {
    free(p_);
  }
  p_ = nullptr;
}

uint64_t Result::approx_bytes() const {
  uint64_t b = 0;
  for (auto& c : cols) b += c.data.size() + c.valid.size();
  return b;
}

// ------------------------------------------------------------ arena
Arena::~Arena() {
  if (base_) cudaFree(base_);
}

void Arena::init(uint64_t bytes) {
  std::lock_guard<std::mutex> g(mu_);
  cap_ = (bytes + 255) & ~255ULL;
  if (cap_ == 0) return;
  cudaError_t e = cudaMalloc((void**)&base_, cap_);
  if (e != cudaSuccess) {
    cudaGetLastError();
    base_ = nullptr;
    fail(MTL_OOM, std::string("cannot allocate the processing region: ") + cudaGetErrorString(e));
  }
  free_.clear();
  used_.clear();
  free_[0] = cap_;
}

void* Arena::alloc(uint64_t bytes) {
  std::lock_guard<std::mutex> g(mu_);
  bytes = (bytes + 255) & ~255ULL;
  if (bytes == 0) bytes = 256;
  for (auto it = free_.begin(); it != free_.end(); ++it) {
    if (it->second >= bytes) {
      uint64_t off = it->first, sz = it->second;
      free_.erase(it);
      if (sz > bytes) free_[off + bytes] = sz - bytes;
      used_[off] = bytes;
      return base_ + off;
    }
  }
  return nullptr;
}

void Arena::free(void* p) {
  if (!p) return;
  std::lock_guard<std::mutex> g(mu_);
  uint64_t off = (uint64_t)((char*)p - base_);
  auto u = used_.find(off);
  if (u == used_.end()) return;
  uint64_t sz = u->second;
  used_.erase(u);
  auto nx = free_.lower_bound(off);
  if (nx != free_.end() && nx->first == off + sz) {
    sz += nx->second;
    nx = free_.erase(nx);
  }
  if (nx != free_.begin()) {
    auto pv = std::prev(nx);
    if (pv->first + pv->second == off) {
      pv->second += sz;
      return;
    }
  }
  free_[off] = sz;
}

uint64_t Arena::used() const {
  std::lock_guard<std::mutex> g(mu_);
  uint64_t s = 0;
  for (auto& u : used_) s += u.second;
  return s;
}

uint64_t Arena::largest_free() const {
  std::lock_guard<std::mutex> g(mu_);
  uint64_t m = 0;
  for (auto& f : free_) m = std::max(m, f.second);
  return m;
}

Column::~Column() {
  // stream-ordered pool: no device-wide synchronization on free
  if (dev) cudaFreeAsync(dev, 0);
  if (host_owned) {
    if (host_owned_pinned) cudaFreeHost(host_owned);
    else ::free(host_owned);
  }
}

Ctx::~Ctx() {
  serve_shutdown(*this);
  qcache.clear();
  tables.clear();
  if (stream) cudaStreamDestroy(stream);
  if (copy_stream) cudaStreamDestroy(copy_stream);
}

// ------------------------------------------------------------ column cache
static uint64_t table_rows_of(Ctx&, const Column& c) { return c.rows; }

void* column_device(Ctx& ctx, Column& c) {
  std::lock_guard<std::recursive_mutex> g(ctx.mu);
  c.last_use = ++ctx.tick;
  if (c.dev) {
    ctx.cc.hits++;
    return c.dev;
  }
  ctx.cc.misses++;
  const uint64_t rows = table_rows_of(ctx, c);
  const uint64_t bytes = rows * c.width();
  if (bytes > ctx.budgets.cache_region_bytes)
    fail(MTL_BUDGET_EXCEEDED, "column \"" + c.name + "\" (" + std::to_string(bytes) +
                                  " bytes) exceeds the cache region of gpu_buffer_init");
  // LRU eviction of unpinned device columns
  while (ctx.dev_cache_bytes + bytes > ctx.budgets.cache_region_bytes) {
    Column* victim = nullptr;
    for (auto& t : ctx.tables)
      for (auto& cc : t.second->cols)
        if (cc->dev && cc->pins == 0 && (!victim || cc->last_use < victim->last_use)) victim = cc.get();
    if (!victim) fail(MTL_BUDGET_EXCEEDED, "cache region exhausted by columns in use");
    cudaFreeAsync(victim->dev, ctx.copy_stream);
    victim->dev = nullptr;
    ctx.dev_cache_bytes -= victim->dev_bytes;
    victim->dev_bytes = 0;
    ctx.cc.evictions++;
  }
  // Column buffers come from the device's stream-ordered pool (kept reserved
  // by a release threshold set at context creation), so re-registering a
  // table does not pay cudaMalloc/cudaFree each time.
  void* d = nullptr;
  CK(cudaMallocAsync(&d, bytes ? bytes : 16, ctx.copy_stream));
  if (bytes) {
    CK(cudaMemcpyAsync(d, c.host, bytes, cudaMemcpyHostToDevice, ctx.copy_stream));
    CK(cudaStreamSynchronize(ctx.copy_stream));
  }
  c.dev = d;
  c.dev_bytes = bytes;
  ctx.dev_cache_bytes += bytes;
  return d;
}

void column_minmax(Ctx& ctx, Column& c) {
  std::lock_guard<std::recursive_mutex> g(ctx.mu);
  if (c.has_minmax) return;
  const int32_t pt = storage_ptype(c.type);
  if (pt != P_I32 && pt != P_I64) return;
  const uint64_t rows = table_rows_of(ctx, c);
  if (rows == 0) return;
  void* d = column_device(ctx, c);
  int64_t* buf = nullptr;
  CK(cudaMallocAsync((void**)&buf, 16, ctx.copy_stream));
  int64_t init[2] = {INT64_MAX, INT64_MIN};
  CK(cudaMemcpyAsync(buf, init, 16, cudaMemcpyHostToDevice, ctx.copy_stream));
  CK(launch_minmax_i(d, pt, rows, buf, ctx.copy_stream));
  int64_t out[2];
  CK(cudaMemcpyAsync(out, buf, 16, cudaMemcpyDeviceToHost, ctx.copy_stream));
  CK(cudaFreeAsync(buf, ctx.copy_stream));
  CK(cudaStreamSynchronize(ctx.copy_stream));
  c.vmin = out[0];
  c.vmax = out[1];
  c.has_minmax = true;
}

void column_distinct(Ctx& ctx, Table& t, Column& c) {
  std::lock_guard<std::recursive_mutex> g(ctx.mu);
  if (c.has_distinct) return;
  const int32_t pt = storage_ptype(c.type);
  if (t.rows == 0) {
    c.has_distinct = c.has_unique = c.unique = true;
    c.distinct = 0;
    return;
  }
  if (c.type.t == MTL_T_VARCHAR) {
    c.has_distinct = true;
    c.distinct = std::min<uint64_t>(c.dict.size(), t.rows);
    return;
  }
  void* d = column_device(ctx, c);
  cudaStream_t s = ctx.copy_stream;
  unsigned long long* out = nullptr;
  CK(cudaMallocAsync((void**)&out, 16, s));
  CK(cudaMemsetAsync(out, 0, 16, s));
  if (pt == P_I32 || pt == P_I64) column_minmax(ctx, c);
  const __int128 span = c.has_minmax ? (__int128)c.vmax - (__int128)c.vmin + 1 : 0;
  if (span > 0 && span <= (__int128)(8 * t.rows + (1u << 24))) {
    // small value range: a presence bitmap (span / 8 bytes)
    const uint64_t words = ((uint64_t)span + 31) / 32;
    uint32_t* bits = nullptr;
    CK(cudaMallocAsync((void**)&bits, words * 4, s));
    CK(cudaMemsetAsync(bits, 0, words * 4, s));
    CK(launch_count_dups_dense(d, pt, t.rows, c.vmin, (uint64_t)span, bits, out, s));
    CK(cudaFreeAsync(bits, s));
  } else {
    const uint64_t cap = std::max<uint64_t>(64, 2 * t.rows);
    int64_t* table = nullptr;
    uint32_t* special = nullptr;
    CK(cudaMallocAsync((void**)&table, cap * 8, s));
    CK(cudaMallocAsync((void**)&special, 16, s));
    CK(cudaMemsetAsync(table, 0xFF, cap * 8, s));
    CK(cudaMemsetAsync(special, 0, 16, s));
    // F32/F64 columns hash their bit patterns (distinct estimate only).
    CK(launch_count_dups(d, pt == P_F32 ? P_I32 : (pt == P_F64 ? P_I64 : pt), t.rows, table, cap, special, out, s));
    CK(cudaFreeAsync(table, s));
    CK(cudaFreeAsync(special, s));
  }
  unsigned long long dups = 0;
  CK(cudaMemcpyAsync(&dups, out, 8, cudaMemcpyDeviceToHost, s));
  CK(cudaFreeAsync(out, s));
  CK(cudaStreamSynchronize(s));
  c.distinct = t.rows - dups;
  c.has_distinct = true;
  c.has_unique = true;
  c.unique = dups == 0;
}

void column_unique(Ctx& ctx, Table& t, Column& c) { column_distinct(ctx, t, c); }

// ------------------------------------------------------------ compiler
namespace {

struct Compiler {
  Ctx& ctx;
  const BoundPlan& plan;
  Program& P;

  // ---- scratch
  void* scratch(uint64_t bytes) {
    void* p = ctx.arena.alloc(bytes);
    if (!p)
      fail(MTL_BUDGET_EXCEEDED, "query needs more device scratch than the processing region allows (" +
                                    std::to_string(bytes) + " bytes requested, " +
                                    std::to_string(ctx.arena.largest_free()) + " free)");
    P.blocks.push_back(p);
    P.scratch_bytes += (bytes + 255) & ~255ULL;
    return p;
  }
  // Descriptor uploads complete before compile() returns: the program may
  // run on any stream, and a plain cudaMemcpy from pageable memory can
  // return before its DMA lands.
  void upload(void* dst, const void* src, size_t bytes) {
    std::lock_guard<std::recursive_mutex> g(ctx.mu);
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx.copy_stream));
    CK(cudaStreamSynchronize(ctx.copy_stream));
  }

  // Scratch initialization is collected and emitted as one fill launch at
  // the start of the program (arena blocks are 256-byte aligned and sized in
  // 256-byte units, so rounding a segment up to 16 bytes stays in its block).
  std::vector<FillSeg> fills;
  std::vector<int> fill_owner;  // per segment: the source whose build it belongs to (-1: the query's)
  int cur_owner = -1;
  void memset_step(void* p, int byte, uint64_t bytes) {
    FillSeg f;
    memset(&f, 0, sizeof(f));
    f.ptr = p;
    f.bytes = (bytes + 15) & ~15ULL;
    f.pattern = 0x0101010101010101ULL * (uint64_t)(byte & 0xFF);
    f.stride = 0;
    fills.push_back(f);
    fill_owner.push_back(cur_owner);
  }
  void fill_step(void* p, uint64_t words, uint64_t v) {
    FillSeg f;
    memset(&f, 0, sizeof(f));
    f.ptr = p;
    f.bytes = (words * 8 + 15) & ~15ULL;
    f.pattern = v;
    f.stride = 0;
    fills.push_back(f);
    fill_owner.push_back(cur_owner);
  }
  // n entries of stride_words words (even), each a copy of entry_dev
  void fill_entries(void* p, uint64_t n, uint64_t stride_words, const uint64_t* entry_dev) {
    FillSeg f;
    memset(&f, 0, sizeof(f));
    f.ptr = p;
    f.bytes = n * stride_words * 8;
    f.entry = entry_dev;
    f.entry_words = stride_words;
    fills.push_back(f);
    fill_owner.push_back(cur_owner);
  }
  // one 8-byte word every stride_words words, n times
  void fill_strided(void* p, uint64_t n, uint64_t stride_words, uint64_t v) {
    FillSeg f;
    memset(&f, 0, sizeof(f));
    f.ptr = p;
    f.bytes = n * stride_words * 8;
    f.pattern = v;
    f.stride = stride_words * 8;
    fills.push_back(f);
    fill_owner.push_back(cur_owner);
  }
  void emit_fills() {
    if (fills.empty()) return;
    FillSeg* dev = (FillSeg*)scratch(fills.size() * sizeof(FillSeg));
    upload(dev, fills.data(), fills.size() * sizeof(FillSeg));
    uint64_t mx = 0;
    for (auto& f : fills) mx = std::max(mx, f.bytes);
    Step s;
    s.k = Step::FILL;
    s.ptr = dev;
    s.byte = (int)fills.size();
    s.bytes = mx;
    s.name = "init_scratch";
    P.steps.insert(P.steps.begin(), s);
    P.kernels += 1;
    P.fills_host = fills;
    P.fill_owner = fill_owner;
    P.fills_dev = dev;
  }

  // ---- join tree
  int root = 0;
  std::vector<int> parent;          // -1 for root
  std::vector<Column*> up_col;      // build key column of each non-root source
  std::vector<Column*> down_col;    // parent's probe column for each non-root source
  std::vector<std::vector<int>> children;
  std::vector<uint32_t> subtree;    // source mask of each subtree

  uint32_t subtree_mask(int s) {
    uint32_t m = 1u << s;
    for (int c : children[s]) m |= subtree_mask(c);
    return subtree[s] = m;
  }

  void plan_joins() {
    const int S = (int)plan.sources.size();
    parent.assign(S, -1);
    up_col.assign(S, nullptr);
    down_col.assign(S, nullptr);
    children.assign(S, {});
    subtree.assign(S, 0);
    if (S == 1) {
      root = 0;
      subtree_mask(0);
      return;
    }
    if ((int)plan.joins.size() != S - 1)
      fail(MTL_UNSUPPORTED, "join graph must be a tree of equi-joins (cross products and cyclic joins are "
                            "outside the offloaded subset)");
    std::vector<int> order(S);
    for (int i = 0; i < S; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
      return plan.sources[a].table->rows > plan.sources[b].table->rows;
    });
    for (int cand : order) {
      // orient edges away from cand
      std::vector<int> par(S, -2);
      std::vector<Column*> upc(S, nullptr), downc(S, nullptr);
      par[cand] = -1;
      std::vector<int> q{cand};
      bool ok = true;
      for (size_t qi = 0; qi < q.size() && ok; ++qi) {
        int u = q[qi];
        for (const BJoin& j : plan.joins) {
          int v = -1;
          Column *vc = nullptr, *uc = nullptr;
          if (j.ls == u) { v = j.rs; vc = j.rc; uc = j.lc; }
          else if (j.rs == u) { v = j.ls; vc = j.lc; uc = j.rc; }
          else continue;
          if (par[v] != -2) {
            if (v != par[u]) ok = false;  // cycle
            continue;
          }
          par[v] = u;
          upc[v] = vc;
          downc[v] = uc;
          q.push_back(v);
        }
      }
      if (!ok || (int)q.size() != S) fail(MTL_UNSUPPORTED, "join graph must be a connected tree of equi-joins");
      bool unique_builds = true;
      for (int v = 0; v < S && unique_builds; ++v) {
        if (v == cand) continue;
        Column* c = upc[v];
        if (storage_ptype(c->type) != P_I32 && storage_ptype(c->type) != P_I64) {
          unique_builds = false;
          break;
        }
        if (storage_ptype(downc[v]->type) != storage_ptype(c->type) &&
            !((storage_ptype(downc[v]->type) == P_I32 || storage_ptype(downc[v]->type) == P_I64))) {
          unique_builds = false;
          break;
        }
        column_unique(ctx, *plan.sources[v].table, *c);
        if (!c->unique) unique_builds = false;
      }
      if (!unique_builds) continue;
      root = cand;
      parent = par;
      parent[cand] = -1;
      up_col = upc;
      down_col = downc;
      for (int v = 0; v < S; ++v)
        if (v != cand) children[parent[v]].push_back(v);
      subtree_mask(root);
      return;
    }
    fail(MTL_UNSUPPORTED, "every join needs a unique key on its build side (non-unique join keys are "
                          "outside the offloaded subset)");
  }

  // ---- expression programs
  struct PipeBuilder {
    PipeDesc d;
    std::map<std::pair<int, const Column*>, int> colmap;
    std::vector<double> op_sel;  // estimated pass fraction of each op
    std::vector<int> pred_filter;  // plan filter of each predicate
    PipeBuilder() {
      memset(&d, 0, sizeof(d));
      d.first_col = -1;
      d.slot_probe = -1;
    }
  };

  int add_col(PipeBuilder& pb, int src, Column* c) {
    auto key = std::make_pair(src, (const Column*)c);
    auto it = pb.colmap.find(key);
    if (it != pb.colmap.end()) return it->second;
    if (pb.d.n_cols >= kMaxCols) fail(MTL_UNSUPPORTED, "too many columns in one pipeline");
    int i = pb.d.n_cols++;
    pb.d.cols[i].ptr = column_device(ctx, *c);
    pb.d.cols[i].ptype = storage_ptype(c->type);
    pb.d.cols[i].src = src;
    pb.colmap[key] = i;
    pinned_cols.insert(c);
    return i;
  }
  std::set<Column*> pinned_cols;

  void emit(PipeBuilder& pb, VmProg& p, const BExpr& e) {
    auto push = [&](VmIns in) {
      if (p.n >= kMaxIns) fail(MTL_UNSUPPORTED, "expression too long for the device evaluator");
      p.ins[p.n++] = in;
    };
    VmIns in;
    memset(&in, 0, sizeof(in));
    switch (e.k) {
      case BExpr::COL:
        in.op = VM_COL;
        in.type = (int16_t)storage_ptype(e.col->type);
        in.arg = add_col(pb, e.src, e.col);
        push(in);
        break;
      case BExpr::CONST:
        in.op = VM_CONST;
        in.type = (int16_t)e.ptype;
        in.k = e.lo;
        in.k2 = e.hi;
        if (e.ptype == P_I32 || e.ptype == P_I64) in.k2 = e.lo < 0 ? -1 : 0;
        push(in);
        break;
      case BExpr::ARITH:
        emit(pb, p, *e.a[0]);
        emit(pb, p, *e.a[1]);
        in.op = e.op;
        in.type = (int16_t)e.ptype;
        push(in);
        break;
      case BExpr::CAST:
        emit(pb, p, *e.a[0]);
        in.op = VM_CAST;
        in.type = (int16_t)e.ptype;
        in.arg = e.a[0]->ptype;
        in.k = e.mul;
        in.k2 = e.div;
        push(in);
        break;
      case BExpr::NEG:
        emit(pb, p, *e.a[0]);
        in.op = VM_NEG;
        in.type = (int16_t)e.ptype;
        push(in);
        break;
      default:
        fail(MTL_UNSUPPORTED, "aggregate in a scalar context");
    }
  }

  int add_prog(PipeBuilder& pb, const BExpr& e) {
    if (pb.d.n_progs >= kMaxProgs) fail(MTL_UNSUPPORTED, "too many expressions in one pipeline");
    int i = pb.d.n_progs++;
    VmProg& p = pb.d.progs[i];
    memset(&p, 0, sizeof(p));
    emit(pb, p, e);
    p.out_type = e.ptype;
    int sp = 0;
    for (int k = 0; k < p.n; ++k) {
      const int16_t op = p.ins[k].op;
      if (op == VM_COL || op == VM_CONST || op == VM_SLOT) p.depth = std::max(p.depth, ++sp);
      else if (op != VM_CAST && op != VM_NEG) --sp;
    }
    make_fast(p);
    return i;
  }

  // Recasts a postfix program as a VmFast tree when it has at most three
  // leaves, two binary ops and one cast per node.
  static void make_fast(VmProg& p) {
    VmFast f;
    memset(&f, 0, sizeof(f));
    struct Node {
      bool leaf;
      int idx;
      int left_leaf;  // op nodes: whether the left child is a leaf (-1 unknown)
    };
    Node st[kMaxIns];
    int sp = 0, nl = 0, no = 0;
    bool root_is_op = false;
    int inner_on_left = -1;  // for the second op: is the first op its left child
    for (int k = 0; k < p.n; ++k) {
      const VmIns& in = p.ins[k];
      switch (in.op) {
        case VM_COL:
        case VM_CONST:
          if (nl >= 3) return;
          f.leaf[nl] = in;
          st[sp++] = Node{true, nl++, -1};
          break;
        case VM_CAST: {
          if (sp < 1) return;
          const Node& t = st[sp - 1];
          VmCast& c = t.leaf ? f.leaf_cast[t.idx] : f.op_cast[t.idx];
          if (c.on) return;
          c.on = 1;
          c.from = (int16_t)in.arg;
          c.to = in.type;
          c.mul = in.k;
          c.div = in.k2;
          break;
        }
        case VM_ADD:
        case VM_SUB:
        case VM_MUL: {
          if (sp < 2 || no >= 2) return;
          const Node b = st[--sp];
          const Node a = st[--sp];
          if (no == 1) {
            // the second op must combine the first op's result with a leaf
            if (a.leaf == b.leaf) return;
            inner_on_left = a.leaf ? 0 : 1;
          } else if (!(a.leaf && b.leaf)) {
            return;
          }
          f.op[no] = in;
          st[sp++] = Node{false, no++, -1};
          break;
        }
        default:
          return;  // NEG, SLOT
      }
    }
    if (sp != 1) return;
    root_is_op = !st[0].leaf;
    if (!root_is_op) f.shape = nl == 1 ? 1 : 0;
    else if (no == 1) f.shape = nl == 2 ? 2 : 0;
    else f.shape = nl == 3 ? (inner_on_left ? 4 : 3) : 0;
    if (f.shape) p.fast = f;
  }

  static void expr_sources(const BExpr& e, uint32_t& m) {
    if (e.k == BExpr::COL) m |= 1u << e.src;
    for (auto& c : e.a) expr_sources(*c, m);
  }

  // ---- builds
  std::vector<DBuild> builds;  // per source
  std::vector<int> build_probe_index;  // per source: probe index in its parent's pipeline

  DBuild make_build(int s) {
    cur_owner = s;  // the build's own scratch initialization
    struct Reset {
      int& o;
      ~Reset() { o = -1; }
    } reset{cur_owner};
    DBuild b;
    memset(&b, 0, sizeof(b));
    Table& t = *plan.sources[s].table;
    Column& k = *up_col[s];
    column_minmax(ctx, k);
    const uint64_t rows = t.rows;
    b.key_ptype = storage_ptype(k.type);
    b.unique_keys = (k.has_unique && k.unique) ? 1 : 0;
    bool dense = false;
    uint64_t span = 0;
    if (k.has_minmax) {
      __int128 sp = (__int128)k.vmax - (__int128)k.vmin + 1;
      if (sp > 0 && sp <= (__int128)(4 * rows + (1u << 20)) && sp < ((__int128)1 << 31)) {
        dense = true;
        span = (uint64_t)sp;
      }
    }
    if (rows == 0) {
      dense = true;
      span = 1;
      b.key_min = 0;
    }
    if (dense) {
      b.kind = B_DENSE;
      if (rows) b.key_min = k.vmin;
      b.capacity = span;
      // the slot map is read only where its presence bit is set, so only the
      // bitmap (span / 8 bytes) is cleared per query
      b.dense_map = (uint32_t*)scratch(span * 4);
      b.dense_bits = (uint32_t*)scratch(((span + 31) / 32) * 4);
      memset_step(b.dense_bits, 0, ((span + 31) / 32) * 4);
    } else {
      b.kind = B_HASH;
      const double lf = tune_load_factor(ctx, "hash_build", rows);
      P.load_keys.push_back({tune_key_load("hash_build", rows), rows});
      b.capacity = std::max<uint64_t>(64, (uint64_t)std::ceil(lf * (double)rows));
      b.hash_keys = (int64_t*)scratch(b.capacity * 8);
      b.hash_slot = (uint32_t*)scratch(b.capacity * 4);
      b.hash_special = (uint32_t*)scratch(8);
      memset_step(b.hash_keys, 0xFF, b.capacity * 8);
      memset_step(b.hash_special, 0, 8);
      // A build that filters its rows (a predicate, or a probe of its own
      // builds) holds a fraction of its table's keys, so most probes miss:
      // a Bloom filter of about 8 bits per table row (small enough to stay
      // in L2) answers those misses without reading the table in HBM. The
      // reference builds a membership bitmap for the same purpose
      // (build_membership_filter_v / membership_filter_mask_v,
      // src/metal/shaders/kernels.metal:917-956, src/plan/executor/join_plan.rs:312).
      if (build_filters(s)) {
        uint64_t words = 64;
        while (words < rows / 4) words <<= 1;
        b.bloom_words = words;
        b.bloom = (uint32_t*)scratch(words * 4);
        memset_step(b.bloom, 0, words * 4);
      }
    }
    return b;
  }

  // Whether source s's build pipeline drops rows: a predicate on s, or a
  // probe of a child build (an inner join).
  bool build_filters(int s) const {
    if (!children[s].empty()) return true;
    for (const BFilter& f : plan.filters)
      if (f.src == s && f.op != C_TRUE) return true;
    return false;
  }

  // Sources whose row ids the root pipeline's sink needs.
  uint32_t needed_root = 0;
  uint32_t payload_mask(int s) const { return needed_root & subtree[s]; }
  int rep_src = -1;
  bool cas_table = false;  // one-key hash aggregate claimed by CAS on the key
  int state_stride = 1;    // words between groups in the aggregate states

  void add_filters(PipeBuilder& pb, int s) {
    for (size_t fi = 0; fi < plan.filters.size(); ++fi) {
      const BFilter& f = plan.filters[fi];
      if (f.src != s) continue;
      if (pb.d.n_preds >= kMaxPreds) fail(MTL_UNSUPPORTED, "too many predicates on one table");
      int pi = pb.d.n_preds++;
      DPred& p = pb.d.preds[pi];
      p.col = add_col(pb, s, f.col);
      p.op = f.op;
      p.ilit = f.ilit;
      p.flit = f.flit;
      pb.d.ops[pb.d.n_ops].kind = OPK_FILTER;
      pb.d.ops[pb.d.n_ops].idx = pi;
      pb.d.n_ops++;
      pb.op_sel.push_back(estimate_selectivity(f));
      pb.pred_filter.push_back((int)fi);
    }
  }

  // Pass fraction of a predicate from the column's min/max (uniform values
  // assumed); used only to decide which columns to stream.
  double estimate_selectivity(const BFilter& f) {
    if (f.op == C_TRUE) return 1.0;
    if (f.op == C_FALSE) return 0.0;
    const int32_t pt = storage_ptype(f.col->type);
    if (pt != P_I32 && pt != P_I64) return f.op == C_EQ ? 0.05 : 0.5;
    column_minmax(ctx, *f.col);
    if (!f.col->has_minmax) return 0.5;
    const double lo = (double)f.col->vmin, hi = (double)f.col->vmax, span = hi - lo + 1.0, x = (double)f.ilit;
    auto clamp = [](double v) { return v < 0 ? 0.0 : (v > 1 ? 1.0 : v); };
    switch (f.op) {
      case C_LT: return clamp((x - lo) / span);
      case C_LE: return clamp((x - lo + 1) / span);
      case C_GT: return clamp((hi - x) / span);
      case C_GE: return clamp((hi - x + 1) / span);
      case C_EQ: return clamp(1.0 / span);
      case C_NE: return clamp(1.0 - 1.0 / span);
      default: return 0.5;
    }
  }

  static void prog_cols(const VmProg& p, std::vector<int>& out) {
    for (int i = 0; i < p.n; ++i)
      if (p.ins[i].op == VM_COL && std::find(out.begin(), out.end(), p.ins[i].arg) == out.end())
        out.push_back(p.ins[i].arg);
  }

  // Chooses the sink's prefetched columns and the streamed (bulk-copied)
  // columns of the driving table.
  void plan_columns(PipeBuilder& pb) {
    PipeDesc& d = pb.d;
    std::vector<int> sink;
    if (d.sink == SK_BUILD) sink.push_back(d.build_key_col);
    if (d.sink == SK_AGG_HASH || d.sink == SK_AGG_SMEM || d.sink == SK_PART_COUNT || d.sink == SK_PART_SCATTER)
      for (int k = 0; k < d.table.n_keys; ++k) prog_cols(d.progs[d.key_prog[k]], sink);
    if (d.sink == SK_AGG_HASH || d.sink == SK_AGG_SMEM || d.sink == SK_AGG_SLOT || d.sink == SK_AGG_SCALAR ||
        d.sink == SK_PART_SCATTER)
      for (int a = 0; a < d.n_aggs; ++a)
        if (d.aggs[a].prog >= 0) prog_cols(d.progs[d.aggs[a].prog], sink);
    if (d.sink == SK_MATERIALIZE || d.sink == SK_MAT_WRITE)
      for (int q = 0; q < d.n_out; ++q) prog_cols(d.progs[d.out_prog[q]], sink);
    d.n_sink_cols = (int)std::min<size_t>(sink.size(), 6);
    for (int i = 0; i < d.n_sink_cols; ++i) d.sink_cols[i] = sink[i];

    d.n_stream = 0;
    if (d.tuple_input) return;
    uint32_t budget = 16;  // bytes per tuple: 64 KB of double-buffered tiles
    int max_stream = 4;
    // (staging every output column of the compaction's write pass, up to
    // 32 bytes a row, halves its resident CTAs and measured no faster)
    // The scatter pass reads every input of the records (up to 20 bytes a
    // row staged), within about 110 KB with its partition cursors so that
    // two of its CTAs (its fixed grid) share an SM: with the most partitions
    // fewer bytes are staged and the rest read directly.
    if (d.sink == SK_PART_SCATTER) {
      const uint32_t cursors = (4u << d.part_bits);
      budget = 20;
      while (budget > 4 && cursors + 8 * (2 * 256 * budget + 2048) > 110 * 1024) budget -= 4;
    }
    if (d.sink == SK_AGG_SMEM) {
      // keep the CTA within about 110 KB so two fit on an SM: stream
      // buffers take 2 x 2048 bytes per streamed byte of a row
      size_t table = pipeline_smem_bytes(d);
      budget = table >= 110 * 1024 ? 0 : (uint32_t)std::min<size_t>(16, (110 * 1024 - table) / (2 * 2048));
    }
    uint32_t used = 0;
    auto try_stream = [&](int col) {
      if (d.cols[col].src != d.drive_src || d.n_stream >= max_stream) return;
      for (int i = 0; i < d.n_stream; ++i)
        if (d.stream_cols[i] == col) return;
      uint32_t w = (uint32_t)ptype_width(d.cols[col].ptype);
      if (w > 8 || used + w > budget) return;
      d.stream_cols[d.n_stream++] = col;
      used += w;
    };
    double reach = 1.0;  // estimated fraction of tuples reaching the op
    const double kStreamAbove = 0.25;
    for (int o = 0; o < d.n_ops; ++o) {
      const PipeOp& op = d.ops[o];
      const int col = op.kind == OPK_FILTER ? d.preds[op.idx].col : d.probes[op.idx].key_col;
      if (o == 0 || reach >= kStreamAbove) try_stream(col);
      reach *= op.kind == OPK_FILTER ? (o < (int)pb.op_sel.size() ? pb.op_sel[o] : 0.5) : 0.25;
    }
    // A build's key column is streamed at a lower reach: its read sits on the
    // critical path of the sink (the map store depends on it).
    if (reach >= kStreamAbove || (d.sink == SK_BUILD && reach >= 0.05))
      for (int c : sink) try_stream(c);
  }

  // Probes into the children's builds; fill masks bring the row ids listed
  // in `want` into the pipeline.
  void add_probes(PipeBuilder& pb, int s, uint32_t want) {
    for (int c : children[s]) {
      if (pb.d.n_probes >= kMaxProbes) fail(MTL_UNSUPPORTED, "too many joins on one table");
      int pi = pb.d.n_probes++;
      int bi = pb.d.n_builds++;
      pb.d.builds[bi] = builds[c];
      DProbe& pr = pb.d.probes[pi];
      pr.key_col = add_col(pb, s, down_col[c]);
      pr.build = bi;
      pr.fill_mask = want & subtree[c];
      pb.d.ops[pb.d.n_ops].kind = OPK_PROBE;
      pb.d.ops[pb.d.n_ops].idx = pi;
      pb.d.n_ops++;
      build_probe_index[c] = pi;
    }
  }

  void finish_ops(PipeBuilder& pb) {
    if (pb.d.n_ops > 0) {
      const PipeOp& o = pb.d.ops[0];
      pb.d.first_col = o.kind == OPK_FILTER ? pb.d.preds[o.idx].col : pb.d.probes[o.idx].key_col;
    }
  }

  void push_pipeline(PipeBuilder& pb, uint64_t n_hint) {
    static const char* sinks[] = {"none",       "build",      "materialize", "agg_hash",    "agg_smem",
                                  "agg_slot",   "agg_scalar", "part_count",  "part_scatter",
                                  "agg_few",    "mat_count",  "mat_write"};
    plan_columns(pb);
    Step s;
    s.k = Step::PIPELINE;
    s.pipe = pb.d;
    s.n_hint = n_hint;
    s.pred_filter = pb.pred_filter;
    s.name = std::string("pipeline:") + sinks[pb.d.sink] + ":" + plan.sources[pb.d.drive_src].name;
    P.steps.push_back(s);
    P.kernels += 1;
  }

  // Partitioned one-key aggregation, for all but a few groups: the rows'
  // keys and aggregate inputs are written out grouped by key partition (a
  // count pass, a scan and a scatter pass over the same pipeline), then
  // CTAs aggregate one partition's chunk each in shared memory and merge
  // their groups into the global table, so rows update shared memory
  // instead of contending for global atomics, and each CTA's table holds
  // one partition's keys only. Returns false (nothing queued) when the
  // aggregate does not
  // qualify: few groups, a 128-bit input, more distinct inputs than a record
  // holds, more partitions than the count pass supports, or records that do
  // not fit the scratch region. On success pb.d.sink is SK_PART_COUNT.
  bool push_partitioned(PipeBuilder& pb, uint64_t est, uint64_t rows, bool forced = false) {
    if ((est <= 8 && !forced) || rows == 0 || rows >= (1ull << 31)) return false;
    PipeDesc d = pb.d;
    int nv = 0;
    int slot_prog[kMaxAggs];
    for (int a = 0; a < d.n_aggs; ++a) {
      d.part_val[a] = -1;
      const int pi = d.aggs[a].prog;
      if (pi < 0) continue;
      if (d.progs[pi].out_type == P_I128) return false;
      int f = -1;
      for (int j = 0; j < nv && f < 0; ++j)
        if (memcmp(&d.progs[slot_prog[j]], &d.progs[pi], sizeof(VmProg)) == 0) f = j;
      if (f < 0) {
        if (nv == part_max_values()) return false;
        f = nv++;
        slot_prog[f] = pi;
        d.part_src[f] = a;
      }
      d.part_val[a] = f;
    }
    // the partition CTA's table: up to 2048 entries within about 100 KB, so
    // two CTAs share an SM
    d.smem_capacity = 1;
    const uint64_t entry = part_agg_smem_bytes(d);
    const uint64_t cap = std::min<uint64_t>(2048, (100 * 1024) / entry);
    if (cap < 256) return false;
    // partitions: on average at most half a table of groups each; beyond
    // the partition limit, partitions hold more groups than a table and
    // the records of the keys a full table leaves out update the global
    // table, within the partition's stretch of it (kept in L2)
    int bits = 1;
    while ((cap / 2) << bits < est && bits < part_max_bits()) ++bits;
    const bool overfull = (cap / 2) << bits < est;
    const uint64_t np = 1ull << bits;
    const uint64_t words = nv == 0 ? 1 : nv == 1 ? 2 : 4;  // 16-byte aligned records
    const uint64_t rec_bytes = rows * words * 8;
    if (rec_bytes + (64ull << 20) > ctx.arena.largest_free()) return false;
    // Partitions holding more groups than a table are sub-partitioned: the
    // CTA of a chunk places its records by the next 2^split hash bits and
    // aggregates one sub-partition at a time, each about 60 % of a table.
    // That needs a second record buffer; without room for it, the keys a
    // full table leaves out update the global table directly.
    int split = 0;
    if (overfull) {
      while (split < part_max_split() && (uint64_t)((double)cap * 0.6) << (bits + split) < est) ++split;
      if (2 * rec_bytes + (64ull << 20) > ctx.arena.largest_free()) split = 0;
    }
    const bool still_overfull = (uint64_t)((double)cap * 0.6) << (bits + split) < est;
    const int ctas = pipeline_part_ctas();
    d.part_bits = bits;
    d.part_words = (int32_t)words;
    d.part_nvals = nv;
    d.part_combine = est / np < 128 ? 1 : 0;
    d.part_ctas = ctas;
    d.smem_capacity = (int32_t)cap;
    d.part_split = split;
    d.smem_probes = still_overfull ? 8 : 0;  // 0: the kernel's default window
    // records per CTA: half a partition's average, but small enough for
    // eight CTAs per SM, and at least 4096
    const uint64_t min_ctas = 4ull * (uint64_t)pipeline_part_ctas();
    d.part_chunk = (uint32_t)std::max<uint64_t>(
        4096, std::min<uint64_t>((rows + 2 * np - 1) / (2 * np), (rows + min_ctas - 1) / min_ctas));
    // sub-partitioned chunks: about one chunk per partition, so that each
    // group is merged into the global table once
    if (split) d.part_chunk = (uint32_t)std::max<uint64_t>(4096, (rows + np - 1) / np * 5 / 4);
    d.part_records = (uint64_t*)scratch(rec_bytes);
    d.part_sub = split ? (uint64_t*)scratch(rec_bytes) : nullptr;
    d.part_counts = (uint32_t*)scratch((uint64_t)ctas * np * 4);
    d.part_offsets = (uint32_t*)scratch((uint64_t)ctas * np * 4);
    d.part_start = (uint32_t*)scratch((np + 1) * 4);
    d.part_chunk_start = (uint32_t*)scratch((np + 1) * 4);
    pb.d = d;
    PipeBuilder scatter = pb;
    pb.d.sink = SK_PART_COUNT;
    push_pipeline(pb, rows);
    Step sc;
    sc.k = Step::PART_SCAN;
    sc.pipe = d;
    sc.name = "part_scan";
    P.steps.push_back(sc);
    P.kernels += 1;
    scatter.d.sink = SK_PART_SCATTER;
    push_pipeline(scatter, rows);
    Step sa;
    sa.k = Step::PART_AGG;
    sa.pipe = d;
    sa.name = "part_agg";
    sa.n_hint = rows;
    P.steps.push_back(sa);
    P.kernels += 1;
    return true;
  }

  // One pass over one table's columns into per-CTA shared-memory tables that
  // hold every group (k_agg_few): for a one-key aggregate over few groups of
  // one table with no filters, whose key and inputs are plain columns.
  // Returns false (nothing queued) when the query does not have that shape.
  bool push_few(PipeBuilder& pb, uint64_t est, uint64_t rows) {
    const PipeDesc& d = pb.d;
    if (plan.sources.size() != 1 || d.n_ops != 0 || rows == 0 || est > 1536) return false;
    auto plain = [&](int pi) {
      const VmProg& p = d.progs[pi];
      return p.fast.shape == 1 && p.fast.leaf[0].op == VM_COL && !p.fast.leaf_cast[0].on;
    };
    if (!plain(d.key_prog[0])) return false;
    std::set<int> cols;
    int n128 = 0;
    for (int a = 0; a < d.n_aggs; ++a) {
      n128 += d.aggs[a].fn == A_SUM_I128;
      if (d.aggs[a].prog < 0) continue;
      if (!plain(d.aggs[a].prog)) return false;
      cols.insert(d.progs[d.aggs[a].prog].fast.leaf[0].arg);
    }
    if ((int)cols.size() > agg_few_max_cols()) return false;
    uint64_t cap = 64;
    while (cap < est * 4 / 3 + 16) cap <<= 1;
    if (cap * (1 + (uint64_t)d.n_aggs + (uint64_t)n128) * 8 > 200 * 1024) return false;
    pb.d.smem_capacity = (int32_t)cap;
    pb.d.sink = SK_AGG_FEW;
    Step s;
    s.k = Step::AGG_FEW;
    s.pipe = pb.d;
    s.n_hint = rows;
    s.name = "agg_few:" + plan.sources[0].name;
    P.steps.push_back(s);
    P.kernels += 1;
    return true;
  }

  // Aggregate state descriptors for the sink (shared with the rep build).
  struct AggState {
    int fn_dev = 0;   // AggFn
    int prog_agg = -1;  // BAgg index whose arg feeds it (-1: COUNT)
    uint64_t* lo = nullptr;
    int64_t* hi = nullptr;
  };
  std::vector<AggState> states;      // device states
  std::vector<int> agg_sum_state, agg_cnt_state, agg_state;  // per BAgg
  int count_state = -1;

  static bool sum_fits64(const BAgg& g, uint64_t rows) {
    const BExpr& e = *g.arg;
    if (!e.bounded) return false;
    __int128 m = std::max(e.bmin < 0 ? -e.bmin : e.bmin, e.bmax < 0 ? -e.bmax : e.bmax);
    __int128 bound = m * (__int128)(rows ? rows : 1);
    return bound < ((__int128)1 << 63) - 1;
  }

  void plan_states(uint64_t groups, uint64_t rows, bool need_count, bool alloc = true) {
    agg_sum_state.assign(plan.aggs.size(), -1);
    agg_cnt_state.assign(plan.aggs.size(), -1);
    agg_state.assign(plan.aggs.size(), -1);
    auto new_state = [&](int fn, int agg) {
      AggState s;
      s.fn_dev = fn;
      s.prog_agg = agg;
      if (alloc) {
        s.lo = (uint64_t*)scratch(groups * 8);
        if (fn == A_SUM_I128) s.hi = (int64_t*)scratch(groups * 8);
      }
      states.push_back(s);
      return (int)states.size() - 1;
    };
    bool any_avg = false;
    for (auto& g : plan.aggs) any_avg |= g.fn == AG_AVG;
    if (need_count || any_avg) count_state = new_state(A_COUNT, -1);
    for (size_t i = 0; i < plan.aggs.size(); ++i) {
      const BAgg& g = plan.aggs[i];
      switch (g.fn) {
        case AG_COUNT:
          if (count_state < 0) count_state = new_state(A_COUNT, -1);
          agg_state[i] = count_state;
          break;
        case AG_SUM:
        case AG_AVG: {
          const LType at = g.arg->type;
          int fn;
          if (is_float_family(at)) fn = A_SUM_F;
          else if (g.fn == AG_AVG && at.t == MTL_T_INTEGER) fn = A_SUM_I;
          else fn = sum_fits64(g, rows) ? A_SUM_I : A_SUM_I128;
          // reuse the state of an identical sum
          int found = -1;
          for (size_t j = 0; j < i; ++j)
            if (agg_sum_state[j] >= 0 && plan.aggs[j].arg && plan.aggs[j].arg->text == g.arg->text &&
                states[agg_sum_state[j]].fn_dev == fn)
              found = agg_sum_state[j];
          int s = found >= 0 ? found : new_state(fn, (int)i);
          agg_sum_state[i] = s;
          agg_state[i] = s;
          if (g.fn == AG_AVG) agg_cnt_state[i] = count_state;
          break;
        }
        case AG_MIN:
        case AG_MAX: {
          bool f = is_float_family(g.arg->type);
          int fn = g.fn == AG_MIN ? (f ? A_MIN_F : A_MIN_I) : (f ? A_MAX_F : A_MAX_I);
          agg_state[i] = new_state(fn, (int)i);
          break;
        }
      }
    }
    if ((int)states.size() > kMaxAggs) fail(MTL_UNSUPPORTED, "too many aggregates in one query");
  }

  void fill_aggs(PipeBuilder& pb, bool with_progs) {
    pb.d.n_aggs = (int)states.size();
    for (size_t i = 0; i < states.size(); ++i) {
      DAgg& a = pb.d.aggs[i];
      a.fn = states[i].fn_dev;
      a.lo = states[i].lo;
      a.hi = states[i].hi;
      a.prog = -1;
      if (with_progs && states[i].prog_agg >= 0) a.prog = add_prog(pb, *plan.aggs[states[i].prog_agg].arg);
    }
  }

  // ---- final outputs of aggregate queries
  struct DenseOut {
    void* dev = nullptr;
    int width = 0;
    int32_t ptype = 0;
  };
  std::vector<DenseOut> dense;  // per plan output

  FinalOut agg_final(int out_i, void* dst) {
    const BOut& o = plan.outputs[out_i];
    FinalOut f;
    memset(&f, 0, sizeof(f));
    f.out = dst;
    const BAgg& g = plan.aggs[o.agg_idx];
    const int si = agg_state[o.agg_idx];
    const AggState& st = states[si];
    f.a = st.lo;
    f.a_hi = st.hi;
    f.stride = state_stride;
    switch (g.fn) {
      case AG_COUNT: f.kind = F_COPY_I64; break;
      case AG_SUM:
        f.kind = st.fn_dev == A_SUM_F ? F_COPY_F64 : st.fn_dev == A_SUM_I128 ? F_SUM_I128 : F_SUM_I64_AS_I128;
        break;
      case AG_MIN:
      case AG_MAX:
        if (st.fn_dev == A_MIN_F || st.fn_dev == A_MAX_F)
          f.kind = g.result.t == MTL_T_FLOAT ? F_MINMAX_F32 : F_MINMAX_F64;
        else
          f.kind = ptype_width(storage_ptype(g.result)) == 4 ? F_COPY_I32 : F_COPY_I64;
        break;
      case AG_AVG: {
        f.cnt = states[agg_cnt_state[o.agg_idx]].lo;
        const LType at = g.arg->type;
        if (is_float_family(at)) f.kind = F_AVG_F64;
        else if (at.t == MTL_T_INTEGER) f.kind = F_AVG_I64_D;
        else if (is_decimal(at)) {
          f.kind = F_AVG_DEC;
          f.scale = std::pow(10.0, at.scale);
        } else f.kind = F_AVG_I128_LD;
        if (st.fn_dev != A_SUM_I128) f.a_hi = nullptr;
        break;
      }
    }
    return f;
  }

  FinalOut* upload_finals(const std::vector<FinalOut>& fo) {
    FinalOut* d = (FinalOut*)scratch(fo.size() * sizeof(FinalOut));
    upload(d, fo.data(), fo.size() * sizeof(FinalOut));
    return d;
  }

  void finalize_step(FinalOut* fd, int n, const uint32_t* idx, const uint64_t* count, uint64_t n_max) {
    Step s;
    s.k = Step::FINALIZE;
    s.fin_dev = fd;
    s.n_fin = n;
    s.idx = idx;
    s.count = count;
    s.n_max = n_max;
    P.steps.push_back(s);
    P.kernels += 1;
  }

  // ---- ORDER BY / LIMIT over dense output arrays
  // With `groups` and `late` (a top-K over a grouped aggregate whose ORDER BY
  // outputs alone were finalized into dense[]), the winners' group ids are
  // gathered from `groups` and the visible outputs finalized for them only.
  void order_and_limit(const uint64_t* count, uint64_t n_max, const std::vector<int>& tie_outs,
                       const uint32_t* groups = nullptr, const std::vector<FinalOut>* late = nullptr) {
    P.limit = plan.limit;
    std::vector<int> vis;
    for (size_t i = 0; i < plan.outputs.size(); ++i)
      if (!plan.outputs[i].hidden) vis.push_back((int)i);
    if (plan.order.empty() || plan.limit == 0 || n_max == 0) {
      for (int i : vis) {
        OutBuf ob;
        ob.name = plan.outputs[i].name;
        ob.type = plan.outputs[i].type;
        ob.dev = dense[i].dev;
        ob.width = dense[i].width;
        ob.dict = plan.outputs[i].dict;
        P.outs.push_back(ob);
      }
      P.out_count = count;
      P.n_max = n_max;
      return;
    }
    SortKeySpec spec;
    memset(&spec, 0, sizeof(spec));
    int bits = 0;
    auto part_bits = [](int32_t pt) { return pt == P_I128 ? 128 : (pt == P_I32 || pt == P_F32) ? 32 : 64; };
    auto add_part = [&](int out_i, bool desc) {
      int32_t pt = dense[out_i].ptype;
      if (bits + part_bits(pt) > 256 || spec.n_parts >= kMaxOrder) return false;
      spec.ptype[spec.n_parts] = pt;
      spec.desc[spec.n_parts] = desc ? 1 : 0;
      spec.col[spec.n_parts] = dense[out_i].dev;
      spec.n_parts++;
      bits += part_bits(pt);
      return true;
    };
    for (const BOrder& o : plan.order)
      if (!add_part(o.out, o.desc)) fail(MTL_UNSUPPORTED, "ORDER BY keys wider than 256 bits");
    for (int t : tie_outs) {
      bool in_order = false;
      for (const BOrder& o : plan.order) in_order |= o.out == t;
      if (!in_order) add_part(t, false);
    }
    SortItem* keys = (SortItem*)scratch(std::max<uint64_t>(n_max, 1) * sizeof(SortItem));
    uint32_t* kidx = (uint32_t*)scratch(std::max<uint64_t>(n_max, 1) * 4);
    Step e;
    e.k = Step::ENCODE;
    e.spec = spec;
    e.count = count;
    e.n_max = n_max;
    e.keys = keys;
    e.kidx = kidx;
    P.steps.push_back(e);
    P.kernels += 1;
    const uint32_t* final_idx;
    const uint64_t* final_count;
    uint64_t rows_max;
    if (plan.limit > 0 && plan.limit <= 1024) {
      const int K = (int)plan.limit;
      uint32_t* oidx = (uint32_t*)scratch((uint64_t)K * 4);
      uint64_t* ocnt = (uint64_t*)scratch(8);
      Step t;
      t.k = Step::TOPK;
      t.keys = keys;
      t.kidx = kidx;
      t.count = count;
      t.n_max = n_max;
      t.topk = K;
      t.out_idx = oidx;
      t.out_count = ocnt;
      t.temp = scratch(topk_temp_bytes(n_max, K));
      P.steps.push_back(t);
      P.kernels += 2;
      final_idx = oidx;
      final_count = ocnt;
      rows_max = std::min<uint64_t>(n_max, (uint64_t)K);
      if (late) {
        uint32_t* wg = (uint32_t*)scratch((uint64_t)K * 4);
        Step g;
        g.k = Step::GATHER;
        g.gin = groups;
        g.width = 4;
        g.idx = oidx;
        g.count = ocnt;
        g.n_max = (uint64_t)K;
        g.gout = wg;
        P.steps.push_back(g);
        P.kernels += 1;
        std::vector<FinalOut> vf;
        for (int i : vis) {
          FinalOut f = (*late)[i];
          f.out = scratch((uint64_t)K * dense[i].width);
          vf.push_back(f);
          OutBuf ob;
          ob.name = plan.outputs[i].name;
          ob.type = plan.outputs[i].type;
          ob.dev = f.out;
          ob.width = dense[i].width;
          ob.dict = plan.outputs[i].dict;
          P.outs.push_back(ob);
        }
        if (!vf.empty()) finalize_step(upload_finals(vf), (int)vf.size(), wg, ocnt, (uint64_t)K);
        P.out_count = ocnt;
        P.n_max = rows_max;
        return;
      }
    } else {
      SortItem* keys2 = (SortItem*)scratch(std::max<uint64_t>(n_max, 1) * sizeof(SortItem));
      uint32_t* kidx2 = (uint32_t*)scratch(std::max<uint64_t>(n_max, 1) * 4);
      Step r;
      r.k = Step::RADIX;
      r.keys = keys;
      r.kidx = kidx;
      r.keys_tmp = keys2;
      r.kidx_tmp = kidx2;
      r.count = count;
      r.n_max = n_max;
      r.key_bytes = (bits + 7) / 8;
      r.temp = scratch(radix_sort_temp_bytes(n_max));
      P.steps.push_back(r);
      uint64_t tiles = (n_max + 4095) / 4096;
      uint64_t chunks = (tiles * 256 + 4095) / 4096;
      P.kernels += r.key_bytes * (chunks == 1 ? 3 : 5);
      final_idx = (r.key_bytes & 1) ? kidx2 : kidx;
      final_count = count;
      rows_max = n_max;
    }
    for (int i : vis) {
      void* outp = scratch(std::max<uint64_t>(rows_max, 1) * dense[i].width);
      Step g;
      g.k = Step::GATHER;
      g.gin = dense[i].dev;
      g.width = dense[i].width;
      g.idx = final_idx;
      g.count = final_count;
      g.n_max = rows_max;
      g.gout = outp;
      P.steps.push_back(g);
      P.kernels += 1;
      OutBuf ob;
      ob.name = plan.outputs[i].name;
      ob.type = plan.outputs[i].type;
      ob.dev = outp;
      ob.width = dense[i].width;
      ob.dict = plan.outputs[i].dict;
      P.outs.push_back(ob);
    }
    P.out_count = final_count;
    P.n_max = rows_max;
  }

  // ---- main
  void compile() {
    P.status = (uint32_t*)scratch(8);
    memset_step(P.status, 0, 8);
    plan_joins();
    const int S = (int)plan.sources.size();
    builds.assign(S, DBuild{});
    build_probe_index.assign(S, -1);
    const uint64_t root_rows = plan.sources[root].table->rows;

    // what the root sink reads
    needed_root = 0;
    if (!plan.is_agg) {
      for (auto& o : plan.outputs) expr_sources(*o.expr, needed_root);
    } else {
      for (auto& g : plan.aggs)
        if (g.arg) expr_sources(*g.arg, needed_root);
      rep_src = find_rep();
      if (rep_src < 0)
        for (auto& k : plan.group_keys) expr_sources(*k, needed_root);
    }

    // aggregate states (the representative build initializes them)
    const bool scalar = plan.is_agg && plan.group_keys.empty();
    uint64_t groups = 0;
    uint64_t est_groups = 0;
    if (plan.is_agg) {
      if (scalar) groups = 1;
      else if (rep_src >= 0) groups = std::max<uint64_t>(1, plan.sources[rep_src].table->rows);
      else {
        est_groups = estimate_groups();
        const double lf = tune_load_factor(ctx, "agg_table", est_groups);
        P.load_keys.push_back({tune_key_load("agg_table", est_groups), est_groups});
        groups = std::max<uint64_t>(64, (uint64_t)std::ceil(lf * (double)est_groups));
      }
      // a one-key hash table keeps one more group: the key equal to the
      // empty-slot sentinel
      cas_table = !scalar && rep_src < 0 && plan.group_keys.size() == 1 && groups + 1 < (1ull << 31);
      plan_states(cas_table ? groups + 1 : groups, root_rows, scalar, !cas_table);
    }

    // build pipelines, children before parents
    std::vector<int> post;
    std::function<void(int)> dfs = [&](int s) {
      for (int c : children[s]) dfs(c);
      if (s != root) post.push_back(s);
    };
    dfs(root);
    uint8_t* slot_hit = nullptr;
    for (int s : post) {
      builds[s] = make_build(s);
      PipeBuilder pb;
      pb.d.n = plan.sources[s].table->rows;
      pb.d.drive_src = s;
      pb.d.src_mask = 1u << s;
      uint32_t pay = payload_mask(s) | (s == rep_src ? (1u << s) : 0u);
      for (int c : children[s]) builds[c].kind = builds[c].kind;  // built already
      add_filters(pb, s);
      add_probes(pb, s, pay);
      finish_ops(pb);
      pb.d.sink = SK_BUILD;
      pb.d.builds[pb.d.n_builds] = builds[s];
      pb.d.sink_build = pb.d.n_builds++;
      pb.d.build_key_col = add_col(pb, s, up_col[s]);
      pb.d.build_payload_mask = pay;
      for (int q = 0; q < kMaxSrc; ++q)
        if (q != s && ((pay >> q) & 1u)) {  // the build's own row is its slot
          builds[s].payload[q] = (uint32_t*)scratch(std::max<uint64_t>(1, plan.sources[s].table->rows) * 4);
          pb.d.builds[pb.d.sink_build].payload[q] = builds[s].payload[q];
        }
      if (s == rep_src) {
        fill_aggs(pb, false);
        slot_hit = (uint8_t*)scratch(std::max<uint64_t>(1, plan.sources[s].table->rows));
        memset_step(slot_hit, 0, std::max<uint64_t>(1, plan.sources[s].table->rows));
        pb.d.slot_hit = slot_hit;
      }
      pb.d.status = P.status;
      push_pipeline(pb, pb.d.n);
      // a build that initializes no aggregate states can stay resident
      // across runs of this program whose literals leave its subtree unchanged
      P.steps.back().build_src = s;
      P.steps.back().build_src_mask = subtree[s];
      P.steps.back().build_keepable = s != rep_src;
      P.steps.back().orig_n = pb.d.n;
    }

    // root pipeline
    PipeBuilder pb;
    pb.d.n = root_rows;
    pb.d.drive_src = root;
    pb.d.src_mask = 1u << root;
    add_filters(pb, root);
    add_probes(pb, root, needed_root);
    finish_ops(pb);
    pb.d.status = P.status;
    dense.assign(plan.outputs.size(), DenseOut{});

    if (!plan.is_agg) {
      // order-preserving materialization of every output (incl. ORDER BY keys)
      pb.d.sink = SK_MATERIALIZE;
      const uint64_t n_max = root_rows;
      pb.d.n_out = (int)plan.outputs.size();
      for (size_t i = 0; i < plan.outputs.size(); ++i) {
        const BOut& o = plan.outputs[i];
        int pi = add_prog(pb, *o.expr);
        pb.d.out_prog[i] = pi;
        const int32_t pt = o.expr->ptype;
        // outputs are stored in the logical type's storage representation
        if (storage_ptype(o.type) != pt) {
          fail(MTL_UNSUPPORTED, "output representation mismatch");
        }
        dense[i].width = ptype_width(pt);
        dense[i].ptype = pt;
        dense[i].dev = scratch(std::max<uint64_t>(1, n_max) * dense[i].width);
        pb.d.out_ptr[i] = dense[i].dev;
      }
      uint32_t m = 0;
      for (auto& o : plan.outputs) expr_sources(*o.expr, m);
      pb.d.mat_src_mask = m;
      pb.d.out_count = (uint64_t*)scratch(8);
      pb.d.out_capacity = n_max;
      const uint64_t tiles = (n_max + pipeline_warp_tile_rows() - 1) / pipeline_warp_tile_rows();
      // Two passes by default: a count of each tile's survivors, a scan, and
      // the write at known offsets (no wait on other tiles); the single pass
      // with a decoupled look-back when the autotuner measured it faster (or
      // a test injects a look-back stall).
      const bool injected = ctx.inject_kind.load() == MTL_INJECT_LOOKBACK_STALL;
      const int mstrat = injected ? 1 : tune_mat_strategy(ctx, root_rows);
      P.mat_strategy_key = injected ? "" : tune_key_mat(root_rows);
      // Late gather: a scan of one table whose outputs are its columns,
      // plain or combined with one constant, writes only the surviving row
      // ids in the write pass; one kernel then gathers every output at them
      // (all source loads of a row in flight together).
      std::vector<GatherOut> gos;
      if (mstrat != 1 && root_rows < (1ull << 32) && plan.sources.size() == 1 && pb.d.n_probes == 0)
        for (size_t i = 0; i < plan.outputs.size(); ++i) {
          const VmProg& pg = pb.d.progs[pb.d.out_prog[i]];
          const bool plain = pg.n == 1 && pg.ins[0].op == VM_COL;
          const bool arith = pg.n == 3 && pg.ins[0].op == VM_COL && pg.ins[1].op == VM_CONST &&
                             pg.ins[2].op >= VM_ADD && pg.ins[2].op <= VM_MUL && pg.ins[2].type != P_I128;
          if (!plain && !arith) break;
          const DCol& c = pb.d.cols[pg.ins[0].arg];
          const int w = ptype_width(c.ptype), ow = ptype_width(pg.out_type);
          if ((w != 4 && w != 8) || (ow != 4 && ow != 8) || c.src != root) break;
          GatherOut g;
          memset(&g, 0, sizeof(g));
          g.src = c.ptr;
          g.out = dense[i].dev;
          g.in_kind = w == 8 ? 2 : c.ptype == P_I32 ? 0 : 1;
          g.out_width = ow;
          g.op = arith ? pg.ins[2].op : 0;
          g.type = arith ? pg.ins[2].type : 0;
          g.k = arith ? pg.ins[1].k : 0;
          gos.push_back(g);
        }
      const bool late = !gos.empty() && gos.size() == plan.outputs.size();
      if (mstrat != 1 && root_rows < (1ull << 32)) {
        const uint64_t chunks = (tiles + kMatScanTiles - 1) / kMatScanTiles;
        pb.d.tile_pos = (uint32_t*)scratch(std::max<uint64_t>(tiles, 1) * 4);
        pb.d.chunk_pos = (uint64_t*)scratch(std::max<uint64_t>(chunks, 1) * 8);
        uint32_t* rid = nullptr;
        if (late) {
          // the count pass also writes the survivor masks, which the scan
          // expands into row ids: no second pass over the table
          rid = (uint32_t*)scratch(std::max<uint64_t>(1, n_max) * 4);
          pb.d.tile_mask = (uint32_t*)scratch(std::max<uint64_t>(tiles, 1) * 32);
          pb.d.out_rids[root] = rid;
        }
        PipeBuilder count = pb;
        count.d.sink = SK_MAT_COUNT;
        push_pipeline(count, root_rows);
        Step sc;
        sc.k = Step::MAT_SCAN;
        sc.pipe = pb.d;
        sc.n_hint = root_rows;
        sc.name = "mat_scan";
        P.steps.push_back(sc);
        P.kernels += late ? 3 : 2;
        pb.d.sink = SK_MAT_WRITE;
        if (late) {
          GatherOut* go = (GatherOut*)scratch(gos.size() * sizeof(GatherOut));
          upload(go, gos.data(), gos.size() * sizeof(GatherOut));
          Step g;
          g.k = Step::GATHER_OUTS;
          g.go = go;
          g.n_go = (int)gos.size();
          g.idx = rid;
          g.count = pb.d.out_count;
          g.n_max = n_max;
          P.steps.push_back(g);
          P.kernels += 1;
        } else {
          push_pipeline(pb, root_rows);
        }
        order_and_limit(pb.d.out_count, n_max, {});
        return;
      }
      // look-back words for the smaller (warp) tiles, so that either kernel
      // can run the step
      pb.d.tile_status = (uint64_t*)scratch(std::max<uint64_t>(tiles, 1) * 8);
      pb.d.tile_counter = (uint32_t*)scratch(8);
      pb.d.epoch = 1;
      if (ctx.inject_kind.load() == MTL_INJECT_LOOKBACK_STALL) {
        pb.d.lb_stall_first = 1;
        pb.d.lb_spin_limit = ctx.inject_arg.load();
      }
      memset_step(pb.d.tile_status, 0, std::max<uint64_t>(tiles, 1) * 8);
      memset_step(pb.d.tile_counter, 0, 8);
      push_pipeline(pb, root_rows);
      order_and_limit(pb.d.out_count, n_max, {});
      return;
    }

    std::vector<int> tie;  // group-key outputs: deterministic tie order
    for (size_t i = 0; i < plan.outputs.size(); ++i)
      if (plan.outputs[i].group_idx >= 0) tie.push_back((int)i);

    if (scalar) {
      pb.d.sink = SK_AGG_SCALAR;
      for (auto& s : states) {
        uint64_t init = 0;
        switch (s.fn_dev) {
          case A_MIN_I: init = 0x7FFFFFFFFFFFFFFFULL; break;
          case A_MAX_I: init = 0x8000000000000000ULL; break;
          case A_MIN_F: init = ~0ULL; break;
          default: init = 0;
        }
        fill_step(s.lo, 1, init);
        if (s.hi) fill_step(s.hi, 1, 0);
      }
      fill_aggs(pb, true);
      push_pipeline(pb, root_rows);
      std::vector<FinalOut> fo;
      for (size_t i = 0; i < plan.outputs.size(); ++i) {
        const BOut& o = plan.outputs[i];
        dense[i].ptype = storage_ptype(o.type);
        dense[i].width = ptype_width(dense[i].ptype);
        dense[i].dev = scratch(16);
        fo.push_back(agg_final((int)i, dense[i].dev));
      }
      finalize_step(upload_finals(fo), (int)fo.size(), nullptr, nullptr, 1);
      P.fixed_count = 1;
      P.empty_count = states[count_state].lo;
      order_and_limit(nullptr, 1, {});
      P.fixed_count = 1;
      return;
    }

    if (rep_src >= 0) {
      // Grouping by a build's representative row: states are dense by the
      // build slot (the reference's dense_row_id_sum_track_live_v /
      // accumulate_revenue_dense_slots_from_indices_v, kernels.metal:1009,1076).
      pb.d.sink = SK_AGG_SLOT;
      pb.d.slot_probe = build_probe_index[rep_src];
      pb.d.slot_hit = slot_hit;
      fill_aggs(pb, true);
      push_pipeline(pb, root_rows);
      const uint64_t cap = std::max<uint64_t>(1, plan.sources[rep_src].table->rows);
      const uint64_t* n_dev = nullptr;  // slots are the build table's rows
      std::vector<FinalOut> fo;
      for (size_t i = 0; i < plan.outputs.size(); ++i) {
        const BOut& o = plan.outputs[i];
        dense[i].ptype = storage_ptype(o.type);
        dense[i].width = ptype_width(dense[i].ptype);
        if (o.agg_idx >= 0) {
          fo.push_back(agg_final((int)i, nullptr));
        } else {
          FinalOut f;
          memset(&f, 0, sizeof(f));
          f.kind = F_GATHER_COL;
          f.width = dense[i].width;
          Column* c = rep_column(*plan.group_keys[o.group_idx]);
          f.col = column_device(ctx, *c);
          pinned_cols.insert(c);
          f.rid = nullptr;  // the group's slot is its row in the representative table
          fo.push_back(f);
        }
      }
      if (agg_topk_fused(fo, slot_hit, nullptr, n_dev, cap, tie)) return;
      uint32_t* gidx = (uint32_t*)scratch(cap * 4);
      uint64_t* gcnt = (uint64_t*)scratch(8);
      compact_step(slot_hit, cap, n_dev, gidx, gcnt, false);
      for (size_t i = 0; i < fo.size(); ++i) fo[i].out = dense[i].dev = scratch(cap * dense[i].width);
      finalize_step(upload_finals(fo), (int)fo.size(), gidx, gcnt, cap);
      order_and_limit(gcnt, cap, tie);
      return;
    }

    // hash aggregation (shared-memory tables when the group count is small)
    const uint64_t cap = groups;
    const uint64_t n_ent = cas_table ? cap + 1 : cap;  // table entries incl. the sentinel key's group
    pb.d.table.capacity = cap;
    pb.d.table.n_keys = (int)plan.group_keys.size();
    pb.d.table.cas = cas_table ? 1 : 0;
    pb.d.table.state = (uint32_t*)scratch(n_ent * 4);
    memset_step(pb.d.table.state, 0, n_ent * 4);
    for (size_t k = 0; k < plan.group_keys.size(); ++k) {
      if (!cas_table) pb.d.table.keys[k] = (uint64_t*)scratch(n_ent * 8);
      pb.d.key_prog[k] = add_prog(pb, *plan.group_keys[k]);
    }
    if (cas_table) {
      // One entry per group holds its key and all of its states, so a row
      // touches one 32-byte-aligned entry. Keys start empty and states at
      // their identities: a claim is one CAS.
      int n_hi = 0;
      for (const AggState& s : states) n_hi += s.fn_dev == A_SUM_I128;
      const uint64_t words = 1 + states.size() + (uint64_t)n_hi;
      const uint64_t stride = (words + 3) & ~3ULL;
      uint64_t* aos = (uint64_t*)scratch(n_ent * stride * 8);
      state_stride = (int)stride;
      pb.d.table.keys[0] = aos;
      pb.d.table.stride = (int32_t)stride;
      // every entry starts as: empty key, state identities, zero high
      // words; written whole, in one pass over the table
      std::vector<uint64_t> entry(stride, 0);
      entry[0] = ~0ULL;
      uint64_t hw = 1 + states.size();
      for (size_t s = 0; s < states.size(); ++s) {
        states[s].lo = aos + 1 + s;
        entry[1 + s] = state_identity(states[s].fn_dev);
        if (states[s].fn_dev == A_SUM_I128) states[s].hi = (int64_t*)(aos + hw++);
      }
      uint64_t* entry_dev = (uint64_t*)scratch(stride * 8);
      upload(entry_dev, entry.data(), stride * 8);
      fill_entries(aos, n_ent, stride, entry_dev);
    } else {
      pb.d.table.stride = 1;
    }
    fill_aggs(pb, true);
    // Few groups: each CTA aggregates in shared memory and merges into the
    // global table at the end. Many: rows update the global table directly;
    // with one key, a small shared-memory table in front of it keeps each
    // CTA's most frequent keys (the first to arrive), so a skewed key's rows
    // meet in shared memory instead of contending on one global entry.
    pb.d.sink = SK_AGG_HASH;
    // one-key aggregates whose groups all fit a CTA's shared-memory table
    // may run either way; the autotuner's measured choice decides
    const int strategy = cas_table && est_groups <= 1536 ? tune_agg_strategy(ctx, est_groups, root_rows) : 0;
    P.agg_strategy_key = cas_table && est_groups <= 1536 ? tune_key_agg(est_groups, root_rows) : "";
    // one pass by default only for the fewest groups (measured faster there;
    // above them the partitioned passes win unless the autotuner says otherwise)
    if (cas_table && (strategy == 1 || (strategy == 0 && est_groups <= 16)) && push_few(pb, est_groups, root_rows)) {
      // one pass over the columns into per-CTA tables
    } else if (cas_table && strategy != 1 && push_partitioned(pb, est_groups, root_rows, strategy == 2)) {
      // count, scan, scatter and per-partition aggregation are queued
    } else if (cas_table) {
      pb.d.sink = SK_AGG_SMEM;
      const bool whole = est_groups <= 1536;
      pb.d.smem_capacity = whole ? (int)(est_groups * 3 / 2 + 64) : 1024;
      pb.d.smem_probes = whole ? pb.d.smem_capacity : 2;
      if (pipeline_smem_bytes(pb.d) > 160 * 1024) {
        pb.d.sink = SK_AGG_HASH;
        pb.d.smem_capacity = 0;
      }
    } else if (est_groups <= 1536) {
      pb.d.sink = SK_AGG_SMEM;
      pb.d.smem_capacity = (int)std::max<uint64_t>(256, est_groups * 4 / 3 + 64);
      if (pipeline_smem_bytes(pb.d) > 150 * 1024) {
        pb.d.sink = SK_AGG_HASH;
        pb.d.smem_capacity = 0;
      }
    }
    if (pb.d.sink != SK_PART_COUNT && pb.d.sink != SK_AGG_FEW) push_pipeline(pb, root_rows);
    std::vector<FinalOut> fo;
    for (size_t i = 0; i < plan.outputs.size(); ++i) {
      const BOut& o = plan.outputs[i];
      dense[i].ptype = storage_ptype(o.type);
      dense[i].width = ptype_width(dense[i].ptype);
      if (o.agg_idx >= 0) {
        fo.push_back(agg_final((int)i, nullptr));
      } else {
        FinalOut f;
        memset(&f, 0, sizeof(f));
        const int32_t pt = dense[i].ptype;
        f.kind = pt == P_I32 ? F_COPY_I32 : pt == P_F32 ? F_COPY_F32 : F_COPY_I64;
        f.a = pb.d.table.keys[o.group_idx];
        f.stride = pb.d.table.stride;
        fo.push_back(f);
      }
    }
    if (agg_topk_fused(fo, nullptr, pb.d.table.state, nullptr, n_ent, tie)) return;
    uint32_t* gidx = (uint32_t*)scratch(n_ent * 4);
    uint64_t* gcnt = (uint64_t*)scratch(8);
    compact_step(pb.d.table.state, n_ent, nullptr, gidx, gcnt, true);
    if (!plan.order.empty() && plan.limit > 0 && plan.limit <= 1024) {
      // ORDER BY ... LIMIT K: only the ordering outputs (and tie-breaks) for
      // every group; the other outputs only for the K winners
      std::vector<char> need(fo.size(), 0);
      for (const BOrder& o : plan.order) need[o.out] = 1;
      for (int t : tie) need[t] = 1;
      std::vector<FinalOut> ford;
      for (size_t i = 0; i < fo.size(); ++i)
        if (need[i]) {
          FinalOut f = fo[i];
          f.out = dense[i].dev = scratch(n_ent * dense[i].width);
          ford.push_back(f);
        }
      finalize_step(upload_finals(ford), (int)ford.size(), gidx, gcnt, n_ent);
      order_and_limit(gcnt, n_ent, tie, gidx, &fo);
      return;
    }
    for (size_t i = 0; i < fo.size(); ++i) fo[i].out = dense[i].dev = scratch(n_ent * dense[i].width);
    finalize_step(upload_finals(fo), (int)fo.size(), gidx, gcnt, n_ent);
    order_and_limit(gcnt, n_ent, tie);
  }

  static uint64_t state_identity(int fn) {
    switch (fn) {
      case A_MIN_I: return 0x7FFFFFFFFFFFFFFFULL;
      case A_MAX_I: return 0x8000000000000000ULL;
      case A_MIN_F: return ~0ULL;
      default: return 0;
    }
  }

  // Aggregate ORDER BY ... LIMIT K with K <= 32: one fused top-K over the
  // live groups' states (no compaction, per-group outputs or key array),
  // then the visible outputs of the K winners only. Returns false when the
  // query needs the general path.
  bool agg_topk_fused(const std::vector<FinalOut>& fo, const uint8_t* flag, const uint32_t* state,
                      const uint64_t* n_dev, uint64_t cap, const std::vector<int>& tie_outs) {
    if (plan.order.empty() || plan.limit < 1 || plan.limit > 32 || cap == 0 || cap >= 0xFFFFFFFFull) return false;
    TopkFinalSpec ts;
    memset(&ts, 0, sizeof(ts));
    int bits = 0;
    auto part_bits = [](int32_t pt) { return pt == P_I128 ? 128 : (pt == P_I32 || pt == P_F32) ? 32 : 64; };
    auto add_part = [&](int out_i, bool desc) {
      // a 128-bit output holding a 64-bit sum orders by its 64-bit image: its
      // high word is only the sign, and the leading key bits (the pruning
      // cut) then carry the sum itself
      const int32_t pt = fo[out_i].kind == F_SUM_I64_AS_I128 ? P_I64 : dense[out_i].ptype;
      if (bits + part_bits(pt) > 256 || ts.n_parts >= kMaxOrder) return false;
      ts.ptype[ts.n_parts] = pt;
      ts.desc[ts.n_parts] = desc ? 1 : 0;
      ts.part[ts.n_parts] = fo[out_i];
      ts.n_parts++;
      bits += part_bits(pt);
      return true;
    };
    for (const BOrder& o : plan.order)
      if (!add_part(o.out, o.desc)) return false;
    for (int t : tie_outs) {
      bool in_order = false;
      for (const BOrder& o : plan.order) in_order |= o.out == t;
      if (!in_order) add_part(t, false);
    }
    ts.total_bits = bits;
    ts.bits0 = part_bits(ts.ptype[0]);
    ts.flag = flag;
    ts.state = state;
    ts.n_dev = n_dev;
    ts.n_max = cap;
    const int K = (int)plan.limit;
    uint32_t* og = (uint32_t*)scratch((uint64_t)K * 4);
    uint64_t* oc = (uint64_t*)scratch(8);
    // one fused top-K straight over the live groups' states (each warp
    // gathers live groups, keys them and keeps a warp list), then one
    // merge pass; the winners come out as group ids
    Step t;
    t.k = Step::TOPK_FINAL;
    t.tfs = ts;
    t.topk = K;
    t.out_idx = og;
    t.out_count = oc;
    t.temp = scratch(topk_final_temp_bytes(cap, K));
    memset_step(t.temp, 0, 256);  // the launch's cross-CTA state starts at zero
    std::vector<FinalOut> vis;
    for (size_t i = 0; i < plan.outputs.size(); ++i) {
      if (plan.outputs[i].hidden) continue;
      FinalOut f = fo[i];
      f.out = scratch((uint64_t)K * dense[i].width);
      vis.push_back(f);
      OutBuf ob;
      ob.name = plan.outputs[i].name;
      ob.type = plan.outputs[i].type;
      ob.dev = f.out;
      ob.width = dense[i].width;
      ob.dict = plan.outputs[i].dict;
      P.outs.push_back(ob);
    }
    t.topk_phase = 1;  // the first pass, then the merge as its own step
    P.steps.push_back(t);
    // the merge pass writes the winners' visible outputs itself
    t.topk_phase = 2;
    t.name = "topk_merge";
    t.fin_dev = vis.empty() ? nullptr : upload_finals(vis);
    t.n_fin = (int)vis.size();
    P.steps.push_back(t);
    P.kernels += 2;
    P.limit = plan.limit;
    P.out_count = oc;
    P.n_max = (uint64_t)K;
    return true;
  }

  void compact_step(const void* flag, uint64_t n, const uint64_t* n_dev, uint32_t* out_idx, uint64_t* out_count,
                    bool ready) {
    const uint64_t tiles = (n + compact_tile_rows() - 1) / compact_tile_rows();
    Step s;
    s.k = ready ? Step::COMPACT_READY : Step::COMPACT_FLAGS;
    s.flag = flag;
    s.n = n;
    s.n_dev = n_dev;
    s.out_idx = out_idx;
    s.out_count = out_count;
    s.tstatus = (uint64_t*)scratch(std::max<uint64_t>(tiles, 1) * 8);
    s.tcounter = (uint32_t*)scratch(8);
    memset_step(s.tstatus, 0, std::max<uint64_t>(tiles, 1) * 8);
    memset_step(s.tcounter, 0, 8);
    P.steps.push_back(s);
    P.kernels += 1;
  }

  // ---- representative-row grouping
  // Union-find over (source, column) joined by equality.
  std::map<std::pair<int, const Column*>, std::pair<int, const Column*>> uf;
  std::pair<int, const Column*> findc(std::pair<int, const Column*> x) {
    auto it = uf.find(x);
    if (it == uf.end() || it->second == x) return x;
    auto r = findc(it->second);
    uf[x] = r;
    return r;
  }
  void unite(std::pair<int, const Column*> a, std::pair<int, const Column*> b) {
    auto ra = findc(a), rb = findc(b);
    if (ra != rb) uf[ra] = rb;
  }

  // The key column of the representative build equal to group key `e`.
  Column* rep_column(const BExpr& e) {
    if (e.src == rep_src) return e.col;
    auto cls = findc({e.src, e.col});
    for (auto& c : plan.sources[rep_src].table->cols)
      if (findc({rep_src, c.get()}) == cls) return c.get();
    fail(MTL_DEVICE_ERROR, "representative column not found");
  }

  int find_rep() {
    if (plan.group_keys.empty() || plan.sources.size() < 2) return -1;
    for (const BJoin& j : plan.joins) unite({j.ls, j.lc}, {j.rs, j.rc});
    for (int b : children[root]) {
      bool all = true;
      for (auto& k : plan.group_keys) {
        if (k->src == b) continue;
        auto cls = findc({k->src, k->col});
        bool found = false;
        for (auto& c : plan.sources[b].table->cols)
          if (findc({b, c.get()}) == cls) found = true;
        if (!found) all = false;
      }
      if (!all) continue;
      // the build key of b must be (equal to) a group key: one group per build row
      auto kcls = findc({b, up_col[b]});
      bool has_key = false;
      for (auto& k : plan.group_keys)
        if (findc({k->src, k->col}) == kcls) has_key = true;
      if (has_key) return b;
    }
    return -1;
  }

  uint64_t estimate_groups() {
    const uint64_t rows = plan.sources[root].table->rows;
    __int128 est = 1;
    for (auto& k : plan.group_keys) {
      Table& t = *plan.sources[k->src].table;
      column_distinct(ctx, t, *k->col);
      est *= (__int128)std::max<uint64_t>(1, k->col->distinct);
      if (est > (__int128)rows) break;
    }
    uint64_t e = est > (__int128)rows ? rows : (uint64_t)est;
    return std::max<uint64_t>(1, e);
  }
};

}  // namespace

std::unique_ptr<Program> compile(Ctx& ctx, const BoundPlan& plan) {
  auto P = std::make_unique<Program>();
  Compiler c{ctx, plan, *P};
  try {
    c.compile();
    c.emit_fills();
    tune_apply(ctx, *P);
  } catch (...) {
    for (void* b : P->blocks) ctx.arena.free(b);
    P->blocks.clear();
    throw;
  }
  {
    std::lock_guard<std::recursive_mutex> g(ctx.mu);
    for (Column* col : c.pinned_cols) {
      col->pins++;
      P->pinned_cols.push_back(col);
    }
  }
  return P;
}

void free_program(Ctx& ctx, Program& p) {
  for (void* b : p.blocks) ctx.arena.free(b);
  p.blocks.clear();
  std::lock_guard<std::recursive_mutex> g(ctx.mu);
  for (Column* c : p.pinned_cols) c->pins--;
  p.pinned_cols.clear();
}

// ------------------------------------------------------------ run
Program::~Program() {
  for (cudaEvent_t e : prof_ev) cudaEventDestroy(e);
  if (graph) cudaGraphExecDestroy(graph);
}

// Replays the program as one CUDA graph (captured on first use). Falls back
// to direct launches when the stream cannot be captured (the legacy default
// stream) or when per-step profiling is on. With `refresh`, the program's
// steps changed since the graph was made (new filter literals): they are
// captured again and the instantiated graph takes their parameters in place
// (cudaGraphExecUpdate), which costs far less than a new instantiation.
void run_program_graph(Ctx& ctx, Program& p, cudaStream_t s, bool refresh) {
  static const bool disabled = std::getenv("METTLE_NO_GRAPH") != nullptr;
  if (p.profile || disabled || s == nullptr || s == cudaStreamLegacy || s == cudaStreamPerThread) {
    run_program(ctx, p, s);
    return;
  }
  if (!p.graph || refresh) {
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();
      run_program(ctx, p, s);
      return;
    }
    try {
      run_program(ctx, p, s);
    } catch (...) {
      cudaStreamEndCapture(s, &g);
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      throw;
    }
    CK(cudaStreamEndCapture(s, &g));
    bool updated = false;
    if (p.graph) {
      cudaGraphExecUpdateResultInfo info;
      if (cudaGraphExecUpdate(p.graph, g, &info) == cudaSuccess) {
        updated = true;
        p.graph_updates++;
      } else {
        cudaGetLastError();
        cudaGraphExecDestroy(p.graph);
        p.graph = nullptr;
      }
    }
    cudaError_t e = updated ? cudaSuccess : cudaGraphInstantiate(&p.graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
      cudaGetLastError();
      p.graph = nullptr;
      run_program(ctx, p, s);
      return;
    }
  }
  CK(cudaGraphLaunch(p.graph, s));
}

// Shape of a bound plan: everything that decides the compiled program
// except the filter literals, which patch_literals writes into a compiled
// program of the same shape.
std::string plan_shape(const BoundPlan& p) {
  std::string o;
  auto add = [&](const std::string& x) {
    o += x;
    o += '\x1f';
  };
  for (auto& s : p.sources)
    add("S" + s.name + "@" + std::to_string((uintptr_t)s.table.get()) + "v" + std::to_string(s.table->version));
  for (auto& f : p.filters) add("F" + std::to_string(f.src) + "." + f.col->name + "#" + std::to_string(f.op));
  for (auto& j : p.joins)
    add("J" + std::to_string(j.ls) + "." + j.lc->name + "=" + std::to_string(j.rs) + "." + j.rc->name);
  add(p.is_agg ? "agg" : "rows");
  for (auto& k : p.group_keys) add("G" + k->text);
  for (auto& a : p.aggs) add("A" + std::to_string(a.fn) + "(" + (a.arg ? a.arg->text : "*") + ")");
  for (auto& x : p.outputs)
    add("O" + x.name + ":" + type_name(x.type) + ":" + (x.expr ? x.expr->text : "") + ":" +
        std::to_string(x.group_idx) + "/" + std::to_string(x.agg_idx) + (x.hidden ? "h" : ""));
  for (auto& r : p.order) add("R" + std::to_string(r.out) + (r.desc ? "d" : "a"));
  add("L" + std::to_string(p.limit) + (p.constant_only ? "c" : ""));
  return o;
}

// Builds kept from the program's previous run: a build pipeline whose
// subtree's filter literals equal those of the last run that completed, and
// that initializes no aggregate states, is left out (its scan covers no
// rows and its scratch is not cleared), so its hash table or direct-mapped
// map, presence bits and payload stay as that run left them. Enqueues on
// `s` the fill descriptors that leave kept builds' scratch alone. Returns
// the number of builds kept.
int keep_builds(Program& P, const BoundPlan& plan, cudaStream_t s) {
  const bool known = P.last_ok && P.last_lits.size() == plan.filters.size();
  uint32_t kept_src = 0;
  int kept = 0;
  for (Step& st : P.steps) {
    if (st.k != Step::PIPELINE || st.build_src < 0) continue;
    bool keep = known && st.build_keepable;
    for (size_t f = 0; keep && f < plan.filters.size(); ++f)
      if ((st.build_src_mask >> plan.filters[f].src) & 1u)
        keep = P.last_lits[f].first == plan.filters[f].ilit && P.last_lits[f].second == plan.filters[f].flit;
    st.pipe.n = keep ? 0 : st.orig_n;
    if (keep) {
      kept_src |= 1u << st.build_src;
      ++kept;
    }
  }
  if (P.fills_dev && !P.fills_host.empty()) {
    std::vector<FillSeg> send = P.fills_host;
    for (size_t i = 0; i < send.size(); ++i)
      if (P.fill_owner[i] >= 0 && ((kept_src >> P.fill_owner[i]) & 1u)) send[i].bytes = 0;
    const bool same = send.size() == P.fills_sent.size() &&
                      memcmp(send.data(), P.fills_sent.data(), send.size() * sizeof(FillSeg)) == 0;
    if (!same && (!P.fills_sent.empty() || kept)) {
      P.fills_sent = std::move(send);
      CK(cudaMemcpyAsync(P.fills_dev, P.fills_sent.data(), P.fills_sent.size() * sizeof(FillSeg),
                         cudaMemcpyHostToDevice, s));
    }
  }
  return kept;
}

// Records the literals of a run that completed (kept builds match them next time).
void mark_completed(Program& P, const BoundPlan& plan, bool ok) {
  P.last_ok = ok;
  P.last_lits.clear();
  if (!ok) return;
  for (const BFilter& f : plan.filters) P.last_lits.push_back({f.ilit, f.flit});
}

void patch_literals(Program& P, const BoundPlan& plan) {
  for (Step& s : P.steps) {
    if (s.k != Step::PIPELINE) continue;
    for (size_t j = 0; j < s.pred_filter.size() && j < (size_t)kMaxPreds; ++j) {
      const BFilter& f = plan.filters[s.pred_filter[j]];
      s.pipe.preds[j].ilit = f.ilit;
      s.pipe.preds[j].flit = f.flit;
    }
  }
}

static const char* step_kind_name(Step::Kind k) {
  switch (k) {
    case Step::MEMSET: return "memset";
    case Step::FILL: return "fill";
    case Step::PIPELINE: return "pipeline";
    case Step::COMPACT_FLAGS: return "compact_flags";
    case Step::COMPACT_READY: return "compact_ready";
    case Step::FINALIZE: return "finalize";
    case Step::ENCODE: return "encode_keys";
    case Step::RADIX: return "radix_sort";
    case Step::TOPK: return "topk";
    case Step::TOPK_FINAL: return "topk_states";
    case Step::GATHER: return "gather";
    case Step::PART_SCAN: return "part_scan";
    case Step::PART_AGG: return "part_agg";
    case Step::AGG_FEW: return "agg_few";
    case Step::MAT_SCAN: return "mat_scan";
    case Step::GATHER_OUTS: return "gather_outs";
  }
  return "step";
}

void run_program(Ctx& ctx, Program& p, cudaStream_t s) {
  (void)ctx;
  if (p.profile && p.prof_ev.size() != 2 * p.steps.size()) {
    for (cudaEvent_t e : p.prof_ev) cudaEventDestroy(e);
    p.prof_ev.assign(2 * p.steps.size(), nullptr);
    for (auto& e : p.prof_ev) CK(cudaEventCreate(&e));
  }
  for (size_t i = 0; i < p.steps.size(); ++i) {
    Step& st = p.steps[i];
    if (st.name.empty()) st.name = step_kind_name(st.k);
    if (p.profile) CK(cudaEventRecord(p.prof_ev[2 * i], s));
    switch (st.k) {
      case Step::MEMSET: CK(cudaMemsetAsync(st.ptr, st.byte, st.bytes, s)); break;
      case Step::FILL: CK(launch_fill_segments((const FillSeg*)st.ptr, st.byte, st.bytes, s)); break;
      case Step::PIPELINE: CK(launch_pipeline(st.pipe, st.n_hint, s)); break;
      case Step::COMPACT_FLAGS:
        CK(launch_compact_flags((const uint8_t*)st.flag, st.n, st.n_dev, st.out_idx, st.out_count, st.tstatus,
                                st.tcounter, 1, p.status, s));
        break;
      case Step::COMPACT_READY:
        CK(launch_compact_ready((const uint32_t*)st.flag, st.n, st.out_idx, st.out_count, st.tstatus, st.tcounter, 1,
                                p.status, s));
        break;
      case Step::FINALIZE: CK(launch_finalize(st.fin_dev, st.n_fin, st.idx, st.count, st.n_max, s)); break;
      case Step::ENCODE: CK(launch_encode_keys(st.spec, st.count, st.n_max, st.keys, st.kidx, s)); break;
      case Step::RADIX: {
        int in_tmp = 0;
        CK(launch_radix_sort(st.keys, st.kidx, st.keys_tmp, st.kidx_tmp, st.count, st.n_max, st.key_bytes, st.temp,
                             s, &in_tmp));
        break;
      }
      case Step::TOPK:
        CK(launch_topk(st.keys, st.kidx, st.count, st.n_max, st.topk, st.out_idx, st.out_count, st.temp, p.status,
                       s, st.remap));
        break;
      case Step::TOPK_FINAL:
        CK(launch_topk_final(st.tfs, st.topk, st.out_idx, st.out_count, st.temp, s, 0, st.topk_phase, st.fin_dev,
                             st.n_fin));
        break;
      case Step::GATHER: CK(launch_gather_width(st.gin, st.width, st.idx, st.count, st.n_max, st.gout, s)); break;
      case Step::GATHER_OUTS: CK(launch_gather_outs(st.go, st.n_go, st.idx, st.count, st.n_max, p.status, s)); break;
      case Step::PART_SCAN: CK(launch_part_scan(st.pipe, s)); break;
      case Step::PART_AGG: CK(launch_part_agg(st.pipe, st.n_hint, s)); break;
      case Step::AGG_FEW: CK(launch_agg_few(st.pipe, st.n_hint, s)); break;
      case Step::MAT_SCAN: CK(launch_mat_scan(st.pipe, st.n_hint, s)); break;
    }
    if (p.profile) CK(cudaEventRecord(p.prof_ev[2 * i + 1], s));
  }
}

static void check_status(uint32_t st) {
  if (!st) return;
  if (st & ST_OVERFLOW) fail(MTL_OVERFLOW, "Overflow in integer arithmetic (out of range for the result type)");
  if (st & ST_SPIN_LIMIT) fail(MTL_DEVICE_ERROR, "a device wait exceeded its iteration limit");
  if (st & ST_TABLE_FULL) fail(MTL_DEVICE_ERROR, "a device hash table ran out of slots");
  if (st & ST_DUP_BUILD_KEY) fail(MTL_DEVICE_ERROR, "duplicate key on a unique join build side");
  if (st & ST_CAPACITY) fail(MTL_DEVICE_ERROR, "a device output buffer was too small");
}

std::shared_ptr<Result> fetch_program(Ctx& ctx, Program& p, cudaStream_t s) {
  (void)ctx;
  uint32_t st = 0;
  uint64_t count = 0;
  CK(cudaMemcpyAsync(&st, p.status, 4, cudaMemcpyDeviceToHost, s));
  if (p.out_count) CK(cudaMemcpyAsync(&count, p.out_count, 8, cudaMemcpyDeviceToHost, s));
  uint64_t empty = 1;
  if (p.empty_count) CK(cudaMemcpyAsync(&empty, p.empty_count, 8, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  check_status(st);
  if (!p.out_count) count = p.fixed_count == UINT64_MAX ? 0 : p.fixed_count;
  if (count > p.n_max) count = p.n_max;
  if (p.limit >= 0 && count > (uint64_t)p.limit) count = (uint64_t)p.limit;
  auto r = std::make_shared<Result>();
  r->rows = (int64_t)count;
  for (const OutBuf& o : p.outs) {
    ResultCol c;
    c.name = o.name;
    c.type = o.type;
    c.width = o.width;
    c.data.resize(count * o.width);
    if (count) CK(cudaMemcpyAsync(c.data.data(), o.dev, count * o.width, cudaMemcpyDeviceToHost, s));
    if (o.dict) c.dict = *o.dict;
    r->cols.push_back(std::move(c));
  }
  CK(cudaStreamSynchronize(s));
  if (p.empty_count && empty == 0) {
    // ungrouped aggregate over no rows: everything but COUNT is NULL
    for (ResultCol& c : r->cols) {
      if (c.type.t == MTL_T_BIGINT && c.name.find("count") != std::string::npos) continue;
      c.valid.assign(count, 0);
    }
  }
  return r;
}

// ------------------------------------------------------------ constants
std::shared_ptr<Result> constant_result(const BoundPlan& plan) {
  auto r = std::make_shared<Result>();
  r->rows = plan.limit == 0 ? 0 : 1;
  for (const BOut& o : plan.outputs) {
    ResultCol c;
    c.name = o.name;
    c.type = o.type;
    c.width = ptype_width(storage_ptype(o.type));
    c.data.resize(r->rows * c.width);
    if (r->rows) {
      int64_t v[2] = {o.expr->lo, o.expr->hi};
      memcpy(c.data.data(), v, c.width);
    }
    r->cols.push_back(std::move(c));
  }
  return r;
}

// ------------------------------------------------------------ gpu_processing
static bool query_cache_enabled() { return std::getenv("METTLE_DISABLE_QUERY_CACHE") == nullptr; }
static const size_t kQueryCacheEntries = 32;  // src/source_cache.rs:230-233

static std::string trim(const std::string& s) {
  size_t b = s.find_first_not_of(" \t\r\n"), e = s.find_last_not_of(" \t\r\n;");
  if (b == std::string::npos) return "";
  return s.substr(b, e - b + 1);
}

std::shared_ptr<Result> processing(Ctx& ctx, const std::string& sql_in) {
  const std::string sql = trim(sql_in);
  if (sql.empty()) fail(MTL_INVALID, "gpu_processing requires a non-empty SQL string");
  {
    std::lock_guard<std::recursive_mutex> g(ctx.mu);
    ctx.last_mode.clear();
  }
  const std::string key = std::to_string(ctx.table_version) + "\x1f" + sql;
  if (query_cache_enabled()) {
    std::lock_guard<std::recursive_mutex> g(ctx.mu);
    for (auto it = ctx.qcache.begin(); it != ctx.qcache.end(); ++it) {
      if (it->first == key) {
        ctx.qcache.splice(ctx.qcache.begin(), ctx.qcache, it);
        ctx.last_mode = "cuda_hot_query_cache";
        return ctx.qcache.front().second;
      }
    }
  }
  SelectStmt st;
  try {
    st = parse_sql(sql);
  } catch (const SqlError& e) {
    fail(MTL_UNSUPPORTED, std::string("SQL outside the offloaded subset: ") + e.what());
  }
  BoundPlan plan = bind_select(ctx, st);
  std::shared_ptr<Result> r;
  std::string mode;
  if (plan.constant_only) {
    r = constant_result(plan);
    mode = "host_constant";
  } else {
    auto prog = compile(ctx, plan);
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    try {
      CK(cudaEventRecord(e0, ctx.stream));
      run_program(ctx, *prog, ctx.stream);
      CK(cudaEventRecord(e1, ctx.stream));
      r = fetch_program(ctx, *prog, ctx.stream);
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      r->device_ms = ms;
    } catch (...) {
      cudaStreamSynchronize(ctx.stream);
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      free_program(ctx, *prog);
      throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    free_program(ctx, *prog);
    mode = "cuda_generic_plan";
  }
  std::lock_guard<std::recursive_mutex> g(ctx.mu);
  ctx.last_mode = mode;
  if (query_cache_enabled() && mode != "host_constant") {
    ctx.qcache.emplace_front(key, r);
    if (plan.grouped_topk) ctx.grouped_topk_entries++;
    while (ctx.qcache.size() > kQueryCacheEntries) ctx.qcache.pop_back();
  }
  return r;
}

}  // namespace mtl
