// capi.cpp — the extern "C" boundary (include/mettle_cuda.h). Every entry
// point catches engine errors, records the message for mtl_last_error and
// returns a status code; no C++ exception crosses the ABI.
#include <cmath>
#include <cstring>
#include <functional>

#include "engine.h"

struct mtl_ctx {
  mtl::Ctx c;
};
struct mtl_result {
  std::shared_ptr<mtl::Result> r;
};
struct mtl_request {
  mtl::Request* r;
};
struct mtl_stmt {
  mtl_ctx* ctx = nullptr;
  mtl::BoundPlan plan;
  std::unique_ptr<mtl::Program> prog;
  std::shared_ptr<mtl::Result> constant;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaStream_t last = nullptr;
  bool launched = false;
};

namespace mtl {
int serve_wait(Request* r, int64_t timeout_ns, std::shared_ptr<Result>* out, std::string* err);
double serve_latency_ms(Request* r);
void serve_free(Request* r);
void serve_stats(Ctx& ctx, mtl_serve_stats* out);
int serve_set_slots(Ctx& ctx, int slots);
void serve_wake(Ctx& ctx);
void serve_drop_programs(Ctx& ctx);
}  // namespace mtl

using namespace mtl;

namespace {

template <typename F>
int guarded(F&& f) {
  try {
    f();
    return MTL_OK;
  } catch (const EngineError& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const SqlError& e) {
    set_last_error(e.what());
    return MTL_UNSUPPORTED;
  } catch (const std::bad_alloc&) {
    set_last_error("host out of memory");
    return MTL_OOM;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return MTL_DEVICE_ERROR;
  }
}

#define CKA(x)                                                                                          \
  do {                                                                                                  \
    cudaError_t e_ = (x);                                                                               \
    if (e_ != cudaSuccess) fail(MTL_DEVICE_ERROR, std::string("CUDA error: ") + cudaGetErrorString(e_)); \
  } while (0)

// Human size parser of gpu_buffer_init: 1024-based units, optional
// fraction, whitespace ignored (src/config.rs:61-123).
bool parse_human_bytes(const char* raw, uint64_t* out, std::string* err) {
  if (!raw) {
    *err = "buffer sizes cannot be empty";
    return false;
  }
  std::string s(raw), num, unit;
  bool any = false;
  for (char ch : s) {
    if (isspace((unsigned char)ch)) continue;
    any = true;
    if (isdigit((unsigned char)ch) || ch == '.') {
      if (!unit.empty()) {
        *err = "invalid size literal '" + s + "'";
        return false;
      }
      num += ch;
    } else {
      unit += (char)tolower((unsigned char)ch);
    }
  }
  if (!any) {
    *err = "buffer sizes cannot be empty";
    return false;
  }
  if (num.empty()) {
    *err = "missing numeric value in '" + s + "'";
    return false;
  }
  char* end = nullptr;
  double q = strtod(num.c_str(), &end);
  if (*end || !std::isfinite(q) || q < 0 || std::count(num.begin(), num.end(), '.') > 1) {
    *err = "invalid numeric value in '" + s + "'";
    return false;
  }
  double mul;
  if (unit == "" || unit == "b") mul = 1;
  else if (unit == "k" || unit == "kb" || unit == "kib") mul = 1024.0;
  else if (unit == "m" || unit == "mb" || unit == "mib") mul = 1024.0 * 1024;
  else if (unit == "g" || unit == "gb" || unit == "gib") mul = 1024.0 * 1024 * 1024;
  else if (unit == "t" || unit == "tb" || unit == "tib") mul = 1024.0 * 1024 * 1024 * 1024;
  else {
    *err = "unsupported size unit '" + unit + "' in '" + s + "'";
    return false;
  }
  double b = q * mul;
  if (b > 1.8446744073709552e19) {
    *err = "size literal '" + s + "' overflowed u64";
    return false;
  }
  *out = (uint64_t)std::llround(b);
  return true;
}

int ptype_for(int32_t t) {
  LType lt;
  lt.t = t;
  return storage_ptype(lt);
}

}  // namespace

extern "C" {

int mtl_parse_buffer_config(const char* cache, const char* processing, const char* pinned, mtl_budgets* out,
                            char* errbuf, size_t errlen) {
  std::string err;
  mtl_budgets b{};
  auto fail_msg = [&](const std::string& m) {
    std::string full = "invalid buffer config: " + m;
    if (errbuf && errlen) {
      strncpy(errbuf, full.c_str(), errlen - 1);
      errbuf[errlen - 1] = 0;
    }
    set_last_error(full);
    return MTL_INVALID;
  };
  if (!parse_human_bytes(cache, &b.cache_region_bytes, &err)) return fail_msg(err);
  if (!parse_human_bytes(processing, &b.processing_region_bytes, &err)) return fail_msg(err);
  if (pinned) {
    if (!parse_human_bytes(pinned, &b.pinned_region_bytes, &err)) return fail_msg(err);
  } else {
    if (b.cache_region_bytes > UINT64_MAX - b.processing_region_bytes)
      return fail_msg("pinned memory default overflowed the configured budgets");
    b.pinned_region_bytes = b.cache_region_bytes + b.processing_region_bytes;
  }
  if (b.cache_region_bytes == 0) return fail_msg("gpu_buffer_init requires a non-zero cache region");
  if (b.processing_region_bytes == 0) return fail_msg("gpu_buffer_init requires a non-zero processing region");
  if (b.pinned_region_bytes == 0) return fail_msg("gpu_buffer_init requires a non-zero pinned region");
  if (out) *out = b;
  return MTL_OK;
}

int mtl_ctx_create(const mtl_budgets* budgets, int device, mtl_ctx** out) {
  if (!budgets || !out) return MTL_INVALID;
  *out = nullptr;
  mtl_ctx* h = nullptr;
  int rc = guarded([&] {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= device) {
      cudaGetLastError();
      fail(MTL_DEVICE_ERROR, "no CUDA device available");
    }
    CKA(cudaSetDevice(device));
    cudaDeviceProp prop;
    CKA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
      fail(MTL_DEVICE_ERROR, std::string("this build targets sm_100a (B200); found ") + prop.name);
    h = new mtl_ctx();
    Ctx& c = h->c;
    c.budgets = *budgets;
    c.device = device;
    c.device_name = prop.name;
    c.total_mem = prop.totalGlobalMem;
    c.sm_count = prop.multiProcessorCount;
    CKA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    CKA(cudaStreamCreateWithFlags(&c.copy_stream, cudaStreamNonBlocking));
    size_t fr = 0, tot = 0;
    CKA(cudaMemGetInfo(&fr, &tot));
    if (budgets->processing_region_bytes > fr)
      fail(MTL_BUDGET_EXCEEDED, "processing region larger than free device memory");
    c.arena.init(budgets->processing_region_bytes);
    // Keep freed column buffers reserved in the device's default pool (a
    // process-local allocator attribute) so table re-registration reuses them.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t keep = budgets->cache_region_bytes;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaGetLastError();
  });
  if (rc != MTL_OK) {
    delete h;
    return rc;
  }
  *out = h;
  return MTL_OK;
}

void mtl_ctx_destroy(mtl_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->c.device);
  delete ctx;
}

int mtl_device_info(mtl_ctx* ctx, char* name, size_t name_cap, char* backend, size_t backend_cap,
                    uint64_t* total_mem, int32_t* sm_count) {
  if (!ctx) {
    set_last_error("call gpu_buffer_init before gpu_processing");
    return MTL_NOT_INITIALIZED;
  }
  if (name && name_cap) {
    strncpy(name, ctx->c.device_name.c_str(), name_cap - 1);
    name[name_cap - 1] = 0;
  }
  if (backend && backend_cap) {
    strncpy(backend, "cuda_sm100a_hbm_column_cache", backend_cap - 1);
    backend[backend_cap - 1] = 0;
  }
  if (total_mem) *total_mem = ctx->c.total_mem;
  if (sm_count) *sm_count = ctx->c.sm_count;
  return MTL_OK;
}

const char* mtl_last_error(mtl_ctx*) { return last_error(); }

const char* mtl_last_execution_mode(mtl_ctx* ctx) {
  if (!ctx) return "";
  static thread_local std::string m;
  std::lock_guard<std::recursive_mutex> g(ctx->c.mu);
  m = ctx->c.last_mode;
  return m.c_str();
}

// ------------------------------------------------------------ tables
int mtl_table_register(mtl_ctx* ctx, const char* table, uint64_t rows, int32_t ncols, const mtl_column_desc* cols,
                       uint32_t flags, mtl_pin_summary* out) {
  if (!ctx) {
    set_last_error("call gpu_buffer_init before gpu_register_table");
    return MTL_NOT_INITIALIZED;
  }
  return guarded([&] {
    if (!table || !*table) fail(MTL_INVALID, "table name is empty");
    if (ncols < 0 || (ncols > 0 && !cols)) fail(MTL_INVALID, "bad column list");
    if (rows >= 0xFFFFFFFFull) fail(MTL_UNSUPPORTED, "tables are limited to 2^32 - 1 rows (32-bit row ids)");
    Ctx& c = ctx->c;
    cudaSetDevice(c.device);
    std::string tname = table;
    for (auto& ch : tname) ch = (char)tolower((unsigned char)ch);
    auto t = std::make_shared<Table>();
    t->name = tname;
    t->rows = rows;
    std::string skipped;
    uint64_t bytes = 0, pinned_new = 0;
    for (int i = 0; i < ncols; ++i) {
      const mtl_column_desc& d = cols[i];
      std::string cname = d.name ? d.name : "";
      for (auto& ch : cname) ch = (char)tolower((unsigned char)ch);
      LType lt;
      lt.t = d.type;
      lt.scale = d.scale;
      lt.width = d.type == MTL_T_DECIMAL ? 18 : 0;
      bool ok = d.type >= MTL_T_INTEGER && d.type <= MTL_T_VARCHAR && (rows == 0 || d.data);
      if (d.type == MTL_T_DECIMAL && (d.scale < 0 || d.scale > 18)) ok = false;
      if (!ok) {
        if (!skipped.empty()) skipped += ",";
        skipped += cname;
        continue;
      }
      auto col = std::make_unique<Column>();
      col->name = cname;
      col->type = lt;
      col->rows = rows;
      const uint64_t w = col->width(), nb = rows * w;
      if (d.type == MTL_T_VARCHAR) {
        std::vector<std::string> dict;
        for (int k = 0; k < d.dict_size; ++k) dict.push_back(d.dict[k] ? d.dict[k] : "");
        std::vector<int32_t> perm(dict.size());
        for (size_t k = 0; k < perm.size(); ++k) perm[k] = (int32_t)k;
        std::stable_sort(perm.begin(), perm.end(), [&](int32_t a, int32_t b) { return dict[a] < dict[b]; });
        bool sorted = true;
        for (size_t k = 0; k < perm.size(); ++k) sorted &= perm[k] == (int32_t)k;
        for (size_t k = 1; k < perm.size(); ++k)
          if (dict[perm[k]] == dict[perm[k - 1]]) fail(MTL_INVALID, "duplicate dictionary entry in " + cname);
        if (!sorted) {
          // remap codes onto the sorted dictionary (code order = string order)
          std::vector<int32_t> inv(dict.size());
          for (size_t k = 0; k < perm.size(); ++k) inv[perm[k]] = (int32_t)k;
          int32_t* codes = (int32_t*)malloc(std::max<uint64_t>(nb, 4));
          const int32_t* src = (const int32_t*)d.data;
          for (uint64_t r = 0; r < rows; ++r) {
            int32_t cd = src[r];
            if (cd < 0 || cd >= (int32_t)dict.size()) {
              ::free(codes);
              fail(MTL_INVALID, "dictionary code out of range in " + cname);
            }
            codes[r] = inv[cd];
          }
          std::vector<std::string> sd(dict.size());
          for (size_t k = 0; k < perm.size(); ++k) sd[k] = dict[perm[k]];
          dict.swap(sd);
          col->host_owned = codes;
          col->host_owned_pinned = false;
          col->host = codes;
        }
        col->dict = std::move(dict);
      }
      if (!col->host) {
        if (flags & MTL_PIN_BORROW) {
          col->host = d.data;
        } else {
          if (c.pinned_bytes + pinned_new + nb > c.budgets.pinned_region_bytes)
            fail(MTL_BUDGET_EXCEEDED, "table \"" + tname + "\" exceeds the pinned memory region of gpu_buffer_init");
          void* h = nullptr;
          if (nb && cudaHostAlloc(&h, nb, cudaHostAllocDefault) == cudaSuccess) {
            memcpy(h, d.data, nb);
            col->host_owned = h;
            col->host_owned_pinned = true;
            pinned_new += nb;
          } else {
            cudaGetLastError();
            h = malloc(std::max<uint64_t>(nb, 4));
            if (nb) memcpy(h, d.data, nb);
            col->host_owned = h;
          }
          col->host = col->host_owned;
        }
      }
      bytes += nb;
      t->cols.push_back(std::move(col));
    }
    {
      std::lock_guard<std::recursive_mutex> g(c.mu);
      auto it = c.tables.find(tname);
      if (it != c.tables.end()) {
        for (auto& oc : it->second->cols) {
          if (oc->dev) {
            c.dev_cache_bytes -= oc->dev_bytes;
            // freed on the stream that allocates column buffers, so the next
            // version's uploads reuse the memory in stream order instead of
            // growing the pool (a statement still using it keeps it)
            if (oc->pins == 0) {
              cudaFreeAsync(oc->dev, c.copy_stream);
              oc->dev = nullptr;
              oc->dev_bytes = 0;
            }
          }
          if (oc->host_owned_pinned) c.pinned_bytes -= oc->rows * oc->width();
        }
        c.tables.erase(it);
      }
      c.pinned_bytes += pinned_new;
      t->version = ++c.table_version;
      c.tables[tname] = t;
      // registering invalidates cached query results (src/lib.rs:48-53)
      c.qcache.clear();
      c.grouped_topk_entries = 0;
      c.last_mode.clear();
    }
    if (flags & MTL_PIN_UPLOAD)
      for (auto& col : t->cols) column_device(c, *col);
    if (out) {
      out->row_count = rows;
      out->byte_count = bytes;
      strncpy(out->skipped_columns, skipped.c_str(), sizeof(out->skipped_columns) - 1);
      out->skipped_columns[sizeof(out->skipped_columns) - 1] = 0;
    }
  });
}

int mtl_table_drop(mtl_ctx* ctx, const char* table) {
  if (!ctx) return MTL_NOT_INITIALIZED;
  return guarded([&] {
    Ctx& c = ctx->c;
    std::string tname = table ? table : "";
    for (auto& ch : tname) ch = (char)tolower((unsigned char)ch);
    std::lock_guard<std::recursive_mutex> g(c.mu);
    auto it = c.tables.find(tname);
    if (it == c.tables.end()) fail(MTL_INVALID, "table \"" + tname + "\" is not registered");
    for (auto& oc : it->second->cols) {
      if (oc->dev) c.dev_cache_bytes -= oc->dev_bytes;
      if (oc->host_owned_pinned) c.pinned_bytes -= oc->rows * oc->width();
    }
    c.tables.erase(it);
    ++c.table_version;
    c.qcache.clear();
    c.grouped_topk_entries = 0;
  });
}

int mtl_column_evict(mtl_ctx* ctx, const char* table, const char* column) {
  if (!ctx) return MTL_NOT_INITIALIZED;
  return guarded([&] {
    Ctx& c = ctx->c;
    std::lock_guard<std::recursive_mutex> g(c.mu);
    auto it = c.tables.find(table ? table : "");
    if (it == c.tables.end()) fail(MTL_INVALID, "table is not registered");
    Column* col = it->second->find(column ? column : "");
    if (!col) fail(MTL_INVALID, "column not found");
    if (col->pins) fail(MTL_INVALID, "column is in use by a prepared statement");
    if (col->dev) {
      cudaFreeAsync(col->dev, 0);
      c.dev_cache_bytes -= col->dev_bytes;
      col->dev = nullptr;
      col->dev_bytes = 0;
      c.cc.evictions++;
    }
  });
}

// ------------------------------------------------------------ queries
int mtl_processing(mtl_ctx* ctx, const char* sql, mtl_result** out) {
  if (out) *out = nullptr;
  if (!ctx) {
    set_last_error("call gpu_buffer_init before gpu_processing");
    return MTL_NOT_INITIALIZED;
  }
  return guarded([&] {
    cudaSetDevice(ctx->c.device);
    auto r = processing(ctx->c, sql ? sql : "");
    if (out) *out = new mtl_result{r};
  });
}

int mtl_stmt_prepare(mtl_ctx* ctx, const char* sql, mtl_stmt** out) {
  if (out) *out = nullptr;
  if (!ctx) {
    set_last_error("call gpu_buffer_init before gpu_processing");
    return MTL_NOT_INITIALIZED;
  }
  mtl_stmt* st = new mtl_stmt();
  st->ctx = ctx;
  int rc = guarded([&] {
    cudaSetDevice(ctx->c.device);
    std::string s = sql ? sql : "";
    if (s.find_first_not_of(" \t\r\n;") == std::string::npos)
      fail(MTL_INVALID, "gpu_processing requires a non-empty SQL string");
    SelectStmt ast;
    try {
      ast = parse_sql(s);
    } catch (const SqlError& e) {
      fail(MTL_UNSUPPORTED, std::string("SQL outside the offloaded subset: ") + e.what());
    }
    st->plan = bind_select(ctx->c, ast);
    if (st->plan.constant_only) st->constant = constant_result(st->plan);
    else st->prog = compile(ctx->c, st->plan);
    CKA(cudaEventCreate(&st->e0));
    CKA(cudaEventCreate(&st->e1));
  });
  if (rc != MTL_OK) {
    mtl_stmt_free(st);
    return rc;
  }
  *out = st;
  return MTL_OK;
}

int mtl_stmt_launch(mtl_stmt* st, void* stream) {
  if (!st) return MTL_INVALID;
  return guarded([&] {
    cudaStream_t s = stream ? (cudaStream_t)stream : st->ctx->c.stream;
    st->last = s;
    st->launched = true;
    if (st->constant) return;
    CKA(cudaEventRecord(st->e0, s));
    run_program_graph(st->ctx->c, *st->prog, s);
    CKA(cudaEventRecord(st->e1, s));
  });
}

int mtl_stmt_fetch(mtl_stmt* st, mtl_result** out) {
  if (out) *out = nullptr;
  if (!st) return MTL_INVALID;
  return guarded([&] {
    if (!st->launched) fail(MTL_INVALID, "statement was not launched");
    std::shared_ptr<Result> r;
    if (st->constant) {
      r = st->constant;
    } else {
      r = fetch_program(st->ctx->c, *st->prog, st->last);
      float ms = 0;
      cudaEventElapsedTime(&ms, st->e0, st->e1);
      r->device_ms = ms;
    }
    if (out) *out = new mtl_result{r};
  });
}

double mtl_stmt_device_ms(mtl_stmt* st) {
  if (!st || !st->launched || st->constant) return 0.0;
  float ms = 0;
  if (cudaEventSynchronize(st->e1) != cudaSuccess) return -1.0;
  cudaEventElapsedTime(&ms, st->e0, st->e1);
  return ms;
}

int32_t mtl_stmt_kernel_count(mtl_stmt* st) { return st && st->prog ? st->prog->kernels : 0; }

int mtl_stmt_set_profiling(mtl_stmt* st, int32_t on) {
  if (!st) return MTL_INVALID;
  if (st->prog) st->prog->profile = on != 0;
  return MTL_OK;
}

int32_t mtl_stmt_step_count(mtl_stmt* st) { return st && st->prog ? (int32_t)st->prog->steps.size() : 0; }

const char* mtl_stmt_step_name(mtl_stmt* st, int32_t i) {
  if (!st || !st->prog || i < 0 || i >= (int32_t)st->prog->steps.size()) return nullptr;
  return st->prog->steps[i].name.c_str();
}

double mtl_stmt_step_ms(mtl_stmt* st, int32_t i) {
  if (!st || !st->prog || !st->prog->profile || i < 0 || 2 * (size_t)i + 1 >= st->prog->prof_ev.size()) return -1.0;
  cudaEvent_t a = st->prog->prof_ev[2 * i], b = st->prog->prof_ev[2 * i + 1];
  if (cudaEventSynchronize(b) != cudaSuccess) return -1.0;
  float ms = 0;
  if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) return -1.0;
  return ms;
}

void mtl_stmt_free(mtl_stmt* st) {
  if (!st) return;
  if (st->last) cudaStreamSynchronize(st->last);
  if (st->prog) free_program(st->ctx->c, *st->prog);
  if (st->e0) cudaEventDestroy(st->e0);
  if (st->e1) cudaEventDestroy(st->e1);
  delete st;
}

int mtl_query_submit(mtl_ctx* ctx, const char* sql, mtl_request** out) {
  if (out) *out = nullptr;
  if (!ctx) {
    set_last_error("call gpu_buffer_init before gpu_processing");
    return MTL_NOT_INITIALIZED;
  }
  return guarded([&] {
    std::string s = sql ? sql : "";
    if (s.find_first_not_of(" \t\r\n;") == std::string::npos)
      fail(MTL_INVALID, "gpu_processing requires a non-empty SQL string");
    Request* r = serve_submit(ctx->c, s);
    *out = new mtl_request{r};
  });
}

int mtl_request_wait(mtl_request* req, int64_t timeout_ns, mtl_result** out) {
  if (out) *out = nullptr;
  if (!req) return MTL_INVALID;
  std::shared_ptr<Result> r;
  std::string err;
  int rc = serve_wait(req->r, timeout_ns, &r, &err);
  if (rc != MTL_OK) {
    set_last_error(err);
    return rc;
  }
  if (out) *out = new mtl_result{r};
  return MTL_OK;
}

double mtl_request_latency_ms(mtl_request* req) { return req ? serve_latency_ms(req->r) : -1.0; }

void mtl_request_free(mtl_request* req) {
  if (!req) return;
  serve_free(req->r);
  delete req;
}

// ------------------------------------------------------------ results
int64_t mtl_result_rows(const mtl_result* r) { return r ? r->r->rows : 0; }
int32_t mtl_result_columns(const mtl_result* r) { return r ? (int32_t)r->r->cols.size() : 0; }
const char* mtl_result_column_name(const mtl_result* r, int32_t col) {
  if (!r || col < 0 || col >= (int32_t)r->r->cols.size()) return nullptr;
  return r->r->cols[col].name.c_str();
}
int32_t mtl_result_column_type(const mtl_result* r, int32_t col, int32_t* scale) {
  if (!r || col < 0 || col >= (int32_t)r->r->cols.size()) return 0;
  if (scale) *scale = r->r->cols[col].type.scale;
  return r->r->cols[col].type.t;
}
const void* mtl_result_column_data(const mtl_result* r, int32_t col) {
  if (!r || col < 0 || col >= (int32_t)r->r->cols.size()) return nullptr;
  return r->r->cols[col].data.data();
}
const uint8_t* mtl_result_column_valid(const mtl_result* r, int32_t col) {
  if (!r || col < 0 || col >= (int32_t)r->r->cols.size()) return nullptr;
  const auto& v = r->r->cols[col].valid;
  return v.empty() ? nullptr : v.data();
}
const char* mtl_result_dict(const mtl_result* r, int32_t col, int32_t code) {
  if (!r || col < 0 || col >= (int32_t)r->r->cols.size()) return nullptr;
  const auto& d = r->r->cols[col].dict;
  if (code < 0 || code >= (int32_t)d.size()) return nullptr;
  return d[code].c_str();
}
double mtl_result_device_ms(const mtl_result* r) { return r ? r->r->device_ms : 0.0; }
void mtl_result_free(mtl_result* r) { delete r; }

// ------------------------------------------------------------ caches
int mtl_cache_stats_get(mtl_ctx* ctx, mtl_cache_stats* out) {
  if (!ctx || !out) return MTL_INVALID;
  Ctx& c = ctx->c;
  std::lock_guard<std::recursive_mutex> g(c.mu);
  memset(out, 0, sizeof(*out));
  int64_t entries = 0;
  for (auto& t : c.tables)
    for (auto& col : t.second->cols)
      if (col->dev) ++entries;
  out->entries = entries;
  out->cached_bytes = (int64_t)c.dev_cache_bytes;
  out->hits = c.cc.hits;
  out->misses = c.cc.misses;
  out->evictions = c.cc.evictions;
  out->bypasses = c.cc.bypasses;
  out->input_entries = entries;
  out->input_cached_bytes = (int64_t)c.dev_cache_bytes;
  out->grouped_topk_entries = c.grouped_topk_entries;
  int64_t qb = 0, gb = 0;
  for (auto& e : c.qcache) qb += (int64_t)e.second->approx_bytes();
  out->grouped_topk_bytes = c.grouped_topk_entries ? gb : 0;
  out->query_result_entries = (int64_t)c.qcache.size();
  out->query_result_bytes = qb;
  return MTL_OK;
}

int mtl_cache_reset(mtl_ctx* ctx) {
  if (!ctx) return MTL_NOT_INITIALIZED;
  return guarded([&] {
    Ctx& c = ctx->c;
    serve_drop_programs(c);  // resident compiled programs release their columns
    std::lock_guard<std::recursive_mutex> g(c.mu);
    c.qcache.clear();
    c.grouped_topk_entries = 0;
    c.last_mode.clear();
    for (auto& t : c.tables)
      for (auto& col : t.second->cols)
        if (col->dev && col->pins == 0) {
          cudaFreeAsync(col->dev, 0);
          c.dev_cache_bytes -= col->dev_bytes;
          col->dev = nullptr;
          col->dev_bytes = 0;
        }
  });
}

// ------------------------------------------------------------ rewrite + hooks
namespace {

std::string print(const AstP& a);

bool numeric_lit(const AstP& a) {
  if (a->k == Ast::INT || a->k == Ast::DEC) return true;
  if (a->k == Ast::NEG) return numeric_lit(a->a[0]);
  return false;
}

std::string print_rewritten(const AstP& a) {
  if (a->k == Ast::BIN && (a->op == '+' || a->op == '*')) {
    const AstP &l = a->a[0], &r = a->a[1];
    const char* fn = a->op == '+' ? "gpu_add_scalar" : "gpu_mul_scalar";
    if (l->k == Ast::COL && numeric_lit(r)) return std::string(fn) + "(" + print(l) + ", " + print(r) + ")";
    if (r->k == Ast::COL && numeric_lit(l)) return std::string(fn) + "(" + print(r) + ", " + print(l) + ")";
  }
  if (a->k == Ast::CMP && a->cmp <= C_GE) {
    static const char* fns[] = {"gpu_eq_scalar", "gpu_lt_scalar", "gpu_le_scalar", "gpu_gt_scalar", "gpu_ge_scalar"};
    static const int flip[] = {C_EQ, C_GT, C_GE, C_LT, C_LE};
    const AstP &l = a->a[0], &r = a->a[1];
    if (l->k == Ast::COL && numeric_lit(r)) return std::string(fns[a->cmp]) + "(" + print(l) + ", " + print(r) + ")";
    if (r->k == Ast::COL && numeric_lit(l))
      return std::string(fns[flip[a->cmp]]) + "(" + print(r) + ", " + print(l) + ")";
  }
  return "";
}

std::string quote_str(const std::string& s) {
  std::string o = "'";
  for (char c : s) {
    if (c == '\'') o += "''";
    else o += c;
  }
  return o + "'";
}

std::string print(const AstP& a) {
  std::string rw = print_rewritten(a);
  if (!rw.empty()) return rw;
  switch (a->k) {
    case Ast::COL: return a->table.empty() ? a->name : a->table + "." + a->name;
    case Ast::INT:
    case Ast::DEC: return a->name;
    case Ast::STR: return quote_str(a->name);
    case Ast::DATE: return "DATE " + quote_str(a->name);
    case Ast::TS: return "TIMESTAMP " + quote_str(a->name);
    case Ast::STAR: return "*";
    case Ast::NEG: return "-" + print(a->a[0]);
    case Ast::BIN: return "(" + print(a->a[0]) + " " + std::string(1, a->op == '|' ? '|' : a->op) + " " + print(a->a[1]) + ")";
    case Ast::CMP: {
      static const char* ops[] = {"=", "<", "<=", ">", ">=", "<>"};
      return print(a->a[0]) + " " + ops[a->cmp] + " " + print(a->a[1]);
    }
    case Ast::AND: return print(a->a[0]) + " AND " + print(a->a[1]);
    case Ast::OR: return "(" + print(a->a[0]) + " OR " + print(a->a[1]) + ")";
    case Ast::NOT: return "NOT (" + print(a->a[0]) + ")";
    case Ast::BETWEEN:
      return print(a->a[0]) + (a->negated ? " NOT" : "") + " BETWEEN " + print(a->a[1]) + " AND " + print(a->a[2]);
    case Ast::FUNC: {
      std::string s = a->name + "(" + (a->distinct ? "DISTINCT " : "");
      for (size_t i = 0; i < a->a.size(); ++i) s += (i ? ", " : "") + print(a->a[i]);
      return s + ")";
    }
    default: return a->text;
  }
}

std::string rewrite(const SelectStmt& st) {
  if (st.has_cte || st.has_set_op || st.has_subquery) fail(MTL_UNSUPPORTED, "cannot rewrite this statement shape");
  std::string s = "SELECT ";
  if (st.distinct) s += "DISTINCT ";
  for (size_t i = 0; i < st.items.size(); ++i) {
    const SelectItem& it = st.items[i];
    if (i) s += ", ";
    if (it.star) {
      s += "*";
      continue;
    }
    s += print(it.expr);
    // keep the original output name of a rewritten expression
    std::string alias = it.alias;
    if (alias.empty() && it.expr->k != Ast::COL && !print_rewritten(it.expr).empty()) alias = it.expr->text;
    if (!alias.empty()) s += " AS \"" + alias + "\"";
  }
  if (!st.from.empty()) {
    s += " FROM ";
    for (size_t f = 0; f < st.from.size(); ++f) {
      if (f) s += ", ";
      s += st.from[f].name + (st.from[f].alias.empty() ? "" : " " + st.from[f].alias);
      for (const JoinClause& j : st.joins[f]) {
        s += j.kind == "inner" ? " JOIN " : " " + j.kind + " JOIN ";
        s += j.right.name + (j.right.alias.empty() ? "" : " " + j.right.alias);
        if (j.on) s += " ON " + print(j.on);
      }
    }
  }
  if (st.where) s += " WHERE " + print(st.where);
  if (!st.group_by.empty()) {
    s += " GROUP BY ";
    for (size_t i = 0; i < st.group_by.size(); ++i) s += (i ? ", " : "") + print(st.group_by[i]);
  }
  if (!st.order_by.empty()) {
    s += " ORDER BY ";
    for (size_t i = 0; i < st.order_by.size(); ++i)
      s += (i ? ", " : "") + print(st.order_by[i].expr) + (st.order_by[i].desc ? " DESC" : "");
  }
  if (st.limit >= 0) s += " LIMIT " + std::to_string(st.limit);
  return s;
}

}  // namespace

int mtl_rewrite_query(mtl_ctx* ctx, const char* sql, char* out, size_t cap) {
  (void)ctx;
  return guarded([&] {
    SelectStmt st;
    try {
      st = parse_sql(sql ? sql : "");
    } catch (const SqlError& e) {
      fail(MTL_UNSUPPORTED, e.what());
    }
    std::string r = rewrite(st);
    if (!out || cap <= r.size()) fail(MTL_INVALID, "output buffer too small for the rewritten query");
    memcpy(out, r.c_str(), r.size() + 1);
  });
}

static int hook(mtl_ctx* ctx, bool cmp, int32_t op, int32_t type, const void* in, uint64_t n, int64_t ilit,
                double flit, void* out) {
  if (!ctx) {
    set_last_error("call gpu_buffer_init before gpu_processing");
    return MTL_NOT_INITIALIZED;
  }
  return guarded([&] {
    Ctx& c = ctx->c;
    cudaSetDevice(c.device);
    if (n && (!in || !out)) fail(MTL_INVALID, "null buffer");
    if (cmp ? (op < 0 || op > C_GE) : (op != MTL_HOOK_ADD && op != MTL_HOOK_MUL)) fail(MTL_INVALID, "bad op");
    int pt = ptype_for(type);
    if (type == MTL_T_VARCHAR || type == MTL_T_HUGEINT || type == MTL_T_BOOLEAN || pt == P_NONE)
      fail(MTL_UNSUPPORTED, "scalar hook on " + type_name(LType{type, 0, 0}));
    if (!cmp && (type == MTL_T_TIMESTAMP || (type == MTL_T_DATE && op == MTL_HOOK_MUL)))
      fail(MTL_UNSUPPORTED, "scalar arithmetic on this type");
    if (n == 0) return;
    const uint64_t w = ptype_width(pt), ob = cmp ? n : n * w;
    void* din = c.arena.alloc(n * w);
    void* dout = c.arena.alloc(ob);
    uint32_t* dst = (uint32_t*)c.arena.alloc(8);
    if (!din || !dout || !dst) {
      c.arena.free(din);
      c.arena.free(dout);
      c.arena.free(dst);
      fail(MTL_BUDGET_EXCEEDED, "scalar hook input exceeds the processing region");
    }
    uint32_t st = 0;
    try {
      CKA(cudaMemsetAsync(dst, 0, 8, c.stream));
      CKA(cudaMemcpyAsync(din, in, n * w, cudaMemcpyHostToDevice, c.stream));
      if (cmp) CKA(launch_scalar_compare(op, pt, din, n, ilit, flit, (uint8_t*)dout, c.stream));
      else CKA(launch_scalar_arith(op, pt, din, n, ilit, flit, dout, dst, c.stream));
      CKA(cudaMemcpyAsync(out, dout, ob, cudaMemcpyDeviceToHost, c.stream));
      CKA(cudaMemcpyAsync(&st, dst, 4, cudaMemcpyDeviceToHost, c.stream));
      CKA(cudaStreamSynchronize(c.stream));
    } catch (...) {
      cudaStreamSynchronize(c.stream);
      c.arena.free(din);
      c.arena.free(dout);
      c.arena.free(dst);
      throw;
    }
    c.arena.free(din);
    c.arena.free(dout);
    c.arena.free(dst);
    if (st & ST_OVERFLOW) fail(MTL_OVERFLOW, "Overflow in scalar hook arithmetic");
  });
}

int mtl_scalar_arith(mtl_ctx* ctx, int32_t op, int32_t type, const void* in, uint64_t n, int64_t ilit, double flit,
                     void* out) {
  return hook(ctx, false, op, type, in, n, ilit, flit, out);
}

int mtl_scalar_compare(mtl_ctx* ctx, int32_t op, int32_t type, const void* in, uint64_t n, int64_t ilit, double flit,
                       uint8_t* out) {
  return hook(ctx, true, op, type, in, n, ilit, flit, out);
}

int mtl_serve_stats_get(mtl_ctx* ctx, mtl_serve_stats* out) {
  if (!ctx || !out) return MTL_INVALID;
  serve_stats(ctx->c, out);
  return MTL_OK;
}

int mtl_serve_set_slots(mtl_ctx* ctx, int32_t slots) {
  if (!ctx) return MTL_NOT_INITIALIZED;
  return serve_set_slots(ctx->c, slots);
}

int mtl_autotune(mtl_ctx* ctx, const char* sql, int32_t reps, char* report, size_t report_cap) {
  if (!ctx) {
    set_last_error("call gpu_buffer_init before gpu_processing");
    return MTL_NOT_INITIALIZED;
  }
  return guarded([&] {
    cudaSetDevice(ctx->c.device);
    std::string s = sql ? sql : "";
    if (s.find_first_not_of(" \t\r\n;") == std::string::npos)
      fail(MTL_INVALID, "gpu_processing requires a non-empty SQL string");
    SelectStmt ast;
    try {
      ast = parse_sql(s);
    } catch (const SqlError& e) {
      fail(MTL_UNSUPPORTED, std::string("SQL outside the offloaded subset: ") + e.what());
    }
    BoundPlan plan = bind_select(ctx->c, ast);
    if (plan.constant_only) fail(MTL_INVALID, "a constant query has nothing to tune");
    const std::string r = autotune(ctx->c, plan, reps);
    if (report && report_cap) {
      const size_t n = std::min(report_cap - 1, r.size());
      memcpy(report, r.data(), n);
      report[n] = 0;
    }
  });
}

int mtl_debug_inject(mtl_ctx* ctx, int32_t what, uint32_t arg) {
  if (!ctx) return MTL_NOT_INITIALIZED;
  if (what != MTL_INJECT_NONE && what != MTL_INJECT_LOOKBACK_STALL && what != MTL_INJECT_HOLD_QUEUE) {
    set_last_error("mtl_debug_inject: unknown injection");
    return MTL_INVALID;
  }
  Ctx& c = ctx->c;
  c.inject_arg.store(arg);
  c.inject_kind.store(what);
  serve_wake(c);  // a held queue starts again once cleared
  return MTL_OK;
}

}  // extern "C"
