// serve.cpp — the serving loop behind gpu_processing.
//
// The reference executes one query at a time at DuckDB bind time with
// set_max_threads(1) (src/processing.rs:59-75). Here requests are queued and
// run by `slots` workers, each with its own CUDA stream, so requests that
// arrive while others are on the GPU overlap on the device. A request is
// admitted when its device scratch fits in the processing region next to
// the requests already running (its compile step allocates from the region
// arena; on a shortfall it waits for running requests to release memory, and
// is rejected only if it cannot fit even alone). Small requests (root table
// at most kSmallRows rows) that are queued together are taken as one batch
// by one worker and launched back to back on its stream.
//
// Compiled programs stay resident between requests: a finished request's
// program (its device scratch, its descriptors and its instantiated CUDA
// graph) is kept, keyed by the shape of its plan (everything but the filter
// literals). A later request of the same shape takes the idle program,
// gets its literals patched into the pipeline descriptors, and replays the
// graph after a parameter update (cudaGraphExecUpdate): no parse-to-launch
// compilation, no descriptor uploads, no graph instantiation. Idle programs
// are evicted (least recently used first) when a new compile needs their
// memory, and the cache holds at most kMaxPrograms programs and half the
// processing region. Join builds stay resident with their program: a build
// whose subtree's literals are those of the program's last completed run
// (and that initializes no aggregate states) is not rebuilt (keep_builds).
#include <chrono>
#include <cstring>

#include "engine.h"

namespace mtl {

constexpr uint64_t kSmallRows = 1ull << 20;
constexpr int kBatchMax = 16;
constexpr size_t kMaxPrograms = 48;

// A compiled program kept for reuse by later requests of the same shape.
struct CachedProgram {
  std::string shape;
  std::unique_ptr<Program> prog;
  // the tables the program reads: kept alive while it is cached (their
  // device columns stay pinned); a table replaced since makes it stale
  std::vector<std::shared_ptr<Table>> tables;
  bool busy = false;
  uint64_t last_use = 0;
};

struct Request {
  std::string sql;
  std::mutex mu;
  std::condition_variable cv;
  bool done = false;
  int status = MTL_OK;
  std::string err;
  std::shared_ptr<Result> result;
  std::chrono::steady_clock::time_point t_submit, t_done;
  bool small = false;
  // compiled state while running
  BoundPlan plan;
  std::unique_ptr<Program> prog;    // compiled for this request
  CachedProgram* cached = nullptr;  // or borrowed from the program cache
  std::string shape;
  Program* program() { return cached ? cached->prog.get() : prog.get(); }
};

struct ServeState {
  std::mutex mu;
  std::condition_variable cv;       // queue and memory
  std::deque<Request*> queue;
  std::vector<std::thread> workers;
  std::vector<cudaStream_t> streams;
  bool stop = false;
  int slots = 4;
  std::atomic<int64_t> submitted{0}, completed{0}, rejected{0}, in_flight{0}, admitted_bytes{0}, batched{0};
  std::atomic<int64_t> reuses{0}, builds_kept{0};
  // program cache (guarded by mu)
  std::list<CachedProgram> programs;
  uint64_t program_bytes = 0;
  uint64_t tick = 0;
};

static void drop_locked(Ctx& ctx, ServeState& S, std::list<CachedProgram>::iterator it) {
  S.program_bytes -= it->prog->scratch_bytes;
  free_program(ctx, *it->prog);
  S.programs.erase(it);
}

// Frees idle cached programs that read a table replaced or dropped since.
static void evict_stale_locked(Ctx& ctx, ServeState& S) {
  std::lock_guard<std::recursive_mutex> g(ctx.mu);
  for (auto it = S.programs.begin(); it != S.programs.end();) {
    bool stale = false;
    for (auto& t : it->tables) {
      auto cur = ctx.tables.find(t->name);
      stale |= cur == ctx.tables.end() || cur->second != t;
    }
    auto nx = std::next(it);
    if (stale && !it->busy) drop_locked(ctx, S, it);
    it = nx;
  }
}

// Frees the least recently used idle cached program; false when none is idle.
static bool evict_one_locked(Ctx& ctx, ServeState& S) {
  auto victim = S.programs.end();
  for (auto it = S.programs.begin(); it != S.programs.end(); ++it)
    if (!it->busy && (victim == S.programs.end() || it->last_use < victim->last_use)) victim = it;
  if (victim == S.programs.end()) return false;
  drop_locked(ctx, S, victim);
  return true;
}

static void finish(ServeState& S, Request* r, int status, const std::string& err) {
  {
    std::lock_guard<std::mutex> g(r->mu);
    r->status = status;
    r->err = err;
    r->done = true;
    r->t_done = std::chrono::steady_clock::now();
  }
  r->cv.notify_all();
  S.completed++;
  if (status == MTL_BUDGET_EXCEEDED) S.rejected++;
}

// Binds and compiles; waits for memory when other requests hold it.
// Returns false (request finished) on error.
static bool prepare(Ctx& ctx, ServeState& S, Request* r) {
  try {
    SelectStmt st;
    try {
      st = parse_sql(r->sql);
    } catch (const SqlError& e) {
      fail(MTL_UNSUPPORTED, std::string("SQL outside the offloaded subset: ") + e.what());
    }
    r->plan = bind_select(ctx, st);
    if (r->plan.constant_only) {
      r->result = constant_result(r->plan);
      finish(S, r, MTL_OK, "");
      return false;
    }
    r->shape = plan_shape(r->plan);
    {
      std::lock_guard<std::mutex> lk(S.mu);
      evict_stale_locked(ctx, S);
      for (CachedProgram& c : S.programs)
        if (!c.busy && c.shape == r->shape) {
          c.busy = true;
          c.last_use = ++S.tick;
          r->cached = &c;
          break;
        }
    }
    if (r->cached) {
      patch_literals(*r->cached->prog, r->plan);
      S.reuses++;
      S.admitted_bytes += (int64_t)r->cached->prog->scratch_bytes;
      return true;
    }
    for (;;) {
      try {
        r->prog = compile(ctx, r->plan);
        S.admitted_bytes += (int64_t)r->prog->scratch_bytes;
        return true;
      } catch (const EngineError& e) {
        if (e.code != MTL_BUDGET_EXCEEDED) throw;
        std::unique_lock<std::mutex> lk(S.mu);
        // idle cached programs give their memory back first
        if (evict_one_locked(ctx, S)) continue;
        // Only this request holds no memory: it can never fit.
        if (S.admitted_bytes.load() == 0) throw;
        // woken when a running request releases its memory
        S.cv.wait_for(lk, std::chrono::milliseconds(500));
        if (S.stop) throw;
      }
    }
  } catch (const EngineError& e) {
    finish(S, r, e.code, e.what());
  } catch (const std::exception& e) {
    finish(S, r, MTL_DEVICE_ERROR, e.what());
  }
  return false;
}

// Returns a request's program: a borrowed one goes back to the cache idle; a
// fresh one joins the cache when there is room, else it is freed.
static void release(Ctx& ctx, ServeState& S, Request* r, bool ok) {
  std::unique_lock<std::mutex> lk(S.mu);
  if (r->cached) {
    S.admitted_bytes -= (int64_t)r->cached->prog->scratch_bytes;
    r->cached->busy = false;
    r->cached->last_use = ++S.tick;
    r->cached = nullptr;
  } else if (r->prog) {
    const uint64_t b = r->prog->scratch_bytes;
    S.admitted_bytes -= (int64_t)b;
    const uint64_t cap = ctx.budgets.processing_region_bytes / 2;
    while (ok && (S.programs.size() >= kMaxPrograms || S.program_bytes + b > cap) && evict_one_locked(ctx, S)) {
    }
    if (ok && S.programs.size() < kMaxPrograms && S.program_bytes + b <= cap) {
      S.programs.emplace_back();
      CachedProgram& c = S.programs.back();
      c.shape = r->shape;
      c.prog = std::move(r->prog);
      for (const Source& src : r->plan.sources) c.tables.push_back(src.table);
      c.last_use = ++S.tick;
      S.program_bytes += b;
    } else {
      free_program(ctx, *r->prog);
      r->prog.reset();
    }
  }
  lk.unlock();
  S.cv.notify_all();
}

// Runs a batch on the worker's stream: every request's program is enqueued
// back to back (a reused program replays its graph after a parameter
// update; a fresh one is launched directly and captured when it is reused),
// then the results are fetched in order.
static void run_batch(Ctx& ctx, ServeState& S, std::vector<Request*>& batch, cudaStream_t s) {
  std::vector<Request*> ready;
  for (Request* r : batch)
    if (prepare(ctx, S, r)) ready.push_back(r);
  if (ready.empty()) return;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  try {
    cudaEventRecord(e0, s);
    for (Request* r : ready) {
      if (r->cached) {
        S.builds_kept += keep_builds(*r->program(), r->plan, s);
        run_program_graph(ctx, *r->program(), s, /*refresh=*/true);
      } else {
        run_program(ctx, *r->program(), s);
      }
    }
    cudaEventRecord(e1, s);
    if (ready.size() > 1) S.batched++;
  } catch (const EngineError& e) {
    cudaStreamSynchronize(s);
    for (Request* r : ready) {
      if (r->program()) mark_completed(*r->program(), r->plan, false);
      release(ctx, S, r, false);
      finish(S, r, e.code, e.what());
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return;
  }
  float ms = 0;
  for (Request* r : ready) {
    try {
      r->result = fetch_program(ctx, *r->program(), s);
      if (ms == 0) cudaEventElapsedTime(&ms, e0, e1);
      r->result->device_ms = ms / (float)ready.size();
      mark_completed(*r->program(), r->plan, true);
      release(ctx, S, r, true);
      finish(S, r, MTL_OK, "");
    } catch (const EngineError& e) {
      mark_completed(*r->program(), r->plan, false);
      release(ctx, S, r, false);
      finish(S, r, e.code, e.what());
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
}

static void worker(Ctx* ctx, ServeState* S, int slot) {
  cudaSetDevice(ctx->device);
  cudaStream_t s = S->streams[slot];
  for (;;) {
    std::vector<Request*> batch;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      // (failure injection can hold the queue: nothing starts until it is cleared)
      S->cv.wait(lk, [&] {
        return S->stop || (!S->queue.empty() && ctx->inject_kind.load() != MTL_INJECT_HOLD_QUEUE);
      });
      if (S->stop && S->queue.empty()) return;
      Request* r = S->queue.front();
      S->queue.pop_front();
      batch.push_back(r);
      if (r->small) {
        while (!S->queue.empty() && (int)batch.size() < kBatchMax && S->queue.front()->small) {
          batch.push_back(S->queue.front());
          S->queue.pop_front();
        }
      }
    }
    S->in_flight += (int64_t)batch.size();
    run_batch(*ctx, *S, batch, s);
    S->in_flight -= (int64_t)batch.size();
  }
}

void serve_init(Ctx& ctx) {
  std::lock_guard<std::recursive_mutex> g(ctx.mu);
  if (ctx.serve) return;
  ctx.serve = new ServeState();
  ServeState& S = *ctx.serve;
  S.streams.resize(S.slots);
  for (int i = 0; i < S.slots; ++i) cudaStreamCreateWithFlags(&S.streams[i], cudaStreamNonBlocking);
  for (int i = 0; i < S.slots; ++i) S.workers.emplace_back(worker, &ctx, &S, i);
}

void serve_shutdown(Ctx& ctx) {
  if (!ctx.serve) return;
  ServeState& S = *ctx.serve;
  {
    std::lock_guard<std::mutex> g(S.mu);
    S.stop = true;
  }
  S.cv.notify_all();
  for (auto& t : S.workers) t.join();
  for (cudaStream_t s : S.streams) cudaStreamSynchronize(s);
  {
    std::lock_guard<std::mutex> g(S.mu);
    while (!S.programs.empty()) drop_locked(ctx, S, S.programs.begin());
  }
  for (cudaStream_t s : S.streams) cudaStreamDestroy(s);
  delete ctx.serve;
  ctx.serve = nullptr;
}

static bool is_small(Ctx& ctx, const std::string& sql) {
  try {
    SelectStmt st = parse_sql(sql);
    std::lock_guard<std::recursive_mutex> g(ctx.mu);
    uint64_t rows = 0;
    for (auto& f : st.from) {
      auto it = ctx.tables.find(f.name);
      if (it != ctx.tables.end()) rows = std::max(rows, it->second->rows);
    }
    for (auto& js : st.joins)
      for (auto& j : js) {
        auto it = ctx.tables.find(j.right.name);
        if (it != ctx.tables.end()) rows = std::max(rows, it->second->rows);
      }
    return rows <= kSmallRows;
  } catch (...) {
    return false;
  }
}

Request* serve_submit(Ctx& ctx, const std::string& sql) {
  serve_init(ctx);
  ServeState& S = *ctx.serve;
  Request* r = new Request();
  r->sql = sql;
  r->t_submit = std::chrono::steady_clock::now();
  r->small = is_small(ctx, sql);
  S.submitted++;
  {
    std::lock_guard<std::mutex> g(S.mu);
    S.queue.push_back(r);
  }
  S.cv.notify_all();
  return r;
}

// ------------------------------------------------------------ C ABI helpers
int serve_wait(Request* r, int64_t timeout_ns, std::shared_ptr<Result>* out, std::string* err) {
  std::unique_lock<std::mutex> lk(r->mu);
  if (timeout_ns < 0) {
    r->cv.wait(lk, [&] { return r->done; });
  } else if (!r->cv.wait_for(lk, std::chrono::nanoseconds(timeout_ns), [&] { return r->done; })) {
    *err = "request did not finish within the timeout";
    return MTL_TIMEOUT;
  }
  *err = r->err;
  if (r->status == MTL_OK) *out = r->result;
  return r->status;
}

double serve_latency_ms(Request* r) {
  std::lock_guard<std::mutex> g(r->mu);
  if (!r->done) return -1.0;
  return std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
}

void serve_free(Request* r) {
  {
    std::unique_lock<std::mutex> lk(r->mu);
    r->cv.wait(lk, [&] { return r->done; });
  }
  delete r;
}

void serve_stats(Ctx& ctx, mtl_serve_stats* out) {
  memset(out, 0, sizeof(*out));
  if (!ctx.serve) return;
  ServeState& S = *ctx.serve;
  out->submitted = S.submitted;
  out->completed = S.completed;
  out->rejected = S.rejected;
  out->in_flight = S.in_flight;
  {
    std::lock_guard<std::mutex> g(S.mu);
    out->queued = (int64_t)S.queue.size();
  }
  out->admitted_bytes = S.admitted_bytes;
  out->batched_launches = S.batched;
  out->program_reuses = S.reuses;
  out->builds_kept = S.builds_kept;
  {
    std::lock_guard<std::mutex> g(S.mu);
    out->cached_programs = (int64_t)S.programs.size();
    for (auto& c : S.programs) out->graph_updates += c.prog->graph_updates;
  }
}

// Wakes the workers (after a change of the queue-holding injection). The
// serving state's lock is taken without the context's (the workers take
// them in the other order).
void serve_wake(Ctx& ctx) {
  ServeState* S;
  {
    std::lock_guard<std::recursive_mutex> g(ctx.mu);
    S = ctx.serve;
  }
  if (!S) return;
  { std::lock_guard<std::mutex> q(S->mu); }
  S->cv.notify_all();
}

// Frees every idle resident program (gpu_cache_reset).
void serve_drop_programs(Ctx& ctx) {
  ServeState* S;
  {
    std::lock_guard<std::recursive_mutex> g(ctx.mu);
    S = ctx.serve;
  }
  if (!S) return;
  std::lock_guard<std::mutex> q(S->mu);
  while (evict_one_locked(ctx, *S)) {
  }
}

int serve_set_slots(Ctx& ctx, int slots) {
  if (slots < 1 || slots > 64) return MTL_INVALID;
  serve_shutdown(ctx);
  std::lock_guard<std::recursive_mutex> g(ctx.mu);
  ctx.serve = new ServeState();
  ServeState& S = *ctx.serve;
  S.slots = slots;
  S.streams.resize(slots);
  for (int i = 0; i < slots; ++i) cudaStreamCreateWithFlags(&S.streams[i], cudaStreamNonBlocking);
  for (int i = 0; i < slots; ++i) S.workers.emplace_back(worker, &ctx, &S, i);
  return MTL_OK;
}

}  // namespace mtl
