// tune.cpp — the launch-shape autotuner.
//
// The reference fixes its launch shapes: one thread per row and a constant
// threadgroup size (src/metal/shaders/compiler.rs:69-91), a hash capacity of
// the next power of two above twice the build rows
// (src/plan/executor/join_plan.rs:300-303). Here three knobs are measured on
// the device and the best choice is kept per device:
//   * CTAs per SM of a pipeline's grid (the pipelines are persistent
//     grid-stride kernels; fewer resident CTAs can cut contention on shared
//     tables and L2 lines, more hide more latency);
//   * the tile group: consecutive 256-row warp-tiles a warp takes per step of
//     its stride (the rows a warp covers between strides, so the tile each
//     warp streams is 256, 512 or 1024 rows);
//   * the hash load factor: the capacity of open-addressing join tables and
//     one-key aggregate tables relative to their rows (fewer probes against
//     more bytes to clear and to miss in L2).
// A choice is keyed by the kind of step and the size class of its input
// (log2 of its rows) plus what shapes its per-row work (bytes streamed per
// row, probes), so one tuning run serves every query of that shape and size.
// mtl_autotune runs a query's program once per candidate, times the step
// with CUDA events (the program's profiling mode) and keeps the fastest;
// the table is written to a file per device and read back by every context
// on that device.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>

#include <sys/stat.h>

#include "engine.h"

namespace mtl {

static void mkdir_one(const std::string& d) { ::mkdir(d.c_str(), 0755); }

static std::string sanitize(const std::string& s) {
  std::string o;
  for (char c : s) o += (isalnum((unsigned char)c) ? c : '_');
  return o;
}

std::string tune_file_path(const Ctx& ctx) {
  if (const char* f = std::getenv("METTLE_TUNE_FILE")) return f;
  std::string dir;
  if (const char* d = std::getenv("METTLE_TUNE_DIR")) dir = d;
  else if (const char* h = std::getenv("HOME")) dir = std::string(h) + "/.cache/mettle_b200";
  else dir = "/tmp/mettle_b200";
  return dir + "/autotune_" + sanitize(ctx.device_name) + "_sm" + std::to_string(ctx.sm_count) + ".txt";
}

static int log2_class(uint64_t n) {
  int b = 0;
  while ((1ull << b) < n && b < 63) ++b;
  return b;
}

std::string tune_key_pipeline(const Step& s) {
  const PipeDesc& d = s.pipe;
  uint32_t stream = 0;
  for (int i = 0; i < d.n_stream && i < kMaxStream; ++i) stream += (uint32_t)ptype_width(d.cols[d.stream_cols[i]].ptype);
  // the step name without the table: "pipeline:<sink>"
  std::string kind = s.name.substr(0, s.name.rfind(':'));
  std::ostringstream k;
  k << kind << "/n" << log2_class(s.n_hint) << "/s" << stream << "/p" << d.n_probes << "/a" << d.n_aggs;
  return k.str();
}

std::string tune_key_load(const char* what, uint64_t rows) {
  return std::string(what) + "/n" + std::to_string(log2_class(rows));
}

// ------------------------------------------------------------ the table
static void tune_load_locked(Ctx& ctx) {
  if (ctx.tune_loaded) return;
  ctx.tune_loaded = true;
  std::ifstream f(tune_file_path(ctx));
  std::string key;
  double a, b;
  while (f >> key >> a >> b) ctx.tune[key] = {a, b};
}

static void tune_save_locked(Ctx& ctx) {
  const std::string path = tune_file_path(ctx);
  const size_t slash = path.rfind('/');
  if (slash != std::string::npos) {
    const std::string dir = path.substr(0, slash);
    // create the directory one level at a time (existing levels are fine)
    for (size_t i = 1; i <= dir.size(); ++i)
      if (i == dir.size() || dir[i] == '/') mkdir_one(dir.substr(0, i));
  }
  std::ofstream f(path + ".tmp");
  for (auto& e : ctx.tune) f << e.first << " " << e.second.first << " " << e.second.second << "\n";
  f.close();
  std::rename((path + ".tmp").c_str(), path.c_str());
}

bool tune_lookup(Ctx& ctx, const std::string& key, double* a, double* b) {
  std::lock_guard<std::recursive_mutex> g(ctx.mu);
  tune_load_locked(ctx);
  auto it = ctx.tune.find(key);
  if (it == ctx.tune.end()) return false;
  *a = it->second.first;
  *b = it->second.second;
  return true;
}

static void tune_store(Ctx& ctx, const std::string& key, double a, double b) {
  std::lock_guard<std::recursive_mutex> g(ctx.mu);
  tune_load_locked(ctx);
  ctx.tune[key] = {a, b};
}

// A pipeline step's launch shape: CTAs per SM (0: as many as fit) and the
// rows a warp takes per step. Order-preserving compaction runs 1024-row CTA
// tiles or 256-row warp tiles; the other sinks take groups of 256-row tiles.
static void set_shape(Step& s, int grid_per_sm, int tile_rows) {
  s.pipe.grid_per_sm = grid_per_sm;
  if (s.pipe.sink == SK_MATERIALIZE) {
    s.pipe.mat_warp_tiles = tile_rows == 256 ? 1 : 0;
  } else {
    const int g = tile_rows / 256;
    s.pipe.tile_group = g == 2 || g == 4 ? g : 1;
  }
}

static std::vector<int> tile_candidates(const Step& s) {
  if (s.pipe.sink == SK_MATERIALIZE) return {1024, 256};
  return {256, 512, 1024};
}

// Applies the table's launch shapes to a compiled program's pipelines. The
// two partition passes must cover the same tiles per CTA, so they keep the
// default shape.
void tune_apply(Ctx& ctx, Program& p) {
  for (Step& s : p.steps) {
    if (s.k != Step::PIPELINE) continue;
    if (s.pipe.sink == SK_PART_COUNT || s.pipe.sink == SK_PART_SCATTER) continue;
    double a = 0, b = 0;
    if (tune_lookup(ctx, tune_key_pipeline(s), &a, &b)) set_shape(s, (int)a, (int)b);
  }
}

// A load factor forced by the tuning run of this thread (0: none).
static thread_local double t_force_load_factor = 0;

double tune_load_factor(Ctx& ctx, const char* what, uint64_t rows) {
  if (t_force_load_factor > 0) return t_force_load_factor;
  double a = 0, b = 0;
  if (tune_lookup(ctx, tune_key_load(what, rows), &a, &b) && a >= 1.25 && a <= 8) return a;
  return 2.0;
}

std::string tune_key_agg(uint64_t groups, uint64_t rows) {
  return "agg_one_key/g" + std::to_string(log2_class(groups)) + "/n" + std::to_string(log2_class(rows));
}

// A strategy forced by the tuning run of this thread (0: none).
static thread_local int t_force_agg_strategy = 0;

int tune_agg_strategy(Ctx& ctx, uint64_t groups, uint64_t rows) {
  if (t_force_agg_strategy) return t_force_agg_strategy;
  double a = 0, b = 0;
  if (tune_lookup(ctx, tune_key_agg(groups, rows), &a, &b) && (a == 1 || a == 2)) return (int)a;
  return 0;
}

std::string tune_key_mat(uint64_t rows) { return "materialize_strategy/n" + std::to_string(log2_class(rows)); }

static thread_local int t_force_mat_strategy = 0;

int tune_mat_strategy(Ctx& ctx, uint64_t rows) {
  if (t_force_mat_strategy) return t_force_mat_strategy;
  double a = 0, b = 0;
  if (tune_lookup(ctx, tune_key_mat(rows), &a, &b) && (a == 1 || a == 2)) return (int)a;
  return 0;
}

// ------------------------------------------------------------ tuning runs
namespace {

// Device ms of each step of one run (profiling mode), the minimum over `reps`.
std::vector<double> run_steps(Ctx& ctx, Program& p, cudaStream_t s, int reps) {
  std::vector<double> best(p.steps.size(), 1e30);
  p.profile = true;
  for (int r = 0; r < reps; ++r) {
    run_program(ctx, p, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) fail(MTL_DEVICE_ERROR, "autotune run failed");
    for (size_t i = 0; i < p.steps.size(); ++i) {
      float ms = 0;
      cudaEventElapsedTime(&ms, p.prof_ev[2 * i], p.prof_ev[2 * i + 1]);
      best[i] = std::min(best[i], (double)ms);
    }
  }
  p.profile = false;
  return best;
}

double total(const std::vector<double>& v) {
  double t = 0;
  for (double x : v) t += x;
  return t;
}

}  // namespace

std::string autotune(Ctx& ctx, const BoundPlan& plan, int reps) {
  std::ostringstream rep;
  cudaStream_t s = ctx.stream;
  reps = std::max(1, std::min(reps, 20));
  // hash load factor first: it changes the program (capacities)
  bool has_hash = false;
  std::vector<std::pair<std::string, uint64_t>> load_keys;
  {
    auto probe = compile(ctx, plan);
    for (const Step& st : probe->steps) {
      if (st.k != Step::PIPELINE) continue;
      for (int b = 0; b < st.pipe.n_builds; ++b)
        if (st.pipe.builds[b].kind == B_HASH) has_hash = true;
      if (st.pipe.table.cas) has_hash = true;
    }
    load_keys = probe->load_keys;
    free_program(ctx, *probe);
  }
  if (has_hash && !load_keys.empty()) {
    const double cands[] = {1.5, 2.0, 3.0};
    double best_t = 1e30, best_lf = 2.0;
    for (double lf : cands) {
      t_force_load_factor = lf;
      std::unique_ptr<Program> p;
      try {
        p = compile(ctx, plan);
      } catch (...) {
        t_force_load_factor = 0;
        throw;
      }
      t_force_load_factor = 0;
      double t = 1e30;
      try {
        t = total(run_steps(ctx, *p, s, reps));
      } catch (...) {
        free_program(ctx, *p);
        throw;
      }
      free_program(ctx, *p);
      rep << "load_factor " << lf << ": " << t << " ms\n";
      if (t < best_t) {
        best_t = t;
        best_lf = lf;
      }
    }
    for (auto& k : load_keys) tune_store(ctx, k.first, best_lf, 0);
    rep << "chose load factor " << best_lf << "\n";
  }
  // one-key aggregate over few groups: one pass into shared-memory tables
  // against the partitioned passes; order-preserving compaction: one pass
  // with a look-back against two passes
  std::string agg_key, mat_key;
  {
    auto probe = compile(ctx, plan);
    agg_key = probe->agg_strategy_key;
    mat_key = probe->mat_strategy_key;
    free_program(ctx, *probe);
  }
  if (!mat_key.empty()) {
    double best_t = 1e30;
    int best = 2;
    for (int strat : {2, 1}) {
      t_force_mat_strategy = strat;
      std::unique_ptr<Program> p;
      try {
        p = compile(ctx, plan);
      } catch (...) {
        t_force_mat_strategy = 0;
        throw;
      }
      t_force_mat_strategy = 0;
      double t = 1e30;
      try {
        t = total(run_steps(ctx, *p, s, reps));
      } catch (...) {
        free_program(ctx, *p);
        throw;
      }
      free_program(ctx, *p);
      rep << "compaction " << (strat == 1 ? "in one pass (look-back)" : "in two passes (count, scan, write)") << ": "
          << t << " ms\n";
      if (t < best_t * 0.98) {
        best_t = t;
        best = strat;
      }
    }
    tune_store(ctx, mat_key, best, 0);
  }
  if (!agg_key.empty()) {
    double best_t = 1e30;
    int best = 2;
    for (int strat : {1, 2}) {
      t_force_agg_strategy = strat;
      std::unique_ptr<Program> p;
      try {
        p = compile(ctx, plan);
      } catch (...) {
        t_force_agg_strategy = 0;
        throw;
      }
      t_force_agg_strategy = 0;
      double t = 1e30;
      try {
        t = total(run_steps(ctx, *p, s, reps));
      } catch (...) {
        free_program(ctx, *p);
        throw;
      }
      free_program(ctx, *p);
      rep << "one-key aggregate " << (strat == 1 ? "in shared memory (one pass)" : "partitioned") << ": " << t
          << " ms\n";
      if (t < best_t) {
        best_t = t;
        best = strat;
      }
    }
    tune_store(ctx, agg_key, best, 0);
  }
  // launch shapes, one pipeline step at a time
  auto p = compile(ctx, plan);
  try {
    tune_apply(ctx, *p);
    for (size_t i = 0; i < p->steps.size(); ++i) {
      Step& st = p->steps[i];
      if (st.k != Step::PIPELINE || st.pipe.sink == SK_PART_COUNT || st.pipe.sink == SK_PART_SCATTER) continue;
      double best_t = 1e30;
      int best_g = 0, best_rows = tile_candidates(st)[0];
      for (int g : {0, 1, 2, 3, 4}) {  // 0: as many as fit
        for (int rows : tile_candidates(st)) {
          set_shape(st, g, rows);
          const double t = run_steps(ctx, *p, s, reps)[i];
          if (t < best_t * 0.995) {  // ties keep the earlier (default) shape
            best_t = t;
            best_g = g;
            best_rows = rows;
          }
        }
      }
      set_shape(st, best_g, best_rows);
      tune_store(ctx, tune_key_pipeline(st), best_g, best_rows);
      rep << st.name << " [" << tune_key_pipeline(st) << "]: ctas_per_sm " << (best_g ? std::to_string(best_g) : "max")
          << ", tile " << best_rows << " rows, " << best_t << " ms\n";
    }
  } catch (...) {
    free_program(ctx, *p);
    throw;
  }
  free_program(ctx, *p);
  {
    std::lock_guard<std::recursive_mutex> g(ctx.mu);
    tune_save_locked(ctx);
  }
  rep << "saved to " << tune_file_path(ctx) << "\n";
  return rep.str();
}

}  // namespace mtl
