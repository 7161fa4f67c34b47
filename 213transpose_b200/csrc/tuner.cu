// Autotuner: times the applicable plan families of a shape on the device,
// then, for the winning family, its block or band size and the kernel
// variants of its passes (column strips staged or cluster-local, their width,
// single- or double-buffered, staged or double-buffered rows, TMA or register tile swaps, bulk
// walker ring depth or the register walker), one choice at a time, and caches
// the winner per exact shape and per shape class.  A class is (element size,
// log2 of d1, d2 and d3, log2 of gcd(d1,d2)); a class entry keeps the family
// and the variants, and the planner re-derives the block or band size for
// each concrete shape.  The cache persists as a text file, one entry per line.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <tuple>

#include "plan.h"

namespace t213 {
namespace {

struct ClassKey {
  int eb, l1, l2, l3, lg;
  bool operator<(const ClassKey &o) const {
    return std::tie(eb, l1, l2, l3, lg) < std::tie(o.eb, o.l1, o.l2, o.l3, o.lg);
  }
};

struct Entry {
  int kind = T213_PLAN_AUTO;
  int64_t t = 0;
  int var = 0;  // Variant::packed()
};

int ilog2(int64_t x) {
  int r = 0;
  while (x > 1) {
    x >>= 1;
    r++;
  }
  return r;
}

ClassKey class_of(int64_t d1, int64_t d2, int64_t d3, int eb) {
  return ClassKey{eb, ilog2(d1), ilog2(d2), ilog2(d3), ilog2(ext_gcd(d1, d2, nullptr))};
}

std::mutex g_mu;
std::map<ClassKey, Entry> g_cache;                                     // per shape class
std::map<std::tuple<int64_t, int64_t, int64_t, int>, Entry> g_exact;  // per exact shape, wins

}  // namespace

int tuner_lookup_internal(int64_t d1, int64_t d2, int64_t d3, int eb, int *kind, int64_t *t, Variant *v) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto ex = g_exact.find(std::make_tuple(d1, d2, d3, eb));
  if (ex != g_exact.end()) {
    *kind = ex->second.kind;
    *t = ex->second.t;
    if (v) *v = Variant::unpack(ex->second.var);
    return T213_OK;
  }
  auto it = g_cache.find(class_of(d1, d2, d3, eb));
  if (it == g_cache.end()) return T213_ERR_NOT_READY;
  *kind = it->second.kind;
  *t = 0;
  if (v) *v = Variant::unpack(it->second.var);
  return T213_OK;
}

}  // namespace t213

using namespace t213;

extern "C" {

int t213_tuner_lookup(int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes, int32_t *plan_kind, int64_t *t) {
  if (!plan_kind || !t) return T213_ERR_INVALID_ARGUMENT;
  int k = 0;
  int rc = tuner_lookup_internal(d1, d2, d3, elem_bytes, &k, t, nullptr);
  *plan_kind = rc == T213_OK ? k : T213_PLAN_AUTO;
  return rc;
}

int t213_tuner_clear(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_cache.clear();
  g_exact.clear();
  return T213_OK;
}

int t213_tuner_save(const char *path) {
  if (!path) return T213_ERR_INVALID_ARGUMENT;
  FILE *f = fopen(path, "w");
  if (!f) {
    set_error(std::string("cannot write ") + path);
    return T213_ERR_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  fprintf(f, "# t213 tuner cache\n# class eb log2(d1) log2(d2) log2(d3) log2(gcd) plan_kind variant\n");
  fprintf(f, "# shape d1 d2 d3 eb plan_kind t variant\n");
  for (auto &kv : g_cache)
    fprintf(f, "class %d %d %d %d %d %d %d\n", kv.first.eb, kv.first.l1, kv.first.l2, kv.first.l3, kv.first.lg,
            kv.second.kind, kv.second.var);
  for (auto &kv : g_exact)
    fprintf(f, "shape %lld %lld %lld %d %d %lld %d\n", (long long)std::get<0>(kv.first),
            (long long)std::get<1>(kv.first), (long long)std::get<2>(kv.first), std::get<3>(kv.first), kv.second.kind,
            (long long)kv.second.t, kv.second.var);
  fclose(f);
  return T213_OK;
}

int t213_tuner_load(const char *path) {
  if (!path) return T213_ERR_INVALID_ARGUMENT;
  FILE *f = fopen(path, "r");
  if (!f) {
    set_error(std::string("cannot read ") + path);
    return T213_ERR_INVALID_ARGUMENT;
  }
  char line[256];
  std::lock_guard<std::mutex> lk(g_mu);
  while (fgets(line, sizeof line, f)) {
    if (line[0] == '#') continue;
    ClassKey k;
    int kind = 0, eb = 0, var = 0;
    long long a, b, c, t = 0;
    // older files have no variant (and no block size on shape lines)
    const int nc = sscanf(line, "class %d %d %d %d %d %d %d", &k.eb, &k.l1, &k.l2, &k.l3, &k.lg, &kind, &var);
    if (nc >= 6 && kind >= T213_PLAN_AUTO && kind <= T213_PLAN_SLICE) {
      g_cache[k] = Entry{kind, 0, nc == 7 ? var : 0};
      continue;
    }
    var = 0;
    const int ns = sscanf(line, "shape %lld %lld %lld %d %d %lld %d", &a, &b, &c, &eb, &kind, &t, &var);
    if (ns >= 5 && kind >= T213_PLAN_AUTO && kind <= T213_PLAN_SLICE)
      g_exact[std::make_tuple((int64_t)a, (int64_t)b, (int64_t)c, eb)] =
          Entry{kind, ns >= 6 ? (int64_t)t : 0, ns == 7 ? var : 0};
  }
  fclose(f);
  return T213_OK;
}

int t213_tune_shape(void *scratch_data, int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes, t213_stream_t stream,
                    int32_t *chosen_plan, int64_t *chosen_t) {
  if (!scratch_data || d1 <= 0 || d2 <= 0 || d3 <= 0) {
    set_error("tuning needs a device buffer of the tensor's size and positive sizes");
    return T213_ERR_INVALID_ARGUMENT;
  }
  cudaStream_t st = (cudaStream_t)stream;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  // one warm-up, then the best of three; a plan that does not build or run
  // scores infinity
  auto time_plan = [&](int kind, int64_t t, const Variant &v, int64_t *built_t) -> double {
    int rc = T213_OK;
    std::shared_ptr<Plan> P = get_plan_variant(d1, d2, d3, elem_bytes, kind, t, v, &rc);
    if (!P) return 1e30;
    if (built_t) *built_t = P->t;
    if (run_plan(*P, (char *)scratch_data, st, nullptr) != T213_OK) return 1e30;
    double best = 1e30;
    for (int r = 0; r < 3; r++) {
      cudaEventRecord(a, st);
      run_plan(*P, (char *)scratch_data, st, nullptr);
      cudaEventRecord(b, st);
      cudaEventSynchronize(b);
      float ms = 0;
      cudaEventElapsedTime(&ms, a, b);
      best = std::min(best, (double)ms);
    }
    return best;
  };
  // 1) the family, each with its planner-chosen block size and default kernels
  const int kinds[] = {T213_PLAN_BLOCKS, T213_PLAN_BANDS, T213_PLAN_BANDS_T, T213_PLAN_C2R, T213_PLAN_R2C,
                       T213_PLAN_SKINNY, T213_PLAN_SLICE};
  double best_ms = 1e30;
  Entry best;
  for (int kind : kinds) {
    int64_t t = 0;
    const double ms = time_plan(kind, 0, Variant{}, &t);
    if (ms < best_ms) {
      best_ms = ms;
      best = Entry{kind, t, 0};
    }
  }
  if (best.kind == T213_PLAN_AUTO) {
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaGetLastError();
    set_error("no plan applies to this shape");
    return T213_ERR_UNSUPPORTED;
  }
  // 2) the block or band size: half the planner's choice, if it builds
  if ((best.kind == T213_PLAN_BLOCKS || best.kind == T213_PLAN_BANDS || best.kind == T213_PLAN_BANDS_T) &&
      best.t >= 16 && best.t % 2 == 0) {
    const double ms = time_plan(best.kind, best.t / 2, Variant{}, nullptr);
    if (ms < best_ms) {
      best_ms = ms;
      best.t /= 2;
    }
  }
  // 3) the kernel variants of the passes the plan has, one choice at a time
  {
    int rc = T213_OK;
    std::shared_ptr<Plan> P = get_plan(d1, d2, d3, elem_bytes, best.kind, best.t, &rc);
    bool has[8] = {false, false, false, false, false, false, false, false};
    if (P)
      for (const PassDesc &q : P->passes) has[q.type] = true;
    struct Knob {
      int type;
      int8_t Variant::*field;
      std::vector<int8_t> values;
    };
    const Knob knobs[] = {{PT_COL, &Variant::col, {1, 2, 3, 4, 5}},
                          {PT_ROW, &Variant::row, {2, 3}},
                          {PT_TILE, &Variant::tile, {1, 2}},
                          {PT_SEG, &Variant::seg, {2, 3}}};
    Variant cur;
    for (const Knob &kb : knobs) {
      if (!has[kb.type]) continue;
      for (int8_t val : kb.values) {
        Variant v = cur;
        v.*kb.field = val;
        const double ms = time_plan(best.kind, best.t, v, nullptr);
        if (ms < best_ms * 0.98) {  // a variant has to win clearly to displace the default
          best_ms = ms;
          cur = v;
        }
      }
    }
    best.var = cur.packed();
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e, "tuning");
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_cache[class_of(d1, d2, d3, elem_bytes)] = Entry{best.kind, 0, best.var};
    g_exact[std::make_tuple(d1, d2, d3, (int)elem_bytes)] = best;
  }
  if (chosen_plan) *chosen_plan = best.kind;
  if (chosen_t) *chosen_t = best.t;
  return T213_OK;
}

}  // extern "C"
