// Autotuner: times the applicable plan families of a shape on the device and
// caches the winner per shape class.  A class is (element size, log2 of d1,
// d2 and d3, log2 of gcd(d1,d2)); the cached entry stores the plan family only,
// and the planner re-derives the block or band size for each concrete shape.
// The cache persists as a text file, one class per line.
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
std::map<ClassKey, int> g_cache;                                     // per shape class
std::map<std::tuple<int64_t, int64_t, int64_t, int>, int> g_exact;  // per exact shape, wins

}  // namespace

int tuner_lookup_internal(int64_t d1, int64_t d2, int64_t d3, int eb, int *kind, int64_t *t) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto ex = g_exact.find(std::make_tuple(d1, d2, d3, eb));
  if (ex != g_exact.end()) {
    *kind = ex->second;
    *t = 0;
    return T213_OK;
  }
  auto it = g_cache.find(class_of(d1, d2, d3, eb));
  if (it == g_cache.end()) return T213_ERR_NOT_READY;
  *kind = it->second;
  *t = 0;
  return T213_OK;
}

}  // namespace t213

using namespace t213;

extern "C" {

int t213_tuner_lookup(int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes, int32_t *plan_kind, int64_t *t) {
  if (!plan_kind || !t) return T213_ERR_INVALID_ARGUMENT;
  int k = 0;
  int rc = tuner_lookup_internal(d1, d2, d3, elem_bytes, &k, t);
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
  fprintf(f, "# t213 tuner cache\n# class eb log2(d1) log2(d2) log2(d3) log2(gcd) plan_kind\n");
  fprintf(f, "# shape d1 d2 d3 eb plan_kind\n");
  for (auto &kv : g_cache)
    fprintf(f, "class %d %d %d %d %d %d\n", kv.first.eb, kv.first.l1, kv.first.l2, kv.first.l3, kv.first.lg,
            kv.second);
  for (auto &kv : g_exact)
    fprintf(f, "shape %lld %lld %lld %d %d\n", (long long)std::get<0>(kv.first), (long long)std::get<1>(kv.first),
            (long long)std::get<2>(kv.first), std::get<3>(kv.first), kv.second);
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
  int n = 0;
  std::lock_guard<std::mutex> lk(g_mu);
  while (fgets(line, sizeof line, f)) {
    if (line[0] == '#') continue;
    ClassKey k;
    int kind, eb;
    long long a, b, c;
    if (sscanf(line, "class %d %d %d %d %d %d", &k.eb, &k.l1, &k.l2, &k.l3, &k.lg, &kind) == 6 &&
        kind >= T213_PLAN_AUTO && kind <= T213_PLAN_IDENTITY) {
      g_cache[k] = kind;
      n++;
    } else if (sscanf(line, "shape %lld %lld %lld %d %d", &a, &b, &c, &eb, &kind) == 5 && kind >= T213_PLAN_AUTO &&
               kind <= T213_PLAN_IDENTITY) {
      g_exact[std::make_tuple((int64_t)a, (int64_t)b, (int64_t)c, eb)] = kind;
      n++;
    }
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
  const int kinds[] = {T213_PLAN_BLOCKS, T213_PLAN_BANDS, T213_PLAN_BANDS_T, T213_PLAN_C2R, T213_PLAN_R2C,
                       T213_PLAN_SKINNY};
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  double best_ms = 1e30;
  int best_kind = T213_PLAN_AUTO;
  int64_t best_t = 0;
  for (int kind : kinds) {
    int rc = T213_OK;
    std::shared_ptr<Plan> P = get_plan(d1, d2, d3, elem_bytes, kind, 0, &rc);
    if (!P) continue;
    // one warm-up, then the best of three
    if (run_plan(*P, (char *)scratch_data, st, nullptr) != T213_OK) continue;
    double ms_best = 1e30;
    for (int r = 0; r < 3; r++) {
      cudaEventRecord(a, st);
      run_plan(*P, (char *)scratch_data, st, nullptr);
      cudaEventRecord(b, st);
      cudaEventSynchronize(b);
      float ms = 0;
      cudaEventElapsedTime(&ms, a, b);
      ms_best = std::min(ms_best, (double)ms);
    }
    if (ms_best < best_ms) {
      best_ms = ms_best;
      best_kind = kind;
      best_t = P->t;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e, "tuning");
  if (best_kind == T213_PLAN_AUTO) {
    set_error("no plan applies to this shape");
    return T213_ERR_UNSUPPORTED;
  }
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_cache[class_of(d1, d2, d3, elem_bytes)] = best_kind;
    g_exact[std::make_tuple(d1, d2, d3, (int)elem_bytes)] = best_kind;
  }
  if (chosen_plan) *chosen_plan = best_kind;
  if (chosen_t) *chosen_t = best_t;
  return T213_OK;
}

}  // extern "C"
