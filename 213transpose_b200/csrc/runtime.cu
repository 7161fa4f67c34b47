// Host runtime of the in-place 213 transpose: error reporting, device
// properties, per-stream workspaces, per-pass timing, the planner, and the
// C ABI declared in include/t213.h.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <list>
#include <map>
#include <tuple>

#include "plan.h"

namespace t213 {

// ------------------------------------------------------------------ errors --
namespace {
thread_local std::string tl_error;
}
void set_error(const std::string &msg) { tl_error = msg; }
const std::string &last_error() { return tl_error; }
int cuda_status(cudaError_t e, const char *where) {
  set_error(std::string(where) + ": " + cudaGetErrorString(e));
  cudaGetLastError();
  return e == cudaErrorMemoryAllocation ? T213_ERR_OUT_OF_MEMORY : T213_ERR_CUDA;
}

// ------------------------------------------------------------------ device --
const DevInfo &dev_info() {
  static std::mutex mu;
  static std::map<int, DevInfo> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(dev);
  if (it != cache.end()) return it->second;
  DevInfo d;
  d.id = dev;
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess) d.sms = v;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) == cudaSuccess) d.smem_optin = v;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) == cudaSuccess) d.smem_per_sm = v;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxThreadsPerMultiProcessor, dev) == cudaSuccess) d.max_threads_sm = v;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrComputeCapabilityMajor, dev) == cudaSuccess) d.cc_major = v;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrComputeCapabilityMinor, dev) == cudaSuccess) d.cc_minor = v;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrL2CacheSize, dev) == cudaSuccess) d.l2_bytes = v;
  cudaGetLastError();
  return cache.emplace(dev, d).first->second;
}

// --------------------------------------------------------------- workspace --
namespace {
std::mutex g_ws_mu;
std::map<std::pair<int, cudaStream_t>, std::pair<char *, size_t>> g_ws;
}  // namespace

char *workspace(cudaStream_t st, size_t bytes, int *status) {
  const int dev = dev_info().id;
  std::lock_guard<std::mutex> lk(g_ws_mu);
  auto &w = g_ws[{dev, st}];
  if (w.first && w.second >= bytes) return w.first;
  if (w.first) {
    // cudaFree does not promise to wait for kernels in flight: finish the
    // stream's earlier work (the only user of this buffer) first
    cudaStreamSynchronize(st);
    cudaFree(w.first);
    w.first = nullptr;
    w.second = 0;
  }
  size_t want = std::max<size_t>(bytes, (size_t)1 << 20);
  want = (want + ((size_t)1 << 20) - 1) & ~(((size_t)1 << 20) - 1);
  char *p = nullptr;
  cudaError_t e = cudaMalloc(&p, want);
  if (e != cudaSuccess) {
    *status = cuda_status(e, "workspace cudaMalloc");
    return nullptr;
  }
  w.first = p;
  w.second = want;
  return p;
}

int *device_status_word(int *status) {
  static std::mutex mu;
  static std::map<int, int *> words;
  const int dev = dev_info().id;
  std::lock_guard<std::mutex> lk(mu);
  auto it = words.find(dev);
  if (it != words.end()) return it->second;
  int *p = nullptr;
  cudaError_t e = cudaMalloc(&p, 256);
  if (e == cudaSuccess) e = cudaMemset(p, 0, 256);
  // the memset runs on the legacy stream, which kernels on non-blocking
  // streams do not wait for: let it land before any pass can record a status
  if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  if (e != cudaSuccess) {
    *status = cuda_status(e, "status word");
    return nullptr;
  }
  words[dev] = p;
  return p;
}

void release_stream_workspace(cudaStream_t st) {
  const int dev = dev_info().id;
  std::lock_guard<std::mutex> lk(g_ws_mu);
  auto it = g_ws.find({dev, st});
  if (it == g_ws.end()) return;
  cudaStreamSynchronize(st);
  if (it->second.first) cudaFree(it->second.first);
  g_ws.erase(it);
}

static void release_workspaces() {
  const int dev = dev_info().id;
  std::lock_guard<std::mutex> lk(g_ws_mu);
  for (auto it = g_ws.begin(); it != g_ws.end();) {
    if (it->first.first == dev) {
      if (it->second.first) cudaFree(it->second.first);
      it = g_ws.erase(it);
    } else {
      ++it;
    }
  }
}

// ----------------------------------------------------------- launch cache --
namespace {
std::mutex g_lc_mu;
std::map<std::tuple<const void *, int64_t, int, int>, int> g_attr_done;
std::map<std::tuple<const void *, int, int64_t, int, int>, int> g_occ;
}  // namespace

bool kernel_attr_once(const void *kern, int64_t smem, int cluster) {
  // The dynamic shared-memory attribute is an upper bound: raise it when a
  // launch needs more than any earlier one, never lower it.
  const int dev = dev_info().id;
  std::lock_guard<std::mutex> lk(g_lc_mu);
  auto key = std::make_tuple(kern, (int64_t)0, 0, dev);
  auto it = g_attr_done.find(key);
  const int64_t have = it == g_attr_done.end() ? -1 : it->second;
  if (smem > have) {
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return false;
    g_attr_done[key] = (int)smem;
  }
  if (cluster > 8) {
    auto ck = std::make_tuple(kern, (int64_t)1, 1, dev);
    if (!g_attr_done.count(ck)) {
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) return false;
      g_attr_done[ck] = 1;
    }
  }
  return true;
}

int occupancy_cached(const void *kern, int threads, int64_t smem, int cluster, int *out) {
  const int dev = dev_info().id;
  {
    std::lock_guard<std::mutex> lk(g_lc_mu);
    auto it = g_occ.find(std::make_tuple(kern, threads, smem, cluster, dev));
    if (it != g_occ.end()) {
      *out = it->second;
      return T213_OK;
    }
  }
  int v = 0;
  if (cluster <= 1) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kern, threads, (size_t)smem) != cudaSuccess || v < 1) {
      cudaGetLastError();
      v = 1;
    }
  } else {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(cluster * 8), 1, 1);
    cfg.blockDim = dim3(threads, 1, 1);
    cfg.dynamicSmemBytes = (size_t)smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaOccupancyMaxActiveClusters(&v, kern, &cfg) != cudaSuccess || v < 1) {
      cudaGetLastError();
      v = std::max(1, dev_info().sms / cluster);
    }
  }
  std::lock_guard<std::mutex> lk(g_lc_mu);
  g_occ[std::make_tuple(kern, threads, smem, cluster, dev)] = v;
  *out = v;
  return T213_OK;
}

// ------------------------------------------------------------------ timing --
namespace {
std::atomic<bool> g_timing{false};
std::mutex g_tmu;
struct TimingRec {
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
  double total_ms = 0;
  int64_t launches = 0;
};
std::map<std::string, TimingRec> g_trec;
}  // namespace

bool pass_timing_on() { return g_timing.load(); }

PassTimer::PassTimer(const char *n, cudaStream_t s) : name(n), st(s) {
  if (!g_timing.load()) return;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) {
    a = b = nullptr;
    cudaGetLastError();
    return;
  }
  cudaEventRecord(a, st);
}

PassTimer::~PassTimer() {
  if (!a) return;
  cudaEventRecord(b, st);
  std::lock_guard<std::mutex> lk(g_tmu);
  g_trec[name].pending.push_back({a, b});
}

// ---------------------------------------------------------------- planning --
int64_t ext_gcd(int64_t a, int64_t b, int64_t *mmi) {
  // gcd and the inverse of a modulo b (0 if gcd != 1), extended Euclid
  int64_t x = 0, lastx = 1, origb = b;
  while (b != 0) {
    int64_t q = a / b, nb = a % b;
    a = b;
    b = nb;
    int64_t nx = lastx - q * x;
    lastx = x;
    x = nx;
  }
  if (mmi) *mmi = (a == 1) ? (lastx < 0 ? lastx + origb : lastx) : 0;
  return a;
}

const char *PassDesc::name() const {
  switch (type) {
    case PT_COL:
      return "col_gather";
    case PT_ROW:
      return "row_gather";
    case PT_SEG:
      return "segment_cycles";
    case PT_TILE:
      return "tile_swap";
    case PT_BAND:
      return "band_transpose";
    case PT_SLICE:
      return "slice";
  }
  return "?";
}

namespace {

PassDesc col_pass(int kind, std::initializer_list<int64_t> prm, int64_t m, int64_t n) {
  PassDesc p;
  p.type = PT_COL;
  p.fn.kind = kind;
  int q = 0;
  for (int64_t v : prm) p.fn.p[q++] = v;
  p.m = m;
  p.n = n;
  return p;
}

PassDesc row_pass(int kind, std::initializer_list<int64_t> prm, int64_t m, int64_t n) {
  PassDesc p = col_pass(kind, prm, m, n);
  p.type = PT_ROW;
  return p;
}

// Items per chunk for the walker: pieces of a segment (16-byte words, team of
// up to 256 threads) times slices.
int64_t items_per_chunk(int64_t seg_bytes, int64_t d3) {
  int team = seg_cycles_team(seg_bytes, 16);
  int64_t words = std::max<int64_t>(1, seg_bytes / 16);
  return std::max<int64_t>(1, (words + team - 1) / team) * std::max<int64_t>(1, d3);
}

int add_seg_pass(Plan &P, const PermSpec &ps, int64_t seg_bytes, bool skip_identity) {
  int st = T213_OK;
  PassDesc p;
  p.type = PT_SEG;
  p.perm = ps;
  p.seg_bytes = seg_bytes;
  p.table = get_cycle_table(ps, items_per_chunk(seg_bytes, P.d3), &st);
  if (!p.table) return st;
  if (skip_identity && p.table->n_chunks == 0) return T213_OK;
  P.passes.push_back(p);
  return T213_OK;
}

// Fraction of the copy bandwidth a segment-cycle pass reaches, by segment
// size (bulk-copy walker from 1 KB up, register walker below).
double seg_eff(int64_t seg_bytes) {
  if (seg_bytes >= 4096) return 0.88;
  if (seg_bytes >= 1024) return 0.8;
  if (seg_bytes >= 512) return 0.65;  // bulk walker when 16-byte aligned: 0.72 at 704 B
  if (seg_bytes >= 256) return 0.5;   // 0.61 at 480 B
  if (seg_bytes >= 128) return 0.3;
  if (seg_bytes >= 64) return 0.18;
  return 0.08;
}

std::string fmt_plan(const Plan &P) {
  VariantScope vs(P.var);  // the pass descriptions show the kernels this plan's variant picks
  static const char *kn[] = {"auto", "c2r", "r2c", "skinny", "blocks", "bands", "bands_t", "identity", "slice"};
  std::string s = kn[P.kind >= 0 && P.kind <= 8 ? P.kind : 0];
  char buf[256];
  if (P.t) {
    snprintf(buf, sizeof buf, " t=%lld", (long long)P.t);
    s += buf;
  }
  s += ":";
  for (const PassDesc &p : P.passes) {
    s += " ";
    switch (p.type) {
      case PT_COL:
        {
          const std::string d = describe_col_gather_fn(p.fn, p.m, p.n, P.eb, nullptr);
          snprintf(buf, sizeof buf, "%s(fn=%d)%s", d.substr(0, d.find('[')).c_str(), p.fn.kind,
                   d.substr(d.find('[')).c_str());
        }
        break;
      case PT_ROW:
        snprintf(buf, sizeof buf, "row_gather(fn=%d)%s", p.fn.kind, describe_row_gather(p.m, p.n, P.eb, nullptr).substr(10).c_str());
        break;
      case PT_SLICE:
        snprintf(buf, sizeof buf, "%s", describe_slice(p.m, p.n, P.eb, P.d3).c_str());
        break;
      case PT_SEG:
        snprintf(buf, sizeof buf, "segment_cycles(S=%lld seg=%lldB cycles=%lld chunks=%lld carry=%lld maxlen=%lld)",
                 (long long)p.perm.S, (long long)p.seg_bytes, (long long)p.table->n_cycles,
                 (long long)p.table->n_chunks, (long long)p.table->n_carry, (long long)p.table->max_len);
        break;
      case PT_TILE:
        snprintf(buf, sizeof buf, "tile_swap(t=%lld)", (long long)p.t);
        break;
      case PT_BAND:
        snprintf(buf, sizeof buf, "band_transpose(%lldx%lld)", (long long)p.R, (long long)p.C);
        break;
    }
    s += buf;
  }
  return s;
}

// C2R on an m x n slice (m = d2 rows, n = d1 columns): src/transpose.cu:30-47
// and src/skinny.cu:313-333.  The column op is always the fused column
// shuffle: on B200 a 32-column strip of any realistic height fits a thread-
// block cluster's shared memory, which replaces the reference's 48 KB switch
// to post-rotation + row scatter.
void c2r_passes(Plan &P, int64_t m, int64_t n, bool skinny) {
  int64_t t, c = ext_gcd(m, n, &t), k;
  if (c > 1)
    ext_gcd(m / c, n / c, &k);
  else
    k = t;
  if (c > 1) {
    if (skinny)
      P.passes.push_back(col_pass(T213_FN_C2R_FUSED_PREOP, {m, n / c}, m, n));
    else
      P.passes.push_back(col_pass(T213_FN_C2R_PREROTATOR, {n / c}, m, n));
  }
  P.passes.push_back(row_pass(skinny ? T213_FN_C2R_LONG_SHUFFLE : T213_FN_C2R_SHUFFLE, {m, n, c, k}, m, n));
  P.passes.push_back(col_pass(T213_FN_C2R_FUSED_POSTOP, {m, n, c}, m, n));
}

// R2C with the passes on the m x n output view: src/transpose.cu:58-89,
// src/skinny.cu:344-363.
void r2c_passes(Plan &P, int64_t m, int64_t n, bool skinny) {
  int64_t t, c = ext_gcd(n, m, &t), q;
  if (c > 1)
    ext_gcd(n / c, m / c, &q);
  else
    q = t;
  P.passes.push_back(col_pass(T213_FN_R2C_FUSED_PREOP, {m / c, c, m, q}, m, n));
  P.passes.push_back(row_pass(T213_FN_R2C_SHUFFLE, {m, n, c, 0}, m, n));
  if (c > 1) {
    if (skinny)
      P.passes.push_back(col_pass(T213_FN_R2C_FUSED_POSTOP, {m, n / c}, m, n));
    else
      P.passes.push_back(col_pass(T213_FN_R2C_POSTROTATOR, {n / c, m}, m, n));
  }
}

// Fraction of the copy rate a gather pass reaches, by variant, from B200
// measurements: cluster-local column strips 0.5-0.64, staged column strips
// 0.3-0.45, DSMEM-clustered columns about 0.25; staged rows 0.6-0.8.  Rows
// longer than shared memory, gathered from a global scratch copy, about 0.17
// (DSMEM-clustered rows 0.06); columns taller than a 16-CTA cluster, from a
// scratch copy, about 0.06 (C2R on (344, 359054, 4) fp32).
double gather_cost(const PassDesc &p, int eb) {
  if (p.type == PT_COL) {
    std::string d = describe_col_gather_fn(p.fn, p.m, p.n, eb, nullptr);
    if (d.find("[local") != std::string::npos) return 1 / 0.6;
    if (d.find("scratch") != std::string::npos) return 1 / 0.06;
    if (d.find("cluster=1 ") != std::string::npos) return 1 / 0.4;
    return 1 / 0.25;
  }
  std::string d = describe_row_gather(p.m, p.n, eb, nullptr);
  if (d.find("scratch") != std::string::npos) return 1 / 0.17;
  if (d.find("cluster") != std::string::npos) return 1 / 0.06;
  return 1 / 0.65;
}

int64_t largest_divisor_le(int64_t x, int64_t limit) {
  // largest divisor of x that is <= limit
  int64_t best = 1;
  for (int64_t f = 1; f * f <= x; f++) {
    if (x % f) continue;
    if (f <= limit) best = std::max(best, f);
    if (x / f <= limit) best = std::max(best, x / f);
  }
  return best;
}

// Candidate block / band sizes.
int64_t pick_block_t(int64_t m, int64_t n) { return ext_gcd(m, n, nullptr); }
int64_t pick_band_t(int64_t m, int64_t n, int eb) {
  // t | m, band t x n fits shared memory; a whole slice up to 96 KB is one band
  if (band_smem_bytes(m, n, eb) <= 96 * 1024) return m;
  int64_t per_row = band_smem_bytes(1, n, eb);
  if (per_row > band_smem_limit()) return 0;
  return largest_divisor_le(m, band_smem_limit() / per_row);
}
int64_t pick_band_t_t(int64_t m, int64_t n, int eb) {
  // t | n, band m x t fits shared memory
  int64_t lim = band_smem_limit() / std::max<int64_t>(1, m * eb);
  if (lim < 1) return 0;
  return largest_divisor_le(n, lim);
}

// Fraction of the copy bandwidth the square-block tile pass reaches (measured
// on (8192, 6144, d3) blocks of t = 2048): the TMA kernel's 64-wide fp32
// tiles 0.91, the register kernel's 32-wide tiles 0.90 (8-byte) and 0.93
// (16-byte) but 0.72 for 4-byte elements, whose 32-wide rows are only 128
// bytes; the element-wise kernel about 0.35.
double tile_eff(int64_t t, int eb) {
  if (eb == 4 && t % 64 == 0) return 0.91;
  if ((eb == 8 || eb == 16) && t % 32 == 0) return 0.9;
  if (eb == 4 && t % 32 == 0) return 0.72;
  return 0.35;
}

int build_plan(Plan &P, int kind, int64_t t) {
  const int64_t d1 = P.d1, d2 = P.d2, d3 = P.d3;
  const int eb = P.eb;
  const int64_t m = d2, n = d1;
  P.kind = kind;
  P.t = 0;
  P.passes.clear();
  switch (kind) {
    case T213_PLAN_IDENTITY:
      if (d1 != 1 && d2 != 1) {
        set_error("identity plan needs d1 == 1 or d2 == 1");
        return T213_ERR_UNSUPPORTED;
      }
      return T213_OK;
    case T213_PLAN_C2R:
      c2r_passes(P, m, n, false);
      return T213_OK;
    case T213_PLAN_R2C:
      r2c_passes(P, d1, d2, false);  // output view: d1 rows x d2 columns
      return T213_OK;
    case T213_PLAN_SKINNY:
      if (d2 <= 32 && d2 < d1) {
        c2r_passes(P, m, n, true);
        return T213_OK;
      }
      if (d1 <= 32) {
        r2c_passes(P, d1, d2, true);
        return T213_OK;
      }
      set_error("skinny plan needs min(d1,d2) <= 32");
      return T213_ERR_UNSUPPORTED;
    case T213_PLAN_BLOCKS: {
      if (t <= 0) t = pick_block_t(m, n);
      if (m % t || n % t) {
        set_error("block size must divide gcd(d1,d2)");
        return T213_ERR_UNSUPPORTED;
      }
      P.t = t;
      PassDesc tp;
      tp.type = PT_TILE;
      tp.t = t;
      tp.m = m;
      tp.n = n;
      P.passes.push_back(tp);
      PermSpec ps;
      ps.kind = 0;
      ps.A = m / t;
      ps.Mid = t;
      ps.C = n / t;
      ps.S = m * n / t;
      if (ps.A == 1 && ps.C == 1) return T213_OK;
      return add_seg_pass(P, ps, t * eb, true);
    }
    case T213_PLAN_BANDS: {
      if (t <= 0) t = pick_band_t(m, n, eb);
      if (t <= 0 || m % t || !band_fits(t, n, eb)) {
        set_error("band size must divide d2 and a t x d1 band must fit shared memory");
        return T213_ERR_UNSUPPORTED;
      }
      P.t = t;
      PassDesc bp;
      bp.type = PT_BAND;
      bp.R = t;
      bp.C = n;
      bp.bands = m / t;
      P.passes.push_back(bp);
      PermSpec ps;
      ps.kind = 0;
      ps.A = m / t;
      ps.Mid = 1;
      ps.C = n;
      ps.S = (m / t) * n;
      return add_seg_pass(P, ps, t * eb, true);
    }
    case T213_PLAN_SLICE: {
      if (!slice_fits(m, n, eb)) {
        set_error("slice plan needs a slice that fits a 16-CTA cluster's shared memory");
        return T213_ERR_UNSUPPORTED;
      }
      PassDesc sp;
      sp.type = PT_SLICE;
      sp.m = m;
      sp.n = n;
      P.passes.push_back(sp);
      return T213_OK;
    }
    case T213_PLAN_BANDS_T: {
      if (t <= 0) t = pick_band_t_t(m, n, eb);
      if (t <= 0 || n % t || !band_fits(m, t, eb)) {
        set_error("band size must divide d1 and a d2 x t band must fit shared memory");
        return T213_ERR_UNSUPPORTED;
      }
      P.t = t;
      PermSpec ps;
      ps.kind = 0;
      ps.A = m;
      ps.Mid = 1;
      ps.C = n / t;
      ps.S = m * (n / t);
      int st = add_seg_pass(P, ps, t * eb, true);
      if (st) return st;
      PassDesc bp;
      bp.type = PT_BAND;
      bp.R = m;
      bp.C = t;
      bp.bands = n / t;
      P.passes.push_back(bp);
      return T213_OK;
    }
  }
  set_error("unknown plan kind");
  return T213_ERR_INVALID_ARGUMENT;
}

double plan_cost(const Plan &P) {
  double c = 0;
  for (const PassDesc &p : P.passes) {
    switch (p.type) {
      case PT_COL:
      case PT_ROW:
        c += gather_cost(p, P.eb);
        break;
      case PT_SEG: {
        c += 1.0 / seg_eff(p.seg_bytes) * (double)p.table->moved / std::max<int64_t>(1, p.perm.S);
        break;
      }
      case PT_TILE:
        c += 1 / tile_eff(p.t, P.eb);
        break;
      case PT_BAND:
        c += 1 / 0.5;
        break;
      case PT_SLICE:
        c += 1 / 0.6;
        break;
    }
  }
  return c;
}

// Cheap estimate used to rank candidates before any cycle table is built.
double estimate_cost(int kind, int64_t m, int64_t n, int64_t t, int eb, int64_t d3) {
  (void)d3;
  const double S_limit = 4.0e6;  // first-call host cycle walk stays around 20 ms
  switch (kind) {
    case T213_PLAN_BLOCKS: {
      if (t <= 0 || t * eb < 16) return 1e9;
      const double tile = 1 / tile_eff(t, eb);
      if (m == n && m == t) return tile;
      double S = (double)m * (double)n / (double)t;
      if (S > S_limit) return 1e9;
      return tile + 1 / seg_eff(t * eb);
    }
    case T213_PLAN_BANDS:
    case T213_PLAN_BANDS_T: {
      if (t <= 0 || t * eb < 32) return 1e9;
      double S = (double)m * (double)n / (double)t;
      if (S > S_limit) return 1e9;
      if ((kind == T213_PLAN_BANDS && t == m) || (kind == T213_PLAN_BANDS_T && t == n)) return 1 / 0.5;
      return 1 / 0.5 + 1 / seg_eff(t * eb);
    }
  }
  return 1e9;
}

struct PlanKey {
  int64_t d1, d2, d3;
  int eb, kind;
  int64_t t;
  int dev;
  int var = 0;  // Variant::packed()
  bool operator<(const PlanKey &o) const {
    return std::tie(d1, d2, d3, eb, kind, t, dev, var) < std::tie(o.d1, o.d2, o.d3, o.eb, o.kind, o.t, o.dev, o.var);
  }
};

// LRU cache of plans (front = most recently used).  Evicting a plan can drop
// the last reference to its cycle tables; their device memory is then freed
// only after a device-wide synchronisation (see CycleTable).
// Heap objects that are never destroyed: at process exit the plans (and the
// CUDA resources of their cycle tables) are left to the driver's teardown
// instead of being released by static destructors in an unspecified order.
std::mutex &g_plan_mu = *new std::mutex;
auto &g_plan_lru = *new std::list<std::pair<PlanKey, std::shared_ptr<Plan>>>;
auto &g_plans = *new std::map<PlanKey, std::list<std::pair<PlanKey, std::shared_ptr<Plan>>>::iterator>;
constexpr size_t kPlanCacheMax = 1024;

std::shared_ptr<Plan> new_plan(int64_t d1, int64_t d2, int64_t d3, int eb) {
  auto P = std::make_shared<Plan>();
  P->d1 = d1;
  P->d2 = d2;
  P->d3 = d3;
  P->eb = eb;
  return P;
}

}  // namespace

int tuner_lookup_internal(int64_t d1, int64_t d2, int64_t d3, int eb, int *kind, int64_t *t, Variant *v);

std::shared_ptr<Plan> get_plan_variant(int64_t d1, int64_t d2, int64_t d3, int eb, int kind, int64_t t,
                                       const Variant &v, int *status) {
  std::shared_ptr<Plan> base = get_plan(d1, d2, d3, eb, kind, t, status);
  if (!base || !v.any()) return base;
  PlanKey key{d1, d2, d3, eb, kind, t, dev_info().id, v.packed()};
  std::lock_guard<std::mutex> lk(g_plan_mu);
  auto it = g_plans.find(key);
  if (it != g_plans.end()) {
    g_plan_lru.splice(g_plan_lru.begin(), g_plan_lru, it->second);
    return it->second->second;
  }
  auto P = std::make_shared<Plan>(*base);
  P->var = v;
  P->desc = fmt_plan(*P);  // the pass descriptions under this variant
  char buf[64];
  snprintf(buf, sizeof buf, " [variant col=%d row=%d tile=%d seg=%d]", v.col, v.row, v.tile, v.seg);
  P->desc += buf;
  g_plan_lru.emplace_front(key, P);
  g_plans[key] = g_plan_lru.begin();
  while (g_plan_lru.size() > kPlanCacheMax) {
    g_plans.erase(g_plan_lru.back().first);
    g_plan_lru.pop_back();
  }
  return P;
}

bool plan_cached(int64_t d1, int64_t d2, int64_t d3, int eb, int kind, int64_t t) {
  PlanKey key{d1, d2, d3, eb, kind, t, dev_info().id};
  std::lock_guard<std::mutex> lk(g_plan_mu);
  return g_plans.find(key) != g_plans.end();
}

std::shared_ptr<Plan> get_plan(int64_t d1, int64_t d2, int64_t d3, int eb, int kind, int64_t t, int *status) {
  *status = T213_OK;
  const int dev = dev_info().id;
  if (kind == T213_PLAN_AUTO) {
    int tk = 0;
    int64_t tt = 0;
    Variant tv;
    if (tuner_lookup_internal(d1, d2, d3, eb, &tk, &tt, &tv) == T213_OK && tk != T213_PLAN_AUTO) {
      auto p = get_plan_variant(d1, d2, d3, eb, tk, tt, tv, status);
      if (!p && tt) p = get_plan_variant(d1, d2, d3, eb, tk, 0, tv, status);  // block size of another shape
      if (p) return p;
      *status = T213_OK;
    }
  }
  PlanKey key{d1, d2, d3, eb, kind, t, dev};
  {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    auto it = g_plans.find(key);
    if (it != g_plans.end()) {
      g_plan_lru.splice(g_plan_lru.begin(), g_plan_lru, it->second);
      return it->second->second;
    }
  }
  std::shared_ptr<Plan> best;
  if (kind != T213_PLAN_AUTO) {
    best = new_plan(d1, d2, d3, eb);
    int st = build_plan(*best, kind, t);
    if (st) {
      *status = st;
      return nullptr;
    }
    best->est_cost = plan_cost(*best);
  } else {
    const int64_t m = d2, n = d1;
    if (d1 == 1 || d2 == 1 || d1 == 0 || d2 == 0 || d3 == 0) {
      best = new_plan(d1, d2, d3, eb);
      best->kind = T213_PLAN_IDENTITY;
    } else {
      // rank the cheap estimates first; build only the winners
      struct Cand {
        int kind;
        int64_t t;
        double est;
      };
      std::vector<Cand> cands;
      int64_t tb = pick_block_t(m, n);
      cands.push_back({T213_PLAN_BLOCKS, tb, estimate_cost(T213_PLAN_BLOCKS, m, n, tb, eb, d3)});
      int64_t tr = pick_band_t(m, n, eb);
      cands.push_back({T213_PLAN_BANDS, tr, estimate_cost(T213_PLAN_BANDS, m, n, tr, eb, d3)});
      int64_t tc = pick_band_t_t(m, n, eb);
      cands.push_back({T213_PLAN_BANDS_T, tc, estimate_cost(T213_PLAN_BANDS_T, m, n, tc, eb, d3)});
      // The one-pass cluster plan (T213_PLAN_SLICE) wins where launch latency
      // dominates: small tensors whose rows are 16-byte multiples both ways.
      // Measured on B200: fp32 (256, 128, 64) 0.0126 ms against 0.0190 for
      // BLOCKS; fp32 (512, 384, 16) 0.0192 against 0.0244 (clusters of 4, one
      // wave).  Its element-wise form (other alignments) won on fp64
      // (45, 600, 2) (0.015 against 0.025 ms) but lost badly on 1-byte
      // (1000, 999, 1) (0.26 against 0.15 ms).  So it is ranked for tensors
      // up to 16 MB with aligned rows only, and is otherwise taken when
      // forced or chosen by the tuner.
      if (slice_fits(m, n, eb) && (n * eb) % 16 == 0 && (m * eb) % 16 == 0 && d1 * d2 * d3 * eb <= (16ll << 20))
        cands.push_back({T213_PLAN_SLICE, 0, 1.0});
      // The Catanzaro decomposition both ways: the reference's dispatcher
      // takes C2R when d1 >= d2, else R2C (src/transpose.cu:117-123); here
      // both are costed, since which one keeps its rows inside shared
      // memory decides the faster one for tall or wide slices.
      for (int k : {T213_PLAN_C2R, T213_PLAN_R2C}) {
        Plan tmp;
        tmp.d1 = d1;
        tmp.d2 = d2;
        tmp.d3 = d3;
        tmp.eb = eb;
        build_plan(tmp, k, 0);
        // ties go to the reference's choice
        const bool ref_choice = (k == T213_PLAN_C2R) == (d1 >= d2);
        cands.push_back({k, 0, plan_cost(tmp) * (ref_choice ? 1.0 : 1.0001)});
      }
      std::sort(cands.begin(), cands.end(), [](const Cand &a, const Cand &b) { return a.est < b.est; });
      for (const Cand &c : cands) {
        if (c.est >= 1e8) continue;
        auto P = new_plan(d1, d2, d3, eb);
        if (build_plan(*P, c.kind, c.t) == T213_OK) {
          P->est_cost = plan_cost(*P);
          best = P;
          break;
        }
      }
      if (!best) {
        *status = T213_ERR_UNSUPPORTED;
        set_error("no plan applies to this shape");
        return nullptr;
      }
    }
  }
  best->desc = fmt_plan(*best);
  {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    auto it = g_plans.find(key);
    if (it == g_plans.end()) {
      g_plan_lru.push_front({key, best});
      g_plans[key] = g_plan_lru.begin();
      while (g_plan_lru.size() > kPlanCacheMax) {
        g_plans.erase(g_plan_lru.back().first);
        g_plan_lru.pop_back();
      }
    }
  }
  return best;
}

std::shared_ptr<Plan> make_c2r_plan(int64_t d1, int64_t d2, int64_t d3, int eb, bool skinny, int *status) {
  *status = T213_OK;
  auto P = new_plan(d1, d2, d3, eb);
  P->kind = skinny ? T213_PLAN_SKINNY : T213_PLAN_C2R;
  c2r_passes(*P, d2, d1, skinny);
  P->desc = fmt_plan(*P);
  return P;
}

std::shared_ptr<Plan> make_r2c_plan(int64_t d1, int64_t d2, int64_t d3, int eb, bool skinny, int *status) {
  *status = T213_OK;
  auto P = new_plan(d1, d2, d3, eb);
  P->kind = skinny ? T213_PLAN_SKINNY : T213_PLAN_R2C;
  r2c_passes(*P, d2, d1, skinny);
  P->desc = fmt_plan(*P);
  return P;
}

size_t plan_workspace_bytes(const Plan &p) {
  size_t w = 0;
  for (const PassDesc &q : p.passes)
    if (q.type == PT_SEG && q.table) w = std::max(w, seg_cycles_carry_bytes(*q.table, p.d3, q.seg_bytes));
  return w;
}

namespace {
thread_local Variant t_variant;
}  // namespace

const Variant &current_variant() { return t_variant; }
VariantScope::VariantScope(const Variant &v) : saved(t_variant) { t_variant = v; }
VariantScope::~VariantScope() { t_variant = saved; }

// Slices per group when a plan runs its passes group by group
// (T213_SLICE_GROUP_MB: the group's size in MB; unset or 0: all slices in
// one group).  Every pass of a group runs before the next group starts, so a
// pass finds part of what the previous pass wrote still in L2.
int64_t slice_group(const Plan &P) {
  static const int64_t mb = [] {
    const char *v = std::getenv("T213_SLICE_GROUP_MB");
    return v ? (int64_t)std::atoll(v) : 0;
  }();
  const int64_t slice_bytes = P.d1 * P.d2 * P.eb;
  if (mb <= 0 || slice_bytes <= 0 || P.d3 <= 1) return std::max<int64_t>(1, P.d3);
  return std::max<int64_t>(1, std::min<int64_t>(P.d3, (mb << 20) / slice_bytes));
}

int run_plan(const Plan &P, char *data, cudaStream_t st, LaunchStats *ls) {
  const int64_t slice_bytes = P.d1 * P.d2 * P.eb;
  VariantScope vs(P.var);
  const int64_t group = slice_group(P);
  for (int64_t k0 = 0; k0 < P.d3; k0 += group) {
    const int64_t g = std::min<int64_t>(group, P.d3 - k0);
    char *gd = data + k0 * slice_bytes;
    for (const PassDesc &p : P.passes) {
      PassTimer tm(p.name(), st);
      int rc = T213_OK;
      switch (p.type) {
        case PT_COL:
          rc = launch_col_gather(p.fn, gd, g, p.m, p.n, P.eb, st, ls);
          break;
        case PT_ROW:
          rc = launch_row_gather(p.fn, gd, g, p.m, p.n, P.eb, st, ls);
          break;
        case PT_TILE:
          rc = launch_tile_swap(gd, g, p.m, p.n, p.t, P.eb, st, ls);
          break;
        case PT_BAND:
          rc = launch_band_transpose(gd, g * p.bands, p.R, p.C, P.eb, st, ls);
          break;
        case PT_SEG:
          rc = launch_seg_cycles(*p.table, gd, g, slice_bytes, p.seg_bytes, st, ls, nullptr, 0);
          break;
        case PT_SLICE:
          rc = launch_slice(gd, g, p.m, p.n, P.eb, st, ls);
          break;
      }
      if (rc) return rc;
    }
  }
  return T213_OK;
}

}  // namespace t213

// =========================================================================
// C ABI
// =========================================================================
using namespace t213;

namespace {

int check_args(const void *data, int64_t d1, int64_t d2, int64_t d3, int32_t eb) {
  if (d1 < 0 || d2 < 0 || d3 < 0) {
    set_error("negative dimension");
    return T213_ERR_INVALID_ARGUMENT;
  }
  if (eb != 1 && eb != 2 && eb != 4 && eb != 8 && eb != 16) {
    set_error("element size must be 1, 2, 4, 8 or 16 bytes");
    return T213_ERR_UNSUPPORTED;
  }
  const double vol = (double)d1 * (double)d2 * (double)d3 * (double)eb;
  if (vol >= 9.0e18) {
    set_error("tensor too large");
    return T213_ERR_INVALID_ARGUMENT;
  }
  if (vol > 0 && !data) {
    set_error("data is NULL");
    return T213_ERR_INVALID_ARGUMENT;
  }
  if (((uintptr_t)data) % (uintptr_t)std::min(eb, 16)) {
    set_error("data is not aligned to its element size");
    return T213_ERR_INVALID_ARGUMENT;
  }
  return T213_OK;
}

int prefetch_if_managed(void *data, size_t bytes, cudaStream_t st) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, data) != cudaSuccess) {
    cudaGetLastError();
    set_error("data is not a CUDA device or managed pointer");
    return T213_ERR_INVALID_ARGUMENT;
  }
  if (at.type == cudaMemoryTypeManaged) {
    cudaError_t e = cudaMemPrefetchAsync(data, bytes, dev_info().id, st);
    if (e != cudaSuccess) return cuda_status(e, "cudaMemPrefetchAsync");
  } else if (at.type != cudaMemoryTypeDevice) {
    set_error("data must be device or managed memory (use t213_transpose_host for host buffers)");
    return T213_ERR_INVALID_ARGUMENT;
  }
  return T213_OK;
}

int run_shape(void *data, int64_t d1, int64_t d2, int64_t d3, int32_t eb, int kind, int64_t t,
              cudaStream_t st, int which /*0 auto/with_plan, 1 c2r, 2 r2c, 3 skinny c2r, 4 skinny r2c*/) {
  int rc = check_args(data, d1, d2, d3, eb);
  if (rc) return rc;
  if (d1 == 0 || d2 == 0 || d3 == 0) return T213_OK;
  rc = prefetch_if_managed(data, (size_t)(d1 * d2 * d3 * eb), st);
  if (rc) return rc;
  std::shared_ptr<Plan> P;
  switch (which) {
    case 0:
      P = get_plan(d1, d2, d3, eb, kind, t, &rc);
      break;
    case 1:
      P = make_c2r_plan(d1, d2, d3, eb, false, &rc);
      break;
    case 2:
      P = make_r2c_plan(d1, d2, d3, eb, false, &rc);
      break;
    case 3:
      if (d2 > 32) {
        set_error("skinny C2R needs d2 <= 32");
        return T213_ERR_INVALID_ARGUMENT;
      }
      P = make_c2r_plan(d1, d2, d3, eb, true, &rc);
      break;
    case 4:
      if (d2 > 32) {
        set_error("skinny R2C needs d2 <= 32");
        return T213_ERR_INVALID_ARGUMENT;
      }
      P = make_r2c_plan(d1, d2, d3, eb, true, &rc);
      break;
  }
  if (!P) return rc ? rc : T213_ERR_UNSUPPORTED;
  return run_plan(*P, (char *)data, st, nullptr);
}

int run_single_pass(int type, int32_t fn_kind, const int64_t *prm, int32_t np, void *data, int64_t d3,
                    int64_t d2, int64_t d1, int32_t eb, cudaStream_t st) {
  int rc = check_args(data, d1, d2, d3, eb);
  if (rc) return rc;
  if (np < 0 || np > 4 || (np > 0 && !prm)) {
    set_error("functor parameters: 0..4 values");
    return T213_ERR_INVALID_ARGUMENT;
  }
  FnSpec f;
  f.kind = fn_kind;
  for (int q = 0; q < np; q++) f.p[q] = prm[q];
  for (int q = 0; q < np; q++)
    if (f.p[q] < 0) {
      set_error("functor parameters must be non-negative");
      return T213_ERR_INVALID_ARGUMENT;
    }
  if (d1 == 0 || d2 == 0 || d3 == 0) return T213_OK;
  rc = prefetch_if_managed(data, (size_t)(d1 * d2 * d3 * eb), st);
  if (rc) return rc;
  const int64_t m = d2, n = d1;
  // divisor-type parameters must be positive
  auto need_pos = [&](std::initializer_list<int> idx) -> bool {
    for (int q : idx)
      if (f.p[q] <= 0) return false;
    return true;
  };
  switch (type) {
    case PT_COL: {
      bool ok = true;
      switch (fn_kind) {
        case T213_FN_C2R_PREROTATOR:
        case T213_FN_C2R_POSTROTATOR:
        case T213_FN_R2C_PREROTATOR:
          ok = need_pos({0});
          break;
        case T213_FN_R2C_POSTROTATOR:
          ok = need_pos({0});
          break;
        case T213_FN_C2R_FUSED_PREOP:
        case T213_FN_R2C_FUSED_POSTOP:
          ok = need_pos({0, 1}) && f.p[0] == m;
          break;
        case T213_FN_C2R_FUSED_POSTOP:
          ok = need_pos({0}) && f.p[0] == m;
          break;
        case T213_FN_R2C_FUSED_PREOP:
          ok = need_pos({0, 1, 2}) && f.p[2] == m;
          break;
        default:
          set_error("functor kind is not a rotator or column shuffler");
          return T213_ERR_INVALID_ARGUMENT;
      }
      if (!ok) {
        set_error("functor parameters do not match the slice (m must equal d2, divisors positive)");
        return T213_ERR_INVALID_ARGUMENT;
      }
      PassTimer tm("col_gather", st);
      return launch_col_gather(f, (char *)data, d3, m, n, eb, st, nullptr);
    }
    case PT_ROW: {
      if (fn_kind != T213_FN_C2R_SHUFFLE && fn_kind != T213_FN_C2R_LONG_SHUFFLE && fn_kind != T213_FN_R2C_SHUFFLE) {
        set_error("functor kind is not a row shuffler");
        return T213_ERR_INVALID_ARGUMENT;
      }
      if (!need_pos({0, 1, 2}) || f.p[0] != m || f.p[1] != n) {
        set_error("row shuffler parameters must be (m=d2, n=d1, c>0, k)");
        return T213_ERR_INVALID_ARGUMENT;
      }
      PassTimer tm("row_gather", st);
      return launch_row_gather(f, (char *)data, d3, m, n, eb, st, nullptr);
    }
    case PT_SEG: {
      if (fn_kind != T213_FN_C2R_POSTPERMUTER && fn_kind != T213_FN_R2C_PREPERMUTER) {
        set_error("functor kind is not a row permuter");
        return T213_ERR_INVALID_ARGUMENT;
      }
      if (!need_pos({0, 1, 2}) || f.p[0] != m || f.p[1] != n || m % f.p[2] || n % f.p[2]) {
        set_error("row permuter parameters must be (m=d2, n=d1, c) with c dividing both");
        return T213_ERR_INVALID_ARGUMENT;
      }
      PermSpec ps;
      ps.kind = fn_kind;
      ps.fn = f;
      ps.S = m;
      const int64_t seg = n * eb;
      std::shared_ptr<CycleTable> ct = get_cycle_table(ps, items_per_chunk(seg, d3), &rc);
      if (!ct) return rc;
      PassTimer tm("segment_cycles", st);
      return launch_seg_cycles(*ct, (char *)data, d3, m * n * eb, seg, st, nullptr, nullptr, 0);
    }
  }
  return T213_ERR_INVALID_ARGUMENT;
}

}  // namespace

extern "C" {

const char *t213_status_string(int status) {
  switch (status) {
    case T213_OK:
      return "ok";
    case T213_ERR_INVALID_ARGUMENT:
      return "invalid argument";
    case T213_ERR_UNSUPPORTED:
      return "unsupported";
    case T213_ERR_CUDA:
      return "CUDA error";
    case T213_ERR_OUT_OF_MEMORY:
      return "out of device memory";
    case T213_ERR_TIMEOUT:
      return "device-side wait timed out";
    case T213_ERR_BUDGET:
      return "request exceeds the HBM budget";
    case T213_ERR_NOT_READY:
      return "not ready";
  }
  return "unknown status";
}

const char *t213_last_error(void) { return last_error().c_str(); }

const char *t213_version(void) { return "213transpose_b200 1.0 (sm_100a)"; }

int t213_transpose(void *data, int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes, t213_stream_t stream) {
  return run_shape(data, d1, d2, d3, elem_bytes, T213_PLAN_AUTO, 0, (cudaStream_t)stream, 0);
}

int t213_transpose_with_plan(void *data, int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes, int32_t plan_kind,
                             int64_t t, t213_stream_t stream) {
  if (plan_kind < T213_PLAN_AUTO || plan_kind > T213_PLAN_SLICE || t < 0) {
    set_error("bad plan kind or block size");
    return T213_ERR_INVALID_ARGUMENT;
  }
  return run_shape(data, d1, d2, d3, elem_bytes, plan_kind, t, (cudaStream_t)stream, 0);
}

int t213_permute(void *data, int32_t rank, const int64_t *dims, const int32_t *perm, int32_t elem_bytes,
                 t213_stream_t stream) {
  if (rank < 0 || rank > 32 || (rank > 0 && (!dims || !perm))) {
    set_error("t213_permute: rank must be 0..32 with dims and perm given");
    return T213_ERR_INVALID_ARGUMENT;
  }
  std::vector<int> seen(rank, 0);
  double vol = 1;
  for (int i = 0; i < rank; i++) {
    if (dims[i] < 0 || perm[i] < 0 || perm[i] >= rank || seen[perm[i]]++) {
      set_error("t213_permute: dims must be >= 0 and perm a permutation of 0..rank-1");
      return T213_ERR_INVALID_ARGUMENT;
    }
    vol *= (double)dims[i];
  }
  if (vol * elem_bytes >= 9.0e18) {
    set_error("tensor too large");
    return T213_ERR_INVALID_ARGUMENT;
  }
  const int rc0 = check_args(data, vol > 0 ? 1 : 0, 1, 1, elem_bytes);  // element size, NULL, alignment
  if (rc0) return rc0;
  if (vol == 0 || rank < 2) return T213_OK;
  // Leading axes the permutation keeps in place become part of the element:
  // up to 16 bytes the 213 plans move it as one element; from 64 bytes on,
  // a 213 step of such elements is a single segment-cycle pass (one read and
  // one write of the tensor) as long as its cycle table stays small.
  const double total_bytes = vol * elem_bytes;
  int64_t E = elem_bytes;
  int q0 = 0;
  while (q0 < rank - 1 && perm[q0] == q0) {
    const int64_t E2 = E * dims[q0];
    const bool small = E2 <= 16 && (E2 & (E2 - 1)) == 0;
    const bool seg = E2 >= 64 && total_bytes / (double)E2 <= 4.0e6;
    if (!small && !seg) break;
    E = E2;
    q0++;
  }
  // cur[q]: the input axis now at position q (fastest first) among axes
  // q0..rank-1.  For k from the slowest position down, bring perm[k] to
  // position k by rotating the prefix [q0, k]: the group [q0, p] (ending with
  // that axis) moves behind the group [p+1, k], which is one 213 transpose
  // with d1 = the first group's volume, d2 = the second's and d3 = everything
  // slower.
  std::vector<int> cur(rank);
  for (int i = 0; i < rank; i++) cur[i] = i;
  for (int k = rank - 1; k > q0; k--) {
    int p = q0;
    while (cur[p] != perm[k]) p++;
    if (p == k) continue;
    int64_t g1 = 1, g2 = 1, g3 = 1;
    for (int q = q0; q <= p; q++) g1 *= dims[cur[q]];
    for (int q = p + 1; q <= k; q++) g2 *= dims[cur[q]];
    for (int q = k + 1; q < rank; q++) g3 *= dims[cur[q]];
    int rc;
    if (E <= 16) {
      rc = run_shape(data, g1, g2, g3, (int32_t)E, T213_PLAN_AUTO, 0, (cudaStream_t)stream, 0);
    } else if (g1 == 1 || g2 == 1) {
      rc = T213_OK;  // the memory layout does not change
    } else {
      // segments of E bytes: [g2][g1] -> [g1][g2] in each of the g3 slices
      PermSpec ps;
      ps.kind = 0;
      ps.A = g2;
      ps.Mid = 1;
      ps.C = g1;
      ps.S = g1 * g2;
      rc = T213_OK;
      auto ct = get_cycle_table(ps, items_per_chunk(E, g3), &rc);
      if (!ct) return rc;
      if (ct->n_chunks > 0)
        rc = launch_seg_cycles(*ct, (char *)data, g3, g1 * g2 * E, E, (cudaStream_t)stream, nullptr, nullptr, 0);
    }
    if (rc) return rc;
    std::rotate(cur.begin() + q0, cur.begin() + p + 1, cur.begin() + k + 1);
  }
  return T213_OK;
}

int t213_c2r_transpose(void *data, int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes, t213_stream_t stream) {
  return run_shape(data, d1, d2, d3, elem_bytes, 0, 0, (cudaStream_t)stream, 1);
}

int t213_r2c_transpose(void *data, int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes, t213_stream_t stream) {
  return run_shape(data, d1, d2, d3, elem_bytes, 0, 0, (cudaStream_t)stream, 2);
}

int t213_skinny_c2r_transpose(void *data, int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes,
                              t213_stream_t stream) {
  return run_shape(data, d1, d2, d3, elem_bytes, 0, 0, (cudaStream_t)stream, 3);
}

int t213_skinny_r2c_transpose(void *data, int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes,
                              t213_stream_t stream) {
  return run_shape(data, d1, d2, d3, elem_bytes, 0, 0, (cudaStream_t)stream, 4);
}

int t213_rotate(int32_t fn_kind, const int64_t *fn_params, int32_t n_params, void *data, int64_t d3, int64_t d2,
                int64_t d1, int32_t elem_bytes, t213_stream_t stream) {
  if (fn_kind < T213_FN_C2R_PREROTATOR || fn_kind > T213_FN_R2C_POSTROTATOR) {
    set_error("functor kind is not a rotator");
    return T213_ERR_INVALID_ARGUMENT;
  }
  return run_single_pass(PT_COL, fn_kind, fn_params, n_params, data, d3, d2, d1, elem_bytes, (cudaStream_t)stream);
}

int t213_row_shuffle(int32_t fn_kind, const int64_t *fn_params, int32_t n_params, void *data, int64_t d3,
                     int64_t d2, int64_t d1, int32_t elem_bytes, t213_stream_t stream) {
  return run_single_pass(PT_ROW, fn_kind, fn_params, n_params, data, d3, d2, d1, elem_bytes, (cudaStream_t)stream);
}

int t213_col_shuffle(int32_t fn_kind, const int64_t *fn_params, int32_t n_params, void *data, int64_t d3,
                     int64_t d2, int64_t d1, int32_t elem_bytes, t213_stream_t stream) {
  if (fn_kind < T213_FN_C2R_FUSED_PREOP || fn_kind > T213_FN_R2C_FUSED_POSTOP) {
    set_error("functor kind is not a column shuffler");
    return T213_ERR_INVALID_ARGUMENT;
  }
  return run_single_pass(PT_COL, fn_kind, fn_params, n_params, data, d3, d2, d1, elem_bytes, (cudaStream_t)stream);
}

int t213_scatter_permute(int32_t fn_kind, const int64_t *fn_params, int32_t n_params, void *data, int64_t d3,
                         int64_t d2, int64_t d1, int32_t elem_bytes, t213_stream_t stream) {
  return run_single_pass(PT_SEG, fn_kind, fn_params, n_params, data, d3, d2, d1, elem_bytes, (cudaStream_t)stream);
}

int t213_plan_describe(int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes, int32_t plan_kind, int64_t t,
                       char *buf, size_t buflen) {
  int rc = check_args((void *)16, d1, d2, d3, elem_bytes);
  if (rc) return rc;
  if (!buf || buflen == 0) {
    set_error("buffer is NULL");
    return T213_ERR_INVALID_ARGUMENT;
  }
  std::shared_ptr<Plan> P = get_plan(d1, d2, d3, elem_bytes, plan_kind, t, &rc);
  if (!P) return rc;
  snprintf(buf, buflen, "%s", P->desc.c_str());
  return T213_OK;
}

int t213_plan_launches(int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes, int32_t plan_kind, int64_t t,
                       int32_t *launches) {
  int rc = check_args((void *)16, d1, d2, d3, elem_bytes);
  if (rc) return rc;
  if (!launches) return T213_ERR_INVALID_ARGUMENT;
  std::shared_ptr<Plan> P = get_plan(d1, d2, d3, elem_bytes, plan_kind, t, &rc);
  if (!P) return rc;
  int n = 0;
  const int64_t group = slice_group(*P);
  for (int64_t k0 = 0; k0 < d3; k0 += group) {
    const int64_t g = std::min<int64_t>(group, d3 - k0);
    for (const PassDesc &p : P->passes) {
      switch (p.type) {
        case PT_COL:
          n += count_col_gather(g, p.m, p.n, elem_bytes);
          break;
        case PT_ROW:
          n += count_row_gather(g, p.m, p.n, elem_bytes);
          break;
        case PT_SEG:
          n += (p.table->n_chunks > 0) + (p.table->n_carry > 0);
          break;
        default:
          n += 1;
      }
    }
  }
  *launches = n;
  return T213_OK;
}

int t213_device_status(t213_stream_t stream, int32_t *device_status) {
  if (!device_status) return T213_ERR_INVALID_ARGUMENT;
  int rc = T213_OK;
  int *w = device_status_word(&rc);
  if (!w) return rc;
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_status(e, "cudaStreamSynchronize");
  int v = 0;
  if ((e = cudaMemcpy(&v, w, sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess) return cuda_status(e, "status read");
  if (v && (e = cudaMemsetAsync(w, 0, sizeof(int), (cudaStream_t)stream)) == cudaSuccess)
    e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_status(e, "status reset");
  *device_status = v;
  return T213_OK;
}

int t213_pass_timing_enable(int32_t enable) {
  g_timing.store(enable != 0);
  return T213_OK;
}

int t213_pass_timing_read(const char *pass_name, double *total_ms, int64_t *launches) {
  if (!pass_name || !total_ms || !launches) return T213_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(g_tmu);
  TimingRec &r = g_trec[pass_name];
  for (auto &pr : r.pending) {
    cudaEventSynchronize(pr.second);
    float ms = 0;
    if (cudaEventElapsedTime(&ms, pr.first, pr.second) == cudaSuccess) r.total_ms += ms;
    cudaEventDestroy(pr.first);
    cudaEventDestroy(pr.second);
    r.launches++;
  }
  r.pending.clear();
  cudaGetLastError();
  *total_ms = r.total_ms;
  *launches = r.launches;
  return T213_OK;
}

int t213_pass_timing_reset(void) {
  std::lock_guard<std::mutex> lk(g_tmu);
  for (auto &kv : g_trec)
    for (auto &pr : kv.second.pending) {
      cudaEventSynchronize(pr.second);
      cudaEventDestroy(pr.first);
      cudaEventDestroy(pr.second);
    }
  g_trec.clear();
  cudaGetLastError();
  return T213_OK;
}

int t213_release_cache(void) {
  cudaDeviceSynchronize();
  {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    g_plans.clear();
    g_plan_lru.clear();
  }
  release_workspaces();
  flush_deferred_frees();
  return T213_OK;
}

}  // extern "C"
