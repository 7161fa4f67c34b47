// Launchers of the row-gather and column-gather passes: variant choice
// (single CTA, thread-block cluster, global-scratch fallback), access width,
// index width, and the functor dispatch.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "k_gather.cuh"
#include "k_slice.cuh"
#include "plan.h"

namespace t213 {

namespace {

constexpr int64_t kSmemCap = 220 * 1024;     // per-CTA unit budget (opt-in max is 227 KB)
constexpr int64_t kSmemTarget = 104 * 1024;  // prefer two CTAs per SM
constexpr int kMaxCluster = 16;

// Column-gather functor dispatch (rotators and column shufflers).
template <typename U, typename Fn>
bool with_col_fn(const FnSpec &f, int64_t m, Fn &&fn) {
  switch (f.kind) {
    case T213_FN_C2R_PREROTATOR:
      return fn(RotGather<U, RotC2RPre<U>>(RotC2RPre<U>(f.p[0]), m));
    case T213_FN_C2R_POSTROTATOR:
      return fn(RotGather<U, RotC2RPost<U>>(RotC2RPost<U>(f.p[0]), m));
    case T213_FN_R2C_PREROTATOR:
      return fn(RotGather<U, RotR2CPre<U>>(RotR2CPre<U>(f.p[0]), m));
    case T213_FN_R2C_POSTROTATOR:
      return fn(RotGather<U, RotR2CPost<U>>(RotR2CPost<U>(f.p[0], f.p[1]), m));
    case T213_FN_C2R_FUSED_PREOP:
      return fn(ColC2RFusedPre<U>(f.p[0], f.p[1]));
    case T213_FN_C2R_FUSED_POSTOP:
      return fn(ColC2RFusedPost<U>(f.p[0], f.p[1], f.p[2]));
    case T213_FN_R2C_FUSED_PREOP:
      return fn(ColR2CFusedPre<U>(f.p[0], f.p[1], f.p[2], f.p[3]));
    case T213_FN_R2C_FUSED_POSTOP:
      return fn(ColR2CFusedPost<U>(f.p[0], f.p[1]));
  }
  return false;
}

template <typename U, typename Fn>
bool with_row_fn(const FnSpec &f, Fn &&fn) {
  switch (f.kind) {
    case T213_FN_C2R_SHUFFLE:
    case T213_FN_C2R_LONG_SHUFFLE:
      return fn(RowC2RShuffle<U>(f.p[0], f.p[1], f.p[2], f.p[3]));
    case T213_FN_R2C_SHUFFLE:
      return fn(RowR2CShuffle<U>(f.p[0], f.p[1], f.p[2]));
  }
  return false;
}

int aligned16(const void *p, int64_t pitch_bytes) {
  return (((uintptr_t)p | (uint64_t)pitch_bytes) & 15) == 0;
}

// Access word of the gather kernels: 16 bytes when the base and the pitch
// allow, 8 bytes for 4-byte elements on an 8-byte pitch (half the
// instructions of 4-byte words), else the element.  T213_AW_MAX (4, 8 or 16)
// caps it, for measuring the widths against each other.
int pick_aw(int eb, const void *data, int64_t pitch_bytes, int64_t extra_bytes) {
  if (eb >= 16) return 16;
  static const int cap = [] {
    const char *v = std::getenv("T213_AW_MAX");
    return v && std::atoi(v) > 0 ? std::atoi(v) : 16;
  }();
  if (eb >= 4 && cap >= 16 && aligned16(data, pitch_bytes) && (extra_bytes & 15) == 0) return 16;
  if (eb == 4 && cap >= 8 && ((((uintptr_t)data | (uint64_t)pitch_bytes | (uint64_t)extra_bytes) & 7) == 0)) return 8;
  return eb;
}

int64_t round_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

// ----------------------------------------------------------- column config --
struct ColCfg {
  int aw = 4;
  int64_t W = 0, WS = 0;  // strip width and smem row stride (elements)
  int K = 1;              // cluster size; 0 = scratch fallback
  int64_t H = 0;          // rows per CTA
  int64_t smem = 0;
  int64_t group_w = 0;    // scratch fallback: columns per copy
};

int env_int(const char *name) {
  const char *v = std::getenv(name);
  return v ? std::atoi(v) : 0;
}

ColCfg col_config(int64_t m, int64_t n, int eb, const void *data) {
  ColCfg c;
  c.aw = pick_aw(eb, data, n * eb, 0);
  const int64_t P = c.aw / eb;
  // T213_COL_WBYTES / T213_COL_CLUSTER force a strip width (bytes) and a
  // cluster size, for measuring the variants against each other
  if (const int fw = env_int("T213_COL_WBYTES")) {
    const int fk = std::max(1, std::min(kMaxCluster, env_int("T213_COL_CLUSTER")));
    const int64_t W = round_up(std::min<int64_t>(std::max<int64_t>(P, fw / eb), round_up(n, P)), P);
    const int64_t WS = (W * eb) % 128 == 0 ? W + P : W;
    const int64_t H = (m + fk - 1) / fk;
    if (H * WS * eb <= kSmemCap) {
      c.W = W;
      c.WS = WS;
      c.K = fk;
      c.H = fk == 1 ? m : H;
      c.smem = c.H * WS * eb;
      return c;
    }
  }
  auto strip = [&](int64_t wbytes, bool widen) -> int64_t {
    int64_t W = std::max<int64_t>(P, wbytes / eb);
    if (widen) {  // short columns: widen so a unit is worth ~48 KB
      int64_t want = (48 * 1024) / std::max<int64_t>(1, m * eb);
      if (want > W) W = want / W * W;
    }
    W = std::min<int64_t>(W, round_up(n, P));
    return round_up(W, P);
  };
  auto stride = [&](int64_t W) { return (W * eb) % 128 == 0 ? W + P : W; };
  // 1) one CTA holds the whole strip: the widest strip that fits
  for (int64_t wbytes : {(int64_t)128, (int64_t)64, (int64_t)32, (int64_t)16}) {
    const int64_t W = strip(wbytes, wbytes == 128);
    if (wbytes < 128 && W * eb > wbytes && W > P) continue;
    const int64_t WS = stride(W);
    if (m * WS * eb <= kSmemCap) {
      c.W = W;
      c.WS = WS;
      c.K = 1;
      c.H = m;
      c.smem = m * WS * eb;
      return c;
    }
  }
  // 2) a thread-block cluster shares a 128-byte strip through DSMEM
  for (int64_t wbytes : {(int64_t)128, (int64_t)32}) {
    const int64_t W = strip(wbytes, false);
    const int64_t WS = stride(W);
    const int64_t bytes = m * WS * eb;
    int K = (int)((bytes + kSmemTarget - 1) / kSmemTarget);
    if (K > kMaxCluster) K = (int)((bytes + kSmemCap - 1) / kSmemCap);
    if (K <= kMaxCluster) {
      c.W = W;
      c.WS = WS;
      c.K = K;
      c.H = (m + K - 1) / K;
      c.smem = c.H * WS * eb;
      return c;
    }
  }
  // 3) scratch fallback: copy groups of columns to the workspace
  c.K = 0;
  c.W = std::max<int64_t>(P, 128 / eb);
  c.group_w = std::max<int64_t>(c.W, (int64_t)(256ll << 20) / std::max<int64_t>(1, m * eb) / c.W * c.W);
  c.group_w = std::min<int64_t>(c.group_w, round_up(n, P));
  return c;
}

// ------------------------------------------------- cluster-local columns --
// Which form a column functor has (k_col_local): 1 = offset of the functor
// itself, identity maps; 2 = C2R fused post-op (+j offsets, output rows through
// the inverse post-permuter); 3 = R2C fused pre-op (-j offsets, source rows
// through the pre-permuter); 0 = not handled.
int local_form(int kind) {
  switch (kind) {
    case T213_FN_C2R_PREROTATOR:
    case T213_FN_C2R_POSTROTATOR:
    case T213_FN_R2C_PREROTATOR:
    case T213_FN_R2C_POSTROTATOR:
    case T213_FN_C2R_FUSED_PREOP:
    case T213_FN_R2C_FUSED_POSTOP:
      return 1;
    case T213_FN_C2R_FUSED_POSTOP:
      return 2;
    case T213_FN_R2C_FUSED_PREOP:
      return 3;
  }
  return 0;
}

struct LocalCfg {
  bool ok = false;
  int aw = 4, K = 1;
  int64_t W = 0, WS = 0, H = 0, halo = 0, smem = 0;  // smem: one strip buffer
  bool u64 = false;
  bool db = false;  // double-buffered kernel (two strip buffers)
  // k_col_local_peel: 16-byte accesses although the pitch is not a 16-byte
  // multiple; SB = slot stride in bytes, max_slots = slots of one strip buffer
  bool peel = false;
  int64_t SB = 0, max_slots = 0;
};

// Largest (dmax - dmin) over the strips of width W: the key offsets of one
// strip, unwrapped around the strip's first column, as the kernel computes
// them.  O(n) functor evaluations, cached per (functor, m, n, W).
template <typename Off>
int64_t strip_span(Off off, int64_t m, int64_t n, int64_t W) {
  int64_t worst = 0;
  for (int64_t j0 = 0; j0 < n; j0 += W) {
    const int64_t r0 = (int64_t)off((uint64_t)j0);
    int64_t lo = 0, hi = 0;
    for (int64_t w = 1; w < W && j0 + w < n; w++) {
      int64_t d = (int64_t)off((uint64_t)(j0 + w)) - r0;
      if (2 * d > m) d -= m;
      if (2 * d <= -m) d += m;
      lo = std::min(lo, d);
      hi = std::max(hi, d);
    }
    worst = std::max(worst, hi - lo);
    if (worst > kColHaloMax) break;
  }
  return worst;
}

int64_t local_span(const FnSpec &f, int64_t m, int64_t n, int64_t W) {
  static std::mutex mu;
  static std::map<std::tuple<int, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t, int64_t>, int64_t> cache;
  const auto key = std::make_tuple(f.kind, f.p[0], f.p[1], f.p[2], f.p[3], m, n, W);
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  int64_t span = kColHaloMax + 1;
  const int form = local_form(f.kind);
  if (form == 2) {
    span = strip_span(OffAffine<uint64_t, false>{FastDiv<uint64_t>((uint64_t)m)}, m, n, W);
  } else if (form == 3) {
    span = strip_span(OffAffine<uint64_t, true>{FastDiv<uint64_t>((uint64_t)m)}, m, n, W);
  } else if (form == 1) {
    with_col_fn<uint64_t>(f, m, [&](auto fn) -> bool {
      using F = decltype(fn);
      span = strip_span(OffOfCol<uint64_t, F>{fn}, m, n, W);
      return true;
    });
  }
  std::lock_guard<std::mutex> lk(mu);
  if (cache.size() > 4096) cache.clear();
  cache[key] = span;
  return span;
}

int64_t gcd64(int64_t a, int64_t b) {
  while (b) {
    const int64_t t = a % b;
    a = b;
    b = t;
  }
  return a;
}

// The forms hold for the decomposition's own parameters: the functor's m is
// the matrix's, c = gcd(m, n') (the post-permuter is then a bijection whose
// inverse is the pre-permuter with q = b^-1 mod a), and the pre-permuter's q
// is a unit mod a.  Other parameters keep plain gather semantics through the
// staged kernel.
bool local_params_ok(const FnSpec &f, int64_t m) {
  switch (f.kind) {
    case T213_FN_C2R_FUSED_PREOP:
    case T213_FN_R2C_FUSED_POSTOP:
      return f.p[0] == m && f.p[1] > 0;
    case T213_FN_C2R_FUSED_POSTOP:
      return f.p[0] == m && f.p[1] > 0 && f.p[2] > 0 && f.p[2] == gcd64(m, f.p[1]);
    case T213_FN_R2C_FUSED_PREOP:
      return f.p[2] == m && f.p[0] > 0 && f.p[1] > 0 && f.p[0] * f.p[1] == m && f.p[3] >= 0 &&
             gcd64(f.p[3] % f.p[0], f.p[0]) == 1;
  }
  return true;  // rotators: any amount is a rotation of the m-row column
}

LocalCfg local_col_config(const FnSpec &f, int64_t m, int64_t n, int eb, const void *data) {
  LocalCfg c;
  const char *var = std::getenv("T213_COL_VARIANT");
  const Variant &pv = current_variant();
  if (pv.col == 1 || (pv.col == 0 && var && std::strcmp(var, "old") == 0)) return c;
  if (!local_form(f.kind) || m <= 0 || n <= 0 || !local_params_ok(f, m)) return c;
  c.aw = pick_aw(eb, data, n * eb, 0);
  const int64_t P = c.aw / eb;
  // strip width: a power of two of access words, at most 32 of them (the
  // kernel's fast path gives each lane one word of a row) and 256 elements
  auto width = [&](int64_t wbytes) {
    int64_t words = 1;
    while (words < 32 && 2 * words * c.aw <= wbytes && 2 * words * P <= 256) words *= 2;
    return std::min<int64_t>(words * P, round_up(n, P));
  };
  // index width: the functor's own bound, and the permutation maps' products
  // (below a * a with a = m / gcd)
  c.u64 = !fits32(f, m, n) || (double)m * (double)m >= 2.0e9;
  // double-buffered kernel (T213_COL_DB or the pinned variant): 1 keeps the
  // strip sizes below, 2 halves them (twice the cluster size) so two CTAs
  // share an SM
  const int dbmode = pv.col == 3 ? 1 : pv.col == 4 ? 2 : env_int("T213_COL_DB");
  const int64_t buf_cap = dbmode ? kSmemCap / 2 - 64 : kSmemCap;
  const int64_t whole_cap =
      std::min<int64_t>(buf_cap, (env_int("T213_COL_WHOLE_KB") > 0 ? env_int("T213_COL_WHOLE_KB") : 104) * 1024);
  // narrow access words for 4- and 8-byte elements (the pitch or the base is
  // not 16-byte aligned): the peeled kernel moves the same strips with
  // 16-byte accesses (variant col=5 or T213_COL_PEEL=0 keep the word-width
  // kernel)
  const char *pe = std::getenv("T213_COL_PEEL");
  if ((eb == 4 || eb == 8) && c.aw < 16 && (reinterpret_cast<uintptr_t>(data) % (uintptr_t)eb) == 0 && !dbmode &&
      pv.col != 5 && !(pe && std::atoi(pe) == 0)) {
    c.peel = true;
    c.aw = 16;
    auto slot_bytes = [](int64_t wb) { return wb + 16 + 1; };  // blocks of a slot + its byte in the offset table
    if (m * slot_bytes(128) <= whole_cap && env_int("T213_COL_LOCAL_K") <= 1 && pv.col != 2) {
      int64_t wb = 128;
      const int64_t target = std::max<int64_t>(128, (48 * 1024) / m);
      while (2 * wb <= 512 && 2 * wb <= target && 2 * wb <= round_up(n * eb, 16)) wb *= 2;
      while (wb > 128 && m * slot_bytes(wb) > whole_cap) wb /= 2;
      c.W = wb / eb;
      c.WS = c.W;
      c.SB = wb + 16;
      c.K = 1;
      c.H = m;
      c.halo = 0;
      c.max_slots = m;
      c.smem = m * c.SB + round_up(m, 16);
      c.ok = true;
      return c;
    }
    struct Try {
      int64_t wbytes, kb;
    };
    std::vector<Try> tries;
    if (env_int("T213_COL_LOCAL_WBYTES") >= 64 || env_int("T213_COL_LOCAL_SMEM_KB") > 0)
      tries.push_back({env_int("T213_COL_LOCAL_WBYTES") >= 64 ? env_int("T213_COL_LOCAL_WBYTES") : 128,
                       env_int("T213_COL_LOCAL_SMEM_KB") > 0 ? env_int("T213_COL_LOCAL_SMEM_KB") : 100});
    else if (pv.col == 2)
      tries = {{256, 110}, {256, 200}, {128, 100}, {128, 200}, {64, 200}};
    else  // 110 KB: the most that still lets two CTAs share an SM (fp32 (7919, 6151, 2): clusters of 9
          // instead of 10, column pass 0.245 -> 0.228 ms; clusters that leave one CTA per SM are slower)
      tries = {{128, 110}, {128, 200}, {64, 200}};
    for (const Try &t : tries) {
      if (t.wbytes != 64 && t.wbytes != 128 && t.wbytes != 256 && t.wbytes != 512) continue;
      c.W = t.wbytes / eb;
      c.WS = c.W;
      c.SB = t.wbytes + 16;
      c.halo = local_span(f, m, n, c.W);
      if (c.halo > kColHaloMax) continue;
      const int64_t hmax = std::max<int64_t>(1, (t.kb * 1024) / slot_bytes(t.wbytes) - c.halo);
      c.K = (int)std::min<int64_t>(kMaxCluster + 1, (m + hmax - 1) / hmax);
      if (env_int("T213_COL_LOCAL_K") > 1) c.K = env_int("T213_COL_LOCAL_K");
      if (c.K > kMaxCluster || c.K < 2) continue;
      c.H = (m + c.K - 1) / c.K;
      c.max_slots = c.H + c.halo;
      c.smem = c.max_slots * c.SB + round_up(c.max_slots, 16);
      if (c.smem > buf_cap) continue;
      c.ok = true;
      return c;
    }
    // no peeled strip fits: the word-width kernel below
    c.peel = false;
    c.aw = pick_aw(eb, data, n * eb, 0);
    c.SB = c.max_slots = 0;
  }
  if (m * 128 <= whole_cap && env_int("T213_COL_LOCAL_K") <= 1 && pv.col != 2) {
    // whole strips in one CTA: at least 128-byte rows, widened to about
    // 48 KB per strip (at most 256 columns), no halo
    c.W = width(std::max<int64_t>(128, (48 * 1024) / m));
    while (c.W > P && m * c.W * eb > whole_cap) c.W /= 2;
    c.WS = c.W;
    c.K = 1;
    c.H = m;
    c.halo = 0;
    c.smem = m * c.WS * eb;
    c.ok = true;
    c.db = dbmode != 0;
    return c;
  }
  // tall strips: 128-byte strips over a cluster of up to 16 CTAs of about
  // 100 KB each; taller columns take narrower strips and fuller CTAs (still
  // far ahead of the DSMEM-gathering and global-scratch variants)
  struct Try {
    int64_t wbytes, kb;
  };
  std::vector<Try> tries;
  if (env_int("T213_COL_LOCAL_WBYTES") > 0 || env_int("T213_COL_LOCAL_SMEM_KB") > 0)
    tries.push_back({env_int("T213_COL_LOCAL_WBYTES") > 0 ? env_int("T213_COL_LOCAL_WBYTES") : 128,
                     env_int("T213_COL_LOCAL_SMEM_KB") > 0 ? env_int("T213_COL_LOCAL_SMEM_KB") : 100});
  else if (pv.col == 2)  // 256-byte strips: longer DRAM bursts, fewer CTAs per SM
    tries = {{256, 110}, {256, 200}, {128, 100}, {128, 200}, {64, 200}, {32, 200}, {16, 200}};
  else if (dbmode == 2)
    tries = {{128, 50}, {128, 110}, {64, 110}, {32, 110}, {16, 110}};
  else if (dbmode)
    tries = {{128, 100}, {128, 110}, {64, 110}, {32, 110}, {16, 110}};
  else  // 110 KB per CTA, as for the peeled strips (fp32 (4096, 5003, 4) column pass 0.154 -> 0.140 ms,
        // (6144, 7001, 2) 0.161 -> 0.151 ms, fp64 (3000, 9001, 2) unchanged)
    tries = {{128, 110}, {128, 200}, {64, 200}, {32, 200}, {16, 200}};
  for (const Try &t : tries) {
    c.W = width(t.wbytes);
    c.WS = c.W;  // the gather's diagonal reads step by WS +- 1 words: no padding needed
    c.halo = local_span(f, m, n, c.W);
    if (c.halo > kColHaloMax) continue;
    const int64_t row_bytes = c.WS * eb;
    const int64_t hmax = std::max<int64_t>(1, (t.kb * 1024) / row_bytes - c.halo);
    c.K = (int)std::min<int64_t>(kMaxCluster + 1, (m + hmax - 1) / hmax);
    if (env_int("T213_COL_LOCAL_K") > 1) c.K = env_int("T213_COL_LOCAL_K");
    if (c.K > kMaxCluster || c.K < 2) continue;
    c.H = (m + c.K - 1) / c.K;
    c.smem = (c.H + c.halo) * row_bytes;
    if (c.smem > buf_cap) continue;
    c.ok = true;
    c.db = dbmode != 0;
    return c;
  }
  return c;
}

// --------------------------------------------------------------- row config --
struct RowCfg {
  int aw = 4;
  int K = 1;          // 0 = scratch fallback
  int rows_per_unit = 1;
  int64_t part = 0;   // elements per CTA when clustered
  int64_t smem = 0;
  int64_t group_rows = 0;
  bool pipe = false;  // k_row_pipe: two buffers of buf_bytes
  int64_t buf_bytes = 0;
  bool peel = false;  // k_row_gather_peel: 16-byte accesses although the pitch is not a 16-byte multiple
};

RowCfg row_config(int64_t m, int64_t n, int eb, const void *data) {
  RowCfg r;
  r.aw = pick_aw(eb, data, n * eb, 0);
  const int64_t P = r.aw / eb;
  const int64_t row_bytes = n * eb;
  // Double-buffered units of whole rows (k_row_pipe, T213_ROW_STAGE_KB per
  // buffer), on request with T213_ROW_VARIANT=pipe.  Measured on B200 it is
  // not the default: the staged kernel's two or three resident CTAs per SM
  // already overlap one CTA's loads with another's gather (fp64 (7919, 6151,
  // 2) C2R shuffle 0.345 ms staged against 0.388 ms double-buffered; R2C
  // shuffle 0.291 against 0.284 ms; fp32 (8192, 6143, 2) 0.212 against 0.209).
  const char *var = std::getenv("T213_ROW_VARIANT");
  const Variant &pv = current_variant();
  const int64_t stage = (env_int("T213_ROW_STAGE_KB") > 0 ? env_int("T213_ROW_STAGE_KB") : 48) * 1024;
  const int64_t cap = std::max<int64_t>(stage, (kSmemCap / 2) / 16 * 16);
  const bool pipe = pv.row == 2 || (pv.row == 0 && var && std::strcmp(var, "pipe") == 0);
  if (pipe && row_bytes <= cap) {
    r.K = 1;
    r.pipe = true;
    r.rows_per_unit = (int)std::max<int64_t>(1, std::min<int64_t>(m, stage / row_bytes));
    r.buf_bytes = round_up(r.rows_per_unit * row_bytes, 16);
    r.smem = 2 * r.buf_bytes;
    return r;
  }
  if (row_bytes <= kSmemCap) {
    r.K = 1;
    int64_t rpu = std::max<int64_t>(1, (48 * 1024) / row_bytes);
    rpu = std::min<int64_t>(rpu, m);
    r.rows_per_unit = (int)std::max<int64_t>(1, rpu);
    r.smem = r.rows_per_unit * row_bytes;
    // narrow access words (the pitch or the base is not 16-byte aligned): the
    // peeled kernel moves the same bytes with 16-byte accesses (variant row=3
    // or T213_ROW_PEEL=0 keep the word-width kernel).  Measured on B200, for
    // elements of 4 bytes or less only: C2R row pass of fp32 (7919, 6151, 2)
    // 0.170 against 0.220 ms, (6151, 7919, 2) 0.143 against 0.199, (3951,
    // 3210, 4) 0.131 against 0.166; fp64 (7919, 6151, 2) 0.294 against 0.281
    // (8-byte words already carry most of the gain).
    const char *pe = std::getenv("T213_ROW_PEEL");
    r.peel = r.aw < 16 && eb <= 4 && pv.row != 3 && !(pe && std::atoi(pe) == 0);
    return r;
  }
  // Rows longer than shared memory: copied to the stream's workspace in
  // groups of about T213_ROW_GROUP_MB (default 64) and gathered from there,
  // mostly out of L2.  Measured on B200 this beats splitting each row over a
  // thread-block cluster and gathering element by element through DSMEM
  // (T213_ROW_VARIANT=cluster): 3.4-3.6 ms against 10.1 ms for the R2C row
  // pass of (89, 675165, 8) fp32, 3.7 against 7.9 ms on (344, 359054, 4).
  int K = (int)((row_bytes + kSmemTarget - 1) / kSmemTarget);
  if (K > kMaxCluster) K = (int)((row_bytes + kSmemCap - 1) / kSmemCap);
  if (K <= kMaxCluster && var && std::strcmp(var, "cluster") == 0) {
    r.K = K;
    r.part = round_up((n + K - 1) / K, P);
    r.smem = r.part * eb;
    return r;
  }
  r.K = 0;
  const int64_t group_mb = env_int("T213_ROW_GROUP_MB") > 0 ? env_int("T213_ROW_GROUP_MB") : 64;
  r.group_rows = std::max<int64_t>(1, (group_mb << 20) / row_bytes);
  return r;
}

template <typename Kern>
int prep_kernel(Kern kern, int64_t smem, int K) {
  if (!kernel_attr_once((const void *)kern, smem, K)) return cuda_status(cudaGetLastError(), "cudaFuncSetAttribute");
  return T213_OK;
}

// Grid size: resident CTAs (or clusters x K), capped by the number of units.
template <typename Kern>
int64_t persistent_grid(Kern kern, int threads, int64_t smem, int K, int64_t units) {
  const DevInfo &d = dev_info();
  int v = 1;
  occupancy_cached((const void *)kern, threads, smem, K, &v);
  if (K <= 1) return std::max<int64_t>(1, std::min<int64_t>((int64_t)v * d.sms, units));
  return std::max<int64_t>(1, std::min<int64_t>(v, units)) * K;
}

template <typename Kern, typename... Args>
int launch_k(Kern kern, int64_t grid, int threads, int64_t smem, int K, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid, 1, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = (size_t)smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  if (K > 1) {
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = K;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
  }
  cudaError_t e = cudaLaunchKernelEx(&cfg, kern, args...);
  if (e != cudaSuccess) return cuda_status(e, "cudaLaunchKernelEx");
  return T213_OK;
}

}  // namespace

int col_local_form(const FnSpec &f, int64_t m) {
  if (m <= 0 || !local_params_ok(f, m)) return 0;
  return local_form(f.kind);
}

bool fits32(const FnSpec &f, int64_t m, int64_t n) {
  const int64_t lim = (int64_t)1 << 31;
  // generous common bound: every functor's intermediates are below about
  // 3*m*n + 3*(m+n); the c2r shuffle also forms k*b' with k, b' < b, and the
  // r2c permuters form products below a*a and c*m.
  if (m <= 0 || n <= 0) return true;
  if (m > lim / 4 || n > lim / 4) return false;
  if ((double)m * (double)n * 3.0 + 3.0 * (double)(m + n) >= (double)lim) return false;
  for (int q = 0; q < 4; q++)
    if (f.p[q] < 0 || f.p[q] >= lim / 4) return false;
  if (f.kind == T213_FN_C2R_SHUFFLE || f.kind == T213_FN_C2R_LONG_SHUFFLE) {
    int64_t c = f.p[2] > 0 ? f.p[2] : 1;
    int64_t b = f.p[1] / c;
    if ((double)b * (double)b >= (double)lim) return false;
    if ((double)f.p[1] * (double)(f.p[0] + 1) + f.p[0] >= (double)lim) return false;
  }
  if (f.kind == T213_FN_R2C_FUSED_PREOP || f.kind == T213_FN_R2C_PREPERMUTER) {
    double a = (double)f.p[0], c = (double)f.p[1], mm = (double)f.p[2];
    if (f.kind == T213_FN_R2C_PREPERMUTER) {
      mm = (double)f.p[0];
      c = (double)f.p[2];
      a = mm / std::max(1.0, c);
    }
    if (a * (a + 1) >= (double)lim || c * (mm + c) >= (double)lim) return false;
  }
  if (f.kind == T213_FN_C2R_FUSED_POSTOP || f.kind == T213_FN_C2R_POSTPERMUTER) {
    double mm = (double)f.p[0], nn = (double)f.p[1], c = (double)f.p[2];
    if (mm * nn + nn >= (double)lim || mm * c >= (double)lim) return false;
  }
  if (f.kind == T213_FN_R2C_SHUFFLE) {
    double mm = (double)f.p[0], nn = (double)f.p[1];
    if (mm * nn + mm + nn >= (double)lim) return false;
  }
  return true;
}

// ------------------------------------------------------------------ column --
std::string describe_col_gather_fn(const FnSpec &f, int64_t m, int64_t n, int eb, const void *data) {
  LocalCfg lc = local_col_config(f, m, n, eb, data);
  if (lc.ok) {
    char buf[160];
    snprintf(buf, sizeof buf, "col_gather[local%s W=%lld cluster=%d halo=%lld smem=%lldK aw=%d%s]",
             lc.db ? " db" : "", (long long)lc.W, lc.K, (long long)lc.halo,
             (long long)((lc.db ? 2 : 1) * lc.smem / 1024), lc.aw, lc.peel ? " peeled" : "");
    return buf;
  }
  return describe_col_gather(m, n, eb, data);
}

std::string describe_col_gather(int64_t m, int64_t n, int eb, const void *data) {
  ColCfg c = col_config(m, n, eb, data);
  char buf[160];
  if (c.K == 0)
    snprintf(buf, sizeof buf, "col_gather[scratch W=%lld group=%lld aw=%d]", (long long)c.W,
             (long long)c.group_w, c.aw);
  else
    snprintf(buf, sizeof buf, "col_gather[W=%lld cluster=%d smem=%lldK aw=%d]", (long long)c.W, c.K,
             (long long)(c.smem / 1024), c.aw);
  return buf;
}

int count_col_gather(int64_t d3, int64_t m, int64_t n, int eb) {
  ColCfg c = col_config(m, n, eb, nullptr);
  if (c.K > 0) return 1;
  int64_t groups = (n + c.group_w - 1) / c.group_w;
  return (int)(2 * groups * d3);
}

namespace {

constexpr int kNoCluster = -1;  // launch_col_local_t: the cluster cannot be resident

// Clusters of K CTAs that can be resident at once (0 if none fits), cached.
int clusters_resident(const void *kern, int threads, int64_t smem, int K) {
  static std::mutex mu;
  static std::map<std::tuple<const void *, int64_t, int, int>, int> cache;
  const int dev = dev_info().id;
  const auto key = std::make_tuple(kern, smem, K, dev);
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)(K * 8), 1, 1);
  cfg.blockDim = dim3(threads, 1, 1);
  cfg.dynamicSmemBytes = (size_t)smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = K;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int v = 0;
  if (cudaOccupancyMaxActiveClusters(&v, kern, &cfg) != cudaSuccess) {
    cudaGetLastError();
    v = 0;
  }
  std::lock_guard<std::mutex> lk(mu);
  cache[key] = v;
  return v;
}

// Calls go(off, F, G) with the key offsets and the row maps of the functor's
// cluster-local form (local_form).
template <typename U, typename Go>
void with_local_maps(const FnSpec &f, int64_t m, Go &&go) {
  const int form = local_form(f.kind);
  if (form == 1) {
    with_col_fn<U>(f, m, [&](auto fn) -> bool {
      go(OffOfCol<U, decltype(fn)>{fn}, MapId<U>{}, MapId<U>{});
      return true;
    });
  } else if (form == 2) {  // p = {m, n', c}
    const int64_t cc = f.p[2] > 0 ? f.p[2] : 1, a = m / cc, b = f.p[1] / cc;
    int64_t binv = 0;
    if (a > 1) {
      ext_gcd(b % a, a, &binv);
      binv %= a;
      if (binv < 0) binv += a;
    }
    go(OffAffine<U, false>{FastDiv<U>((uint64_t)m)}, MapId<U>{}, PermR2CPre<U>(m, cc, binv));
  } else {  // form 3, p = {a, c, m, q}
    const int64_t cc = f.p[1] > 0 ? f.p[1] : 1, a = f.p[0] > 0 ? f.p[0] : 1;
    const int64_t q = ((f.p[3] % a) + a) % a;
    go(OffAffine<U, true>{FastDiv<U>((uint64_t)m)}, PermR2CPre<U>(m, cc, q), MapId<U>{});
  }
}

// k_col_local for one element size / access width / index width.
template <int EB, int AW, typename U>
int launch_col_local_t(const FnSpec &f, const LocalCfg &c, char *data, int64_t d3, int64_t m, int64_t n,
                       cudaStream_t st) {
  const int64_t n_strips = (n + c.W - 1) / c.W;
  const int64_t units = n_strips * d3;
  int status = T213_OK;
  auto go = [&](auto off, auto F, auto G) {
    using Off = decltype(off);
    using Fs = decltype(F);
    using Gs = decltype(G);
    int *stw = device_status_word(&status);
    if (!stw) return;
    if (c.db) {
      const int64_t buf_elems = (c.smem + 15) / 16 * 16 / EB;
      const int64_t smem2 = 2 * buf_elems * EB;
      if (c.K == 1) {
        auto kern = k_col_local_db<EB, AW, U, Off, Fs, Gs, false>;
        if ((status = prep_kernel(kern, smem2, 1))) return;
        const int64_t grid = persistent_grid(kern, kGatherThreads, smem2, 1, units);
        status = launch_k(kern, grid, kGatherThreads, smem2, 1, st, data, d3, (U)m, (U)n, (U)c.W, (U)c.WS, n_strips,
                          (U)c.H, (int)c.halo, off, F, G, buf_elems, stw);
      } else {
        auto kern = k_col_local_db<EB, AW, U, Off, Fs, Gs, true>;
        if ((status = prep_kernel(kern, smem2, c.K))) return;
        if (clusters_resident((const void *)kern, kGatherThreads, smem2, c.K) < 1) {
          status = kNoCluster;
          return;
        }
        const int64_t grid = persistent_grid(kern, kGatherThreads, smem2, c.K, units);
        status = launch_k(kern, grid, kGatherThreads, smem2, c.K, st, data, d3, (U)m, (U)n, (U)c.W, (U)c.WS,
                          n_strips, (U)c.H, (int)c.halo, off, F, G, buf_elems, stw);
      }
      return;
    }
    if (c.K == 1) {
      auto kern = k_col_local<EB, AW, U, Off, Fs, Gs, false>;
      if ((status = prep_kernel(kern, c.smem, 1))) return;
      const int64_t grid = persistent_grid(kern, kGatherThreads, c.smem, 1, units);
      status = launch_k(kern, grid, kGatherThreads, c.smem, 1, st, data, d3, (U)m, (U)n, (U)c.W, (U)c.WS, n_strips,
                        (U)c.H, (int)c.halo, off, F, G, stw);
    } else {
      auto kern = k_col_local<EB, AW, U, Off, Fs, Gs, true>;
      if ((status = prep_kernel(kern, c.smem, c.K))) return;
      if (clusters_resident((const void *)kern, kGatherThreads, c.smem, c.K) < 1) {
        // no GPC holds such a cluster: the caller takes another variant
        status = kNoCluster;
        return;
      }
      const int64_t grid = persistent_grid(kern, kGatherThreads, c.smem, c.K, units);
      status = launch_k(kern, grid, kGatherThreads, c.smem, c.K, st, data, d3, (U)m, (U)n, (U)c.W, (U)c.WS,
                        n_strips, (U)c.H, (int)c.halo, off, F, G, stw);
    }
  };
  with_local_maps<U>(f, m, go);
  return status;
}

// k_col_local_peel for one element size / index width.
template <int EB, typename U>
int launch_col_peel_t(const FnSpec &f, const LocalCfg &c, char *data, int64_t d3, int64_t m, int64_t n,
                      cudaStream_t st) {
  const int64_t n_strips = (n + c.W - 1) / c.W;
  const int64_t units = n_strips * d3;
  int status = T213_OK;
  auto go = [&](auto off, auto F, auto G) {
    using Off = decltype(off);
    using Fs = decltype(F);
    using Gs = decltype(G);
    int *stw = device_status_word(&status);
    if (!stw) return;
    if (c.K == 1) {
      auto kern = k_col_local_peel<EB, U, Off, Fs, Gs, false>;
      if ((status = prep_kernel(kern, c.smem, 1))) return;
      const int64_t grid = persistent_grid(kern, kGatherThreads, c.smem, 1, units);
      status = launch_k(kern, grid, kGatherThreads, c.smem, 1, st, data, d3, (U)m, (U)n, (U)c.W, (U)c.SB,
                        (U)c.max_slots, n_strips, (U)c.H, (int)c.halo, off, F, G, stw);
    } else {
      auto kern = k_col_local_peel<EB, U, Off, Fs, Gs, true>;
      if ((status = prep_kernel(kern, c.smem, c.K))) return;
      if (clusters_resident((const void *)kern, kGatherThreads, c.smem, c.K) < 1) {
        status = kNoCluster;
        return;
      }
      const int64_t grid = persistent_grid(kern, kGatherThreads, c.smem, c.K, units);
      status = launch_k(kern, grid, kGatherThreads, c.smem, c.K, st, data, d3, (U)m, (U)n, (U)c.W, (U)c.SB,
                        (U)c.max_slots, n_strips, (U)c.H, (int)c.halo, off, F, G, stw);
    }
  };
  with_local_maps<U>(f, m, go);
  return status;
}

}  // namespace

int launch_col_gather(const FnSpec &f, char *data, int64_t d3, int64_t m, int64_t n, int eb,
                      cudaStream_t st, LaunchStats *ls) {
  if (m <= 0 || n <= 0 || d3 <= 0) return T213_OK;
  const LocalCfg lc = local_col_config(f, m, n, eb, data);
  if (lc.ok && lc.peel) {
    int status = T213_ERR_UNSUPPORTED;
    if (eb == 4)
      status = lc.u64 ? launch_col_peel_t<4, uint64_t>(f, lc, data, d3, m, n, st)
                      : launch_col_peel_t<4, uint32_t>(f, lc, data, d3, m, n, st);
    else if (eb == 8)
      status = lc.u64 ? launch_col_peel_t<8, uint64_t>(f, lc, data, d3, m, n, st)
                      : launch_col_peel_t<8, uint32_t>(f, lc, data, d3, m, n, st);
    if (status != kNoCluster) {
      if (ls) ls->launches++;
      return status;
    }
  }
  if (lc.ok && !lc.peel) {
    int status = T213_ERR_UNSUPPORTED;
    auto run = [&](auto EBc, auto AWc) -> bool {
      constexpr int EB = decltype(EBc)::value;
      constexpr int AW = decltype(AWc)::value;
      status = lc.u64 ? launch_col_local_t<EB, AW, uint64_t>(f, lc, data, d3, m, n, st)
                      : launch_col_local_t<EB, AW, uint32_t>(f, lc, data, d3, m, n, st);
      return true;
    };
    dispatch_eb_aw(eb, lc.aw, run);
    if (status != kNoCluster) {
      if (ls) ls->launches++;
      return status;
    }
  }
  ColCfg c = col_config(m, n, eb, data);
  const bool u32 = fits32(f, m, n);
  int status = T213_OK;
  bool known = false;
  auto run = [&](auto EBc, auto AWc) -> bool {
    constexpr int EB = decltype(EBc)::value;
    constexpr int AW = decltype(AWc)::value;
    auto go = [&](auto UT) -> bool {
      using U = decltype(UT);
      return with_col_fn<U>(f, m, [&](auto fn) -> bool {
        using F = decltype(fn);
        known = true;
        if (c.K >= 1) {
          const int64_t n_strips = (n + c.W - 1) / c.W;
          const int64_t units = n_strips * d3;
          if (c.K == 1) {
            auto kern = k_col_gather<EB, AW, F, U, false>;
            if ((status = prep_kernel(kern, c.smem, 1))) return true;
            int64_t grid = persistent_grid(kern, kGatherThreads, c.smem, 1, units);
            status = launch_k(kern, grid, kGatherThreads, c.smem, 1, st, data, d3, (U)m, (U)n, (U)c.W,
                              (U)c.WS, n_strips, (U)c.H, fn);
          } else {
            auto kern = k_col_gather<EB, AW, F, U, true>;
            if ((status = prep_kernel(kern, c.smem, c.K))) return true;
            int64_t grid = persistent_grid(kern, kGatherThreads, c.smem, c.K, units);
            status = launch_k(kern, grid, kGatherThreads, c.smem, c.K, st, data, d3, (U)m, (U)n,
                              (U)c.W, (U)c.WS, n_strips, (U)c.H, fn);
          }
          if (ls) ls->launches++;
          return true;
        }
        // scratch fallback
        const int64_t gw_max = c.group_w;
        char *scr = workspace(st, (size_t)(m * gw_max * eb), &status);
        if (!scr) return true;
        auto kern = k_col_gather_scratch<EB, AW, F, U>;
        const DevInfo &d = dev_info();
        for (int64_t k = 0; k < d3 && status == T213_OK; k++) {
          char *slice = data + k * m * n * eb;
          for (int64_t j = 0; j < n && status == T213_OK; j += gw_max) {
            const int64_t gw = std::min<int64_t>(gw_max, n - j);
            cudaError_t e = cudaMemcpy2DAsync(scr, (size_t)(gw * eb), slice + j * eb, (size_t)(n * eb),
                                              (size_t)(gw * eb), (size_t)m, cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) {
              status = cuda_status(e, "cudaMemcpy2DAsync");
              break;
            }
            int64_t words = m * (gw * eb / AW);
            int64_t grid = std::min<int64_t>((int64_t)d.sms * 4, (words + kGatherThreads - 1) / kGatherThreads);
            status = launch_k(kern, std::max<int64_t>(1, grid), kGatherThreads, 0, 1, st, slice,
                              (const char *)scr, (U)m, (U)n, (U)j, (U)gw, fn);
            if (ls) ls->launches += 2;
          }
        }
        return true;
      });
    };
    return u32 ? go(uint32_t{}) : go(uint64_t{});
  };
  if (!dispatch_eb_aw(eb, c.aw, run)) {
    set_error("unsupported element size");
    return T213_ERR_UNSUPPORTED;
  }
  if (!known) {
    set_error("functor kind is not a column gather");
    return T213_ERR_INVALID_ARGUMENT;
  }
  return status;
}

// --------------------------------------------------------------------- row --
std::string describe_row_gather(int64_t m, int64_t n, int eb, const void *data) {
  RowCfg r = row_config(m, n, eb, data);
  char buf[160];
  if (r.K == 0)
    snprintf(buf, sizeof buf, "row_gather[scratch rows/group=%lld aw=%d]", (long long)r.group_rows, r.aw);
  else if (r.pipe)
    snprintf(buf, sizeof buf, "row_gather[pipelined rows/unit=%d smem=2x%lldK aw=%d]", r.rows_per_unit,
             (long long)(r.buf_bytes / 1024), r.aw);
  else if (r.K == 1)
    snprintf(buf, sizeof buf, "row_gather[rows/unit=%d smem=%lldK aw=%d%s]", r.rows_per_unit,
             (long long)(r.smem / 1024), r.peel ? 16 : r.aw, r.peel ? " peeled" : "");
  else
    snprintf(buf, sizeof buf, "row_gather[cluster=%d part=%lld aw=%d]", r.K, (long long)r.part, r.aw);
  return buf;
}

int count_row_gather(int64_t d3, int64_t m, int64_t n, int eb) {
  RowCfg r = row_config(m, n, eb, nullptr);
  if (r.K > 0) return 1;
  int64_t rows = d3 * m;
  return (int)(2 * ((rows + r.group_rows - 1) / r.group_rows));
}

int launch_row_gather(const FnSpec &f, char *data, int64_t d3, int64_t m, int64_t n, int eb,
                      cudaStream_t st, LaunchStats *ls) {
  if (m <= 0 || n <= 0 || d3 <= 0) return T213_OK;
  RowCfg r = row_config(m, n, eb, data);
  const bool u32 = fits32(f, m, n);
  int status = T213_OK;
  bool known = false;
  const int64_t total_rows = d3 * m;
  auto run = [&](auto EBc, auto AWc) -> bool {
    constexpr int EB = decltype(EBc)::value;
    constexpr int AW = decltype(AWc)::value;
    constexpr int PER = AW / EB;
    auto go = [&](auto UT) -> bool {
      using U = decltype(UT);
      return with_row_fn<U>(f, [&](auto fn) -> bool {
        using F = decltype(fn);
        known = true;
        FastDiv<U> wpr((uint64_t)(n / PER));
        FastDiv<U> md((uint64_t)m);
        if (r.pipe) {
          auto kern = k_row_pipe<EB, AW, F, U>;
          if ((status = prep_kernel(kern, r.smem, 1))) return true;
          const int64_t units = (total_rows + r.rows_per_unit - 1) / r.rows_per_unit;
          int64_t grid = persistent_grid(kern, kGatherThreads, r.smem, 1, units);
          status = launch_k(kern, grid, kGatherThreads, r.smem, 1, st, data, total_rows, (U)m, (U)n,
                            r.rows_per_unit, r.buf_bytes, wpr, md, fn);
          if (ls) ls->launches++;
          return true;
        }
        if (r.K == 1 && r.peel) {
          if constexpr (EB < 16) {
            auto kern = k_row_gather_peel<EB, F, U>;
            const int64_t smem = r.smem + 32;  // the 16-byte blocks that cover a unit
            if ((status = prep_kernel(kern, smem, 1))) return true;
            const int64_t units = (total_rows + r.rows_per_unit - 1) / r.rows_per_unit;
            int64_t grid = persistent_grid(kern, kGatherThreads, smem, 1, units);
            status = launch_k(kern, grid, kGatherThreads, smem, 1, st, data, total_rows, (U)m, (U)n,
                              r.rows_per_unit, FastDiv<U>((uint64_t)n), md, fn);
            if (ls) ls->launches++;
            return true;
          }
        }
        if (r.K == 1) {
          auto kern = k_row_gather<EB, AW, F, U, false>;
          if ((status = prep_kernel(kern, r.smem, 1))) return true;
          const int64_t units = (total_rows + r.rows_per_unit - 1) / r.rows_per_unit;
          int64_t grid = persistent_grid(kern, kGatherThreads, r.smem, 1, units);
          status = launch_k(kern, grid, kGatherThreads, r.smem, 1, st, data, total_rows, (U)m, (U)n,
                            r.rows_per_unit, (U)0, wpr, md, fn);
          if (ls) ls->launches++;
          return true;
        }
        if (r.K > 1) {
          auto kern = k_row_gather<EB, AW, F, U, true>;
          if ((status = prep_kernel(kern, r.smem, r.K))) return true;
          int64_t grid = persistent_grid(kern, kGatherThreads, r.smem, r.K, total_rows);
          status = launch_k(kern, grid, kGatherThreads, r.smem, r.K, st, data, total_rows, (U)m, (U)n, 1,
                            (U)r.part, wpr, md, fn);
          if (ls) ls->launches++;
          return true;
        }
        // scratch fallback: groups of whole rows
        const int64_t row_bytes = n * EB;
        char *scr = workspace(st, (size_t)(r.group_rows * row_bytes), &status);
        if (!scr) return true;
        auto kern = k_row_gather_scratch<EB, AW, F, U>;
        const DevInfo &d = dev_info();
        for (int64_t r0 = 0; r0 < total_rows && status == T213_OK; r0 += r.group_rows) {
          const int64_t nr = std::min<int64_t>(r.group_rows, total_rows - r0);
          cudaError_t e = cudaMemcpyAsync(scr, data + r0 * row_bytes, (size_t)(nr * row_bytes),
                                          cudaMemcpyDeviceToDevice, st);
          if (e != cudaSuccess) {
            status = cuda_status(e, "cudaMemcpyAsync");
            break;
          }
          int64_t grid = std::min<int64_t>((int64_t)d.sms * 4,
                                           (n / PER + kGatherThreads - 1) / kGatherThreads);
          status = launch_k(kern, std::max<int64_t>(1, grid), kGatherThreads, 0, 1, st, data,
                            (const char *)scr, r0, nr, (U)m, (U)n, wpr, fn);
          if (ls) ls->launches += 2;
        }
        return true;
      });
    };
    return u32 ? go(uint32_t{}) : go(uint64_t{});
  };
  if (!dispatch_eb_aw(eb, r.aw, run)) {
    set_error("unsupported element size");
    return T213_ERR_UNSUPPORTED;
  }
  if (!known) {
    set_error("functor kind is not a row shuffle");
    return T213_ERR_INVALID_ARGUMENT;
  }
  return status;
}


// ------------------------------------------------------------------- slice --
namespace {

constexpr int64_t kSliceSmemCap = 220 * 1024;
constexpr int kSliceGroupK = 8;  // cluster size of the batched form's grouped slice launch

struct SliceCfg {
  int K = 0;
  uint32_t H = 0, P = 0;
  int64_t smem = 0;
  bool vec = false;
};

// Cluster size, rows per CTA and padded row pitch for one-pass slices; K = 0
// when the slice does not fit 16 CTAs.  The smallest cluster that holds the
// slice, doubled (up to 8) while the slices still leave SMs idle.
SliceCfg slice_config(int64_t m, int64_t n, int eb, int64_t d3, const void *data) {
  SliceCfg c;
  if (m < 2 || n < 2 || m > (1 << 24) || n > (1 << 24)) return c;
  int64_t P = (n * eb + 15) / 16 * 16;
  if ((P / 16) % 2 == 0) P += 16;  // consecutive rows in different 16-byte bank groups
  auto rows = [&](int K) -> int64_t {
    if (K == 1) return m;
    return ((m + K - 1) / K + 31) / 32 * 32;
  };
  int K = 0;
  for (int k : {1, 2, 4, 8, 16})
    if (rows(k) * P <= kSliceSmemCap) {
      K = k;
      break;
    }
  if (!K) return c;
  (void)d3;  // the launch widens the cluster when slices leave SMs idle
  c.K = K;
  c.H = (uint32_t)rows(K);
  c.P = (uint32_t)P;
  c.smem = (int64_t)c.H * P;
  c.vec = (n * eb) % 16 == 0 && (m * eb) % 16 == 0 && ((uintptr_t)data % 16) == 0;
  return c;
}

}  // namespace

bool slice_fits(int64_t m, int64_t n, int eb) { return slice_config(m, n, eb, 1, nullptr).K > 0; }

bool slice_group_params(int64_t m, int64_t n, int eb, const void *data, uint32_t *H, uint32_t *P, bool *vec) {
  if (m < 2 || n < 2 || m > (1 << 24) || n > (1 << 24)) return false;
  int64_t pitch = (n * eb + 15) / 16 * 16;
  if ((pitch / 16) % 2 == 0) pitch += 16;
  const int64_t rows = ((m + kSliceGroupK - 1) / kSliceGroupK + 31) / 32 * 32;
  if (rows * pitch > kSliceSmemCap) return false;
  *H = (uint32_t)rows;
  *P = (uint32_t)pitch;
  *vec = (n * eb) % 16 == 0 && (m * eb) % 16 == 0 && ((uintptr_t)data % 16) == 0;
  return true;
}

int launch_slice_group(const void *entries, int32_t n_entries, int64_t n_items, int64_t smem, cudaStream_t st) {
  if (n_items <= 0) return T213_OK;
  auto kern = k_slice_group<true>;
  int status = prep_kernel(kern, smem, kSliceGroupK);
  if (status) return status;
  const int res = clusters_resident((const void *)kern, kSliceThreads, smem, kSliceGroupK);
  if (res < 1) return cuda_status(cudaErrorInvalidConfiguration, "slice group cluster cannot be resident");
  const int64_t clusters = std::min<int64_t>(n_items, res);
  return launch_k(kern, clusters * kSliceGroupK, kSliceThreads, smem, kSliceGroupK, st,
                  (const SliceEntry *)entries, n_entries, n_items);
}

std::string describe_slice(int64_t m, int64_t n, int eb, int64_t d3) {
  SliceCfg c = slice_config(m, n, eb, d3, nullptr);
  char buf[96];
  snprintf(buf, sizeof buf, "slice(cluster=%d rows/cta=%u smem=%lldK)", c.K, c.H, (long long)(c.smem / 1024));
  return buf;
}

int launch_slice(char *data, int64_t d3, int64_t m, int64_t n, int eb, cudaStream_t st, LaunchStats *ls) {
  if (d3 <= 0 || m <= 0 || n <= 0) return T213_OK;
  const SliceCfg c0 = slice_config(m, n, eb, d3, data);
  if (!c0.K) {
    set_error("slice does not fit a cluster's shared memory");
    return T213_ERR_UNSUPPORTED;
  }
  int status = T213_ERR_UNSUPPORTED;
  auto go = [&](auto kern) {
    // The cluster size: from the smallest that holds a slice, doubled (up to
    // 8, with at least 32 rows per CTA) while that lowers waves x bytes per
    // CTA, the time of a launch in which every slice costs one CTA's load
    // and write of its share.  E.g. 16 slices of fp32 512 x 384 take 16
    // clusters of 4 (one wave of 198 KB per CTA), not 16 clusters of 8,
    // which would need two waves when 15 of them are resident.
    SliceCfg c = c0;
    auto cost = [&](const SliceCfg &x) -> double {
      int res = 0;
      if (x.K > 1) {
        if (prep_kernel(kern, x.smem, x.K)) return 1e30;
        res = clusters_resident((const void *)kern, kSliceThreads, x.smem, x.K);
      } else {
        if (prep_kernel(kern, x.smem, 1)) return 1e30;
        occupancy_cached((const void *)kern, kSliceThreads, x.smem, 1, &res);
        res *= dev_info().sms;
      }
      if (res < 1) return 1e30;
      return (double)((d3 + res - 1) / res) * (double)x.smem;
    };
    double best = cost(c);
    for (int K = c0.K * 2; K <= 8 && m / K >= 32; K *= 2) {
      SliceCfg x = c0;
      x.K = K;
      x.H = (uint32_t)(((m + K - 1) / K + 31) / 32 * 32);
      x.smem = (int64_t)x.H * x.P;
      const double cx = cost(x);
      if (cx < best) {
        best = cx;
        c = x;
      }
    }
    int64_t clusters = d3;
    if (c.K > 1) {
      const int res = clusters_resident((const void *)kern, kSliceThreads, c.smem, c.K);
      if (res < 1) {
        status = cuda_status(cudaErrorInvalidConfiguration, "slice cluster cannot be resident");
        return;
      }
      clusters = std::min<int64_t>(d3, res);
    } else {
      int per_sm = 1;
      occupancy_cached((const void *)kern, kSliceThreads, c.smem, 1, &per_sm);
      clusters = std::min<int64_t>(d3, (int64_t)std::max(1, per_sm) * dev_info().sms);
    }
    status = launch_k(kern, clusters * c.K, kSliceThreads, c.smem, c.K, st, data, d3, (uint32_t)m, (uint32_t)n, c.H,
                      c.P);
    if (ls) ls->launches++;
  };
  // a cluster kernel when the smallest cluster that holds a slice has more
  // than one CTA, else (one CTA per slice) the plain form
  auto pick = [&](auto EBc) {
    constexpr int EB = decltype(EBc)::value;
    if (c0.vec) {
      if (c0.K > 1 || m / 2 >= 32) go(k_slice<EB, true, true>);
      else go(k_slice<EB, true, false>);
    } else {
      if (c0.K > 1 || m / 2 >= 32) go(k_slice<EB, false, true>);
      else go(k_slice<EB, false, false>);
    }
  };
  switch (eb) {
    case 1: pick(IC<1>{}); break;
    case 2: pick(IC<2>{}); break;
    case 4: pick(IC<4>{}); break;
    case 8: pick(IC<8>{}); break;
    case 16: pick(IC<16>{}); break;
    default:
      set_error("unsupported element size");
      return T213_ERR_UNSUPPORTED;
  }
  return status;
}

}  // namespace t213
