// Launchers of the row-gather and column-gather passes: variant choice
// (single CTA, thread-block cluster, global-scratch fallback), access width,
// index width, and the functor dispatch.
#include <algorithm>
#include <cstdio>

#include "internal.h"
#include "k_gather.cuh"

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

int pick_aw(int eb, const void *data, int64_t pitch_bytes, int64_t extra_bytes) {
  if (eb >= 16) return 16;
  if (eb >= 4 && aligned16(data, pitch_bytes) && (extra_bytes & 15) == 0) return 16;
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

ColCfg col_config(int64_t m, int64_t n, int eb, const void *data) {
  ColCfg c;
  c.aw = pick_aw(eb, data, n * eb, 0);
  const int64_t P = c.aw / eb;
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

// --------------------------------------------------------------- row config --
struct RowCfg {
  int aw = 4;
  int K = 1;          // 0 = scratch fallback
  int rows_per_unit = 1;
  int64_t part = 0;   // elements per CTA when clustered
  int64_t smem = 0;
  int64_t group_rows = 0;
};

RowCfg row_config(int64_t m, int64_t n, int eb, const void *data) {
  RowCfg r;
  r.aw = pick_aw(eb, data, n * eb, 0);
  const int64_t P = r.aw / eb;
  const int64_t row_bytes = n * eb;
  if (row_bytes <= kSmemCap) {
    r.K = 1;
    int64_t rpu = std::max<int64_t>(1, (48 * 1024) / row_bytes);
    rpu = std::min<int64_t>(rpu, m);
    r.rows_per_unit = (int)std::max<int64_t>(1, rpu);
    r.smem = r.rows_per_unit * row_bytes;
    return r;
  }
  int K = (int)((row_bytes + kSmemTarget - 1) / kSmemTarget);
  if (K > kMaxCluster) K = (int)((row_bytes + kSmemCap - 1) / kSmemCap);
  if (K <= kMaxCluster) {
    r.K = K;
    r.part = round_up((n + K - 1) / K, P);
    r.smem = r.part * eb;
    return r;
  }
  r.K = 0;
  r.group_rows = std::max<int64_t>(1, (int64_t)(256ll << 20) / row_bytes);
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

int launch_col_gather(const FnSpec &f, char *data, int64_t d3, int64_t m, int64_t n, int eb,
                      cudaStream_t st, LaunchStats *ls) {
  if (m <= 0 || n <= 0 || d3 <= 0) return T213_OK;
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
  else if (r.K == 1)
    snprintf(buf, sizeof buf, "row_gather[rows/unit=%d smem=%lldK aw=%d]", r.rows_per_unit,
             (long long)(r.smem / 1024), r.aw);
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

}  // namespace t213
