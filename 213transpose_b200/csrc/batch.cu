// Batched form: many tensors of uneven shape and element size transposed by
// one persistent kernel launch (k_batch), captured in a CUDA graph on the
// first execute and replayed after that.  No reference counterpart: the
// reference offers only a loop of plain calls (t213_transpose_looped here).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <tuple>

#include "k_batch.cuh"
#include "k_slice.cuh"
#include "plan.h"

using namespace t213;

struct t213_batch_st {
  int dev = 0;
  std::vector<t213_tensor_desc> tensors;
  std::vector<std::shared_ptr<Plan>> plans;
  std::vector<BPass> h_passes;
  std::vector<BItem> h_items;
  // tensors run by their own plans as graph nodes after the persistent kernel:
  // larger than the direct threshold (bandwidth-bound on their own) or with a
  // plan that does not fit the persistent kernel's shared memory
  std::vector<int> spill;
  BPass *d_passes = nullptr;
  BItem *d_items = nullptr;
  unsigned long long *d_ctrs = nullptr;  // one per pass, then the queue head
  int *d_status = nullptr;
  char *d_carry = nullptr;
  size_t carry_bytes = 0;
  int n_ctrs = 0;
  int grid = 0;
  size_t spill_ws = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t graph_stream = nullptr;
  // the tensors run by their own plans go on this stream, forked from and
  // joined to the caller's, so they overlap the persistent kernel
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  std::string desc;
  int64_t total_bytes = 0;
  // limit of every dependency wait of the persistent kernel (nanoseconds of
  // %globaltimer); lowered only by t213_batch_debug_stall
  uint64_t wait_ns = kWaitNs;
  // small tensors transposed in one pass by a grouped cluster launch before
  // the persistent kernel (their slices fit an 8-CTA cluster's shared memory)
  std::vector<int> sliced;
  SliceEntry *d_slices = nullptr;
  int32_t n_slice_entries = 0;
  int64_t n_slice_items = 0, slice_smem = 0;
};

namespace {

struct BatchTables {
  std::vector<BPass> passes;
  std::vector<BItem> items;
  std::vector<size_t> carry_off;  // per cycle pass with carries (its CARRY and SEG passes share it)
  size_t carry_bytes = 0;
};

// Target bytes read per queue item: small enough that one tensor's pass
// spreads over many SMs (the batch's critical path is the chain of passes of
// its slowest tensor), large enough that the queue overhead stays small.
constexpr int64_t kItemBytes = 256 * 1024;

// Tensors above this size saturate the GPU on their own and keep their
// specialised kernels (graph nodes); smaller ones share the persistent kernel.
int64_t direct_threshold() {
  static int64_t v = [] {
    const char *e = getenv("T213_BATCH_DIRECT_MB");
    return (int64_t)((e ? atof(e) : 32.0) * (1 << 20));
  }();
  return v;
}

int aw_for(int eb, const void *data, int64_t pitch) {
  if (eb >= 16) return 16;
  if (eb >= 4 && ((((uintptr_t)data) | (uint64_t)pitch) % 16 == 0)) return 16;
  if (eb == 4 && ((((uintptr_t)data) | (uint64_t)pitch) % 8 == 0)) return 8;
  return eb;
}

template <typename U>
bool set_col_fn(AnyFn<U> &a, const FnSpec &f, int64_t m) {
  switch (f.kind) {
    case T213_FN_C2R_PREROTATOR:
      a.set(f.kind, RotGather<U, RotC2RPre<U>>(RotC2RPre<U>(f.p[0]), m));
      return true;
    case T213_FN_C2R_POSTROTATOR:
      a.set(f.kind, RotGather<U, RotC2RPost<U>>(RotC2RPost<U>(f.p[0]), m));
      return true;
    case T213_FN_R2C_PREROTATOR:
      a.set(f.kind, RotGather<U, RotR2CPre<U>>(RotR2CPre<U>(f.p[0]), m));
      return true;
    case T213_FN_R2C_POSTROTATOR:
      a.set(f.kind, RotGather<U, RotR2CPost<U>>(RotR2CPost<U>(f.p[0], f.p[1]), m));
      return true;
    case T213_FN_C2R_FUSED_PREOP:
      a.set(f.kind, ColC2RFusedPre<U>(f.p[0], f.p[1]));
      return true;
    case T213_FN_C2R_FUSED_POSTOP:
      a.set(f.kind, ColC2RFusedPost<U>(f.p[0], f.p[1], f.p[2]));
      return true;
    case T213_FN_R2C_FUSED_PREOP:
      a.set(f.kind, ColR2CFusedPre<U>(f.p[0], f.p[1], f.p[2], f.p[3]));
      return true;
    case T213_FN_R2C_FUSED_POSTOP:
      a.set(f.kind, ColR2CFusedPost<U>(f.p[0], f.p[1]));
      return true;
  }
  return false;
}

template <typename U>
bool set_row_fn(AnyFn<U> &a, const FnSpec &f) {
  if (f.kind == T213_FN_R2C_SHUFFLE) {
    a.set(f.kind, RowR2CShuffle<U>(f.p[0], f.p[1], f.p[2]));
    return true;
  }
  if (f.kind == T213_FN_C2R_SHUFFLE || f.kind == T213_FN_C2R_LONG_SHUFFLE) {
    a.set(f.kind, RowC2RShuffle<U>(f.p[0], f.p[1], f.p[2], f.p[3]));
    return true;
  }
  return false;
}

template <typename U>
bool set_perm_fn(AnyFn<U> &a, const PermSpec &p) {
  if (p.kind == 0) {
    a.set(0, SegPerm3<U>(p.A, p.Mid, p.C));
    return true;
  }
  if (p.kind == T213_FN_C2R_POSTPERMUTER) {
    a.set(p.kind, PermC2RPost<U>(p.fn.p[0], p.fn.p[1], p.fn.p[2]));
    return true;
  }
  if (p.kind == T213_FN_R2C_PREPERMUTER) {
    int64_t m = p.fn.p[0], n = p.fn.p[1], c = p.fn.p[2] > 0 ? p.fn.p[2] : 1, q;
    ext_gcd(n / c, m / c, &q);
    a.set(p.kind, PermR2CPre<U>(m, c, q));
    return true;
  }
  return false;
}

// Column strip width for the batch kernel (single CTA, <= kBatchSmem).
bool batch_col_cfg(int64_t m, int64_t n, int eb, int aw, int64_t &W, int64_t &WS) {
  const int64_t P = aw / eb;
  for (int64_t wbytes : {(int64_t)128, (int64_t)64, (int64_t)32, (int64_t)16}) {
    W = std::max<int64_t>(P, wbytes / eb);
    if (wbytes == 128) {
      int64_t want = (32 * 1024) / std::max<int64_t>(1, m * eb);
      if (want > W) W = want / W * W;
    }
    W = std::min<int64_t>(W, (n + P - 1) / P * P);
    W = (W + P - 1) / P * P;
    WS = (W * eb) % 128 == 0 ? W + P : W;
    if (m * WS * eb <= kBatchHalf) return true;
  }
  return false;
}

bool plan_fits_batch(const Plan &p) {
  for (const PassDesc &q : p.passes) {
    switch (q.type) {
      case PT_COL: {
        int64_t W, WS;
        if (!batch_col_cfg(q.m, q.n, p.eb, p.eb, W, WS)) return false;
        break;
      }
      case PT_ROW:
        if (q.n * p.eb > kBatchHalf) return false;
        break;
      case PT_BAND:
        if (q.R * q.C * p.eb > kBatchHalf) return false;
        break;
      case PT_SLICE:  // a cluster launch of its own; no executor in the persistent kernel
        return false;
      default:
        break;
    }
  }
  return true;
}

// Flattens the plans of the tensors (plans[i] null or skip[i] set: left out)
// into the persistent kernel's pass table and its level-ordered item queue,
// and lays out the carry pool the cycle passes need (bind_carry points them
// at it).
int build_batch_tables(const t213_tensor_desc *tensors, int32_t count, const std::vector<std::shared_ptr<Plan>> &plans,
                       const std::vector<char> &skip, BatchTables &T) {
  T.passes.clear();
  T.items.clear();
  T.carry_off.clear();
  T.carry_bytes = 0;
  // ---- passes ------------------------------------------------------------------
  size_t carry_total = 0;
  std::vector<size_t> &carry_off = T.carry_off;
  std::vector<std::vector<int>> tensor_passes(count);
  int rc = T213_OK;
  for (int32_t i = 0; i < count; i++) {
    const t213_tensor_desc &d = tensors[i];
    const std::shared_ptr<Plan> &P = plans[i];
    if (!P || skip[i]) continue;
    const int eb = d.elem_bytes;
    char *data = (char *)d.data;
    const int64_t slice_bytes = d.d1 * d.d2 * eb;
    for (const PassDesc &q : P->passes) {
      BPass bp;
      bp.eb = eb;
      bp.data = data;
      bp.d3 = d.d3;
      bp.slice_bytes = slice_bytes;
      bp.m = q.m;
      bp.n = q.n;
      switch (q.type) {
        case PT_TILE: {
          bp.kind = BK_TILE;
          bp.t = q.t;
          bp.Bm = q.m / q.t;
          bp.Bn = q.n / q.t;
          bp.nt = (q.t + 31) / 32;
          bp.pairs = bp.nt * (bp.nt + 1) / 2;
          bp.tile_vec = eb >= 4 && q.t % 32 == 0 && ((((uintptr_t)data) | (uint64_t)(q.n * eb)) % 16 == 0);
          bp.n_units = d.d3 * bp.Bm * bp.Bn * bp.pairs;
          break;
        }
        case PT_BAND: {
          bp.kind = BK_BAND;
          bp.R = q.R;
          bp.C = q.C;
          const int Q = 16 / eb;
          bp.band_vec = eb >= 2 && eb <= 8 && q.R % Q == 0 && q.C % Q == 0 && ((uintptr_t)data % 16 == 0);
          bp.n_units = d.d3 * q.bands;
          break;
        }
        case PT_COL: {
          bp.kind = BK_COL;
          bp.aw = aw_for(eb, data, q.n * eb);
          int64_t W, WS;
          if (!batch_col_cfg(q.m, q.n, eb, bp.aw, W, WS)) {
            bp.aw = eb;  // narrowest access width always fits (checked by plan_fits_batch)
            batch_col_cfg(q.m, q.n, eb, bp.aw, W, WS);
          }
          bp.W = W;
          bp.WS = WS;
          bp.n_strips = (q.n + W - 1) / W;
          bp.div_w = FastDiv<uint32_t>((uint64_t)(W / (bp.aw / eb)));
          bp.div_wl = FastDiv<uint32_t>((uint64_t)((q.n - (bp.n_strips - 1) * W) / (bp.aw / eb)));
          bp.n_units = d.d3 * bp.n_strips;
          bp.u64 = !fits32(q.fn, q.m, q.n);
          if (bp.u64)
            set_col_fn<uint64_t>(bp.f64, q.fn, q.m);
          else
            set_col_fn<uint32_t>(bp.f32, q.fn, q.m);
          // the cluster-local form: forms 2 and 3 carry the row permuter in
          // place of the functor (their key offsets are +-j mod m); at most
          // 256 columns per strip (the offsets' shared-memory table)
          bp.col_form = W <= kBatchAuxInts && std::getenv("T213_BATCH_COL_GENERIC") == nullptr
                            ? col_local_form(q.fn, q.m)
                            : 0;
          if (bp.col_form == 2 || bp.col_form == 3) {
            int64_t cc, qq;
            if (bp.col_form == 2) {  // p = {m, n', c}: inverse post-permuter, q = b^-1 mod a
              cc = q.fn.p[2] > 0 ? q.fn.p[2] : 1;
              const int64_t a = q.m / cc, b = q.fn.p[1] / cc;
              qq = 0;
              if (a > 1) {
                ext_gcd(b % a, a, &qq);
                qq %= a;
                if (qq < 0) qq += a;
              }
            } else {  // p = {a, c, m, q}: the pre-permuter
              cc = q.fn.p[1] > 0 ? q.fn.p[1] : 1;
              const int64_t a = q.fn.p[0] > 0 ? q.fn.p[0] : 1;
              qq = ((q.fn.p[3] % a) + a) % a;
            }
            if (bp.u64)
              bp.f64.set(T213_FN_R2C_PREPERMUTER, PermR2CPre<uint64_t>(q.m, cc, qq));
            else
              bp.f32.set(T213_FN_R2C_PREPERMUTER, PermR2CPre<uint32_t>(q.m, cc, qq));
          }
          bp.div_m = FastDiv<uint64_t>((uint64_t)q.m);
          bp.div_m32 = FastDiv<uint32_t>((uint64_t)q.m);
          if (bp.col_form && bp.aw < 16) bp.WS = bp.W;  // the diagonal reads are conflict-free unpadded
          break;
        }
        case PT_ROW: {
          bp.kind = BK_ROW;
          bp.aw = aw_for(eb, data, q.n * eb);
          bp.rows_per_unit = std::max<int64_t>(1, std::min<int64_t>(q.m, (64 * 1024) / std::max<int64_t>(1, q.n * eb)));
          bp.n_units = (d.d3 * q.m + bp.rows_per_unit - 1) / bp.rows_per_unit;
          // elements of at most 4 bytes on a pitch that is not a 16-byte
          // multiple: the peeled executor (16-byte words, stepped shuffles);
          // its divisor is then n itself
          bp.row_peel = bp.aw < 16 && eb <= 4 && std::getenv("T213_BATCH_ROW_WORDS") == nullptr &&
                        q.n * eb * bp.rows_per_unit + 32 <= kBatchHalf;
          bp.div_w = FastDiv<uint32_t>((uint64_t)(bp.row_peel ? q.n : q.n / (bp.aw / eb)));
          bp.div_m = FastDiv<uint64_t>((uint64_t)q.m);
          bp.u64 = !fits32(q.fn, q.m, q.n);
          if (bp.u64)
            set_row_fn<uint64_t>(bp.f64, q.fn);
          else
            set_row_fn<uint32_t>(bp.f32, q.fn);
          break;
        }
        case PT_SEG: {
          const CycleTable &ct = *q.table;
          if ((rc = const_cast<CycleTable &>(ct).ensure_uploaded(nullptr)) ||
              (rc = const_cast<CycleTable &>(ct).wait_uploaded()))
            return rc;
          bp.seg_bytes = q.seg_bytes;
          bp.seg_aw = seg_access_width(data, q.seg_bytes, slice_bytes);
          bp.chunks = (const Chunk *)ct.d_chunks;
          bp.carries = (const CarryItem *)ct.d_carry_items;
          bp.n_chunks = ct.n_chunks;
          bp.n_carry = ct.n_carry;
          bp.u64 = !(q.perm.kind == 0 ? (double)q.perm.S < 2.0e9 : fits32(q.perm.fn, q.perm.fn.p[0], q.perm.fn.p[1]));
          if (bp.u64)
            set_perm_fn<uint64_t>(bp.f64, q.perm);
          else
            set_perm_fn<uint32_t>(bp.f32, q.perm);
          if (ct.n_carry > 0) {
            BPass cp = bp;
            cp.kind = BK_CARRY;
            cp.n_units = ct.n_carry * d.d3;
            T.passes.push_back(cp);
            tensor_passes[i].push_back((int)T.passes.size() - 1);
            carry_off.push_back(carry_total);
            carry_total += (size_t)(ct.n_carry * d.d3 * q.seg_bytes + 255) / 256 * 256;
          }
          bp.kind = BK_SEG;
          bp.seg_tma = bp.seg_aw == 16 && q.seg_bytes >= 512;
          bp.piece_bytes = bp.seg_tma ? std::min<int64_t>(q.seg_bytes, kBatchPiece) : 32 * bp.seg_aw;
          bp.pieces = (q.seg_bytes + bp.piece_bytes - 1) / bp.piece_bytes;
          bp.n_units = ct.n_chunks * bp.pieces * d.d3;
          if (ct.n_carry > 0) carry_off.push_back(carry_off.back());  // same buffer as its CARRY pass
          break;
        }
      }
      if (bp.n_units == 0) continue;
      T.passes.push_back(bp);
      tensor_passes[i].push_back((int)T.passes.size() - 1);
    }
  }
  std::vector<int64_t> items_of_pass(T.passes.size(), 0);
  size_t max_levels = 0;
  for (auto &tp : tensor_passes) max_levels = std::max(max_levels, tp.size());
  for (size_t lvl = 0; lvl < max_levels; lvl++) {
    for (int32_t i = 0; i < count; i++) {
      if (lvl >= tensor_passes[i].size()) continue;
      const int pi = tensor_passes[i][lvl];
      BPass &bp = T.passes[pi];
      bp.done_ctr = pi;
      if (lvl > 0) {
        const int prev = tensor_passes[i][lvl - 1];
        bp.dep_ctr = prev;
        bp.dep_target = items_of_pass[prev];
      }
      // units per item: about kItemBytes read per item
      int64_t upi = 1;
      const int eb = bp.eb;
      auto per = [&](int64_t unit_bytes) { return std::max<int64_t>(1, kItemBytes / std::max<int64_t>(1, unit_bytes)); };
      switch (bp.kind) {
        case BK_TILE:
          upi = per(2 * 32 * 32 * eb);
          break;
        case BK_BAND:
          upi = per(bp.R * bp.C * eb);
          break;
        case BK_COL:
          upi = per(bp.m * bp.W * eb);
          break;
        case BK_ROW:
          upi = per(bp.rows_per_unit * bp.n * eb);
          break;
        case BK_CARRY:
          upi = per(bp.seg_bytes);
          break;
        case BK_SEG:
          // one chunk walk per warp: a walk is a chain of dependent loads,
          // so walks are spread over CTAs rather than queued behind each other
          upi = kBatchWarps;
          break;
      }
      for (int64_t u = 0; u < bp.n_units; u += upi) {
        T.items.push_back(BItem{pi, 0, u, std::min(bp.n_units, u + upi)});
        items_of_pass[pi]++;
      }
    }
  }
  T.carry_bytes = carry_total;
  return T213_OK;
}

void bind_carry(std::vector<BPass> &passes, const std::vector<size_t> &carry_off, char *pool) {
  size_t ci = 0;
  for (BPass &bp : passes)
    if ((bp.kind == BK_CARRY || bp.kind == BK_SEG) && bp.n_carry > 0) bp.carry_buf = pool + carry_off[ci++];
}

}  // namespace

namespace t213 {

std::shared_ptr<Plan> group_plan(int64_t d1, int64_t d2, int64_t d3, int eb, int *status, bool search_slice) {
  std::shared_ptr<Plan> P = get_plan(d1, d2, d3, eb, T213_PLAN_AUTO, 0, status);
  if (!P) return nullptr;
  if (plan_fits_batch(*P)) return P;
  // a tensor whose own plan is the one-pass slice plan runs best on its own
  // launch; searching the other families builds their cycle tables, which a
  // caller planning as requests arrive cannot afford
  if (P->kind == T213_PLAN_SLICE && !search_slice) return nullptr;
  // the cheapest other family whose passes fit the persistent kernel's
  // shared memory
  std::shared_ptr<Plan> best;
  for (int k : {T213_PLAN_BLOCKS, T213_PLAN_BANDS, T213_PLAN_BANDS_T, T213_PLAN_C2R, T213_PLAN_R2C,
                T213_PLAN_SKINNY}) {
    int rc2 = T213_OK;
    auto Q = get_plan(d1, d2, d3, eb, k, 0, &rc2);
    if (Q && plan_fits_batch(*Q) && (!best || Q->est_cost < best->est_cost)) best = Q;
  }
  return best;
}

struct GroupExec {
  int dev = 0;
  int64_t cap_passes = 0, cap_items = 0;
  size_t cap_carry = 0;
  BPass *d_passes = nullptr, *h_passes = nullptr;  // device table and its pinned staging
  BItem *d_items = nullptr, *h_items = nullptr;
  unsigned long long *d_ctrs = nullptr;  // one per pass, then the queue head
  int *d_status = nullptr, *h_status = nullptr;
  char *d_carry = nullptr;
  int grid = 0;
  cudaEvent_t done = nullptr;
  bool launched = false;
};

GroupExec *group_exec_create(int64_t max_passes, int64_t max_items, size_t carry_bytes, int *status) {
  *status = T213_OK;
  auto *g = new GroupExec();
  g->dev = dev_info().id;
  g->cap_passes = max_passes;
  g->cap_items = max_items;
  g->cap_carry = carry_bytes;
  cudaError_t e = cudaSuccess;
  if (!e) e = cudaMalloc(&g->d_passes, max_passes * sizeof(BPass));
  if (!e) e = cudaMallocHost(&g->h_passes, max_passes * sizeof(BPass));
  if (!e) e = cudaMalloc(&g->d_items, max_items * sizeof(BItem));
  if (!e) e = cudaMallocHost(&g->h_items, max_items * sizeof(BItem));
  if (!e) e = cudaMalloc(&g->d_ctrs, (max_passes + 1) * sizeof(unsigned long long));
  if (!e) e = cudaMalloc(&g->d_status, 256);
  if (!e) e = cudaMallocHost(&g->h_status, sizeof(int));
  if (!e && carry_bytes) e = cudaMalloc(&g->d_carry, carry_bytes);
  if (!e) e = cudaMemset(g->d_status, 0, 256);
  if (!e) e = cudaEventCreateWithFlags(&g->done, cudaEventDisableTiming);
  if (!e) e = cudaFuncSetAttribute(k_batch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)(kBatchSmem + kBatchBarBytes));
  if (!e) e = cudaDeviceSynchronize();  // the memset ran on the legacy stream
  if (e) {
    *status = cuda_status(e, "group executor");
    group_exec_destroy(g);
    return nullptr;
  }
  *g->h_status = 0;
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch, kBatchThreads,
                                                    (size_t)(kBatchSmem + kBatchBarBytes)) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  g->grid = per_sm * dev_info().sms;
  return g;
}

void group_exec_destroy(GroupExec *g) {
  if (!g) return;
  if (g->done) {
    cudaEventSynchronize(g->done);
    cudaEventDestroy(g->done);
  }
  cudaFree(g->d_passes);
  cudaFreeHost(g->h_passes);
  cudaFree(g->d_items);
  cudaFreeHost(g->h_items);
  cudaFree(g->d_ctrs);
  cudaFree(g->d_status);
  cudaFreeHost(g->h_status);
  cudaFree(g->d_carry);
  delete g;
}

bool group_exec_idle(GroupExec *g) { return !g->launched || cudaEventQuery(g->done) == cudaSuccess; }

int group_exec_status(GroupExec *g) { return *g->h_status; }

int group_exec_run(GroupExec *g, const t213_tensor_desc *tensors, int32_t count, cudaStream_t st) {
  std::vector<std::shared_ptr<Plan>> plans(count);
  for (int32_t i = 0; i < count; i++) {
    const t213_tensor_desc &d = tensors[i];
    if (d.d1 * d.d2 * d.d3 == 0) continue;
    int rc = T213_OK;
    plans[i] = group_plan(d.d1, d.d2, d.d3, d.elem_bytes, &rc, false);
    if (!plans[i]) return T213_ERR_UNSUPPORTED;
  }
  BatchTables T;
  int rc = build_batch_tables(tensors, count, plans, std::vector<char>(count, 0), T);
  if (rc) return rc;
  if ((int64_t)T.passes.size() > g->cap_passes || (int64_t)T.items.size() > g->cap_items ||
      T.carry_bytes > g->cap_carry)
    return T213_ERR_UNSUPPORTED;
  if (T.items.empty()) return T213_OK;
  bind_carry(T.passes, T.carry_off, g->d_carry);
  // the staging is free: the previous launch, and with it its table copies, finished
  memcpy(g->h_passes, T.passes.data(), T.passes.size() * sizeof(BPass));
  memcpy(g->h_items, T.items.data(), T.items.size() * sizeof(BItem));
  cudaError_t e = cudaMemcpyAsync(g->d_passes, g->h_passes, T.passes.size() * sizeof(BPass),
                                  cudaMemcpyHostToDevice, st);
  if (!e) e = cudaMemcpyAsync(g->d_items, g->h_items, T.items.size() * sizeof(BItem), cudaMemcpyHostToDevice, st);
  if (!e) e = cudaMemsetAsync(g->d_ctrs, 0, (T.passes.size() + 1) * sizeof(unsigned long long), st);
  if (e) return cuda_status(e, "group tables");
  k_batch<<<g->grid, kBatchThreads, (size_t)(kBatchSmem + kBatchBarBytes), st>>>(
      g->d_passes, g->d_items, (int64_t)T.items.size(), g->d_ctrs, g->d_ctrs + T.passes.size(), g->d_status,
      kWaitNs);
  e = cudaGetLastError();
  if (!e) e = cudaMemcpyAsync(g->h_status, g->d_status, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (!e) e = cudaMemsetAsync(g->d_status, 0, sizeof(int), st);
  if (!e) e = cudaEventRecord(g->done, st);
  if (e) return cuda_status(e, "group launch");
  g->launched = true;
  return T213_OK;
}

}  // namespace t213

extern "C" {

int t213_transpose_looped(const t213_tensor_desc *tensors, int32_t count, t213_stream_t stream) {
  if (count < 0 || (count > 0 && !tensors)) return T213_ERR_INVALID_ARGUMENT;
  for (int32_t i = 0; i < count; i++) {
    const t213_tensor_desc &d = tensors[i];
    int rc = d.plan_kind == T213_PLAN_AUTO
                 ? t213_transpose(d.data, d.d1, d.d2, d.d3, d.elem_bytes, stream)
                 : t213_transpose_with_plan(d.data, d.d1, d.d2, d.d3, d.elem_bytes, d.plan_kind, 0, stream);
    if (rc) return rc;
  }
  return T213_OK;
}

int t213_batch_create(const t213_tensor_desc *tensors, int32_t count, t213_batch *out) {
  if (!out || count < 0 || (count > 0 && !tensors)) {
    set_error("t213_batch_create: bad arguments");
    return T213_ERR_INVALID_ARGUMENT;
  }
  *out = nullptr;
  auto *B = new t213_batch_st();
  B->dev = dev_info().id;
  B->tensors.assign(tensors, tensors + count);
  int rc = T213_OK;
  auto fail = [&](int code) {
    t213_batch_destroy(B);
    return code;
  };

  // ---- plans ---------------------------------------------------------------
  for (int32_t i = 0; i < count; i++) {
    const t213_tensor_desc &d = tensors[i];
    if (d.d1 < 0 || d.d2 < 0 || d.d3 < 0 || (d.elem_bytes != 1 && d.elem_bytes != 2 && d.elem_bytes != 4 &&
                                              d.elem_bytes != 8 && d.elem_bytes != 16)) {
      set_error("t213_batch_create: bad tensor descriptor");
      return fail(T213_ERR_INVALID_ARGUMENT);
    }
    if (d.d1 * d.d2 * d.d3 > 0 && !d.data) {
      set_error("t213_batch_create: NULL data");
      return fail(T213_ERR_INVALID_ARGUMENT);
    }
    B->total_bytes += d.d1 * d.d2 * d.d3 * d.elem_bytes;
    std::shared_ptr<Plan> P;
    if (d.d1 * d.d2 * d.d3 > 0) {
      P = d.plan_kind == T213_PLAN_AUTO ? group_plan(d.d1, d.d2, d.d3, d.elem_bytes, &rc, true) : nullptr;
      if (!P) P = get_plan(d.d1, d.d2, d.d3, d.elem_bytes, d.plan_kind, 0, &rc);
      if (!P) return fail(rc);
      if (!plan_fits_batch(*P) || d.d1 * d.d2 * d.d3 * d.elem_bytes > direct_threshold()) B->spill.push_back(i);
    }
    B->plans.push_back(P);
  }

  // ---- one-pass slices (on request: T213_BATCH_SLICE=1) ------------------------
  // Measured on the 455 small tensors of the batched workload: 4.76 ms with
  // the 150 that fit taken out of the persistent kernel into one grouped
  // cluster launch, against 4.36 ms without; so it is off by default.
  std::vector<char> skip(count, 0);
  for (int i : B->spill) skip[i] = 1;
  {
    const char *sv = getenv("T213_BATCH_SLICE");
    const bool on = sv && atoi(sv) == 1;
    std::vector<SliceEntry> entries;
    for (int32_t i = 0; i < count && on; i++) {
      const t213_tensor_desc &d = tensors[i];
      if (skip[i] || !B->plans[i] || d.plan_kind != T213_PLAN_AUTO || d.d1 * d.d2 * d.d3 == 0) continue;
      uint32_t H = 0, P = 0;
      bool vec = false;
      // the element-wise form is kept for 8- and 16-byte elements, where it measured faster
      if (!slice_group_params(d.d2, d.d1, d.elem_bytes, d.data, &H, &P, &vec) || !(vec || d.elem_bytes >= 8))
        continue;
      SliceEntry e{};
      e.data = (char *)d.data;
      e.d3 = d.d3;
      e.first_item = B->n_slice_items;
      e.m = (uint32_t)d.d2;
      e.n = (uint32_t)d.d1;
      e.H = H;
      e.P = P;
      e.eb = d.elem_bytes;
      e.vec = vec ? 1 : 0;
      entries.push_back(e);
      B->n_slice_items += d.d3;
      B->slice_smem = std::max<int64_t>(B->slice_smem, (int64_t)H * P);
      B->sliced.push_back(i);
      skip[i] = 1;
    }
    if (!entries.empty()) {
      cudaError_t e = cudaMalloc(&B->d_slices, entries.size() * sizeof(SliceEntry));
      if (e == cudaSuccess)
        e = cudaMemcpy(B->d_slices, entries.data(), entries.size() * sizeof(SliceEntry), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) return fail(cuda_status(e, "batch slice entries"));
      B->n_slice_entries = (int32_t)entries.size();
    }
  }
  BatchTables T;
  if ((rc = build_batch_tables(tensors, count, B->plans, skip, T))) return fail(rc);
  B->h_passes = std::move(T.passes);
  B->h_items = std::move(T.items);
  // carry pool
  if (T.carry_bytes > 0) {
    cudaError_t e = cudaMalloc(&B->d_carry, T.carry_bytes);
    if (e != cudaSuccess) return fail(cuda_status(e, "batch carry pool"));
    B->carry_bytes = T.carry_bytes;
    bind_carry(B->h_passes, T.carry_off, B->d_carry);
  }
  B->n_ctrs = (int)B->h_passes.size();

  // ---- upload --------------------------------------------------------------
  cudaError_t e = cudaSuccess;
  if (!B->h_passes.empty()) {
    e = cudaMalloc(&B->d_passes, B->h_passes.size() * sizeof(BPass));
    if (e == cudaSuccess)
      e = cudaMemcpy(B->d_passes, B->h_passes.data(), B->h_passes.size() * sizeof(BPass), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess && !B->h_items.empty()) {
    e = cudaMalloc(&B->d_items, B->h_items.size() * sizeof(BItem));
    if (e == cudaSuccess)
      e = cudaMemcpy(B->d_items, B->h_items.data(), B->h_items.size() * sizeof(BItem), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMalloc(&B->d_ctrs, (B->n_ctrs + 1) * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&B->d_status, 256);
  if (e == cudaSuccess) e = cudaMemset(B->d_status, 0, 256);
  // the copies and the memset ran on the legacy stream; executes on
  // non-blocking streams are not ordered after it, so let them land here
  if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  if (e != cudaSuccess) return fail(cuda_status(e, "batch upload"));
  // workspace the spilled plans need during capture
  for (int i : B->spill) B->spill_ws = std::max(B->spill_ws, plan_workspace_bytes(*B->plans[i]));
  // grid: resident CTAs of the persistent kernel
  e = cudaFuncSetAttribute(k_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(kBatchSmem + kBatchBarBytes));
  if (e != cudaSuccess) return fail(cuda_status(e, "cudaFuncSetAttribute(k_batch)"));
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch, kBatchThreads,
                                                    (size_t)(kBatchSmem + kBatchBarBytes)) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  // With tensors on their own plans beside it, the persistent kernel takes
  // T213_BATCH_SMS SMs' worth of CTAs (default 96) and leaves the rest to
  // their bandwidth-bound kernels, which run concurrently on a side stream.
  // Measured on the 512-tensor workload: 12.07 ms with all 148 SMs, 11.73 ms
  // with 96, 11.80 with 64, 14.1 with 48 (the persistent kernel's share is
  // bound by its SMs' issue rate, not by latency).
  {
    const char *v = getenv("T213_BATCH_SMS");
    int sms = dev_info().sms;
    if (!B->spill.empty()) sms = std::min(sms, v && atoi(v) > 0 ? atoi(v) : 96);
    B->grid = per_sm * std::max(1, sms);
  }
  if (!B->spill.empty()) {
    if ((e = cudaStreamCreateWithFlags(&B->side, cudaStreamNonBlocking)) ||
        (e = cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming)) ||
        (e = cudaEventCreateWithFlags(&B->join, cudaEventDisableTiming)))
      return fail(cuda_status(e, "batch side stream"));
  }

  char buf[256];
  int64_t direct_bytes = 0;
  for (int i : B->spill) direct_bytes += tensors[i].d1 * tensors[i].d2 * tensors[i].d3 * tensors[i].elem_bytes;
  snprintf(buf, sizeof buf,
           "batch: %d tensors, %.1f MB; one-pass slices: %d tensors; persistent kernel: %d tensors, %zu passes, %zu "
           "items, grid %d x %d threads; graph nodes: %d tensors, %.1f MB",
           count, B->total_bytes / 1e6, (int)B->sliced.size(), count - (int)B->spill.size() - (int)B->sliced.size(),
           B->h_passes.size(), B->h_items.size(), B->grid, kBatchThreads, (int)B->spill.size(), direct_bytes / 1e6);
  B->desc = buf;
  *out = B;
  return T213_OK;
}

static int batch_enqueue(t213_batch B, cudaStream_t st) {
  cudaError_t e;
  if (!B->spill.empty()) {  // fork: the side stream starts after the caller's earlier work
    if ((e = cudaEventRecord(B->fork, st)) || (e = cudaStreamWaitEvent(B->side, B->fork, 0)))
      return cuda_status(e, "batch fork");
  }
  e = cudaMemsetAsync(B->d_ctrs, 0, (B->n_ctrs + 1) * sizeof(unsigned long long), st);
  if (e != cudaSuccess) return cuda_status(e, "batch counters reset");
  if (B->n_slice_entries > 0) {
    int rc = launch_slice_group(B->d_slices, B->n_slice_entries, B->n_slice_items, B->slice_smem, st);
    if (rc) return rc;
  }
  if (!B->h_items.empty()) {
    k_batch<<<B->grid, kBatchThreads, (size_t)(kBatchSmem + kBatchBarBytes), st>>>(
        B->d_passes, B->d_items, (int64_t)B->h_items.size(), B->d_ctrs, B->d_ctrs + B->n_ctrs, B->d_status,
        B->wait_ns);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, "k_batch launch");
  }
  for (int i : B->spill) {
    int rc = run_plan(*B->plans[i], (char *)B->tensors[i].data, B->side, nullptr);
    if (rc) return rc;
  }
  if (!B->spill.empty()) {  // join
    if ((e = cudaEventRecord(B->join, B->side)) || (e = cudaStreamWaitEvent(st, B->join, 0)))
      return cuda_status(e, "batch join");
  }
  return T213_OK;
}

int t213_batch_execute(t213_batch B, t213_stream_t stream) {
  if (!B) return T213_ERR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  if (B->exec && B->graph_stream == st) {
    cudaError_t e = cudaGraphLaunch(B->exec, st);
    return e == cudaSuccess ? T213_OK : cuda_status(e, "cudaGraphLaunch");
  }
  // first execute on this stream: reserve what capture cannot allocate, capture
  if (!B->spill.empty()) {
    int rc = T213_OK;
    if (B->spill_ws && !workspace(B->side, B->spill_ws, &rc)) return rc;
    for (int i : B->spill)
      for (const PassDesc &q : B->plans[i]->passes)
        if (q.table && ((rc = q.table->ensure_uploaded(B->side)) || (rc = q.table->wait_uploaded()))) return rc;
    int *w = device_status_word(&rc);
    if (!w) return rc;
  }
  if (st == nullptr) {
    // the legacy default stream cannot be captured: run without a graph
    return batch_enqueue(B, st);
  }
  if (B->exec) {
    cudaGraphExecDestroy(B->exec);
    B->exec = nullptr;
  }
  if (B->graph) {
    cudaGraphDestroy(B->graph);
    B->graph = nullptr;
  }
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return cuda_status(e, "cudaStreamBeginCapture");
  int rc = batch_enqueue(B, st);
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(st, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return cuda_status(e, "cudaStreamEndCapture");
  B->graph = g;
  e = cudaGraphInstantiate(&B->exec, g, 0);
  if (e != cudaSuccess) return cuda_status(e, "cudaGraphInstantiate");
  B->graph_stream = st;
  e = cudaGraphLaunch(B->exec, st);
  return e == cudaSuccess ? T213_OK : cuda_status(e, "cudaGraphLaunch");
}

int t213_batch_status(t213_batch B, t213_stream_t stream) {
  if (!B) return T213_ERR_INVALID_ARGUMENT;
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_status(e, "cudaStreamSynchronize");
  int v = 0;
  e = cudaMemcpy(&v, B->d_status, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_status(e, "batch status read");
  if (v) {
    if (cudaMemsetAsync(B->d_status, 0, sizeof(int), (cudaStream_t)stream) == cudaSuccess)
      cudaStreamSynchronize((cudaStream_t)stream);
    set_error("a bounded wait of the persistent batch kernel ran out");
  }
  return v;
}

int t213_batch_tune(const t213_tensor_desc *tensors, int32_t count, t213_stream_t stream) {
  if (count < 0 || (count > 0 && !tensors)) return T213_ERR_INVALID_ARGUMENT;
  // every distinct shape once
  std::map<std::tuple<int64_t, int64_t, int64_t, int>, int> rep;
  for (int32_t i = 0; i < count; i++) {
    const t213_tensor_desc &d = tensors[i];
    if (d.d1 <= 1 || d.d2 <= 1 || d.d3 <= 0) continue;
    rep.emplace(std::make_tuple(d.d1, d.d2, d.d3, d.elem_bytes), i);
  }
  int64_t maxb = 0;
  for (auto &kv : rep) {
    const t213_tensor_desc &d = tensors[kv.second];
    maxb = std::max<int64_t>(maxb, d.d1 * d.d2 * d.d3 * d.elem_bytes);
  }
  if (rep.empty()) return T213_OK;
  char *scratch = nullptr;
  cudaError_t e = cudaMalloc(&scratch, (size_t)maxb);
  if (e != cudaSuccess) return cuda_status(e, "tuning scratch");
  int rc = T213_OK;
  for (auto &kv : rep) {
    const t213_tensor_desc &d = tensors[kv.second];
    int32_t kind = 0;
    int64_t t = 0;
    rc = t213_tune_shape(scratch, d.d1, d.d2, d.d3, d.elem_bytes, stream, &kind, &t);
    if (rc) break;
  }
  cudaStreamSynchronize((cudaStream_t)stream);
  cudaFree(scratch);
  return rc;
}

int t213_batch_debug_stall(t213_batch B, int64_t wait_ns, int32_t stall_pass) {
  if (!B || wait_ns <= 0) return T213_ERR_INVALID_ARGUMENT;
  if (stall_pass < 0)
    for (size_t i = 0; i < B->h_passes.size() && stall_pass < 0; i++)
      if (B->h_passes[i].dep_ctr >= 0) stall_pass = (int32_t)i;
  if (stall_pass < 0 || stall_pass >= (int32_t)B->h_passes.size() || B->h_passes[stall_pass].dep_ctr < 0) {
    set_error("t213_batch_debug_stall: no pass with a dependency to stall");
    return T213_ERR_INVALID_ARGUMENT;
  }
  cudaError_t e = cudaDeviceSynchronize();  // no execute may still read the pass table
  if (e != cudaSuccess) return cuda_status(e, "t213_batch_debug_stall");
  // one item more than the predecessor pass has: its counter never gets there
  B->h_passes[stall_pass].dep_target += 1;
  e = cudaMemcpy(B->d_passes + stall_pass, &B->h_passes[stall_pass], sizeof(BPass), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_status(e, "t213_batch_debug_stall upload");
  B->wait_ns = (uint64_t)wait_ns;
  // the captured graph holds the old launch parameters
  if (B->exec) cudaGraphExecDestroy(B->exec);
  if (B->graph) cudaGraphDestroy(B->graph);
  B->exec = nullptr;
  B->graph = nullptr;
  B->graph_stream = nullptr;
  return T213_OK;
}

int t213_batch_describe(t213_batch B, char *buf, size_t buflen) {
  if (!B || !buf || !buflen) return T213_ERR_INVALID_ARGUMENT;
  snprintf(buf, buflen, "%s", B->desc.c_str());
  return T213_OK;
}

int t213_batch_destroy(t213_batch B) {
  if (!B) return T213_OK;
  cudaDeviceSynchronize();  // an execute may still be running; cudaFree does not wait for it
  if (B->exec) cudaGraphExecDestroy(B->exec);
  if (B->graph) cudaGraphDestroy(B->graph);
  if (B->d_passes) cudaFree(B->d_passes);
  if (B->d_items) cudaFree(B->d_items);
  if (B->d_ctrs) cudaFree(B->d_ctrs);
  if (B->d_status) cudaFree(B->d_status);
  if (B->d_carry) cudaFree(B->d_carry);
  if (B->d_slices) cudaFree(B->d_slices);
  if (B->side) {
    release_stream_workspace(B->side);
    cudaStreamDestroy(B->side);
  }
  if (B->fork) cudaEventDestroy(B->fork);
  if (B->join) cudaEventDestroy(B->join);
  delete B;
  return T213_OK;
}

}  // extern "C"
