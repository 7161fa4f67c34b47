// Cycle tables (host) and the launch of the segment-cycle walkers.
//
// The host lists every non-trivial cycle of a segment permutation with a
// visited bitmap (O(S) functor evaluations with the device's own arithmetic)
// and, in the same walk, cuts cycles longer than a target length into chunks
// so the walk spreads over the whole GPU.  Tables are cached per permutation and device
// and uploaded once; they are the "precomputed cycle leaders" of the pass.
#include <algorithm>
#include <cstdlib>
#include <cstdio>
#include <list>
#include <map>

#include "internal.h"
#include "k_cycles.cuh"

namespace t213 {

CycleTable::~CycleTable() {
  if (d_chunks) defer_free(dev, d_chunks);
  if (d_carry_items) defer_free(dev, d_carry_items);
  if (ready) cudaEventDestroy(ready);  // released once the event completes
}

namespace {
// Never destroyed: tables held by other translation units' caches can be
// released during static destruction at exit, after this file's statics.
std::mutex &grave_mu() {
  static std::mutex *m = new std::mutex;
  return *m;
}
std::vector<std::pair<int, void *>> &grave() {
  static auto *v = new std::vector<std::pair<int, void *>>;
  return *v;
}
constexpr size_t kGraveMax = 256;

void flush_locked() {
  auto &g_grave = grave();
  if (g_grave.empty()) return;
  int cur = 0;
  cudaGetDevice(&cur);
  std::vector<int> devs;
  for (auto &e : g_grave)
    if (std::find(devs.begin(), devs.end(), e.first) == devs.end()) devs.push_back(e.first);
  for (int d : devs) {
    cudaSetDevice(d);
    cudaDeviceSynchronize();  // nothing in flight can still read the tables
  }
  for (auto &e : g_grave) {
    cudaSetDevice(e.first);
    cudaFree(e.second);
  }
  g_grave.clear();
  cudaSetDevice(cur);
}
}  // namespace

void defer_free(int dev, void *p) {
  std::lock_guard<std::mutex> lk(grave_mu());
  grave().push_back({dev, p});
  if (grave().size() > kGraveMax) flush_locked();
}

void flush_deferred_frees() {
  std::lock_guard<std::mutex> lk(grave_mu());
  flush_locked();
}

namespace {

// One walk over the positions lists every non-trivial cycle and cuts it into
// chunks as it goes: the chunk length Lc is fixed up front from S (an upper
// bound of the moved positions) so that about 8 walker items exist per
// resident walker team, and the walk records the position at every Lc-th
// step of a cycle.  A cycle of at most Lc moves is one whole chunk (its walker
// reads the start itself); a longer one becomes chunks of Lc moves (the last
// one shorter) whose starts are saved to carry slots before the walkers run.
template <typename P>
int walk_and_chunk(const P &dst, int64_t S, int64_t items_per_chunk, std::vector<Chunk> &chunks,
                   std::vector<CarryItem> &carries, int64_t &n_cycles, int64_t &moved, int64_t &max_len) {
  const DevInfo &d = dev_info();
  const int64_t resident_teams = (int64_t)d.sms * 8;
  // T213_SEG_ITEMS: walker items per resident team (default 2); fewer means
  // longer chunks and fewer carry slots, more means finer load balance.
  // Measured on B200 (whole transpose, ms, 8 / 3 / 2 / 1 items): fp32
  // (8192, 6144, 4) 0.554 / 0.548 / 0.541 / 0.542; int32 (3, 2^22, 8) 0.294 /
  // 0.290 / 0.287 / 0.288; 16-byte (92, 1173128, 1) 1.317 / 1.305 / 1.279 /
  // 1.405; fp32 (2^24, 48, 1) 2.574 / 2.580 / 2.561 / 2.521.
  static const int64_t items_per_team = [] {
    const char *v = std::getenv("T213_SEG_ITEMS");
    return v && std::atoi(v) > 0 ? (int64_t)std::atoi(v) : (int64_t)2;
  }();
  const int64_t target_chunks =
      std::max<int64_t>(1, items_per_team * resident_teams / std::max<int64_t>(1, items_per_chunk));
  const int64_t Lc = std::max<int64_t>(16, (S + target_chunks - 1) / target_chunks);
  std::vector<uint64_t> seen((size_t)((S + 63) / 64), 0);
  std::vector<int64_t> marks;
  n_cycles = moved = max_len = 0;
  for (int64_t p = 0; p < S; p++) {
    if (seen[p >> 6] >> (p & 63) & 1) continue;
    marks.clear();
    int64_t x = p, len = 0, k = 0;
    do {
      if (x < 0 || x >= S || (seen[x >> 6] >> (x & 63) & 1)) {
        set_error("segment map is not a permutation of its index range");
        return T213_ERR_INVALID_ARGUMENT;
      }
      seen[x >> 6] |= 1ull << (x & 63);
      if (k == 0) {
        marks.push_back(x);
        k = Lc;
      }
      k--;
      x = (int64_t)dst(x);
      len++;
    } while (x != p);
    if (len < 2) continue;
    n_cycles++;
    moved += len;
    max_len = std::max(max_len, len);
    if (len <= Lc) {
      chunks.push_back({p, len, -1});
      continue;
    }
    for (size_t i = 0; i < marks.size(); i++) {
      const int64_t l = std::min<int64_t>(Lc, len - (int64_t)i * Lc);
      const int64_t slot = (int64_t)carries.size();
      carries.push_back({marks[i], slot});
      chunks.push_back({marks[i], l, slot});
    }
  }
  std::stable_sort(chunks.begin(), chunks.end(), [](const Chunk &a, const Chunk &b) { return a.len > b.len; });
  return T213_OK;
}

template <typename U, typename Fn>
bool with_perm(const PermSpec &p, Fn &&fn) {
  if (p.kind == 0) return fn(SegPerm3<U>(p.A, p.Mid, p.C));
  if (p.kind == T213_FN_C2R_POSTPERMUTER) return fn(PermC2RPost<U>(p.fn.p[0], p.fn.p[1], p.fn.p[2]));
  if (p.kind == T213_FN_R2C_PREPERMUTER) {
    // q = inverse of b = n/c modulo a = m/c (src/transpose.cu:77-82)
    int64_t m = p.fn.p[0], n = p.fn.p[1], c = p.fn.p[2];
    if (c <= 0) c = 1;
    int64_t a = m / c, b = n / c;
    // extended Euclid for b^{-1} mod a
    int64_t x = 0, lastx = 1, aa = b, bb = a;
    while (bb != 0) {
      int64_t q = aa / bb, nb = aa % bb;
      aa = bb;
      bb = nb;
      int64_t nx = lastx - q * x;
      lastx = x;
      x = nx;
    }
    int64_t q = (aa == 1) ? (lastx < 0 ? lastx + a : lastx) : 0;
    return fn(PermR2CPre<U>(m, c, q));
  }
  return false;
}

bool perm_fits32(const PermSpec &p) {
  if (p.kind == 0) {
    double s = (double)p.A * (double)p.Mid * (double)p.C;
    return s < (double)(1ll << 31);
  }
  return fits32(p.fn, p.fn.p[0], p.fn.p[1]);
}

struct Key {
  PermSpec spec;
  int64_t ipc;
  int dev;
};

// never destroyed, like the plan cache (no CUDA calls from static destructors)
std::mutex &g_mu = *new std::mutex;
auto &g_cache = *new std::list<std::pair<Key, std::shared_ptr<CycleTable>>>;  // front = most recent
constexpr size_t kCacheMax = 256;

}  // namespace

std::shared_ptr<CycleTable> get_cycle_table(const PermSpec &p, int64_t items_per_chunk, int *status) {
  *status = T213_OK;
  const int dev = dev_info().id;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto it = g_cache.begin(); it != g_cache.end(); ++it) {
      if (it->first.dev == dev && it->first.ipc == items_per_chunk && it->first.spec == p) {
        auto v = it->second;
        g_cache.splice(g_cache.begin(), g_cache, it);
        return v;
      }
    }
  }
  std::vector<Chunk> chunks;
  std::vector<CarryItem> carries;
  int64_t moved = 0, max_len = 0, n_cycles = 0;
  int rc = T213_OK;
  bool ok;
  auto build = [&](auto fn) -> bool {
    rc = walk_and_chunk(fn, p.S, items_per_chunk, chunks, carries, n_cycles, moved, max_len);
    return true;
  };
  if (perm_fits32(p))
    ok = with_perm<uint32_t>(p, build);
  else
    ok = with_perm<uint64_t>(p, build);
  if (!ok) {
    set_error("unknown segment permutation kind");
    *status = T213_ERR_INVALID_ARGUMENT;
    return nullptr;
  }
  if (rc != T213_OK) {
    *status = rc;
    return nullptr;
  }
  auto ct = std::make_shared<CycleTable>();
  ct->spec = p;
  ct->dev = dev;
  ct->n_chunks = (int64_t)chunks.size();
  ct->n_carry = (int64_t)carries.size();
  ct->moved = moved;
  ct->n_cycles = n_cycles;
  ct->max_len = max_len;
  ct->h_chunks.assign((const char *)chunks.data(), (const char *)(chunks.data() + chunks.size()));
  ct->h_carry_items.assign((const char *)carries.data(), (const char *)(carries.data() + carries.size()));
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_cache.push_front({Key{p, items_per_chunk, dev}, ct});
    while (g_cache.size() > kCacheMax) g_cache.pop_back();
  }
  return ct;
}

int CycleTable::ensure_uploaded(cudaStream_t st) {
  std::lock_guard<std::mutex> lk(mu);
  if (n_chunks == 0) return T213_OK;
  if (d_chunks) {
    if (ready_seen) return T213_OK;
    cudaError_t q = cudaEventQuery(ready);
    if (q == cudaSuccess) {
      ready_seen = true;
      return T213_OK;
    }
    if (q != cudaErrorNotReady) return cuda_status(q, "cycle table upload");
    if (st == upload_stream) return T213_OK;  // same stream: already ordered
    q = cudaStreamWaitEvent(st, ready, 0);
    return q == cudaSuccess ? T213_OK : cuda_status(q, "cycle table upload wait");
  }
  cudaError_t e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc(&d_chunks, h_chunks.size());
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_chunks, h_chunks.data(), h_chunks.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && n_carry > 0) {
    e = cudaMalloc(&d_carry_items, h_carry_items.size());
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_carry_items, h_carry_items.data(), h_carry_items.size(), cudaMemcpyHostToDevice, st);
  }
  if (e == cudaSuccess) e = cudaEventRecord(ready, st);
  if (e != cudaSuccess) {
    // nothing reads the tables yet; finish the stream before freeing them
    cudaStreamSynchronize(st);
    if (d_chunks) cudaFree(d_chunks);
    if (d_carry_items) cudaFree(d_carry_items);
    if (ready) cudaEventDestroy(ready);
    d_chunks = d_carry_items = nullptr;
    ready = nullptr;
    return cuda_status(e, "cycle table upload");
  }
  upload_stream = st;
  return T213_OK;
}

int CycleTable::wait_uploaded() {
  std::lock_guard<std::mutex> lk(mu);
  if (n_chunks == 0 || ready_seen) return T213_OK;
  if (!ready) {
    set_error("cycle table was never uploaded");
    return T213_ERR_INVALID_ARGUMENT;
  }
  cudaError_t e = cudaEventSynchronize(ready);
  if (e != cudaSuccess) return cuda_status(e, "cycle table upload");
  ready_seen = true;
  return T213_OK;
}

int seg_cycles_team(int64_t seg_bytes, int aw) {
  int64_t words = seg_bytes / aw;
  int64_t team = (words + 31) / 32 * 32;
  return (int)std::max<int64_t>(32, std::min<int64_t>(kCycleThreads, team));
}

size_t seg_cycles_carry_bytes(const CycleTable &ct, int64_t d3, int64_t seg_bytes) {
  return (size_t)(ct.n_carry * d3 * seg_bytes);
}

int launch_seg_cycles(const CycleTable &ct, char *data, int64_t d3, int64_t slice_bytes, int64_t seg_bytes,
                      cudaStream_t st, LaunchStats *ls, char *carry_override, size_t carry_override_bytes) {
  if (ct.n_chunks == 0 || d3 <= 0) return T213_OK;
  {
    int up = const_cast<CycleTable &>(ct).ensure_uploaded(st);
    if (up) return up;
  }
  const int aw = seg_access_width(data, seg_bytes, slice_bytes);
  const int team = seg_cycles_team(seg_bytes, aw);
  const int64_t words = seg_bytes / aw;
  const int64_t pieces = (words + team - 1) / team;
  const DevInfo &d = dev_info();
  int status = T213_OK;
  char *carry = nullptr;
  const size_t cb = seg_cycles_carry_bytes(ct, d3, seg_bytes);
  if (ct.n_carry > 0) {
    if (carry_override) {
      if (carry_override_bytes < cb) {
        set_error("carry buffer too small");
        return T213_ERR_INVALID_ARGUMENT;
      }
      carry = carry_override;
    } else {
      carry = workspace(st, cb, &status);
      if (!carry) return status;
    }
  }
  bool ok = false;
  // 16-byte-aligned segments of at least T213_SEG_BULK_MIN bytes (default 256)
  // take the bulk (TMA) walker, the others the register walker.  Measured on
  // B200: 704-byte segments (BANDS of (92, 1173128, 1) 16-byte) 0.735 ms bulk
  // against 1.967 ms register; 480-byte (BANDS_T of (552630, 125, 1) 16-byte)
  // 0.555 against 1.160 ms.
  const char *bm = std::getenv("T213_SEG_BULK_MIN");
  const Variant &pin = current_variant();
  const int64_t bulk_min =
      pin.seg == 3 ? INT64_MAX : pin.seg ? 256 : (bm && std::atoi(bm) >= 16 ? std::atoi(bm) : 256);
  if (aw == 16 && seg_bytes >= bulk_min) {
    // TMA bulk walker: pieces of up to 16 KB (T213_SEG_PIECE_KB), a ring of
    // 6 buffers (T213_SEG_RING=10 for 10)
    const char *pv = std::getenv("T213_SEG_PIECE_KB");
    const int64_t piece_cap = (pv && std::atoi(pv) > 0 ? std::atoi(pv) : 16) * 1024;
    const char *rv = std::getenv("T213_SEG_RING");
    const int ring = pin.seg == 2 ? 10 : pin.seg == 1 ? kBulkRing : (rv && std::atoi(rv) == 10) ? 10 : kBulkRing;
    const int64_t piece = std::min<int64_t>(seg_bytes, piece_cap);
    const int64_t npieces = (seg_bytes + piece - 1) / piece;
    const int64_t smem = 128 + (int64_t)ring * piece;
    int *stw = device_status_word(&status);
    if (!stw) return status;
    if (ct.n_carry > 0) {
      const int64_t total = ct.n_carry * d3 * (seg_bytes / 16);
      int64_t grid = std::min<int64_t>((int64_t)d.sms * 8, (total + kCycleThreads - 1) / kCycleThreads);
      k_carry_save<16><<<(unsigned)std::max<int64_t>(1, grid), kCycleThreads, 0, st>>>(
          data, slice_bytes, d3, seg_bytes, (const CarryItem *)ct.d_carry_items, ct.n_carry, carry);
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_status(e, "k_carry_save launch");
      if (ls) ls->launches++;
    }
    auto go = [&](auto UT) -> bool {
      using U = decltype(UT);
      return with_perm<U>(ct.spec, [&](auto dst) -> bool {
        using P = decltype(dst);
        auto kern = ring == 10 ? k_seg_cycles_bulk<P, U, 10> : k_seg_cycles_bulk<P, U, kBulkRing>;
        if (!kernel_attr_once((const void *)kern, smem, 1)) {
          status = cuda_status(cudaGetLastError(), "cudaFuncSetAttribute(bulk walker)");
          return true;
        }
        int per_sm = 1;
        occupancy_cached((const void *)kern, 32, smem, 1, &per_sm);
        cudaError_t e;
        const int64_t items = ct.n_chunks * npieces * d3;
        const int64_t grid = std::max<int64_t>(1, std::min<int64_t>((int64_t)per_sm * d.sms, items));
        kern<<<(unsigned)grid, 32, (size_t)smem, st>>>(data, slice_bytes, d3, seg_bytes, piece, npieces,
                                                      (const Chunk *)ct.d_chunks, ct.n_chunks, carry, dst, stw);
        e = cudaGetLastError();
        if (e != cudaSuccess) status = cuda_status(e, "k_seg_cycles_bulk launch");
        if (ls) ls->launches++;
        return true;
      });
    };
    ok = perm_fits32(ct.spec) ? go(uint32_t{}) : go(uint64_t{});
    if (!ok && status == T213_OK) {
      set_error("unknown segment permutation kind");
      return T213_ERR_INVALID_ARGUMENT;
    }
    return status;
  }
  auto run_aw = [&](auto AWc) -> bool {
    constexpr int AW = decltype(AWc)::value;
    if (ct.n_carry > 0) {
      const int64_t total = ct.n_carry * d3 * (seg_bytes / AW);
      int64_t grid = std::min<int64_t>((int64_t)d.sms * 8, (total + kCycleThreads - 1) / kCycleThreads);
      k_carry_save<AW><<<(unsigned)std::max<int64_t>(1, grid), kCycleThreads, 0, st>>>(
          data, slice_bytes, d3, seg_bytes, (const CarryItem *)ct.d_carry_items, ct.n_carry, carry);
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) {
        status = cuda_status(e, "k_carry_save launch");
        return true;
      }
      if (ls) ls->launches++;
    }
    auto go = [&](auto UT) -> bool {
      using U = decltype(UT);
      return with_perm<U>(ct.spec, [&](auto dst) -> bool {
        using P = decltype(dst);
        const int64_t items = ct.n_chunks * pieces * d3;
        const int64_t threads_needed = items * team;
        int64_t grid = std::min<int64_t>((int64_t)d.sms * (d.max_threads_sm / kCycleThreads),
                                         (threads_needed + kCycleThreads - 1) / kCycleThreads);
        grid = std::max<int64_t>(1, grid);
        k_seg_cycles<AW, 8, P, U><<<(unsigned)grid, kCycleThreads, 0, st>>>(
            data, slice_bytes, d3, seg_bytes, team, pieces, (const Chunk *)ct.d_chunks, ct.n_chunks, carry, dst);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) status = cuda_status(e, "k_seg_cycles launch");
        if (ls) ls->launches++;
        return true;
      });
    };
    if (perm_fits32(ct.spec))
      ok = go(uint32_t{});
    else
      ok = go(uint64_t{});
    return true;
  };
  switch (aw) {
    case 16:
      run_aw(IC<16>{});
      break;
    case 8:
      run_aw(IC<8>{});
      break;
    case 4:
      run_aw(IC<4>{});
      break;
    case 2:
      run_aw(IC<2>{});
      break;
    default:
      run_aw(IC<1>{});
      break;
  }
  if (!ok && status == T213_OK) {
    set_error("unknown segment permutation kind");
    return T213_ERR_INVALID_ARGUMENT;
  }
  return status;
}

}  // namespace t213
