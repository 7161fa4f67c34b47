// Serving runtime (include/t213_serve.h): HBM-budget admission into a device
// arena, continuous dispatch of admitted requests onto a stream pool,
// completion polling and latency statistics.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/t213_serve.h"
#include "plan.h"

namespace t213 {
namespace {

// splitmix64 finaliser (Vigna): the fill and the checksums are built on it.
__host__ __device__ __forceinline__ uint64_t smix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Word w (0 or 1) of element e of a request's tensor.
__device__ __forceinline__ uint64_t fill_word(uint64_t seed, uint64_t e, int w) {
  return smix(seed * 0xD1B54A32D192ED03ull ^ (e * 2 + (uint64_t)w));
}

// An element folded to 64 bits (the first eb bytes of its words).
__device__ __forceinline__ uint64_t fold(uint64_t w0, uint64_t w1, int eb) {
  if (eb >= 16) return w0 ^ ((w1 << 17) | (w1 >> 47));
  if (eb == 8) return w0;
  return w0 & ((1ull << (8 * eb)) - 1);
}

__device__ __forceinline__ uint64_t term(uint64_t pos, uint64_t v) { return smix(pos * 0x100000001B3ull ^ v); }

__device__ __forceinline__ void fill_elem(unsigned char *p, int64_t e, int eb, uint64_t seed) {
  const uint64_t w0 = fill_word(seed, (uint64_t)e, 0);
  switch (eb) {
    case 1:
      p[e] = (unsigned char)w0;
      break;
    case 2:
      reinterpret_cast<uint16_t *>(p)[e] = (uint16_t)w0;
      break;
    case 4:
      reinterpret_cast<uint32_t *>(p)[e] = (uint32_t)w0;
      break;
    case 8:
      reinterpret_cast<unsigned long long *>(p)[e] = w0;
      break;
    default: {
      const uint64_t w1 = fill_word(seed, (uint64_t)e, 1);
      reinterpret_cast<uint4 *>(p)[e] = make_uint4((uint32_t)w0, (uint32_t)(w0 >> 32), (uint32_t)w1, (uint32_t)(w1 >> 32));
    }
  }
}

__global__ void k_fill(unsigned char *p, int64_t nel, int eb, uint64_t seed) {
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nel; e += (int64_t)gridDim.x * blockDim.x)
    fill_elem(p, e, eb, seed);
}

__device__ __forceinline__ void reduce_add(uint64_t v, unsigned long long *out) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, (unsigned long long)v);
}

__device__ __forceinline__ uint64_t checksum_term(const unsigned char *p, int64_t e, int eb) {
  uint64_t w0 = 0, w1 = 0;
  switch (eb) {
    case 1:
      w0 = p[e];
      break;
    case 2:
      w0 = reinterpret_cast<const uint16_t *>(p)[e];
      break;
    case 4:
      w0 = reinterpret_cast<const uint32_t *>(p)[e];
      break;
    case 8:
      w0 = reinterpret_cast<const unsigned long long *>(p)[e];
      break;
    default: {
      const uint4 v = reinterpret_cast<const uint4 *>(p)[e];
      w0 = (uint64_t)v.x | ((uint64_t)v.y << 32);
      w1 = (uint64_t)v.z | ((uint64_t)v.w << 32);
    }
  }
  return term((uint64_t)e, fold(w0, w1, eb));
}

__global__ void k_checksum(const unsigned char *p, int64_t nel, int eb, unsigned long long *out) {
  uint64_t acc = 0;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nel; e += (int64_t)gridDim.x * blockDim.x)
    acc += checksum_term(p, e, eb);
  reduce_add(acc, out);
}

// A group of requests handled by one launch each of fill, transpose
// (k_batch) and checksum: blockIdx.y picks the request.
constexpr int kMaxGroup = 64;
struct GroupReq {
  unsigned char *p;
  int64_t nel;
  uint64_t seed;
  int32_t eb, pad;
};
struct GroupArgs {
  GroupReq r[kMaxGroup];
};

// also zeroes the request's checksum accumulator (read by k_checksum_group,
// which runs after the transpose on the same stream)
__global__ void k_fill_group(const GroupArgs a, unsigned long long *sums) {
  const GroupReq R = a.r[blockIdx.y];
  if (blockIdx.x == 0 && threadIdx.x == 0) sums[blockIdx.y] = 0;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < R.nel; e += (int64_t)gridDim.x * blockDim.x)
    fill_elem(R.p, e, R.eb, R.seed);
}

__global__ void k_checksum_group(const GroupArgs a, unsigned long long *sums) {
  const GroupReq R = a.r[blockIdx.y];
  uint64_t acc = 0;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < R.nel; e += (int64_t)gridDim.x * blockDim.x)
    acc += checksum_term(R.p, e, R.eb);
  reduce_add(acc, sums + blockIdx.y);
}

// Checksum a correct 213 transpose must have: output position o holds the
// element filled at source index src(o).
__global__ void k_checksum_expected(int64_t d1, int64_t d2, int64_t d3, int eb, uint64_t seed,
                                    unsigned long long *out) {
  const int64_t nel = d1 * d2 * d3;
  uint64_t acc = 0;
  for (int64_t o = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; o < nel; o += (int64_t)gridDim.x * blockDim.x) {
    const int64_t k = o / (d1 * d2), r = o - k * d1 * d2;
    const int64_t i1 = r / d2, i2 = r - i1 * d2;  // output is (d2 fastest, then d1)
    const uint64_t src = (uint64_t)(k * d1 * d2 + i2 * d1 + i1);
    uint64_t w0 = fill_word(seed, src, 0), w1 = eb >= 16 ? fill_word(seed, src, 1) : 0;
    if (eb < 8) w0 &= (1ull << (8 * eb)) - 1;
    acc += term((uint64_t)o, fold(w0, w1, eb));
  }
  reduce_add(acc, out);
}

// First-fit allocator over the device arena (host bookkeeping only).
class Arena {
 public:
  void reset(int64_t bytes) {
    free_.clear();
    if (bytes > 0) free_[0] = bytes;
    used_ = 0;
  }
  int64_t alloc(int64_t bytes) {
    bytes = (bytes + 255) / 256 * 256;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        const int64_t off = it->first, rest = it->second - bytes;
        free_.erase(it);
        if (rest > 0) free_[off + bytes] = rest;
        used_ += bytes;
        return off;
      }
    }
    return -1;
  }
  void release(int64_t off, int64_t bytes) {
    bytes = (bytes + 255) / 256 * 256;
    used_ -= bytes;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  int64_t used() const { return used_; }

 private:
  std::map<int64_t, int64_t> free_;
  int64_t used_ = 0;
};

int grid_for(int64_t nel) {
  const int64_t g = (nel + 255) / 256;
  return (int)std::max<int64_t>(1, std::min<int64_t>(g, (int64_t)dev_info().sms * 8));
}

}  // namespace
}  // namespace t213

using namespace t213;

// One grouped launch in flight: its executor (tables, k_batch), the
// checksums of its requests and the event after their copies.
struct ServeGroup {
  GroupExec *ex = nullptr;
  unsigned long long *d_sums = nullptr;
  unsigned long long *h_sums = nullptr;  // pinned
  cudaEvent_t ev = nullptr;
  int pending = 0;  // requests of the last launch not yet completed
};

struct t213_server_st {
  int dev = 0;
  char *arena = nullptr;
  int64_t arena_bytes = 0;
  int max_inflight = 64;
  std::vector<cudaStream_t> streams;
  unsigned long long *d_sums = nullptr;
  unsigned long long *h_sums = nullptr;  // pinned mirror
  std::vector<cudaEvent_t> events;
  Arena arena_map;
  std::vector<ServeGroup> groups;
  int64_t group_max_bytes = 0;  // requests up to this size may share a launch
};

namespace {

struct Slot {
  int req = -1;
  int64_t off = 0, bytes = 0;
  cudaEvent_t ev = nullptr;                 // completion of the request
  const unsigned long long *sum = nullptr;  // its checksum, valid after ev
  int group = -1;                           // the ServeGroup it ran in
};

// Copies a finished request's tensor out to the caller's buffer (stream
// ordered, before the completion event).
int enqueue_capture(void *out, const void *p, int64_t bytes, cudaStream_t st) {
  if (!out) return T213_OK;
  cudaError_t e = cudaMemcpyAsync(out, p, (size_t)bytes, cudaMemcpyDeviceToHost, st);
  return e == cudaSuccess ? T213_OK : cuda_status(e, "result copy");
}

int enqueue_request(t213_server s, const t213_request &r, int slot, int64_t off, cudaStream_t st, void *capture) {
  const int64_t nel = r.d1 * r.d2 * r.d3;
  unsigned char *p = (unsigned char *)s->arena + off;
  k_fill<<<grid_for(nel), 256, 0, st>>>(p, nel, r.elem_bytes, r.seed);
  int rc = r.plan_kind == T213_PLAN_AUTO
               ? t213_transpose(p, r.d1, r.d2, r.d3, r.elem_bytes, (t213_stream_t)st)
               : t213_transpose_with_plan(p, r.d1, r.d2, r.d3, r.elem_bytes, r.plan_kind, 0, (t213_stream_t)st);
  if (rc) return rc;
  cudaMemsetAsync(s->d_sums + slot, 0, sizeof(unsigned long long), st);
  k_checksum<<<grid_for(nel), 256, 0, st>>>(p, nel, r.elem_bytes, s->d_sums + slot);
  cudaMemcpyAsync(s->h_sums + slot, s->d_sums + slot, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
  if ((rc = enqueue_capture(capture, p, nel * r.elem_bytes, st))) return rc;
  cudaError_t e = cudaEventRecord(s->events[slot], st);
  if (e != cudaSuccess) return cuda_status(e, "cudaEventRecord");
  e = cudaGetLastError();
  return e == cudaSuccess ? T213_OK : cuda_status(e, "request launch");
}

// Several admitted requests in one launch of each kind: a grouped fill, one
// persistent k_batch over all their transposes, a grouped checksum.
// T213_ERR_UNSUPPORTED if the executor cannot take them; the grouped fill
// has been enqueued then, and the caller runs the requests one by one.
int enqueue_group(t213_server s, ServeGroup &G, const t213_request *reqs, const std::vector<int> &slot_ids,
                  std::vector<Slot> &slots, cudaStream_t st, void *const *capture) {
  const int n = (int)slot_ids.size();
  GroupArgs a{};
  std::vector<t213_tensor_desc> descs(n);
  int64_t max_nel = 0;
  for (int r = 0; r < n; r++) {
    const Slot &S = slots[slot_ids[r]];
    const t213_request &q = reqs[S.req];
    unsigned char *p = (unsigned char *)s->arena + S.off;
    a.r[r] = GroupReq{p, q.d1 * q.d2 * q.d3, q.seed, q.elem_bytes, 0};
    descs[r] = t213_tensor_desc{p, q.d1, q.d2, q.d3, q.elem_bytes, T213_PLAN_AUTO};
    max_nel = std::max(max_nel, q.d1 * q.d2 * q.d3);
  }
  const int gx = (int)std::max<int64_t>(
      1, std::min<int64_t>((max_nel + 255) / 256, std::max<int64_t>(1, (int64_t)dev_info().sms * 8 / n)));
  k_fill_group<<<dim3(gx, n), 256, 0, st>>>(a, G.d_sums);
  int rc = group_exec_run(G.ex, descs.data(), n, st);
  if (rc) return rc;
  k_checksum_group<<<dim3(gx, n), 256, 0, st>>>(a, G.d_sums);
  cudaError_t e = cudaMemcpyAsync(G.h_sums, G.d_sums, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return cuda_status(e, "group checksums");
  for (int r = 0; r < n; r++) {
    const Slot &S = slots[slot_ids[r]];
    if (capture && capture[S.req] && (rc = enqueue_capture(capture[S.req], a.r[r].p, a.r[r].nel * a.r[r].eb, st)))
      return rc;
  }
  e = cudaEventRecord(G.ev, st);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_status(e, "group launch");
  for (int r = 0; r < n; r++) {
    Slot &S = slots[slot_ids[r]];
    S.ev = G.ev;
    S.sum = G.h_sums + r;
    S.group = (int)(&G - s->groups.data());
  }
  G.pending = n;
  return T213_OK;
}

// Requests run one by one, each on the stream with its own event and checksum.
int enqueue_singles(t213_server s, const t213_request *reqs, const std::vector<int> &slot_ids,
                    std::vector<Slot> &slots, cudaStream_t st, void *const *capture) {
  for (int sl : slot_ids) {
    Slot &S = slots[sl];
    int rc = enqueue_request(s, reqs[S.req], sl, S.off, st, capture ? capture[S.req] : nullptr);
    if (rc) return rc;
    S.ev = s->events[sl];
    S.sum = s->h_sums + sl;
    S.group = -1;
  }
  return T213_OK;
}

// Plans requests on worker threads as they arrive, so that the dispatch loop
// only looks plans up: building a new shape's plan (its cycle tables above
// all) takes from microseconds to tens of milliseconds of host time, which a
// single dispatch thread would otherwise spend while the GPU idles.  For a
// request small enough to share a launch it also finds the plan the
// persistent kernel would run, and it notes whether the request's shape had
// to be planned (a cold request) or was found in the plan cache (warm).
class PlannerPool {
 public:
  PlannerPool(int dev, int threads, const t213_request *reqs, int n, int64_t group_max_bytes)
      : reqs_(reqs), planned_(n), groupable_(n, 0), cold_(n, 0) {
    for (auto &f : planned_) f.store(0, std::memory_order_relaxed);
    for (int i = 0; i < threads; i++)
      workers_.emplace_back([this, dev, group_max_bytes] {
        cudaSetDevice(dev);
        for (;;) {
          int ri;
          {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return stop_ || !queue_.empty(); });
            if (queue_.empty()) return;
            ri = queue_.front();
            queue_.pop_front();
          }
          const t213_request &r = reqs_[ri];
          int st = T213_OK;
          if (r.d1 > 0 && r.d2 > 0 && r.d3 > 0 &&
              (r.elem_bytes == 1 || r.elem_bytes == 2 || r.elem_bytes == 4 || r.elem_bytes == 8 ||
               r.elem_bytes == 16)) {
            cold_[ri] = !plan_cached(r.d1, r.d2, r.d3, r.elem_bytes, r.plan_kind, 0);
            get_plan(r.d1, r.d2, r.d3, r.elem_bytes, r.plan_kind, 0, &st);  // errors resurface at dispatch
            const int64_t bytes = r.d1 * r.d2 * r.d3 * r.elem_bytes;
            if (r.plan_kind == T213_PLAN_AUTO && bytes <= group_max_bytes)
              groupable_[ri] = group_plan(r.d1, r.d2, r.d3, r.elem_bytes, &st, false) != nullptr;
          }
          planned_[ri].store(1, std::memory_order_release);
        }
      });
  }
  ~PlannerPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
      queue_.clear();
    }
    cv_.notify_all();
    for (auto &w : workers_) w.join();
  }
  void submit(int ri) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      queue_.push_back(ri);
    }
    cv_.notify_one();
  }
  bool ready(int ri) const { return planned_[ri].load(std::memory_order_acquire) != 0; }
  // valid once ready(ri)
  bool groupable(int ri) const { return groupable_[ri] != 0; }
  bool cold(int ri) const { return cold_[ri] != 0; }

 private:
  const t213_request *reqs_;
  std::vector<std::atomic<int>> planned_;
  std::vector<char> groupable_, cold_;  // written by one worker before planned_ is released
  std::vector<std::thread> workers_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::deque<int> queue_;
  bool stop_ = false;
};

// Planner threads: T213_SERVE_PLANNERS, else all host threads but two (at
// most 16, at least 1).
int planner_threads() {
  const char *v = std::getenv("T213_SERVE_PLANNERS");
  if (v && std::atoi(v) > 0) return std::min(64, std::atoi(v));
  const int hw = (int)std::thread::hardware_concurrency();
  return std::max(1, std::min(16, hw - 2));
}

double percentile(std::vector<double> v, double p) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  size_t k = (size_t)std::min<double>((double)v.size() - 1, std::ceil(p * v.size()) - 1);
  return v[k];
}

}  // namespace

extern "C" {

int t213_server_create(int64_t hbm_budget_bytes, int32_t max_inflight, int32_t n_streams, t213_server *out) {
  if (!out || hbm_budget_bytes <= 0 || max_inflight <= 0 || n_streams <= 0) {
    set_error("t213_server_create: bad arguments");
    return T213_ERR_INVALID_ARGUMENT;
  }
  *out = nullptr;
  auto *s = new t213_server_st();
  s->dev = dev_info().id;
  s->max_inflight = max_inflight;
  size_t free_b = 0, total_b = 0;
  cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
  if (e != cudaSuccess) {
    delete s;
    return cuda_status(e, "cudaMemGetInfo");
  }
  // grouped launches: T213_SERVE_GROUPS executors (default 4, 0 = off) for
  // requests of at most T213_SERVE_GROUP_MB (default 32)
  const char *gv = std::getenv("T213_SERVE_GROUPS");
  const int n_groups = gv ? std::max(0, std::min(16, std::atoi(gv))) : 4;
  const char *gm = std::getenv("T213_SERVE_GROUP_MB");
  s->group_max_bytes = n_groups ? (int64_t)((gm ? atof(gm) : 32.0) * (1 << 20)) : 0;
  const size_t group_carry = (size_t)64 << 20;
  const int64_t margin = ((int64_t)2 << 30) + n_groups * (int64_t)(group_carry + (8 << 20));
  s->arena_bytes = std::min<int64_t>(hbm_budget_bytes, (int64_t)free_b - margin);
  if (s->arena_bytes <= 0) {
    delete s;
    set_error("not enough free device memory for the arena");
    return T213_ERR_OUT_OF_MEMORY;
  }
  auto fail = [&](cudaError_t err, const char *w) {
    int rc = cuda_status(err, w);
    t213_server_destroy(s);
    return rc;
  };
  if ((e = cudaMalloc(&s->arena, (size_t)s->arena_bytes))) return fail(e, "arena cudaMalloc");
  s->arena_map.reset(s->arena_bytes);
  if ((e = cudaMalloc(&s->d_sums, sizeof(unsigned long long) * max_inflight))) return fail(e, "sums");
  if ((e = cudaMallocHost(&s->h_sums, sizeof(unsigned long long) * max_inflight))) return fail(e, "pinned sums");
  for (int i = 0; i < n_streams; i++) {
    cudaStream_t st;
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking))) return fail(e, "stream");
    s->streams.push_back(st);
    int rc = T213_OK;
    if (!workspace(st, (size_t)64 << 20, &rc)) {  // carries of the cycle passes
      t213_server_destroy(s);
      return rc;
    }
  }
  for (int i = 0; i < max_inflight; i++) {
    cudaEvent_t ev;
    if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming))) return fail(e, "event");
    s->events.push_back(ev);
  }
  s->groups.resize(n_groups);
  for (ServeGroup &G : s->groups) {
    int rc = T213_OK;
    G.ex = group_exec_create(1024, 1 << 16, group_carry, &rc);
    if (!G.ex) {
      t213_server_destroy(s);
      return rc;
    }
    if ((e = cudaMalloc(&G.d_sums, sizeof(unsigned long long) * kMaxGroup))) return fail(e, "group sums");
    if ((e = cudaMallocHost(&G.h_sums, sizeof(unsigned long long) * kMaxGroup))) return fail(e, "group sums");
    if ((e = cudaEventCreateWithFlags(&G.ev, cudaEventDisableTiming))) return fail(e, "group event");
  }
  *out = s;
  return T213_OK;
}

int t213_server_run_capture(t213_server s, const t213_request *reqs, int32_t n, t213_serve_stats *stats,
                            uint64_t *checksums, double *latency_ms, void *const *outputs) {
  if (!s || n < 0 || (n > 0 && !reqs)) return T213_ERR_INVALID_ARGUMENT;
  using clk = std::chrono::steady_clock;
  std::vector<int> order(n);
  for (int i = 0; i < n; i++) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return reqs[a].arrival_s < reqs[b].arrival_s; });
  std::vector<double> lat(n, -1.0);
  std::vector<uint64_t> sums(n, 0);
  std::deque<int> pending;
  std::vector<Slot> slots(s->max_inflight);
  std::vector<int> free_slots;
  for (int i = s->max_inflight - 1; i >= 0; i--) free_slots.push_back(i);
  int next = 0, done = 0, rejected = 0, rr = 0;
  int64_t bytes_done = 0, peak = 0, max_inflight = 0, inflight = 0, group_launches = 0, grouped = 0;
  PlannerPool planners(s->dev, planner_threads(), reqs, n, s->group_max_bytes);
  const auto t0 = clk::now();
  auto now_s = [&]() { return std::chrono::duration<double>(clk::now() - t0).count(); };
  std::vector<int> grp;  // slots admitted in this round that may share a launch
  auto flush_group = [&]() -> int {
    if (grp.empty()) return T213_OK;
    cudaStream_t st = s->streams[rr++ % s->streams.size()];
    ServeGroup *G = nullptr;
    if (grp.size() >= 2)
      for (ServeGroup &g : s->groups)
        if (g.pending == 0 && group_exec_idle(g.ex)) {
          G = &g;
          break;
        }
    int rc = G ? enqueue_group(s, *G, reqs, grp, slots, st, outputs) : T213_ERR_UNSUPPORTED;
    if (rc == T213_OK) {
      group_launches++;
      grouped += (int64_t)grp.size();
    } else if (rc == T213_ERR_UNSUPPORTED) {
      rc = enqueue_singles(s, reqs, grp, slots, st, outputs);
    }
    grp.clear();
    return rc;
  };
  while (done + rejected < n) {
    bool progress = false;
    const double t = now_s();
    while (next < n && reqs[order[next]].arrival_s <= t) {
      planners.submit(order[next]);
      pending.push_back(order[next++]);
    }
    // completions
    for (int sl = 0; sl < s->max_inflight; sl++) {
      Slot &S = slots[sl];
      if (S.req < 0) continue;
      cudaError_t q = cudaEventQuery(S.ev);
      if (q == cudaErrorNotReady) continue;
      if (q != cudaSuccess) return cuda_status(q, "request completion");
      if (S.group >= 0) {
        ServeGroup &G = s->groups[S.group];
        if (group_exec_status(G.ex)) {
          set_error("a bounded wait of a grouped serving launch ran out");
          return T213_ERR_TIMEOUT;
        }
        G.pending--;
      }
      lat[S.req] = (now_s() - reqs[S.req].arrival_s) * 1e3;
      sums[S.req] = *S.sum;
      bytes_done += S.bytes;
      s->arena_map.release(S.off, S.bytes);
      S = Slot{};
      free_slots.push_back(sl);
      inflight--;
      done++;
      progress = true;
    }
    // admissions in arrival order among the requests whose plans are ready
    // (a request still being planned is passed over, not waited for; the
    // first one that does not fit the arena stops admission until memory
    // frees up, so large requests are not starved).  Small requests admitted
    // in the same round share one launch of each kernel.
    size_t pi = 0;
    while (pi < pending.size() && pi < 256 && !free_slots.empty()) {
      const int ri = pending[pi];
      const t213_request &r = reqs[ri];
      const int64_t bytes = r.d1 * r.d2 * r.d3 * r.elem_bytes;
      if (bytes > s->arena_bytes || r.d1 < 0 || r.d2 < 0 || r.d3 < 0) {
        pending.erase(pending.begin() + pi);
        rejected++;
        progress = true;
        continue;
      }
      if (bytes == 0) {
        pending.erase(pending.begin() + pi);
        lat[ri] = (now_s() - r.arrival_s) * 1e3;
        done++;
        progress = true;
        continue;
      }
      if (!planners.ready(ri)) {
        pi++;
        continue;
      }
      const int64_t off = s->arena_map.alloc(bytes);
      if (off < 0) break;  // wait for memory to free up
      pending.erase(pending.begin() + pi);
      const int sl = free_slots.back();
      free_slots.pop_back();
      slots[sl] = Slot{ri, off, bytes, nullptr, nullptr, -1};
      inflight++;
      max_inflight = std::max(max_inflight, inflight);
      peak = std::max(peak, s->arena_map.used());
      progress = true;
      if (!s->groups.empty() && planners.groupable(ri)) {
        grp.push_back(sl);
        if ((int)grp.size() == kMaxGroup) {
          int rc = flush_group();
          if (rc) return rc;
        }
        continue;
      }
      cudaStream_t st = s->streams[rr++ % s->streams.size()];
      int rc = enqueue_request(s, r, sl, off, st, outputs ? outputs[ri] : nullptr);
      if (rc) return rc;
      slots[sl].ev = s->events[sl];
      slots[sl].sum = s->h_sums + sl;
    }
    {
      int rc = flush_group();
      if (rc) return rc;
    }
    if (!progress) {
      // nothing to do until the next arrival or completion
      const double wait = next < n ? reqs[order[next]].arrival_s - now_s() : 0.0;
      if (wait > 50e-6)
        std::this_thread::sleep_for(std::chrono::microseconds(20));
      else
        std::this_thread::yield();
    }
  }
  const double wall = now_s();
  std::vector<double> ok, cold, warm;
  for (int i = 0; i < n; i++)
    if (lat[i] >= 0) {
      ok.push_back(lat[i]);
      (planners.cold(i) ? cold : warm).push_back(lat[i]);
    }
  if (stats) {
    *stats = t213_serve_stats{};
    stats->completed = done;
    stats->rejected = rejected;
    stats->bytes_done = bytes_done;
    stats->p50_ms = percentile(ok, 0.50);
    stats->p99_ms = percentile(ok, 0.99);
    double sum = 0;
    for (double v : ok) sum += v;
    stats->mean_ms = ok.empty() ? 0 : sum / ok.size();
    stats->max_ms = ok.empty() ? 0 : *std::max_element(ok.begin(), ok.end());
    stats->wall_s = wall;
    stats->peak_resident_bytes = peak;
    stats->max_inflight = max_inflight;
    stats->cold = (int64_t)cold.size();
    stats->p50_cold_ms = percentile(cold, 0.50);
    stats->p99_cold_ms = percentile(cold, 0.99);
    stats->p50_warm_ms = percentile(warm, 0.50);
    stats->p99_warm_ms = percentile(warm, 0.99);
    stats->group_launches = group_launches;
    stats->grouped_requests = grouped;
  }
  if (checksums) std::copy(sums.begin(), sums.end(), checksums);
  if (latency_ms) std::copy(lat.begin(), lat.end(), latency_ms);
  return T213_OK;
}

int t213_server_run(t213_server s, const t213_request *reqs, int32_t n, t213_serve_stats *stats, uint64_t *checksums,
                    double *latency_ms) {
  return t213_server_run_capture(s, reqs, n, stats, checksums, latency_ms, nullptr);
}

int t213_server_expected_checksum(t213_server s, const t213_request *r, uint64_t *checksum) {
  if (!s || !r || !checksum) return T213_ERR_INVALID_ARGUMENT;
  cudaStream_t st = s->streams[0];
  cudaMemsetAsync(s->d_sums, 0, sizeof(unsigned long long), st);
  const int64_t nel = r->d1 * r->d2 * r->d3;
  k_checksum_expected<<<grid_for(nel), 256, 0, st>>>(r->d1, r->d2, r->d3, r->elem_bytes, r->seed, s->d_sums);
  cudaError_t e = cudaMemcpyAsync(s->h_sums, s->d_sums, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(e, "expected checksum");
  *checksum = s->h_sums[0];
  return T213_OK;
}

int t213_server_run_alone(t213_server s, const t213_request *r, uint64_t *checksum) {
  if (!s || !r || !checksum) return T213_ERR_INVALID_ARGUMENT;
  const int64_t bytes = r->d1 * r->d2 * r->d3 * r->elem_bytes;
  if (bytes > s->arena_bytes) {
    set_error("request larger than the HBM budget");
    return T213_ERR_BUDGET;
  }
  const int64_t off = s->arena_map.alloc(bytes);
  if (off < 0) return T213_ERR_BUDGET;
  int rc = enqueue_request(s, *r, 0, off, s->streams[0], nullptr);
  cudaError_t e = cudaStreamSynchronize(s->streams[0]);
  s->arena_map.release(off, bytes);
  if (rc) return rc;
  if (e != cudaSuccess) return cuda_status(e, "run alone");
  *checksum = s->h_sums[0];
  return T213_OK;
}

int t213_server_destroy(t213_server s) {
  if (!s) return T213_OK;
  for (cudaStream_t st : s->streams) cudaStreamSynchronize(st);
  for (cudaEvent_t ev : s->events) cudaEventDestroy(ev);
  for (ServeGroup &G : s->groups) {
    group_exec_destroy(G.ex);
    if (G.ev) cudaEventDestroy(G.ev);
    if (G.d_sums) cudaFree(G.d_sums);
    if (G.h_sums) cudaFreeHost(G.h_sums);
  }
  for (cudaStream_t st : s->streams) {
    release_stream_workspace(st);
    cudaStreamDestroy(st);
  }
  if (s->arena) cudaFree(s->arena);
  if (s->d_sums) cudaFree(s->d_sums);
  if (s->h_sums) cudaFreeHost(s->h_sums);
  delete s;
  return T213_OK;
}

}  // extern "C"
