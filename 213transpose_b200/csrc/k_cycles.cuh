// Cycle-following movers for permutations of whole segments.
//
// A pass of this kind applies a scatter permutation new[dst(p)] = old[p] to
// the S segments of every slice (a segment is seg_bytes contiguous bytes: a
// whole row for the C2R/R2C row permuters, t elements for the block and band
// plans).  The host lists the non-trivial cycles of dst once per shape and
// cuts long cycles into chunks, so the work can spread over the whole GPU:
//
//   chunk = (start position x_s, len L, carry slot or -1)
//   it writes x_{s+1} .. x_{s+L} with old[x_s] .. old[x_{s+L-1}]
//
// x_{s+L} is either the cycle's own start (a whole cycle, read first by the
// same walker) or the start of the next chunk, whose old value was saved to a
// carry slot by k_carry_save before this kernel started.  So no two walkers
// touch the same position, and each position is read once and written once.
//
// Segments are further cut into pieces of `team` words; every thread walks
// the cycle alone on its own word, reading ahead UNR positions before writing
// them back (positions of one cycle are distinct, so the read-ahead never
// reads a value this walker already overwrote).  No barriers are needed.
#pragma once

#include "common.cuh"
#include "functors.cuh"
#include "tma.cuh"

namespace t213 {

struct Chunk {
  int64_t start;  // position of x_s
  int64_t len;    // number of writes
  int64_t carry;  // carry slot holding old[x_s], or -1 (whole cycle)
};

constexpr int kCycleThreads = 256;

template <int AW, int UNR, typename P, typename U>
__global__ void __launch_bounds__(kCycleThreads)
    k_seg_cycles(char *__restrict__ data, int64_t slice_bytes, int64_t d3, int64_t seg_bytes,
                 int team, int64_t pieces, const Chunk *__restrict__ chunks, int64_t n_chunks,
                 const char *__restrict__ carry, P dst) {
  using W = typename WordT<AW>::type;
  const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = (int)(gtid % team);
  const int64_t team_id = gtid / team;
  const int64_t n_teams = ((int64_t)gridDim.x * blockDim.x) / team;
  if (team_id >= n_teams) return;  // a trailing partial team would repeat team 0's items
  const int64_t per_chunk = pieces * d3;
  const int64_t items = n_chunks * per_chunk;
  for (int64_t it = team_id; it < items; it += n_teams) {
    const int64_t c = it / per_chunk;
    const int64_t rest = it - c * per_chunk;
    const int64_t k = rest / pieces;
    const int64_t pc = rest - k * pieces;
    const int64_t off = (pc * team + lane) * AW;
    if (off >= seg_bytes) continue;
    const Chunk ch = chunks[c];
    char *base = data + k * slice_bytes + off;
    U pos = (U)ch.start;
    W cur;
    if (ch.carry >= 0)
      cur = *reinterpret_cast<const W *>(carry + (ch.carry * d3 + k) * seg_bytes + off);
    else
      cur = __ldcg(reinterpret_cast<const W *>(base + (int64_t)pos * seg_bytes));
    int64_t remaining = ch.len;
    while (remaining > 0) {
      const int cnt = remaining < UNR ? (int)remaining : UNR;
      const bool last_group = remaining == cnt;
      U ps[UNR];
      W nx[UNR];
#pragma unroll
      for (int u = 0; u < UNR; u++) {
        if (u < cnt) {
          pos = dst(pos);
          ps[u] = pos;
        }
      }
#pragma unroll
      for (int u = 0; u < UNR; u++) {
        // the chunk's final position is never read: its old value is either
        // this walker's start or the next chunk's carry
        if (u < cnt && !(last_group && u == cnt - 1))
          nx[u] = __ldcg(reinterpret_cast<const W *>(base + (int64_t)ps[u] * seg_bytes));
      }
#pragma unroll
      for (int u = 0; u < UNR; u++) {
        if (u < cnt) {
          W v = (u == 0) ? cur : nx[u - 1 < 0 ? 0 : u - 1];
          __stcg(reinterpret_cast<W *>(base + (int64_t)ps[u] * seg_bytes), v);
        }
      }
      if (!last_group) cur = nx[UNR - 1];  // not the last group => cnt == UNR
      remaining -= cnt;
    }
  }
}

// Saves old[x_s] of every split chunk (all slices) before the walkers start.
struct CarryItem {
  int64_t pos;
  int64_t slot;
};

template <int AW>
__global__ void __launch_bounds__(kCycleThreads)
    k_carry_save(const char *__restrict__ data, int64_t slice_bytes, int64_t d3, int64_t seg_bytes,
                 const CarryItem *__restrict__ items, int64_t n_items, char *__restrict__ carry) {
  using W = typename WordT<AW>::type;
  const int64_t wps = seg_bytes / AW;
  const int64_t total = n_items * d3 * wps;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t w = t % wps;
    const int64_t r = t / wps;
    const int64_t k = r % d3;
    const int64_t ii = r / d3;
    const CarryItem ci = items[ii];
    const W v = __ldcg(reinterpret_cast<const W *>(data + k * slice_bytes + ci.pos * seg_bytes) + w);
    reinterpret_cast<W *>(carry + (ci.slot * d3 + k) * seg_bytes)[w] = v;
  }
}

// ---------------------------------------------------------------------------
// TMA walker for segments of 16-byte multiples.  One walker per 32-thread CTA;
// lane 0 drives a ring of NB shared-memory buffers with bulk asynchronous
// copies (cp.async.bulk): the piece at x_i is loaded into buffer i % NB, and
// step k stores buffer (k-1) % NB to x_k once x_k's own old value has landed.
// Loads run NB-2 positions ahead of the stores; a buffer is reloaded only
// after the bulk store that read it has finished reading (wait_group.read).
// Every mbarrier wait is bounded; on timeout the walker records
// T213_ERR_TIMEOUT in *status, drains its stores and returns.
// ---------------------------------------------------------------------------
constexpr int kBulkRing = 6;

template <typename P, typename U, int NB = kBulkRing>
__global__ void __launch_bounds__(32)
    k_seg_cycles_bulk(char *__restrict__ data, int64_t slice_bytes, int64_t d3, int64_t seg_bytes,
                      int64_t piece_bytes, int64_t pieces, const Chunk *__restrict__ chunks, int64_t n_chunks,
                      const char *__restrict__ carry, P dst, int *status) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
  char *buf = reinterpret_cast<char *>(smem_raw) + 128;
  if (threadIdx.x != 0) return;
  for (int i = 0; i < NB; i++) mbar_init(&bars[i], 1);
  fence_barrier_init();
  uint32_t parity = 0;  // bit b: parity of the next completion of bars[b]
  bool failed = false;
  const int64_t per_chunk = pieces * d3;
  const int64_t items = n_chunks * per_chunk;
  for (int64_t it = blockIdx.x; it < items && !failed; it += gridDim.x) {
    const int64_t c = it / per_chunk;
    const int64_t rest = it - c * per_chunk;
    const int64_t k = rest / pieces;
    const int64_t pc = rest - k * pieces;
    const Chunk ch = chunks[c];
    const int64_t off = pc * piece_bytes;
    const uint32_t pb = (uint32_t)min(piece_bytes, seg_bytes - off);
    char *base = data + k * slice_bytes + off;
    const int64_t L = ch.len;
    U xi = (U)ch.start;  // position of the newest load issued
    U pos[NB];
    // x_0: from the carry slot (split chunk) or from memory (whole cycle)
    mbar_expect_tx(&bars[0], pb);
    if (ch.carry >= 0)
      bulk_g2s(buf, carry + (ch.carry * d3 + k) * seg_bytes + off, pb, &bars[0]);
    else
      bulk_g2s(buf, base + (int64_t)xi * seg_bytes, pb, &bars[0]);
    pos[0] = xi;
    int64_t issued = 1;
    while (issued < L && issued <= NB - 2) {
      xi = dst(xi);
      const int b = (int)(issued % NB);
      pos[b] = xi;
      mbar_expect_tx(&bars[b], pb);
      bulk_g2s(buf + (int64_t)b * piece_bytes, base + (int64_t)xi * seg_bytes, pb, &bars[b]);
      issued++;
    }
    // loads [waited, issued) are in flight; a timed-out walker drains them
    // (each wait bounded again) before it returns, so no copy still lands in
    // shared memory of an exited CTA
    int64_t waited = 0;
    auto drain = [&]() {
      for (int64_t j = waited; j < issued; j++) {
        const int b = (int)(j % NB);
        if (!mbar_wait(&bars[b], (parity >> b) & 1u)) break;
        parity ^= 1u << b;
      }
    };
    // old value of x_0 in place
    if (!mbar_wait(&bars[0], parity & 1u)) {
      failed = true;
      drain();
      break;
    }
    parity ^= 1u;
    waited = 1;
    U last = pos[0];
    for (int64_t s = 1; s <= L; s++) {
      const int bs = (int)(s % NB);
      const int bp = (int)((s - 1) % NB);
      U target;
      if (s < L) {
        // x_s must be read before it is overwritten
        if (!mbar_wait(&bars[bs], (parity >> bs) & 1u)) {
          failed = true;
          drain();
          break;
        }
        parity ^= 1u << bs;
        waited = s + 1;
        target = pos[bs];
      } else {
        target = dst(last);  // cycle start or the next chunk's start
      }
      fence_proxy_async();
      bulk_s2g(base + (int64_t)target * seg_bytes, buf + (int64_t)bp * piece_bytes, pb);
      bulk_commit();
      last = target;
      if (issued < L) {
        bulk_wait_read<1>();  // the buffer's previous store has read it
        xi = dst(xi);
        const int b = (int)(issued % NB);
        pos[b] = xi;
        mbar_expect_tx(&bars[b], pb);
        bulk_g2s(buf + (int64_t)b * piece_bytes, base + (int64_t)xi * seg_bytes, pb, &bars[b]);
        issued++;
      }
    }
    bulk_wait_read<0>();
  }
  bulk_wait_all<0>();
  if (failed) atomicExch(status, 5 /* T213_ERR_TIMEOUT */);
}

}  // namespace t213
