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

}  // namespace t213
