// Host-side internals shared by the launchers and the runtime.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/t213.h"

namespace t213 {

// ---------------------------------------------------------------- errors --
void set_error(const std::string &msg);
const std::string &last_error();
// Turns a CUDA error into T213_ERR_CUDA with a message.
int cuda_status(cudaError_t e, const char *where);

// ---------------------------------------------------------------- device --
struct DevInfo {
  int id = 0;
  int sms = 148;
  int smem_optin = 227 * 1024;    // per CTA, opt-in maximum
  int smem_per_sm = 228 * 1024;
  int max_threads_sm = 2048;
  int cc_major = 10, cc_minor = 0;
  int l2_bytes = 0;
};
const DevInfo &dev_info();  // the current device, cached

// Per-device status word written by kernels whose bounded waits ran out
// (T213_ERR_TIMEOUT); read and cleared by t213_device_status.
int *device_status_word(int *status);

// ------------------------------------------------------------- workspace --
// Grow-only scratch buffer per (device, stream).  Calls on one stream run in
// order, so they can share it; calls on different streams never do.
char *workspace(cudaStream_t st, size_t bytes, int *status);
// Frees the workspace of one stream (before the stream is destroyed).
void release_stream_workspace(cudaStream_t st);

// Device memory that kernels in flight on any stream may still read (cycle
// tables of evicted plans) is not freed at once: cudaFree does not promise to
// wait for them.  It is parked here and freed after a device-wide
// synchronisation, once enough has accumulated or on t213_release_cache.
void defer_free(int dev, void *p);
void flush_deferred_frees();

// ------------------------------------------------------------- functors --
struct FnSpec {
  int kind = 0;
  int64_t p[4] = {0, 0, 0, 0};
};

// true when every intermediate value of the functor over an m x n slice stays
// below 2^31, so the 32-bit index path is exact.
bool fits32(const FnSpec &f, int64_t m, int64_t n);

template <int V>
using IC = std::integral_constant<int, V>;

// (element bytes, access width) -> compile-time pair
template <typename Fn>
bool dispatch_eb_aw(int eb, int aw, Fn &&fn) {
  switch (eb) {
    case 1:
      return fn(IC<1>{}, IC<1>{});
    case 2:
      return fn(IC<2>{}, IC<2>{});
    case 4:
      return aw == 16 ? fn(IC<4>{}, IC<16>{}) : aw == 8 ? fn(IC<4>{}, IC<8>{}) : fn(IC<4>{}, IC<4>{});
    case 8:
      return aw == 16 ? fn(IC<8>{}, IC<16>{}) : fn(IC<8>{}, IC<8>{});
    case 16:
      return fn(IC<16>{}, IC<16>{});
  }
  return false;
}

// access width for segment moves: any power of two up to 16 dividing the
// segment size, the slice pitch and the base address
inline int seg_access_width(const void *base, int64_t seg_bytes, int64_t slice_bytes) {
  uint64_t a = (uint64_t)(uintptr_t)base | (uint64_t)seg_bytes | (uint64_t)slice_bytes;
  if ((a & 15) == 0) return 16;
  if ((a & 7) == 0) return 8;
  if ((a & 3) == 0) return 4;
  if ((a & 1) == 0) return 2;
  return 1;
}

// Per-kernel launch facts cached across calls: the shared-memory attribute is
// set once per (kernel, bytes), and the resident-CTA count per SM is queried
// once per (kernel, threads, bytes, cluster).
bool kernel_attr_once(const void *kern, int64_t smem, int cluster);
int occupancy_cached(const void *kern, int threads, int64_t smem, int cluster, int *per_sm_or_clusters);

// ------------------------------------------------------------- launchers --
struct LaunchStats {
  int launches = 0;
};

// Kernel choices a plan may pin; 0 leaves a launcher's default (its
// environment override, else its built-in rule).  The autotuner searches them
// per shape class.
struct Variant {
  int8_t col = 0;   // column passes: 1 staged strips (no cluster-local form), 2 cluster-local 256-byte strips,
                    // 3 cluster-local double-buffered, 4 the same with half-size buffers (two CTAs per SM),
                    // 5 word-width cluster-local strips where the default takes 16-byte accesses over an
                    // unaligned pitch (k_col_local_peel)
  int8_t row = 0;   // row passes: 1 staged rows, 2 double-buffered rows (k_row_pipe), 3 word-width staged rows
                    // where the default takes 16-byte accesses over an unaligned pitch (k_row_gather_peel)
  int8_t tile = 0;  // tile swaps: 1 TMA ring, 2 register tiles (k_tile_swap_vec)
  int8_t seg = 0;   // segment cycles: 1 bulk walker ring of 6, 2 ring of 10, 3 register walker
  bool any() const { return col || row || tile || seg; }
  int packed() const { return (col & 15) | (row & 15) << 4 | (tile & 15) << 8 | (seg & 15) << 12; }
  static Variant unpack(int v) {
    Variant x;
    x.col = (int8_t)(v & 15);
    x.row = (int8_t)(v >> 4 & 15);
    x.tile = (int8_t)(v >> 8 & 15);
    x.seg = (int8_t)(v >> 12 & 15);
    return x;
  }
};
// The variant of the plan this host thread is launching (set by run_plan).
const Variant &current_variant();
struct VariantScope {
  explicit VariantScope(const Variant &v);
  ~VariantScope();
  Variant saved;
};

// Column gather new[i][j] = old[f(i,j)][j] over d3 slices of m x n.
int launch_col_gather(const FnSpec &f, char *data, int64_t d3, int64_t m, int64_t n, int eb,
                      cudaStream_t st, LaunchStats *ls);
// Row gather new[i][j] = old[i][f(i,j)].
int launch_row_gather(const FnSpec &f, char *data, int64_t d3, int64_t m, int64_t n, int eb,
                      cudaStream_t st, LaunchStats *ls);
// Which cluster-local form a column functor with these parameters has (the
// column kernels evaluate it as key offsets and row maps): 1 offsets of the
// functor itself with identity maps, 2 the C2R fused post-op (+j offsets,
// output rows through the inverse post-permuter), 3 the R2C fused pre-op (-j
// offsets, source rows through the pre-permuter); 0 none.
int col_local_form(const FnSpec &f, int64_t m);
// Describes the variant launch_col_gather / launch_row_gather would pick.
std::string describe_col_gather(int64_t m, int64_t n, int eb, const void *data);
// The variant launch_col_gather picks for this functor (the cluster-local
// kernel when the functor's form and the strip halo allow it).
std::string describe_col_gather_fn(const FnSpec &f, int64_t m, int64_t n, int eb, const void *data);
std::string describe_row_gather(int64_t m, int64_t n, int eb, const void *data);
// Number of launches the gathers enqueue.
int count_col_gather(int64_t d3, int64_t m, int64_t n, int eb);
int count_row_gather(int64_t d3, int64_t m, int64_t n, int eb);

// Square-block transposes (t x t blocks of an m x n slice) and band transposes.
int launch_tile_swap(char *data, int64_t d3, int64_t m, int64_t n, int64_t t, int eb, cudaStream_t st,
                     LaunchStats *ls);
int launch_band_transpose(char *data, int64_t n_bands, int64_t R, int64_t C, int eb, cudaStream_t st,
                          LaunchStats *ls);
int64_t band_smem_bytes(int64_t R, int64_t C, int eb);
// One-pass transpose of slices held whole in a cluster's shared memory.
int launch_slice(char *data, int64_t d3, int64_t m, int64_t n, int eb, cudaStream_t st, LaunchStats *ls);
bool slice_fits(int64_t m, int64_t n, int eb);
std::string describe_slice(int64_t m, int64_t n, int eb, int64_t d3);
// Grouped one-pass slices (the batched form): the rows per CTA H and padded
// pitch P of a slice split over an 8-CTA cluster (false if it does not fit),
// and one launch of the grouped kernel over device SliceEntry records.
bool slice_group_params(int64_t m, int64_t n, int eb, const void *data, uint32_t *H, uint32_t *P, bool *vec);
int launch_slice_group(const void *entries, int32_t n_entries, int64_t n_items, int64_t smem, cudaStream_t st);
int64_t band_smem_limit();
bool band_fits(int64_t R, int64_t C, int eb);

// ------------------------------------------------------------ cycle tables --
// A permutation of segment indices: either a segment 3-D rearrangement
// [A][Mid][C] -> [C][Mid][A] or one of the row permuters (FnSpec).
struct PermSpec {
  int kind = 0;  // 0 = SegPerm3, else T213_FN_*_PERMUTER
  int64_t A = 0, Mid = 0, C = 0;
  FnSpec fn;
  int64_t S = 0;  // positions per slice
  bool operator==(const PermSpec &o) const {
    return kind == o.kind && A == o.A && Mid == o.Mid && C == o.C && S == o.S &&
           fn.kind == o.fn.kind && fn.p[0] == o.fn.p[0] && fn.p[1] == o.fn.p[1] &&
           fn.p[2] == o.fn.p[2] && fn.p[3] == o.fn.p[3];
  }
};

struct CycleTable {
  PermSpec spec;
  int64_t n_chunks = 0, n_carry = 0, moved = 0, n_cycles = 0, max_len = 0;
  std::vector<char> h_chunks, h_carry_items;  // host copies (Chunk[], CarryItem[])
  void *d_chunks = nullptr;                   // device copies, uploaded on first launch
  void *d_carry_items = nullptr;
  int dev = 0;
  std::mutex mu;
  // The upload is stream-ordered: a synchronous cudaMemcpy from pageable
  // memory may return before its DMA lands, and work on non-blocking streams
  // is not ordered after the legacy stream, so a walker could read a table
  // that is not there yet.  The first call copies on `st` and records `ready`;
  // later calls from other streams make their stream wait on `ready` until
  // the event is seen complete.
  cudaEvent_t ready = nullptr;
  cudaStream_t upload_stream = nullptr;
  bool ready_seen = false;
  int ensure_uploaded(cudaStream_t st);
  // Blocks the host until the upload has landed (set-up paths that capture
  // graphs afterwards call this so captured work needs no event wait).
  int wait_uploaded();
  ~CycleTable();
};

// Builds (or fetches from the cache) the cycle table of a permutation, sized
// for `pieces_x_slices` work items per chunk.  Synchronous on first build.
std::shared_ptr<CycleTable> get_cycle_table(const PermSpec &p, int64_t items_per_chunk, int *status);

// Moves segments of seg_bytes along the cycles of the table, all d3 slices.
// Uses the stream's workspace for carries.
int launch_seg_cycles(const CycleTable &ct, char *data, int64_t d3, int64_t slice_bytes,
                      int64_t seg_bytes, cudaStream_t st, LaunchStats *ls, char *carry_override,
                      size_t carry_override_bytes);
size_t seg_cycles_carry_bytes(const CycleTable &ct, int64_t d3, int64_t seg_bytes);
int seg_cycles_team(int64_t seg_bytes, int aw);

// ----------------------------------------------------------------- timing --
// Per-pass CUDA-event timing (enabled by t213_pass_timing_enable).
struct PassTimer {
  const char *name;
  cudaStream_t st;
  cudaEvent_t a = nullptr, b = nullptr;
  PassTimer(const char *n, cudaStream_t s);
  ~PassTimer();
};
bool pass_timing_on();

}  // namespace t213
