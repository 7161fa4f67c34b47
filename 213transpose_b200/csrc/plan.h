// Plans: the sequence of passes that transposes one (d1,d2,d3) shape.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "internal.h"

namespace t213 {

enum PassType { PT_COL = 1, PT_ROW = 2, PT_SEG = 3, PT_TILE = 4, PT_BAND = 5, PT_SLICE = 6 };

struct PassDesc {
  PassType type = PT_COL;
  FnSpec fn;             // PT_COL / PT_ROW: the index functor
  int64_t m = 0, n = 0;  // matrix view of a slice (rows, columns)
  PermSpec perm;         // PT_SEG
  int64_t seg_bytes = 0;
  std::shared_ptr<CycleTable> table;
  int64_t t = 0;                     // PT_TILE: block side
  int64_t R = 0, C = 0, bands = 0;   // PT_BAND: band shape, bands per slice
  const char *name() const;
};

struct Plan {
  int kind = 0;
  int64_t t = 0;
  int64_t d1 = 0, d2 = 0, d3 = 0;
  int eb = 0;
  std::vector<PassDesc> passes;
  std::string desc;
  double est_cost = 0;  // heuristic, in units of one full read+write sweep
  Variant var;          // kernel choices pinned by the tuner (default: none)
};

// Builds the plan of a family (T213_PLAN_*; AUTO picks).  t = 0 lets the
// planner choose the block/band size.  Cached per device.
std::shared_ptr<Plan> get_plan(int64_t d1, int64_t d2, int64_t d3, int eb, int kind, int64_t t, int *status);
// The plan of a family and block size with kernel variants pinned (a cached
// copy of get_plan's plan); the plain plan when v pins nothing.
std::shared_ptr<Plan> get_plan_variant(int64_t d1, int64_t d2, int64_t d3, int eb, int kind, int64_t t,
                                       const Variant &v, int *status);
// Whether get_plan would find this exact key in the cache (nothing is built).
bool plan_cached(int64_t d1, int64_t d2, int64_t d3, int eb, int kind, int64_t t);
// Runs a plan on `data` (d1*d2*d3*eb bytes) on stream st.
int run_plan(const Plan &p, char *data, cudaStream_t st, LaunchStats *ls);
// Extra device memory a run of the plan needs beyond the tensor (carries and
// scratch fallbacks), in bytes.
size_t plan_workspace_bytes(const Plan &p);

// Explicit C2R / R2C / skinny plans with the reference's argument convention.
std::shared_ptr<Plan> make_c2r_plan(int64_t d1, int64_t d2, int64_t d3, int eb, bool skinny, int *status);
std::shared_ptr<Plan> make_r2c_plan(int64_t d1, int64_t d2, int64_t d3, int eb, bool skinny, int *status);

int64_t ext_gcd(int64_t a, int64_t b, int64_t *mmi);

// ---- grouped launches of the persistent batch kernel (batch.cu) ----------------
// A reusable executor: fixed device tables, carry pool and pinned staging, so
// a group of small tensors is transposed by one k_batch launch without any
// allocation at launch time.  Used by the serving loop.
struct GroupExec;
GroupExec *group_exec_create(int64_t max_passes, int64_t max_items, size_t carry_bytes, int *status);
void group_exec_destroy(GroupExec *g);
// The plan a tensor takes inside the persistent kernel (the automatic choice,
// else the cheapest other family whose passes fit its shared memory); null if
// none fits, and, unless search_slice, when the automatic choice is the
// one-pass slice plan (which runs on its own launch).
std::shared_ptr<Plan> group_plan(int64_t d1, int64_t d2, int64_t d3, int eb, int *status, bool search_slice);
// Enqueues one k_batch launch over the tensors on st (tables copied from the
// executor's pinned staging, counters reset), then copies the kernel's status
// word to the executor's host mirror and records its event.  The executor's
// previous launch must have finished (group_exec_idle).  Returns
// T213_ERR_UNSUPPORTED, with nothing enqueued, when a tensor has no plan that
// fits or the group exceeds the executor's capacity.
int group_exec_run(GroupExec *g, const t213_tensor_desc *tensors, int32_t count, cudaStream_t st);
bool group_exec_idle(GroupExec *g);
// Status word of the last finished launch (0, or T213_ERR_TIMEOUT).
int group_exec_status(GroupExec *g);

}  // namespace t213
