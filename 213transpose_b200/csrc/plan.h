// Plans: the sequence of passes that transposes one (d1,d2,d3) shape.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "internal.h"

namespace t213 {

enum PassType { PT_COL = 1, PT_ROW = 2, PT_SEG = 3, PT_TILE = 4, PT_BAND = 5 };

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
};

// Builds the plan of a family (T213_PLAN_*; AUTO picks).  t = 0 lets the
// planner choose the block/band size.  Cached per device.
std::shared_ptr<Plan> get_plan(int64_t d1, int64_t d2, int64_t d3, int eb, int kind, int64_t t, int *status);
// Runs a plan on `data` (d1*d2*d3*eb bytes) on stream st.
int run_plan(const Plan &p, char *data, cudaStream_t st, LaunchStats *ls);
// Extra device memory a run of the plan needs beyond the tensor (carries and
// scratch fallbacks), in bytes.
size_t plan_workspace_bytes(const Plan &p);

// Explicit C2R / R2C / skinny plans with the reference's argument convention.
std::shared_ptr<Plan> make_c2r_plan(int64_t d1, int64_t d2, int64_t d3, int eb, bool skinny, int *status);
std::shared_ptr<Plan> make_r2c_plan(int64_t d1, int64_t d2, int64_t d3, int eb, bool skinny, int *status);

int64_t ext_gcd(int64_t a, int64_t b, int64_t *mmi);

}  // namespace t213
