/*
 * t213.h — C ABI of the B200-native in-place 213 transpose.
 *
 * A (d1,d2,d3) array has d1 as its fastest axis: element (i1,i2,i3) lives at
 * i1 + d1*i2 + d1*d2*i3.  The 213 transpose swaps the first two axes in place,
 * so after the call that element lives at i2 + d2*i1 + d1*d2*i3.  Each of the
 * d3 slices is a row-major d2 x d1 matrix that is transposed to d1 x d2.
 *
 * Every entry point takes plain pointers and sizes, never throws, never exits,
 * and returns a t213_status.  Work is enqueued on the given CUDA stream
 * (NULL = the legacy default stream) and is asynchronous unless stated
 * otherwise.  The first call for a new shape builds that shape's plan (cycle
 * tables, workspace) and may synchronise the device once; later calls for the
 * same shape only enqueue kernels.
 *
 * Element sizes accepted everywhere: 1, 2, 4, 8 and 16 bytes.  The data is moved
 * bit for bit; the element type never enters the arithmetic.
 *
 * Each declaration names the reference interface it replaces
 * (kaihsin/213transpose, paths relative to that project).
 */
#ifndef T213_H
#define T213_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same object as cudaStream_t; NULL selects the legacy default stream. */
typedef struct CUstream_st *t213_stream_t;

typedef enum t213_status {
  T213_OK = 0,
  T213_ERR_INVALID_ARGUMENT = 1, /* negative size, NULL data with work to do, bad kind */
  T213_ERR_UNSUPPORTED = 2,      /* element size or shape outside what this build handles */
  T213_ERR_CUDA = 3,             /* a CUDA runtime call failed; see t213_last_error() */
  T213_ERR_OUT_OF_MEMORY = 4,    /* workspace allocation failed */
  T213_ERR_TIMEOUT = 5,          /* a bounded device-side wait ran out (batched executor) */
  T213_ERR_BUDGET = 6,           /* serving admission: request larger than the HBM budget */
  T213_ERR_NOT_READY = 7         /* serving poll: nothing finished yet */
} t213_status;

/*
 * Index functors of the C2R/R2C decomposition.  Parameters are passed in the
 * order of the reference constructors (include/equations.h, include/skinny.h).
 * Inside a slice the matrix has m rows and n columns; c = gcd(m,n), a = m/c,
 * b = n/c.
 */
typedef enum t213_fn {
  /* column rotators, new[i][j] = old[(i + r(j)) mod m][j]  (detail::rotate) */
  T213_FN_C2R_PREROTATOR = 1,   /* (b)        r = j / b                 equations.h:78-94   */
  T213_FN_C2R_POSTROTATOR = 2,  /* (m)        r = j mod m               equations.h:97-113  */
  T213_FN_R2C_PREROTATOR = 3,   /* (m)        r = (m - j mod m) mod m   equations.h:159-176 */
  T213_FN_R2C_POSTROTATOR = 4,  /* (b, m)     r = j<b ? 0 : m - j/b     equations.h:196-222 */
  /* row shufflers, new[i][j] = old[i][s_i(j)]  (detail::shuffle_fn, skinny_row_op) */
  T213_FN_C2R_SHUFFLE = 10,      /* (m, n, c, k)                        equations.h:12-54   */
  T213_FN_C2R_LONG_SHUFFLE = 11, /* (m, n, c, k) same map, 64-bit       skinny.h:29-67      */
  T213_FN_R2C_SHUFFLE = 12,      /* (m, n, c, k) k unused               equations.h:178-194 */
  /* column shufflers, new[i][j] = old[f(i,j)][j]  (detail::col_shuffle_fn, skinny_col_op) */
  T213_FN_C2R_FUSED_PREOP = 20,  /* (m, b)                              skinny.h:12-26      */
  T213_FN_C2R_FUSED_POSTOP = 21, /* (m, n, c)                           skinny.h:69-78      */
  T213_FN_R2C_FUSED_PREOP = 22,  /* (a, c, m, q)                        skinny.h:87-107     */
  T213_FN_R2C_FUSED_POSTOP = 23, /* (m, b)                              skinny.h:109-117    */
  /* row permuters, new[p(i)][*] = old[i][*]  (detail::scatter_permute) */
  T213_FN_C2R_POSTPERMUTER = 30, /* (m, n, c) = r2c::scatter_prepermuter equations.h:115-128 */
  T213_FN_R2C_PREPERMUTER = 31   /* (m, n, c) = c2r::scatter_postpermuter equations.h:134-157 */
} t213_fn;

/* Plan families the dispatcher can choose (t213_transpose_with_plan, t213_plan_describe). */
typedef enum t213_plan_kind {
  T213_PLAN_AUTO = 0,      /* tuner cache, else the built-in heuristic                        */
  T213_PLAN_C2R = 1,       /* Catanzaro C2R: [prerotate] row shuffle, column op             */
  T213_PLAN_R2C = 2,       /* inverse order: column op, row shuffle, [postrotate]            */
  T213_PLAN_SKINNY = 3,    /* skinny C2R/R2C for min(d1,d2) <= 32                            */
  T213_PLAN_BLOCKS = 4,    /* t x t square-block transposes + segment cycles (t | gcd)       */
  T213_PLAN_BANDS = 5,     /* band transposes + segment-matrix cycles (t | d2)              */
  T213_PLAN_BANDS_T = 6,   /* segment-matrix cycles + band transposes (t | d1)              */
  T213_PLAN_IDENTITY = 7,  /* d1 == 1 or d2 == 1: the memory layout does not change         */
  T213_PLAN_SLICE = 8      /* one pass: each slice held whole in a thread-block cluster's
                              shared memory (slices up to a few MB)                         */
} t213_plan_kind;

const char *t213_status_string(int status);
/* Detail text of the last failure on the calling thread ("" if none). */
const char *t213_last_error(void);
/* Library version string. */
const char *t213_version(void);

/* ---- public dispatcher ---------------------------------------------------
 * Replaces template<T> void inplace::transpose(T*, int d1, int d2, int d3)
 * (include/transpose.h:17-18, src/transpose.cu:99-124).  Chooses the fastest
 * known plan for the shape.  Accepts plain device pointers and managed
 * pointers (managed memory is prefetched to the current device first, as the
 * reference does at src/transpose.cu:104). */
int t213_transpose(void *data, int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes,
                   t213_stream_t stream);

/* Same, with an explicit plan family (T213_PLAN_*) and block/band size t
 * (0 = planner's choice).  Returns T213_ERR_UNSUPPORTED if the family does not
 * apply to the shape. */
int t213_transpose_with_plan(void *data, int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes,
                             int32_t plan_kind, int64_t t, t213_stream_t stream);

/* In-place permutation of the axes of a rank-N tensor, as a sequence of at
 * most N-1 in-place 213 transposes of grouped axes.  The convention is the
 * reference's rank-N model (TensorUtil, src/tensor_util.cpp:7-23,79-92):
 * dims[0] is the fastest axis, and output axis j (fastest first) is input
 * axis perm[j], so perm = {1, 0, 2} is the 213 transpose.  The reference's
 * GPU library has no rank-N call (its TensorUtil::seq_tt is an out-of-place
 * CPU gather); this entry point is the in-place GPU counterpart.  rank <= 32;
 * perm must be a permutation of 0..rank-1.  Asynchronous on `stream`. */
int t213_permute(void *data, int32_t rank, const int64_t *dims, const int32_t *perm, int32_t elem_bytes,
                 t213_stream_t stream);

/* Replaces template<T> void inplace::c2r::transpose(T*, int d1, int d2, int d3)
 * (include/transpose.h:5-9, src/transpose.cu:30-47): the slice is a d2 x d1
 * row-major matrix (m = d2 rows, n = d1 columns) transposed to d1 x d2 by
 * the C2R passes. */
int t213_c2r_transpose(void *data, int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes,
                       t213_stream_t stream);

/* Replaces template<T> void inplace::r2c::transpose(T*, int d1, int d2, int d3)
 * (include/transpose.h:11-15, src/transpose.cu:70-89).  Inverse of
 * t213_c2r_transpose(d1,d2): it maps a d1 x d2 row-major matrix to d2 x d1.
 * The dispatcher calls it with swapped axes (src/transpose.cu:121). */
int t213_r2c_transpose(void *data, int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes,
                       t213_stream_t stream);

/* Replace detail::c2r::skinny_transpose / detail::r2c::skinny_transpose
 * (include/skinny.h:9-10,84-85, src/skinny.cu:313-363).  Require d2 <= 32. */
int t213_skinny_c2r_transpose(void *data, int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes,
                              t213_stream_t stream);
int t213_skinny_r2c_transpose(void *data, int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes,
                              t213_stream_t stream);

/* ---- pass-level entry points (the reference's detail API) -----------------
 * The slice is viewed as d2 rows x d1 columns, d3 slices.  fn_params holds the
 * functor's constructor arguments (see t213_fn); n_params is their count. */

/* Replaces detail::rotate(F, d3, d2, d1, T*) (include/rotate.h:6-7, src/rotate.cu:237-270). */
int t213_rotate(int32_t fn_kind, const int64_t *fn_params, int32_t n_params, void *data,
                int64_t d3, int64_t d2, int64_t d1, int32_t elem_bytes, t213_stream_t stream);
/* Replaces detail::shuffle_fn(T*, d3, d2, d1, F) (include/shuffle.h:5-6, src/shuffle.cu:66-76)
 * and skinny_row_op (src/skinny.cu:237-280). */
int t213_row_shuffle(int32_t fn_kind, const int64_t *fn_params, int32_t n_params, void *data,
                     int64_t d3, int64_t d2, int64_t d1, int32_t elem_bytes, t213_stream_t stream);
/* Replaces detail::col_shuffle_fn(F, d3, d2, d1, T*) (include/col_shuffle.h:8-9,
 * src/col_shuffle.cu:30-42) and skinny_col_op (src/skinny.cu:282-309). */
int t213_col_shuffle(int32_t fn_kind, const int64_t *fn_params, int32_t n_params, void *data,
                     int64_t d3, int64_t d2, int64_t d1, int32_t elem_bytes, t213_stream_t stream);
/* Replaces detail::scatter_permute(F, d3, d2, d1, T*) (include/permute.h:6-7,
 * src/permute.cu:116-137).  Cycle leaders are computed once per functor and cached. */
int t213_scatter_permute(int32_t fn_kind, const int64_t *fn_params, int32_t n_params, void *data,
                         int64_t d3, int64_t d2, int64_t d1, int32_t elem_bytes,
                         t213_stream_t stream);

/* ---- host buffers -----------------------------------------------------------
 * End-to-end call for data that lives in host memory (the reference's driver
 * passes managed memory that starts on the host, src/test_213inplace.cu:32-47):
 * copies the tensor to the device slice by slice, transposes it, copies it
 * back, overlapping the two directions with the transposes.  Synchronous.
 * Pinned host memory gives full copy bandwidth; pageable memory works too. */
int t213_transpose_host(void *host_data, int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes,
                        t213_stream_t stream);

/* ---- planning / introspection ---------------------------------------------- */
/* Writes a one-line description of the plan chosen for the shape into buf. */
int t213_plan_describe(int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes, int32_t plan_kind,
                       int64_t t, char *buf, size_t buflen);
/* Number of kernel launches the plan for this shape enqueues per call. */
int t213_plan_launches(int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes, int32_t plan_kind,
                       int64_t t, int32_t *launches);
/* Per-pass timing: when enabled, every pass is bracketed by CUDA events on the
 * call's stream; t213_pass_timing_read returns the accumulated milliseconds and
 * launch count of the pass whose name matches (names: "tile_swap",
 * "segment_cycles", "row_gather", "col_gather", "band_transpose",
 * "cycle_carry", "row_copy").  Reading synchronises the recorded events. */
int t213_pass_timing_enable(int32_t enable);
int t213_pass_timing_read(const char *pass_name, double *total_ms, int64_t *launches);
int t213_pass_timing_reset(void);
/* Synchronises the stream, then returns (and clears) the device's status word:
 * T213_OK, or T213_ERR_TIMEOUT if a kernel's bounded wait on an asynchronous
 * copy ran out since the last read. */
int t213_device_status(t213_stream_t stream, int32_t *device_status);
/* Frees cached plans and workspace on the current device. */
int t213_release_cache(void);

/* ---- batched form ------------------------------------------------------------
 * Many tensors of uneven shape and element size transposed by ONE persistent
 * kernel launch that walks a device work list; each tensor's passes are
 * ordered by per-tensor completion counters with bounded waits.  The launch
 * is captured in a CUDA graph on the first execute and replayed after that.
 * No reference counterpart (the reference offers only a loop of plain calls). */
typedef struct t213_tensor_desc {
  void *data;
  int64_t d1, d2, d3;
  int32_t elem_bytes;
  int32_t plan_kind; /* T213_PLAN_AUTO or a forced family */
} t213_tensor_desc;

typedef struct t213_batch_st *t213_batch;

int t213_batch_create(const t213_tensor_desc *tensors, int32_t count, t213_batch *out);
/* One launch for the whole batch (graph replay after the first call). */
int t213_batch_execute(t213_batch batch, t213_stream_t stream);
/* Status word written by the persistent kernel (0 = ok, T213_ERR_TIMEOUT if a
 * bounded wait ran out).  Synchronises the stream. */
int t213_batch_status(t213_batch batch, t213_stream_t stream);
int t213_batch_describe(t213_batch batch, char *buf, size_t buflen);
/* Test hook of the batch's failure path.  Limits every dependency wait of the
 * persistent kernel to wait_ns nanoseconds and makes pass stall_pass (-1: the
 * first pass that has a predecessor) wait for one item more than its
 * predecessor has, so that wait can only end by running out.  The next
 * t213_batch_execute runs with these settings (a captured graph is dropped),
 * its CTAs leave on the timeout, the launch completes, and t213_batch_status
 * then returns T213_ERR_TIMEOUT once.  The batch's tensors are left partly
 * transposed.  Replaces no reference interface: the reference's grid-wide
 * waits (src/memory_ops.cu:18-33, src/skinny.cu:31-60) are unbounded. */
int t213_batch_debug_stall(t213_batch batch, int64_t wait_ns, int32_t stall_pass);
int t213_batch_destroy(t213_batch batch);
/* Autotunes every shape class present in the list (timing the applicable
 * plan families on scratch memory of the class's largest tensor) so that
 * t213_batch_create and the plain call pick the measured winner.
 * Synchronous; the tensors' data are not touched. */
int t213_batch_tune(const t213_tensor_desc *tensors, int32_t count, t213_stream_t stream);
/* Baseline form: the plain call looped over the same list on one stream. */
int t213_transpose_looped(const t213_tensor_desc *tensors, int32_t count, t213_stream_t stream);

/* ---- autotuner ------------------------------------------------------------------
 * Times the candidate plans of a shape class on the device and caches the
 * winner per class; the cache persists as a small text file. */
int t213_tune_shape(void *scratch_data, int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes,
                    t213_stream_t stream, int32_t *chosen_plan, int64_t *chosen_t);
int t213_tuner_load(const char *path);
int t213_tuner_save(const char *path);
int t213_tuner_clear(void);
int t213_tuner_lookup(int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes, int32_t *plan_kind,
                      int64_t *t);

#ifdef __cplusplus
}
#endif

#endif /* T213_H */
