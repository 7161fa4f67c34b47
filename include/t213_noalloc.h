/* A row shuffle that allocates no device memory.
 *
 * No counterpart in the reference: its passes allocate whatever scratch they
 * need.  This entry point exists for callers that must not allocate on the
 * device while they run:
 *   - a process whose device memory is already taken by its own caching
 *     allocator or arena (a framework, or the serving arena of t213_serve.h),
 *     where a cudaMalloc would fail with out-of-memory although the tensor is
 *     resident;
 *   - latency-critical loops, where cudaFree may synchronise the whole device
 *     and stall every other stream.
 */
#ifndef T213_NOALLOC_H_
#define T213_NOALLOC_H_

#include <stdint.h>

#include "t213.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Size of the fixed scratch array compiled into the library (32 MiB). */
#define T213_NOALLOC_SCRATCH_BYTES (32ll << 20)

/* The row shuffle of t213_row_shuffle -- same functor kinds and parameters
 * (m = d2, n = d1, c > 0, k), same layout, same result -- run without any
 * device allocation: whole rows are copied, one group at a time, into a
 * file-scope __device__ scratch array of T213_NOALLOC_SCRATCH_BYTES and
 * gathered back from there.
 *
 * Limit: one row (d1 * elem_bytes bytes) must fit the scratch; a longer row
 * returns T213_ERR_UNSUPPORTED and leaves the data untouched.
 * The scratch is shared by every call on a device: calls that overlap in time
 * (on different streams, or from different host threads) race on it and
 * corrupt each other's results, so serialise them.
 * The first call on each device does the set-up: it looks up the scratch's
 * device address and the device's SM count.  Under CUDA's default lazy module
 * loading this is also when the driver loads the library's module holding
 * the array onto the device, reserving its 32 MiB there.  So make the first
 * call on a device before your own allocator fills the device's memory; an
 * empty call (d1, d2 or d3 zero, valid parameters otherwise) does only the
 * set-up and serves as the warm-up.  Set-up itself is thread-safe; it is the
 * scratch that concurrent calls must not share.
 * Nothing has to start at zero: each call writes every scratch byte it reads.
 * Asynchronous on `stream` like t213_row_shuffle. */
int t213_row_shuffle_noalloc(int32_t fn_kind, const int64_t *fn_params, int32_t n_params, void *data,
                             int64_t d3, int64_t d2, int64_t d1, int32_t elem_bytes, t213_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* T213_NOALLOC_H_ */
