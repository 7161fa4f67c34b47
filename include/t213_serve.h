/*
 * t213_serve.h — serving form of the in-place 213 transpose (no counterpart in
 * kaihsin/213transpose, which offers only the plain call).
 *
 * A server replays an open-loop request schedule against the GPU: each request
 * names a (d1,d2,d3) tensor of elem_bytes elements and an arrival time.  On
 * arrival a request is planned on a host worker thread (T213_SERVE_PLANNERS,
 * default all host threads but two, at most 16), then waits, in arrival order
 * among the planned requests, until its tensor fits the HBM budget (the tensor
 * itself, in place: no scratch copy of the full tensor) and an in-flight slot
 * is free; it is then admitted into a device arena reserved at
 * creation, its tensor is materialised on the device (a seeded fill standing in
 * for the producer), transposed in place on one of the server's streams, and
 * checksummed.  Admitted requests run concurrently on the stream pool while new
 * ones keep arriving and being admitted as memory and slots free up
 * (continuous batching).  Small requests (T213_SERVE_GROUP_MB, default 32 MB)
 * admitted together share launches: one grouped fill, one persistent batch
 * kernel over all their transposes (the executor of the batched form) and one
 * grouped checksum, on T213_SERVE_GROUPS (default 4) reusable executors.
 * Latency is measured on the host from the scheduled arrival to the detected
 * completion of the transpose.
 */
#ifndef T213_SERVE_H
#define T213_SERVE_H

#include <stdint.h>

#include "t213.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct t213_request {
  int64_t d1, d2, d3;
  int32_t elem_bytes;
  int32_t plan_kind;   /* T213_PLAN_AUTO or a forced family */
  double arrival_s;    /* seconds from the start of the run */
  uint64_t seed;       /* content of the tensor */
} t213_request;

typedef struct t213_serve_stats {
  int64_t completed, rejected, bytes_done;
  double p50_ms, p99_ms, mean_ms, max_ms, wall_s;
  int64_t peak_resident_bytes, max_inflight;
  /* cold: requests whose shape was not in the plan cache when they arrived
   * (they waited for planning); warm: the others */
  int64_t cold;
  double p50_cold_ms, p99_cold_ms, p50_warm_ms, p99_warm_ms;
  /* launches of the persistent kernel over several small requests, and the
   * requests they carried */
  int64_t group_launches, grouped_requests;
} t213_serve_stats;

typedef struct t213_server_st *t213_server;

/* Reserves min(hbm_budget_bytes, free device memory - 2 GiB) for the arena. */
int t213_server_create(int64_t hbm_budget_bytes, int32_t max_inflight, int32_t n_streams, t213_server *out);

/* Replays the schedule; blocks until every admitted request has finished.
 * checksums (optional, n entries) receives a position-dependent 64-bit
 * checksum of each transposed tensor (0 for rejected requests); latency_ms
 * (optional, n entries) receives each request's latency (-1 if rejected). */
int t213_server_run(t213_server s, const t213_request *requests, int32_t n, t213_serve_stats *stats,
                    uint64_t *checksums, double *latency_ms);
/* The same, and for every request whose outputs[i] is not NULL the transposed
 * tensor is copied there (d1*d2*d3*elem_bytes bytes of host memory, pinned
 * for an asynchronous copy) before the request counts as complete. */
int t213_server_run_capture(t213_server s, const t213_request *requests, int32_t n, t213_serve_stats *stats,
                            uint64_t *checksums, double *latency_ms, void *const *outputs);

/* The checksum a correct transpose of the request's tensor has, computed on
 * the device from the fill without transposing anything. */
int t213_server_expected_checksum(t213_server s, const t213_request *request, uint64_t *checksum);

/* Runs one request alone (admit, fill, transpose, checksum) and returns its
 * checksum. */
int t213_server_run_alone(t213_server s, const t213_request *request, uint64_t *checksum);

int t213_server_destroy(t213_server s);

#ifdef __cplusplus
}
#endif

#endif /* T213_SERVE_H */
