// Row-gather and column-gather passes.
//
// Row gather    new[i][j] = old[i][src(i,j)]   (row shuffles of C2R / R2C)
// Column gather new[i][j] = old[src(i,j)][j]   (rotations and column shuffles)
//
// Both stage the unit they permute (one or more whole rows; one strip of W
// columns over all m rows) in shared memory, then write it back gathered.  A
// unit that is larger than one CTA's shared memory is spread over a thread-
// block cluster of K CTAs and gathered through distributed shared memory
// (ld.shared::cluster via cooperative_groups::cluster_group::map_shared_rank),
// so every element crosses HBM exactly once in each direction.
//
// Global accesses are AW-byte words (16 when the row pitch and base allow it),
// adjacent threads take adjacent words, and every word is read and written by
// the same CTA within one pass, so a pass is in place without hazards.
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"
#include "functors.cuh"
#include "tma.cuh"

namespace t213 {

namespace cg = cooperative_groups;

constexpr int kGatherThreads = 512;

// ---------------------------------------------------------------------------
// Rows: a CTA (or a cluster) owns `rows_per_unit` consecutive rows of the
// flattened d3*m row space.  rows in one unit are contiguous in memory.
// With a cluster of K CTAs each CTA holds `part` elements of the single row of
// the unit (rows_per_unit == 1 then).
// ---------------------------------------------------------------------------
template <int EB, int AW, typename F, typename U, bool CLUSTER>
__global__ void __launch_bounds__(kGatherThreads)
    k_row_gather(char *__restrict__ data, int64_t total_rows, U m, U n, int rows_per_unit, U part,
                 FastDiv<U> words_per_row, FastDiv<U> mdiv, F fn) {
  using E = typename ElemT<EB>::type;
  using W = typename WordT<AW>::type;
  using P = Pack<AW, EB>;
  constexpr int PER = AW / EB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  E *sm = reinterpret_cast<E *>(smem_raw);

  int rank = 0, K = 1;
  int64_t unit0 = blockIdx.x, ustride = gridDim.x;
  if (CLUSTER) {
    cg::cluster_group cl = cg::this_cluster();
    rank = (int)cl.block_rank();
    K = (int)cl.num_blocks();
    unit0 = blockIdx.x / K;
    ustride = gridDim.x / K;
  }
  const int64_t n_units = (total_rows + rows_per_unit - 1) / rows_per_unit;

  for (int64_t u = unit0; u < n_units; u += ustride) {
    const int64_t r0 = u * rows_per_unit;
    const int nr = (int)min((int64_t)rows_per_unit, total_rows - r0);
    char *ubase = data + r0 * (int64_t)n * EB;
    // ---- stage ---------------------------------------------------------
    // element range of this CTA inside the unit
    int64_t e_lo = 0, e_hi = (int64_t)nr * n;
    if (CLUSTER) {
      e_lo = (int64_t)rank * part;
      e_hi = min((int64_t)(rank + 1) * part, (int64_t)n);
    }
    {
      const W *g = reinterpret_cast<const W *>(ubase + e_lo * EB);
      W *s = reinterpret_cast<W *>(sm);
      const uint32_t nw = (e_hi > e_lo) ? (uint32_t)((e_hi - e_lo) / PER) : 0u;
      if constexpr (AW >= 4) {
#pragma unroll 4
        for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x) cp_async<AW>(s + w, g + w);
        cp_async_wait_all();
      } else {
#pragma unroll 4
        for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x) s[w] = __ldcs(g + w);
      }
    }
    if (CLUSTER)
      cg::this_cluster().sync();
    else
      __syncthreads();
    // ---- gather + write back ----------------------------------------------
    {
      W *g = reinterpret_cast<W *>(ubase + e_lo * EB);
      const uint32_t nw = (e_hi > e_lo) ? (uint32_t)((e_hi - e_lo) / PER) : 0u;
      const U i_base = (U)(r0 % (int64_t)m);
      for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x) {
        // words never straddle rows: PER divides n
        U wg = (U)(w + e_lo / PER);  // word index inside the unit
        U rr = words_per_row.div(wg);
        U j0 = (wg - rr * words_per_row.get()) * PER;
        U i = mdiv.mod(i_base + rr);
        typename P::U pk;
#pragma unroll
        for (int e = 0; e < PER; e++) {
          U sj = fn(i, j0 + e);
          if (CLUSTER) {
            U owner = sj / part;
            U local = sj - owner * part;
            E *remote = cg::this_cluster().map_shared_rank(sm, (int)owner);
            pk.e[e] = remote[local];
          } else {
            pk.e[e] = sm[(int64_t)rr * n + sj];
          }
        }
        __stcs(g + w, pk.w);
      }
    }
    if (CLUSTER)
      cg::this_cluster().sync();
    else
      __syncthreads();
  }
}

// Rows too long for a cluster: the old rows were copied to `scratch` by the
// host (one device-to-device copy per group of rows); this kernel gathers from
// that copy in global memory (L2-resident for groups up to tens of MB).
template <int EB, int AW, typename F, typename U>
__global__ void __launch_bounds__(kGatherThreads)
    k_row_gather_scratch(char *__restrict__ data, const char *__restrict__ scratch, int64_t row0,
                         int64_t nrows, U m, U n, FastDiv<U> words_per_row, F fn) {
  using E = typename ElemT<EB>::type;
  using W = typename WordT<AW>::type;
  using P = Pack<AW, EB>;
  constexpr int PER = AW / EB;
  const E *src = reinterpret_cast<const E *>(scratch);
  const int64_t wpr = words_per_row.get();
  for (int64_t rr = 0; rr < nrows; rr++) {
    W *g = reinterpret_cast<W *>(data + (row0 + rr) * (int64_t)n * EB);
    const E *srow = src + rr * (int64_t)n;
    const U i = (U)((row0 + rr) % (int64_t)m);
    for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < wpr;
         w += (int64_t)gridDim.x * blockDim.x) {
      U j0 = (U)w * PER;
      typename P::U pk;
#pragma unroll
      for (int e = 0; e < PER; e++) pk.e[e] = __ldcg(srow + fn(i, j0 + e));
      __stcs(g + w, pk.w);
    }
  }
}

// ---------------------------------------------------------------------------
// Column strips: unit = (slice k, strip s) covering columns [s*W, s*W+W) of
// all m rows.  A cluster of K CTAs splits the strip by rows: CTA r holds rows
// [r*H, r*H+H).  Shared memory rows have stride WS >= W elements (one access
// word of padding spreads the gathered rows over the banks).
// ---------------------------------------------------------------------------
template <int EB, int AW, typename F, typename U, bool CLUSTER>
__global__ void __launch_bounds__(kGatherThreads)
    k_col_gather(char *__restrict__ data, int64_t d3, U m, U n, U W, U WS, int64_t n_strips, U H, F fn) {
  using E = typename ElemT<EB>::type;
  using Wd = typename WordT<AW>::type;
  using P = Pack<AW, EB>;
  constexpr int PER = AW / EB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  E *sm = reinterpret_cast<E *>(smem_raw);

  int rank = 0, K = 1;
  int64_t unit0 = blockIdx.x, ustride = gridDim.x;
  if (CLUSTER) {
    cg::cluster_group cl = cg::this_cluster();
    rank = (int)cl.block_rank();
    K = (int)cl.num_blocks();
    unit0 = blockIdx.x / K;
    ustride = gridDim.x / K;
  }
  const int64_t n_units = d3 * n_strips;
  const U row_lo = CLUSTER ? (U)rank * H : 0;
  const U row_hi = CLUSTER ? (U)min((int64_t)(rank + 1) * H, (int64_t)m) : m;
  const U rows_here = row_hi > row_lo ? row_hi - row_lo : 0;

  for (int64_t u = unit0; u < n_units; u += ustride) {
    const int64_t k = u / n_strips;
    const U s = (U)(u - k * n_strips);
    const U j0 = s * W;
    const U wn = min(W, n - j0);  // multiple of PER
    const U wpr = wn / PER;       // words per strip row
    char *sbase = data + (k * (int64_t)m * n + j0) * EB;
    const int64_t pitch = (int64_t)n * EB;
    // ---- stage rows [row_lo, row_hi) of the strip --------------------------
    {
      const uint32_t nw = (uint32_t)rows_here * (uint32_t)wpr;
      for (uint32_t t = threadIdx.x; t < nw; t += blockDim.x) {
        uint32_t r = t / (uint32_t)wpr;
        uint32_t w = t - r * (uint32_t)wpr;
        const Wd *gp = reinterpret_cast<const Wd *>(sbase + (int64_t)(row_lo + r) * pitch) + w;
        if constexpr (AW >= 4)
          cp_async<AW>(reinterpret_cast<Wd *>(sm + (int64_t)r * WS) + w, gp);
        else
          reinterpret_cast<Wd *>(sm + (int64_t)r * WS)[w] = __ldcs(gp);
      }
      if constexpr (AW >= 4) cp_async_wait_all();
    }
    if (CLUSTER)
      cg::this_cluster().sync();
    else
      __syncthreads();
    // ---- gather + write back -------------------------------------------------
    {
      const uint32_t nw = (uint32_t)rows_here * (uint32_t)wpr;
      for (uint32_t t = threadIdx.x; t < nw; t += blockDim.x) {
        uint32_t r = t / (uint32_t)wpr;
        uint32_t w = t - r * (uint32_t)wpr;
        U i = row_lo + r;
        typename P::U pk;
#pragma unroll
        for (int e = 0; e < PER; e++) {
          U j = j0 + w * PER + e;
          U si = fn(i, j);
          if (CLUSTER) {
            U owner = si / H;
            U local = si - owner * H;
            E *remote = cg::this_cluster().map_shared_rank(sm, (int)owner);
            pk.e[e] = remote[(int64_t)local * WS + w * PER + e];
          } else {
            pk.e[e] = sm[(int64_t)si * WS + w * PER + e];
          }
        }
        Wd *gp = reinterpret_cast<Wd *>(sbase + (int64_t)i * pitch) + w;
        __stcs(gp, pk.w);
      }
    }
    if (CLUSTER)
      cg::this_cluster().sync();
    else
      __syncthreads();
  }
}

// Column groups too tall for a cluster: the host copied columns
// [j_lo, j_lo+gw) of every row of slice k to `scratch` (row pitch gw elements)
// with one 2-D device-to-device copy; this kernel gathers from that copy.
template <int EB, int AW, typename F, typename U>
__global__ void __launch_bounds__(kGatherThreads)
    k_col_gather_scratch(char *__restrict__ data, const char *__restrict__ scratch, U m, U n,
                         U j_lo, U gw, F fn) {
  using E = typename ElemT<EB>::type;
  using Wd = typename WordT<AW>::type;
  using P = Pack<AW, EB>;
  constexpr int PER = AW / EB;
  const E *src = reinterpret_cast<const E *>(scratch);
  const int64_t wpr = gw / PER;
  const int64_t nw = (int64_t)m * wpr;
  const int64_t pitch = (int64_t)n * EB;
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nw;
       t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = t / wpr;
    const U w = (U)(t - r * wpr);
    const U i = (U)r;
    typename P::U pk;
#pragma unroll
    for (int e = 0; e < PER; e++) {
      U si = fn(i, j_lo + w * PER + e);
      pk.e[e] = __ldcg(src + (int64_t)si * gw + w * PER + e);
    }
    __stcs(reinterpret_cast<Wd *>(data + (int64_t)i * pitch + (int64_t)j_lo * EB) + w, pk.w);
  }
}

}  // namespace t213
