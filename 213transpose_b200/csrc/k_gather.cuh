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

// ---------------------------------------------------------------------------
// Row gather with 16-byte global accesses for rows whose pitch is not a
// multiple of 16 bytes (4-byte elements in rows of odd length, and the like).
// A unit of consecutive rows is one contiguous byte range [b0, b1).  The CTA
// loads the 16-byte blocks that cover it with 16-byte cp.async: up to 15 bytes
// on each side belong to the neighbouring units (or lie past the tensor in
// the same 16-byte block, so in the same page); they are read and never used.
// It writes the range back as 16-byte stores between the first and the last
// 16-byte boundary inside it, and as single elements before and after.  A
// thread takes 16/EB consecutive output elements, finds the row and column of
// the first with one division and steps the rest.
// ---------------------------------------------------------------------------
template <int EB, typename F, typename U>
__global__ void __launch_bounds__(kGatherThreads)
    k_row_gather_peel(char *__restrict__ data, int64_t total_rows, U m, U n, int rows_per_unit, FastDiv<U> ndiv,
                      FastDiv<U> mdiv, F fn) {
  using E = typename ElemT<EB>::type;
  constexpr int PER = 16 / EB;
  static_assert(EB < 16, "16-byte elements are always 16-byte aligned");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const E *sm = reinterpret_cast<const E *>(smem_raw);
  const int64_t n_units = (total_rows + rows_per_unit - 1) / rows_per_unit;
  const int64_t row_bytes = (int64_t)n * EB;
  for (int64_t u = blockIdx.x; u < n_units; u += gridDim.x) {
    const int64_t r0 = u * rows_per_unit;
    const int64_t nr = min((int64_t)rows_per_unit, total_rows - r0);
    const uintptr_t b0 = reinterpret_cast<uintptr_t>(data + r0 * row_bytes);
    const uintptr_t b1 = b0 + (uintptr_t)(nr * row_bytes);
    const uintptr_t a0 = b0 & ~(uintptr_t)15, a1 = (b1 + 15) & ~(uintptr_t)15;
    {
      const uint32_t nv = (uint32_t)((a1 - a0) >> 4);
      const uint4 *g = reinterpret_cast<const uint4 *>(a0);
#pragma unroll 4
      for (uint32_t v = threadIdx.x; v < nv; v += blockDim.x) cp_async<16>(smem_raw + 16 * (size_t)v, g + v);
      cp_async_wait_all();
    }
    __syncthreads();
    const U d0 = (U)((b0 - a0) / EB);  // unit element 0 sits at sm[d0]
    const U i_base = (U)(r0 % (int64_t)m);
    const U total = (U)(nr * (int64_t)n);
    // value of unit element q = rr * n + j
    auto value = [&](U rr, U j, U i) -> E { return sm[d0 + rr * n + fn(i, j)]; };
    auto locate = [&](U q, U &rr, U &j, U &i) {
      rr = ndiv.div(q);
      j = q - rr * n;
      const U ii = i_base + rr;
      i = ii < m ? ii : mdiv.mod(ii);
    };
    // 16-byte stores over [c0, c1)
    const uintptr_t c0 = min((b0 + 15) & ~(uintptr_t)15, b1), c1 = max(b1 & ~(uintptr_t)15, c0);
    const U qh = (U)((c0 - b0) / EB), qt = (U)((c1 - b0) / EB);
    const uint32_t nvec = (uint32_t)((c1 - c0) >> 4);
    uint4 *gout = reinterpret_cast<uint4 *>(c0);
    RowStepper<F, U> step(fn);
    for (uint32_t v = threadIdx.x; v < nvec; v += blockDim.x) {
      U rr, j, i;
      locate(qh + (U)v * PER, rr, j, i);
      union {
        uint4 w;
        E e[PER];
      } pk;
      U s = step.first(i, j);
#pragma unroll
      for (int e = 0; e < PER; e++) {
        if (e > 0) {
          if (++j == n) {  // the word runs into the next row
            j = 0;
            rr++;
            if (++i == m) i = 0;
            s = step.first(i, j);
          } else {
            s = step.next(i, j);
          }
        }
        pk.e[e] = sm[d0 + rr * n + s];
      }
      __stcs(gout + v, pk.w);
    }
    // single elements before c0 and from c1 on
    const U nhead = qh, ntail = total - qt;
    for (U t = threadIdx.x; t < nhead + ntail; t += blockDim.x) {
      const U q = t < nhead ? t : qt + (t - nhead);
      U rr, j, i;
      locate(q, rr, j, i);
      reinterpret_cast<E *>(b0)[q] = value(rr, j, i);
    }
    __syncthreads();  // shared memory is restaged by the next unit
  }
}

// ---------------------------------------------------------------------------
// Row gather with the next unit's load in flight: a unit (one or more whole
// rows, at most half the CTA's shared memory) is copied into one of two
// buffers with cp.async groups while the previous unit is gathered from the
// other buffer and written back, so each CTA keeps its loads and its stores
// going at the same time.  Units are this CTA's, in order; a buffer is
// refilled only after the barrier that ends the gather reading it.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async_commit_grp() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_grp1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

template <int EB, int AW, typename F, typename U>
__global__ void __launch_bounds__(kGatherThreads)
    k_row_pipe(char *__restrict__ data, int64_t total_rows, U m, U n, int rows_per_unit, int64_t buf_bytes,
               FastDiv<U> words_per_row, FastDiv<U> mdiv, F fn) {
  using E = typename ElemT<EB>::type;
  using W = typename WordT<AW>::type;
  using P = Pack<AW, EB>;
  constexpr int PER = AW / EB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int64_t n_units = (total_rows + rows_per_unit - 1) / rows_per_unit;
  const int64_t row_bytes = (int64_t)n * EB;

  auto stage = [&](int64_t u, unsigned char *buf) {
    const int64_t r0 = u * rows_per_unit;
    const int nr = (int)min((int64_t)rows_per_unit, total_rows - r0);
    const W *g = reinterpret_cast<const W *>(data + r0 * row_bytes);
    W *sw = reinterpret_cast<W *>(buf);
    const uint32_t nw = (uint32_t)((int64_t)nr * (n / PER));
#pragma unroll 4
    for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x) {
      if constexpr (AW >= 4)
        cp_async<AW>(sw + w, g + w);
      else
        sw[w] = __ldcs(g + w);
    }
    cp_async_commit_grp();
  };

  int64_t u = blockIdx.x;
  if (u >= n_units) return;
  stage(u, smem_raw);
  for (int it = 0; u < n_units; u += gridDim.x, it++) {
    unsigned char *cur = smem_raw + (it & 1) * buf_bytes;
    const int64_t un = u + gridDim.x;
    if (un < n_units)
      stage(un, smem_raw + ((it + 1) & 1) * buf_bytes);
    else
      cp_async_commit_grp();  // an empty group keeps the wait count uniform
    cp_async_wait_grp1();     // this thread's copies of the current unit have landed
    __syncthreads();          // and every other thread's
    const int64_t r0 = u * rows_per_unit;
    const int nr = (int)min((int64_t)rows_per_unit, total_rows - r0);
    W *g = reinterpret_cast<W *>(data + r0 * row_bytes);
    const E *sm = reinterpret_cast<const E *>(cur);
    const uint32_t nw = (uint32_t)((int64_t)nr * (n / PER));
    const U i_base = (U)(r0 % (int64_t)m);
    for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x) {
      const U rr = words_per_row.div((U)w);
      const U j0 = ((U)w - rr * words_per_row.get()) * PER;
      const U i = mdiv.mod(i_base + rr);
      typename P::U pk;
#pragma unroll
      for (int e = 0; e < PER; e++) pk.e[e] = sm[(int64_t)rr * n + fn(i, j0 + e)];
      __stcs(g + w, pk.w);
    }
    __syncthreads();  // the buffer is restaged two units later
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

// ---------------------------------------------------------------------------
// Cluster-local column gather.  Every column functor of the decomposition has
// one of two forms:
//   src(i, j) = (pi(i) + r(j)) mod m       rotators, fused pre/post-ops of C2R
//                                           and the R2C fused post-op
//   src(i, j) = p((i - j) mod m)           the R2C fused pre-op
// Written in a key space kappa (kappa = pi(i), or kappa = i), the source row of
// output (kappa, column j0 + w) of a strip is F((kappa + r_w) mod m), with F
// the identity or p and r_w = r(j0 + w) (or -(j0 + w)) varying by at most a
// few rows across the W columns of the strip.  So the keys [k0, k1) of one CTA
// need only the source rows F(k0 + r_0 + dmin ... k1 + r_0 + dmax): the CTA's
// share of the strip plus a halo of (dmax - dmin) rows.  The CTAs of a cluster
// split the keys, each loads its rows (halo included) into its own shared
// memory, the cluster barrier orders every load of the strip before any
// store, and each CTA writes its output rows G(kappa) (G = pi^-1 or the
// identity) from its own shared memory.  No element crosses DSMEM; the
// strips can be 128-256 bytes wide however tall the matrix is.  A strip short
// enough for one CTA is held whole instead: slot = key, no halo, and the
// source slot of (kappa, w) is (kappa + r_w) mod m.
//
// The loops keep the index work per element small: a lane owns one word
// (16 bytes, or one element) of every row it touches, evaluates F or G once
// for 32 rows and passes the results around by shuffles, and reads the
// per-column shifts once per strip.
// ---------------------------------------------------------------------------
template <typename U>
struct MapId {
  T213_HD U operator()(U x) const { return x; }
};

// Key offset of column j: the column functor at row 0 (form 1 with pi(0) = 0).
template <typename U, typename F>
struct OffOfCol {
  F f;
  T213_HD U operator()(U j) const { return f((U)0, j); }
};

// Key offset +-(j mod m) (C2R fused post-op: +j; R2C fused pre-op: -j).
template <typename U, bool NEG>
struct OffAffine {
  FastDiv<U> m;
  T213_HD U operator()(U j) const {
    const U r = m.mod(j);
    return NEG ? (r ? m.get() - r : 0) : r;
  }
};

constexpr int kColHaloMax = 64;  // largest halo (dmax - dmin) a strip may need

// The barrier between a strip's loads and its stores in the cluster-local
// column kernels.  Each thread has waited for its own cp.async copies, so
// every global read of the strip has been performed and its value sits in
// shared memory: the cluster barrier only has to order execution (no CTA
// stores before every CTA's reads are done), and a relaxed arrive spares each
// thread the release fence, which would wait for its previous strip's global
// stores to drain.  The CTA barrier before it makes the staged shared memory
// visible to all threads of the CTA.
__device__ __forceinline__ void strip_loaded_barrier() {
  __syncthreads();
  asm volatile("barrier.cluster.arrive.relaxed.aligned;\n\tbarrier.cluster.wait.aligned;" ::: "memory");
}

template <int EB, int AW, typename U, typename Off, typename Fsrc, typename Gout, bool CLUSTER>
__global__ void __launch_bounds__(kGatherThreads)
    k_col_local(char *__restrict__ data, int64_t d3, U m, U n, U W, U WS, int64_t n_strips, U H, int halo, Off off,
                Fsrc F, Gout G, int *status) {
  using E = typename ElemT<EB>::type;
  using Wd = typename WordT<AW>::type;
  using P = Pack<AW, EB>;
  constexpr int PER = AW / EB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  E *sm = reinterpret_cast<E *>(smem_raw);
  __shared__ int s_sh[256];  // per column of the strip: slot shift (halo mode) or key offset r_w (whole mode)
  __shared__ int s_span;
  __shared__ U s_base;

  int rank = 0, K = 1;
  int64_t unit0 = blockIdx.x, ustride = gridDim.x;
  if (CLUSTER) {
    cg::cluster_group cl = cg::this_cluster();
    rank = (int)cl.block_rank();
    K = (int)cl.num_blocks();
    unit0 = blockIdx.x / K;
    ustride = gridDim.x / K;
  }
  // whole mode: one CTA owns every key of the strip, slot = key, no halo
  const bool whole = !CLUSTER && H >= m;
  const int64_t n_units = d3 * n_strips;
  const U k0 = (U)min((int64_t)rank * (int64_t)H, (int64_t)m);
  const U k1 = (U)min((int64_t)k0 + (int64_t)H, (int64_t)m);
  const U nk = k1 - k0;
  const int64_t pitch = (int64_t)n * EB;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;

  for (int64_t u = unit0; u < n_units; u += ustride) {
    const int64_t k = u / n_strips;
    const U s = (U)(u - k * n_strips);
    const U j0 = s * W;
    const U wn = min(W, n - j0);  // multiple of PER
    const uint32_t wpr = (uint32_t)(wn / PER);
    char *sbase = data + (k * (int64_t)m * n + j0) * EB;
    // ---- per-strip column offsets -------------------------------------------
    if (warp == 0) {
      const int64_t mm = (int64_t)m;
      const int64_t r0 = (int64_t)off(j0);
      int dmin = 0, dmax = 0;
      for (U w = lane; w < wn; w += 32) {
        const int64_t rw = (int64_t)off(j0 + w);
        int64_t d = rw - r0;
        if (2 * d > mm) d -= mm;
        if (2 * d <= -mm) d += mm;
        s_sh[w] = whole ? (int)rw : (int)d;
        dmin = min(dmin, (int)d);
        dmax = max(dmax, (int)d);
      }
      for (int o = 16; o > 0; o >>= 1) {
        dmin = min(dmin, __shfl_xor_sync(0xffffffffu, dmin, o));
        dmax = max(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
      }
      __syncwarp();
      if (!whole)
        for (U w = lane; w < wn; w += 32) s_sh[w] -= dmin;
      if (lane == 0) {
        s_span = whole ? 0 : dmax - dmin;
        int64_t b = whole ? 0 : ((int64_t)k0 + r0 + dmin) % mm;
        if (b < 0) b += mm;
        s_base = (U)b;
      }
    }
    __syncthreads();
    // the host sized shared memory for its own scan of every strip's span;
    // a strip that needs more records an error and moves no data
    const bool fits = s_span <= halo;
    if (!fits && threadIdx.x == 0) atomicExch(status, 1 /* T213_ERR_INVALID_ARGUMENT */);
    const U nslots = !fits ? 0 : whole ? m : (nk > 0 ? nk + (U)s_span : 0);
    const U nout = fits ? nk : 0;
    const U base = s_base;
    auto key_of_slot = [&](U sl) -> U {
      U key = base + sl;
      return key >= m ? key - m : key;
    };
    auto slot_of = [&](U o, int sh) -> U {  // source slot of output o for a column with shift sh
      if (whole) {
        U v = k0 + o + (U)sh;  // key + r_w < 2m
        return v >= m ? v - m : v;
      }
      return o + (U)sh;
    };
    if (32 % wpr == 0) {
      // ---- fast path: a lane keeps one word of the strip's rows; the row maps
      // are evaluated once per lane for 32 rows and broadcast by shuffles
      const uint32_t rpi = 32 / wpr, lr = lane / wpr, lw = lane - lr * wpr;
      int sh[PER];
#pragma unroll
      for (int e = 0; e < PER; e++) sh[e] = s_sh[lw * PER + e];
      for (U sb = (U)warp * 32; sb < nslots; sb += (U)nwarps * 32) {
        const U mys = sb + lane;
        const U myrow = mys < nslots ? F(key_of_slot(mys)) : 0;
#pragma unroll 4
        for (uint32_t r = lr; r < 32; r += rpi) {
          const U row = __shfl_sync(0xffffffffu, myrow, r);
          const U sl = sb + r;
          if (sl < nslots) {
            const Wd *gp = reinterpret_cast<const Wd *>(sbase + (int64_t)row * pitch) + lw;
            Wd *dp = reinterpret_cast<Wd *>(sm + (int64_t)sl * WS) + lw;
            if constexpr (AW >= 4)
              cp_async<AW>(dp, gp);
            else
              *dp = __ldcs(gp);
          }
        }
      }
      if constexpr (AW >= 4) cp_async_wait_all();
      // every CTA of the strip has read its rows before anyone writes
      if (CLUSTER)
        strip_loaded_barrier();
      else
        __syncthreads();
      for (U ob = (U)warp * 32; ob < nout; ob += (U)nwarps * 32) {
        const U myo = ob + lane;
        const U myrow = myo < nout ? G(k0 + myo) : 0;
#pragma unroll 4
        for (uint32_t r = lr; r < 32; r += rpi) {
          const U row = __shfl_sync(0xffffffffu, myrow, r);
          const U o = ob + r;
          if (o < nout) {
            typename P::U pk;
#pragma unroll
            for (int e = 0; e < PER; e++) pk.e[e] = sm[(int64_t)slot_of(o, sh[e]) * WS + lw * PER + e];
            __stcs(reinterpret_cast<Wd *>(sbase + (int64_t)row * pitch) + lw, pk.w);
          }
        }
      }
    } else {
      // ---- any strip width (the last, narrower strip) -------------------------
      const uint32_t nw = (uint32_t)nslots * wpr;
      for (uint32_t t = threadIdx.x; t < nw; t += blockDim.x) {
        const uint32_t sl = t / wpr, w = t - sl * wpr;
        const U row = F(key_of_slot((U)sl));
        const Wd *gp = reinterpret_cast<const Wd *>(sbase + (int64_t)row * pitch) + w;
        if constexpr (AW >= 4)
          cp_async<AW>(reinterpret_cast<Wd *>(sm + (int64_t)sl * WS) + w, gp);
        else
          reinterpret_cast<Wd *>(sm + (int64_t)sl * WS)[w] = __ldcs(gp);
      }
      if constexpr (AW >= 4) cp_async_wait_all();
      if (CLUSTER)
        strip_loaded_barrier();
      else
        __syncthreads();
      const uint32_t nwo = (uint32_t)nout * wpr;
      for (uint32_t t = threadIdx.x; t < nwo; t += blockDim.x) {
        const uint32_t o = t / wpr, w = t - o * wpr;
        const U row = G(k0 + (U)o);
        typename P::U pk;
#pragma unroll
        for (int e = 0; e < PER; e++) {
          const int c = (int)(w * PER + e);
          pk.e[e] = sm[(int64_t)slot_of((U)o, s_sh[c]) * WS + c];
        }
        __stcs(reinterpret_cast<Wd *>(sbase + (int64_t)row * pitch) + w, pk.w);
      }
    }
    __syncthreads();  // shared memory and s_sh are reused by the next strip
  }
}

// ---------------------------------------------------------------------------
// k_col_local with 16-byte global accesses for rows whose pitch is not a
// multiple of 16 bytes (4- and 8-byte elements, n odd or n = 2 mod 4).  A strip
// is W * EB = 16 L bytes wide, so its start has the same offset a(row) inside
// a 16-byte block as its row (the strip starts are 16-byte multiples apart).
// A slot of shared memory (stride SB = 16 L + 16 bytes) takes the 16-byte
// blocks covering the strip's bytes of one source row: L of them, or L + 1
// when a(row) != 0; up to 15 bytes on either side belong to the neighbouring
// strips and are read and never used.  Element q of the slot sits at byte
// a + q * EB; a per-slot byte table keeps a.  An output row is written by L
// lanes: lane l takes the 16-byte block that starts h + l * PER elements into
// the row (h = elements before the row's first 16-byte boundary), so every
// lane but the last stores one 16-byte vector; the last lane's block runs
// past the strip by h elements, which are the row's first h elements: it
// stores its elements one by one, those past the strip at the row's start.
// The last strip of a row, when narrower, moves element by element.
// Cluster, halo and key-space logic are those of k_col_local.
// ---------------------------------------------------------------------------
template <int EB, typename U, typename Off, typename Fsrc, typename Gout, bool CLUSTER>
__global__ void __launch_bounds__(kGatherThreads)
    k_col_local_peel(char *__restrict__ data, int64_t d3, U m, U n, U W, U SB, U max_slots, int64_t n_strips, U H,
                     int halo, Off off, Fsrc F, Gout G, int *status) {
  static_assert(EB == 4 || EB == 8, "4- and 8-byte elements");
  using E = typename ElemT<EB>::type;
  constexpr int PER = 16 / EB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char *s_al = smem_raw + (size_t)max_slots * SB;  // per slot: byte offset of element 0
  __shared__ int s_sh[256];
  __shared__ int s_span;
  __shared__ U s_base;

  int rank = 0, K = 1;
  int64_t unit0 = blockIdx.x, ustride = gridDim.x;
  if (CLUSTER) {
    cg::cluster_group cl = cg::this_cluster();
    rank = (int)cl.block_rank();
    K = (int)cl.num_blocks();
    unit0 = blockIdx.x / K;
    ustride = gridDim.x / K;
  }
  const bool whole = !CLUSTER && H >= m;
  const int64_t n_units = d3 * n_strips;
  const U k0 = (U)min((int64_t)rank * (int64_t)H, (int64_t)m);
  const U k1 = (U)min((int64_t)k0 + (int64_t)H, (int64_t)m);
  const U nk = k1 - k0;
  const int64_t pitch = (int64_t)n * EB;
  const uint32_t pm = (uint32_t)(pitch & 15);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const uint32_t L = (uint32_t)(W * EB / 16);  // lanes per row; divides 32 (host: W * EB in {64, 128, 256, 512})
  const uint32_t rpi = 32 / L, lr = lane / L, lw = lane - lr * L;

  for (int64_t u = unit0; u < n_units; u += ustride) {
    const int64_t k = u / n_strips;
    const U s = (U)(u - k * n_strips);
    const U j0 = s * W;
    const U wn = min(W, n - j0);
    char *sbase = data + (k * (int64_t)m * n + j0) * EB;
    // offset of the strip inside a 16-byte block: (cb + row * pm) & 15
    const uint32_t cb = (uint32_t)(reinterpret_cast<uintptr_t>(sbase) & 15);
    if (warp == 0) {
      const int64_t mm = (int64_t)m;
      const int64_t r0 = (int64_t)off(j0);
      int dmin = 0, dmax = 0;
      for (U w = lane; w < wn; w += 32) {
        const int64_t rw = (int64_t)off(j0 + w);
        int64_t d = rw - r0;
        if (2 * d > mm) d -= mm;
        if (2 * d <= -mm) d += mm;
        s_sh[w] = whole ? (int)rw : (int)d;
        dmin = min(dmin, (int)d);
        dmax = max(dmax, (int)d);
      }
      for (int o = 16; o > 0; o >>= 1) {
        dmin = min(dmin, __shfl_xor_sync(0xffffffffu, dmin, o));
        dmax = max(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
      }
      __syncwarp();
      if (!whole)
        for (U w = lane; w < wn; w += 32) s_sh[w] -= dmin;
      if (lane == 0) {
        s_span = whole ? 0 : dmax - dmin;
        int64_t b = whole ? 0 : ((int64_t)k0 + r0 + dmin) % mm;
        if (b < 0) b += mm;
        s_base = (U)b;
      }
    }
    __syncthreads();
    const bool fits = s_span <= halo;
    if (!fits && threadIdx.x == 0) atomicExch(status, 1 /* T213_ERR_INVALID_ARGUMENT */);
    const U nslots = !fits ? 0 : whole ? m : (nk > 0 ? nk + (U)s_span : 0);
    const U nout = fits ? nk : 0;
    const U base = s_base;
    auto key_of_slot = [&](U sl) -> U {
      U key = base + sl;
      return key >= m ? key - m : key;
    };
    auto slot_of = [&](U o, int sh) -> U {
      if (whole) {
        U v = k0 + o + (U)sh;
        return v >= m ? v - m : v;
      }
      return o + (U)sh;
    };
    auto elem = [&](U sl, U q) -> E {
      return *reinterpret_cast<const E *>(smem_raw + (size_t)sl * SB + s_al[sl] + (size_t)q * EB);
    };
    if (wn == W) {
      // ---- loads: L lanes per source row, one more block when unaligned ----
      for (U sb = (U)warp * 32; sb < nslots; sb += (U)nwarps * 32) {
        const U mys = sb + lane;
        const U myrow = mys < nslots ? F(key_of_slot(mys)) : 0;
        if (mys < nslots) s_al[mys] = (unsigned char)((cb + (uint32_t)myrow * pm) & 15u);
#pragma unroll 4
        for (uint32_t r = lr; r < 32; r += rpi) {
          const U row = __shfl_sync(0xffffffffu, myrow, r);
          const U sl = sb + r;
          if (sl < nslots) {
            const uintptr_t A = reinterpret_cast<uintptr_t>(sbase + (int64_t)row * pitch);
            const char *g0 = reinterpret_cast<const char *>(A & ~(uintptr_t)15);
            unsigned char *d0 = smem_raw + (size_t)sl * SB;
            cp_async<16>(d0 + 16 * lw, g0 + 16 * lw);
            if (lw == L - 1 && (A & 15)) cp_async<16>(d0 + 16 * L, g0 + 16 * L);
          }
        }
      }
      cp_async_wait_all();
      if (CLUSTER)
        strip_loaded_barrier();
      else
        __syncthreads();
      // ---- stores: the shifts of the 2 PER - 1 columns a lane may take -----
      int shr[2 * PER - 1];
#pragma unroll
      for (int t = 0; t < 2 * PER - 1; t++) {
        uint32_t q = lw * PER + t;
        if (q >= (uint32_t)W) q -= (uint32_t)W;
        shr[t] = s_sh[q];
      }
      for (U ob = (U)warp * 32; ob < nout; ob += (U)nwarps * 32) {
        const U myo = ob + lane;
        const U myrow = myo < nout ? G(k0 + myo) : 0;
#pragma unroll 2
        for (uint32_t r = lr; r < 32; r += rpi) {
          const U row = __shfl_sync(0xffffffffu, myrow, r);
          const U o = ob + r;
          if (o < nout) {
            char *B = sbase + (int64_t)row * pitch;
            const uint32_t ab = (cb + (uint32_t)row * pm) & 15u;
            const uint32_t h = ((16u - ab) & 15u) / EB;  // elements before the row's first 16-byte boundary
            union {
              uint4 w;
              E e[PER];
            } pk;
#pragma unroll
            for (int e = 0; e < PER; e++) {
              int sh = shr[e];
#pragma unroll
              for (int t = 1; t < PER; t++)
                if (h == (uint32_t)t) sh = shr[t + e];
              U q = (U)(lw * PER + h + e);
              if (q >= W) q -= W;
              pk.e[e] = elem(slot_of(o, sh), q);
            }
            if (lw < L - 1 || h == 0) {
              __stcs(reinterpret_cast<uint4 *>(B + (size_t)(h + lw * PER) * EB), pk.w);
            } else {
#pragma unroll
              for (int e = 0; e < PER; e++) {
                U q = (U)(lw * PER + h + e);
                if (q >= W) q -= W;
                reinterpret_cast<E *>(B)[q] = pk.e[e];
              }
            }
          }
        }
      }
    } else {
      // ---- the narrower last strip: element by element, element q at q * EB --
      const uint32_t nw = (uint32_t)nslots * (uint32_t)wn;
      for (uint32_t t = threadIdx.x; t < nw; t += blockDim.x) {
        const uint32_t sl = t / (uint32_t)wn, q = t - sl * (uint32_t)wn;
        const U row = F(key_of_slot((U)sl));
        if (q == 0) s_al[sl] = 0;
        cp_async<EB>(smem_raw + (size_t)sl * SB + (size_t)q * EB, sbase + (int64_t)row * pitch + (int64_t)q * EB);
      }
      cp_async_wait_all();
      if (CLUSTER)
        strip_loaded_barrier();
      else
        __syncthreads();
      const uint32_t nwo = (uint32_t)nout * (uint32_t)wn;
      for (uint32_t t = threadIdx.x; t < nwo; t += blockDim.x) {
        const uint32_t o = t / (uint32_t)wn, q = t - o * (uint32_t)wn;
        const U row = G(k0 + (U)o);
        reinterpret_cast<E *>(sbase + (int64_t)row * pitch)[q] = elem(slot_of((U)o, s_sh[q]), (U)q);
      }
    }
    __syncthreads();  // shared memory, the slot table and s_sh are reused by the next strip
  }
}

// Double-buffered form of k_col_local: shared memory holds two strips, and
// the loads of a CTA's next strip are issued right after the barrier that
// ends the current strip's loads, so they are in flight while the current
// strip is written back.  One cluster (or CTA) barrier per strip orders (a)
// every load of strip u before any store of strip u, and (b) every store of
// the strip before u (which read the other buffer) before that buffer is
// loaded again.  Strips of one CTA are different columns, so the next strip's
// loads never read what the current strip's stores write.
template <int EB, int AW, typename U, typename Off, typename Fsrc, typename Gout, bool CLUSTER>
__global__ void __launch_bounds__(kGatherThreads)
    k_col_local_db(char *__restrict__ data, int64_t d3, U m, U n, U W, U WS, int64_t n_strips, U H, int halo,
                   Off off, Fsrc F, Gout G, int64_t buf_elems, int *status) {
  using E = typename ElemT<EB>::type;
  using Wd = typename WordT<AW>::type;
  using P = Pack<AW, EB>;
  constexpr int PER = AW / EB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_sh[2][256];
  __shared__ int s_span[2];
  __shared__ U s_base[2];

  int rank = 0, K = 1;
  int64_t unit0 = blockIdx.x, ustride = gridDim.x;
  if (CLUSTER) {
    cg::cluster_group cl = cg::this_cluster();
    rank = (int)cl.block_rank();
    K = (int)cl.num_blocks();
    unit0 = blockIdx.x / K;
    ustride = gridDim.x / K;
  }
  const bool whole = !CLUSTER && H >= m;
  const int64_t n_units = d3 * n_strips;
  const U k0 = (U)min((int64_t)rank * (int64_t)H, (int64_t)m);
  const U k1 = (U)min((int64_t)k0 + (int64_t)H, (int64_t)m);
  const U nk = k1 - k0;
  const int64_t pitch = (int64_t)n * EB;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;

  struct Geo {
    char *sbase;
    U j0, wn;
    uint32_t wpr;
  };
  auto geo = [&](int64_t u) {
    Geo g;
    const int64_t k = u / n_strips;
    const U s = (U)(u - k * n_strips);
    g.j0 = s * W;
    g.wn = min(W, n - g.j0);  // multiple of PER
    g.wpr = (uint32_t)(g.wn / PER);
    g.sbase = data + (k * (int64_t)m * n + g.j0) * EB;
    return g;
  };
  // warp 0: the strip's column offsets into slot b
  auto prep = [&](const Geo &g, int b) {
    const int64_t mm = (int64_t)m;
    const int64_t r0 = (int64_t)off(g.j0);
    int dmin = 0, dmax = 0;
    for (U w = lane; w < g.wn; w += 32) {
      const int64_t rw = (int64_t)off(g.j0 + w);
      int64_t d = rw - r0;
      if (2 * d > mm) d -= mm;
      if (2 * d <= -mm) d += mm;
      s_sh[b][w] = whole ? (int)rw : (int)d;
      dmin = min(dmin, (int)d);
      dmax = max(dmax, (int)d);
    }
    for (int o = 16; o > 0; o >>= 1) {
      dmin = min(dmin, __shfl_xor_sync(0xffffffffu, dmin, o));
      dmax = max(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    }
    __syncwarp();
    if (!whole)
      for (U w = lane; w < g.wn; w += 32) s_sh[b][w] -= dmin;
    if (lane == 0) {
      s_span[b] = whole ? 0 : dmax - dmin;
      int64_t bb = whole ? 0 : ((int64_t)k0 + r0 + dmin) % mm;
      if (bb < 0) bb += mm;
      s_base[b] = (U)bb;
    }
  };
  auto key_of_slot = [&](U sl, U base) -> U {
    U key = base + sl;
    return key >= m ? key - m : key;
  };
  auto slot_of = [&](U o, int sh) -> U {
    if (whole) {
      U v = k0 + o + (U)sh;
      return v >= m ? v - m : v;
    }
    return o + (U)sh;
  };
  // the host sized shared memory for its own scan of every strip's span; a
  // strip that needs more records an error and moves no data
  auto slots_of = [&](int b) -> U {
    if (s_span[b] > halo) return 0;
    return whole ? m : (nk > 0 ? nk + (U)s_span[b] : 0);
  };
  auto load = [&](const Geo &g, int b) {
    E *sm = reinterpret_cast<E *>(smem_raw) + (int64_t)b * buf_elems;
    const U nslots = slots_of(b);
    const U base = s_base[b];
    if (s_span[b] > halo && threadIdx.x == 0) atomicExch(status, 1 /* T213_ERR_INVALID_ARGUMENT */);
    if (32 % g.wpr == 0) {
      const uint32_t rpi = 32 / g.wpr, lr = lane / g.wpr, lw = lane - lr * g.wpr;
      for (U sb = (U)warp * 32; sb < nslots; sb += (U)nwarps * 32) {
        const U mys = sb + lane;
        const U myrow = mys < nslots ? F(key_of_slot(mys, base)) : 0;
        for (uint32_t r = lr; r < 32; r += rpi) {
          const U row = __shfl_sync(0xffffffffu, myrow, r);
          const U sl = sb + r;
          if (sl < nslots) {
            const Wd *gp = reinterpret_cast<const Wd *>(g.sbase + (int64_t)row * pitch) + lw;
            Wd *dp = reinterpret_cast<Wd *>(sm + (int64_t)sl * WS) + lw;
            if constexpr (AW >= 4)
              cp_async<AW>(dp, gp);
            else
              *dp = __ldcs(gp);
          }
        }
      }
    } else {
      const uint32_t nw = (uint32_t)nslots * g.wpr;
      for (uint32_t t = threadIdx.x; t < nw; t += blockDim.x) {
        const uint32_t sl = t / g.wpr, w = t - sl * g.wpr;
        const U row = F(key_of_slot((U)sl, base));
        const Wd *gp = reinterpret_cast<const Wd *>(g.sbase + (int64_t)row * pitch) + w;
        if constexpr (AW >= 4)
          cp_async<AW>(reinterpret_cast<Wd *>(sm + (int64_t)sl * WS) + w, gp);
        else
          reinterpret_cast<Wd *>(sm + (int64_t)sl * WS)[w] = __ldcs(gp);
      }
    }
  };
  auto store = [&](const Geo &g, int b) {
    const E *sm = reinterpret_cast<const E *>(smem_raw) + (int64_t)b * buf_elems;
    const U nout = s_span[b] <= halo ? nk : 0;
    if (32 % g.wpr == 0) {
      const uint32_t rpi = 32 / g.wpr, lr = lane / g.wpr, lw = lane - lr * g.wpr;
      int sh[PER];
#pragma unroll
      for (int e = 0; e < PER; e++) sh[e] = s_sh[b][lw * PER + e];
      for (U ob = (U)warp * 32; ob < nout; ob += (U)nwarps * 32) {
        const U myo = ob + lane;
        const U myrow = myo < nout ? G(k0 + myo) : 0;
        for (uint32_t r = lr; r < 32; r += rpi) {
          const U row = __shfl_sync(0xffffffffu, myrow, r);
          const U o = ob + r;
          if (o < nout) {
            typename P::U pk;
#pragma unroll
            for (int e = 0; e < PER; e++) pk.e[e] = sm[(int64_t)slot_of(o, sh[e]) * WS + lw * PER + e];
            __stcs(reinterpret_cast<Wd *>(g.sbase + (int64_t)row * pitch) + lw, pk.w);
          }
        }
      }
    } else {
      const uint32_t nwo = (uint32_t)nout * g.wpr;
      for (uint32_t t = threadIdx.x; t < nwo; t += blockDim.x) {
        const uint32_t o = t / g.wpr, w = t - o * g.wpr;
        const U row = G(k0 + (U)o);
        typename P::U pk;
#pragma unroll
        for (int e = 0; e < PER; e++) {
          const int c = (int)(w * PER + e);
          pk.e[e] = sm[(int64_t)slot_of((U)o, s_sh[b][c]) * WS + c];
        }
        __stcs(reinterpret_cast<Wd *>(g.sbase + (int64_t)row * pitch) + w, pk.w);
      }
    }
  };
  auto barrier = [&]() {
    if (CLUSTER)
      cg::this_cluster().sync();
    else
      __syncthreads();
  };

  int64_t u = unit0;
  if (u >= n_units) return;  // the same for every CTA of a cluster
  Geo cur = geo(u);
  if (warp == 0) prep(cur, 0);
  __syncthreads();
  load(cur, 0);
  for (int b = 0; u < n_units; u += ustride, b ^= 1) {
    if constexpr (AW >= 4) cp_async_wait_all();  // this strip's loads (the only ones in flight)
    barrier();  // (a) strip u loaded everywhere; (b) the previous strip's stores are done
    const int64_t un = u + ustride;
    Geo nxt;
    if (un < n_units) {
      nxt = geo(un);
      if (warp == 0) prep(nxt, b ^ 1);
      __syncthreads();
      load(nxt, b ^ 1);  // in flight during the stores below
    }
    store(cur, b);
    cur = nxt;
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
