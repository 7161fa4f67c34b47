// One-pass 213 transpose of slices that fit a thread-block cluster's shared
// memory (up to 16 CTAs of about 220 KB: slices of a few MB).
//
// A cluster of K CTAs takes one slice (m = d2 rows of n = d1 elements) at a
// time.  CTA r loads source rows [r*H, (r+1)*H) into its shared memory (row
// pitch P bytes, padded so that consecutive rows start in different 16-byte
// bank groups).  A cluster barrier orders every load of the slice before any
// store.  Then CTA r writes its share of the output (output rows = source
// columns) straight to global memory, reading the source elements from
// whichever CTA holds them through distributed shared memory.  A second
// barrier keeps each CTA's shared memory alive until the whole cluster has
// read it, before the next slice is loaded.  Every element is read from and
// written to global memory once: one sweep, against the two of the in-place
// plans for larger slices.
//
// The vector form (16-byte aligned rows in and out) moves Q x Q element
// blocks, Q = 16 / element bytes: a thread reads Q source rows of 16 bytes,
// transposes them in registers and stores Q output rows of 16 bytes.  A warp
// takes 32/Q row blocks by Q column blocks, so each output row it writes gets
// 32/Q consecutive 16-byte words, and its 32 shared-memory reads fall into 8
// different 16-byte bank groups (4 wavefronts, the minimum for 512 bytes).
// The element form handles every other alignment one element at a time.
#pragma once

#include <cooperative_groups.h>

#include "common.cuh"
#include "tma.cuh"

namespace t213 {

constexpr int kSliceThreads = 512;

// One slice by one cluster (or CTA): load, barrier, write, barrier.  `s` is
// the slice, m x n elements; this CTA is `rank` of K and holds rows
// [rank*H, (rank+1)*H) at pitch P.
template <int EB, bool VEC, bool CLUSTER>
__device__ __forceinline__ void slice_item(char *slice, uint32_t m, uint32_t n, uint32_t H, uint32_t P,
                                           uint32_t rank, uint32_t K, unsigned char *smem_raw) {
  namespace cg = cooperative_groups;
  using E = typename ElemT<EB>::type;
  E *s = reinterpret_cast<E *>(slice);
  const uint32_t r0 = (uint32_t)min((uint64_t)rank * H, (uint64_t)m);
  const uint32_t r1 = (uint32_t)min((uint64_t)r0 + H, (uint64_t)m);
  auto sync = [&]() {
    if constexpr (CLUSTER)
      cg::this_cluster().sync();
    else
      __syncthreads();
  };
  // shared memory of the CTA that holds source row `row`, at that row
  auto row_ptr = [&](uint32_t row) -> const unsigned char * {
    const uint32_t owner = row / H, lr = row - owner * H;
    const unsigned char *base = smem_raw;
    if constexpr (CLUSTER) base = cg::this_cluster().map_shared_rank(smem_raw, owner);
    return base + (size_t)lr * P;
  };
  // ---- load my source rows --------------------------------------------------
  if constexpr (VEC) {
    const uint32_t upr = n * EB / 16;  // 16-byte units per row
    const uint32_t total = (r1 - r0) * upr;
    for (uint32_t t = threadIdx.x; t < total; t += blockDim.x) {
      const uint32_t rr = t / upr, w = t - rr * upr;
      cp_async<16>(smem_raw + (size_t)rr * P + w * 16,
                   reinterpret_cast<const unsigned char *>(s + (int64_t)(r0 + rr) * n) + w * 16);
    }
    cp_async_wait_all();
  } else {
    const uint32_t total = (r1 - r0) * n;
    for (uint32_t t = threadIdx.x; t < total; t += blockDim.x) {
      const uint32_t rr = t / n, c = t - rr * n;
      *reinterpret_cast<E *>(smem_raw + (size_t)rr * P + (size_t)c * EB) = __ldcs(s + (int64_t)(r0 + rr) * n + c);
    }
  }
  sync();  // the whole slice is in the cluster's shared memory
  // ---- write my share of the output -----------------------------------------
  if constexpr (VEC) {
    constexpr uint32_t Q = 16 / EB;
    constexpr uint32_t RBL = 32 / Q;  // row blocks per warp
    const uint32_t CB = n / Q, RB = m / Q;
    const uint32_t cb0 = (uint32_t)((uint64_t)rank * CB / K), cb1 = (uint32_t)((uint64_t)(rank + 1) * CB / K);
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const uint32_t a = lane % RBL, c = lane / RBL;
    const uint32_t ntr = (RB + RBL - 1) / RBL, ntc = (cb1 - cb0 + Q - 1) / Q;
    const uint32_t ntiles = ntr * ntc;
    // U tiles per round: all their distributed shared-memory reads are issued
    // before any of their stores (the compiler cannot move a read of one tile
    // above a store of another, which might alias)
    constexpr uint32_t U = Q >= 8 ? 1 : 8 / Q;
    union V {
      uint4 v;
      E e[Q];
    };
    for (uint32_t t0 = warp; t0 < ntiles; t0 += nw * U) {
      V in[U][Q];
      bool ok[U];
      uint32_t rbs[U], cbs[U];
#pragma unroll
      for (uint32_t q = 0; q < U; q++) {
        const uint32_t tile = t0 + q * nw;
        const uint32_t tr = tile % ntr, tc = tile / ntr;
        rbs[q] = tr * RBL + a;
        cbs[q] = cb0 + tc * Q + c;
        ok[q] = tile < ntiles && rbs[q] < RB && cbs[q] < cb1;
        if (ok[q]) {
#pragma unroll
          for (uint32_t i = 0; i < Q; i++)
            in[q][i].v = *reinterpret_cast<const uint4 *>(row_ptr(rbs[q] * Q + i) + (size_t)cbs[q] * 16);
        }
      }
#pragma unroll
      for (uint32_t q = 0; q < U; q++) {
        if (!ok[q]) continue;
        V out[Q];
#pragma unroll
        for (uint32_t i = 0; i < Q; i++)
#pragma unroll
          for (uint32_t j = 0; j < Q; j++) out[j].e[i] = in[q][i].e[j];
#pragma unroll
        for (uint32_t j = 0; j < Q; j++)
          __stcs(reinterpret_cast<uint4 *>(s + (int64_t)(cbs[q] * Q + j) * m + rbs[q] * Q), out[j].v);
      }
    }
  } else {
    const uint32_t c0 = (uint32_t)((uint64_t)rank * n / K), c1 = (uint32_t)((uint64_t)(rank + 1) * n / K);
    const int64_t o0 = (int64_t)c0 * m, o1 = (int64_t)c1 * m;
    constexpr int U = 8;  // reads issued before the stores, as above
    const int64_t step = (int64_t)blockDim.x;
    for (int64_t ob = o0 + threadIdx.x; ob < o1; ob += step * U) {
      E v[U];
#pragma unroll
      for (int q = 0; q < U; q++) {
        const int64_t o = ob + q * step;
        if (o < o1) {
          const uint32_t i1 = (uint32_t)(o / m), i2 = (uint32_t)(o - (int64_t)i1 * m);
          v[q] = *reinterpret_cast<const E *>(row_ptr(i2) + (size_t)i1 * EB);
        }
      }
#pragma unroll
      for (int q = 0; q < U; q++)
        if (ob + q * step < o1) s[ob + q * step] = v[q];
    }
  }
  sync();  // every CTA's reads of my shared memory are done
}

template <bool CLUSTER>
__device__ __forceinline__ void cluster_coords(uint32_t &rank, uint32_t &K, int64_t &u0, int64_t &ustride) {
  rank = 0;
  K = 1;
  u0 = blockIdx.x;
  ustride = gridDim.x;
  if constexpr (CLUSTER) {
    cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
    rank = cl.block_rank();
    K = cl.num_blocks();
    u0 = blockIdx.x / K;
    ustride = gridDim.x / K;
  }
}

template <int EB, bool VEC, bool CLUSTER>
__global__ void __launch_bounds__(kSliceThreads)
    k_slice(char *__restrict__ data, int64_t d3, uint32_t m, uint32_t n, uint32_t H, uint32_t P) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t rank, K;
  int64_t u0, ustride;
  cluster_coords<CLUSTER>(rank, K, u0, ustride);
  const int64_t slice_bytes = (int64_t)m * n * EB;
  for (int64_t u = u0; u < d3; u += ustride) slice_item<EB, VEC, CLUSTER>(data + u * slice_bytes, m, n, H, P, rank, K, smem_raw);
}

// Many tensors' slices in one launch (the batched form): entry e has d3
// slices of m x n elements of eb bytes, split over the cluster's CTAs as H
// rows at pitch P each.  Items (entry, slice) are numbered in entry order;
// each cluster walks items u0, u0 + stride, ...
struct SliceEntry {
  char *data;
  int64_t d3;
  int64_t first_item;  // items of the entries before this one
  uint32_t m, n, H, P;
  int32_t eb, vec;
};

template <bool CLUSTER>
__global__ void __launch_bounds__(kSliceThreads)
    k_slice_group(const SliceEntry *__restrict__ entries, int32_t n_entries, int64_t n_items) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t rank, K;
  int64_t u0, ustride;
  cluster_coords<CLUSTER>(rank, K, u0, ustride);
  int32_t e = 0;
  for (int64_t it = u0; it < n_items; it += ustride) {
    while (e + 1 < n_entries && entries[e + 1].first_item <= it) e++;  // items only grow
    const SliceEntry E = entries[e];
    char *slice = E.data + (it - E.first_item) * (int64_t)E.m * E.n * E.eb;
    switch (E.eb * 2 + (E.vec ? 1 : 0)) {
      case 2: slice_item<1, false, CLUSTER>(slice, E.m, E.n, E.H, E.P, rank, K, smem_raw); break;
      case 3: slice_item<1, true, CLUSTER>(slice, E.m, E.n, E.H, E.P, rank, K, smem_raw); break;
      case 4: slice_item<2, false, CLUSTER>(slice, E.m, E.n, E.H, E.P, rank, K, smem_raw); break;
      case 5: slice_item<2, true, CLUSTER>(slice, E.m, E.n, E.H, E.P, rank, K, smem_raw); break;
      case 8: slice_item<4, false, CLUSTER>(slice, E.m, E.n, E.H, E.P, rank, K, smem_raw); break;
      case 9: slice_item<4, true, CLUSTER>(slice, E.m, E.n, E.H, E.P, rank, K, smem_raw); break;
      case 16: slice_item<8, false, CLUSTER>(slice, E.m, E.n, E.H, E.P, rank, K, smem_raw); break;
      case 17: slice_item<8, true, CLUSTER>(slice, E.m, E.n, E.H, E.P, rank, K, smem_raw); break;
      case 32: slice_item<16, false, CLUSTER>(slice, E.m, E.n, E.H, E.P, rank, K, smem_raw); break;
      default: slice_item<16, true, CLUSTER>(slice, E.m, E.n, E.H, E.P, rank, K, smem_raw); break;
    }
  }
}

}  // namespace t213
