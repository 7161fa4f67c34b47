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

template <int EB, bool VEC, bool CLUSTER>
__global__ void __launch_bounds__(kSliceThreads)
    k_slice(char *__restrict__ data, int64_t d3, uint32_t m, uint32_t n, uint32_t H, uint32_t P) {
  namespace cg = cooperative_groups;
  using E = typename ElemT<EB>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t rank = 0, K = 1;
  int64_t u0 = blockIdx.x, ustride = gridDim.x;
  if constexpr (CLUSTER) {
    cg::cluster_group cl = cg::this_cluster();
    rank = cl.block_rank();
    K = cl.num_blocks();
    u0 = blockIdx.x / K;
    ustride = gridDim.x / K;
  }
  const uint32_t r0 = (uint32_t)min((uint64_t)rank * H, (uint64_t)m);
  const uint32_t r1 = (uint32_t)min((uint64_t)r0 + H, (uint64_t)m);
  const int64_t slice_elems = (int64_t)m * n;
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

  for (int64_t u = u0; u < d3; u += ustride) {
    E *s = reinterpret_cast<E *>(data) + u * slice_elems;
    // ---- load my source rows ------------------------------------------------
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
    // ---- write my share of the output ---------------------------------------
    if constexpr (VEC) {
      constexpr uint32_t Q = 16 / EB;
      constexpr uint32_t RBL = 32 / Q;  // row blocks per warp
      const uint32_t CB = n / Q, RB = m / Q;
      const uint32_t cb0 = (uint32_t)((uint64_t)rank * CB / K), cb1 = (uint32_t)((uint64_t)(rank + 1) * CB / K);
      const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
      const uint32_t a = lane % RBL, c = lane / RBL;
      const uint32_t ntr = (RB + RBL - 1) / RBL, ntc = (cb1 - cb0 + Q - 1) / Q;
      for (uint32_t tile = warp; tile < ntr * ntc; tile += nw) {
        const uint32_t tr = tile % ntr, tc = tile / ntr;
        const uint32_t rb = tr * RBL + a, cb = cb0 + tc * Q + c;
        if (rb < RB && cb < cb1) {
          union V {
            uint4 v;
            E e[Q];
          } in[Q], out[Q];
#pragma unroll
          for (uint32_t i = 0; i < Q; i++)
            in[i].v = *reinterpret_cast<const uint4 *>(row_ptr(rb * Q + i) + (size_t)cb * 16);
#pragma unroll
          for (uint32_t i = 0; i < Q; i++)
#pragma unroll
            for (uint32_t j = 0; j < Q; j++) out[j].e[i] = in[i].e[j];
#pragma unroll
          for (uint32_t j = 0; j < Q; j++)
            __stcs(reinterpret_cast<uint4 *>(s + (int64_t)(cb * Q + j) * m + rb * Q), out[j].v);
        }
      }
    } else {
      const uint32_t c0 = (uint32_t)((uint64_t)rank * n / K), c1 = (uint32_t)((uint64_t)(rank + 1) * n / K);
      const int64_t o0 = (int64_t)c0 * m, o1 = (int64_t)c1 * m;
      for (int64_t o = o0 + threadIdx.x; o < o1; o += blockDim.x) {
        const uint32_t i1 = (uint32_t)(o / m), i2 = (uint32_t)(o - (int64_t)i1 * m);
        s[o] = *reinterpret_cast<const E *>(row_ptr(i2) + (size_t)i1 * EB);
      }
    }
    sync();  // every CTA's reads of my shared memory are done
  }
}

}  // namespace t213
