// Local transposes used by the block and band plans.
//
// k_tile_swap    transposes every t x t square block of a slice in place
//                (block (I,J) covers rows I*t.., columns J*t.. of the m x n
//                slice).  The block is cut into TS x TS tiles; tile (x,y) and
//                tile (y,x) are read by one CTA and written back transposed
//                into each other's place, so every element is read and written
//                exactly once and no two CTAs touch the same tile.
// k_band_transpose transposes contiguous R x C bands in place through
//                shared memory (a band is at most one CTA's shared memory).
#pragma once

#include "common.cuh"

namespace t213 {

constexpr int kTileThreads = 256;

// Pair index p in [0, nt*(nt+1)/2) -> (x, y) with x <= y, row-major over the
// upper triangle: row x holds nt - x pairs.
__host__ __device__ __forceinline__ void tri_decode(int64_t p, int64_t nt, int64_t &x, int64_t &y) {
  // x = largest r with start(r) = r*nt - r*(r-1)/2 <= p
  double disc = (2.0 * nt + 1.0) * (2.0 * nt + 1.0) - 8.0 * (double)p;
  int64_t r = (int64_t)(((2.0 * nt + 1.0) - sqrt(disc)) * 0.5);
  if (r < 0) r = 0;
  if (r > nt - 1) r = nt - 1;
  while (r > 0 && r * nt - r * (r - 1) / 2 > p) r--;
  while (r + 1 < nt && (r + 1) * nt - (r + 1) * r / 2 <= p) r++;
  x = r;
  y = r + (p - (r * nt - r * (r - 1) / 2));
}

template <int EB, int TS>
__global__ void __launch_bounds__(kTileThreads)
    k_tile_swap(char *__restrict__ data, int64_t n, int64_t slice_elems, int64_t d3, int64_t t,
                int64_t Bm, int64_t Bn, int64_t nt) {
  using E = typename ElemT<EB>::type;
  __shared__ E tA[TS][TS + 1];
  __shared__ E tB[TS][TS + 1];
  E *d = reinterpret_cast<E *>(data);
  const int64_t pairs = nt * (nt + 1) / 2;
  const int64_t per_slice = Bm * Bn * pairs;
  const int64_t total = d3 * per_slice;
  for (int64_t u = blockIdx.x; u < total; u += gridDim.x) {
    const int64_t k = u / per_slice;
    int64_t r = u - k * per_slice;
    const int64_t blk = r / pairs;
    const int64_t p = r - blk * pairs;
    const int64_t I = blk / Bn, J = blk - (blk / Bn) * Bn;
    int64_t x, y;
    tri_decode(p, nt, x, y);
    E *s = d + k * slice_elems + (I * t) * n + J * t;  // block origin
    // tile A at tile coords (x,y): rows x*TS.., cols y*TS..; tile B at (y,x)
    const int64_t ar = x * TS, ac = y * TS;
    const int64_t hA = min((int64_t)TS, t - ar), wA = min((int64_t)TS, t - ac);
    for (int e = threadIdx.x; e < TS * TS; e += blockDim.x) {
      const int uu = e / TS, vv = e % TS;
      if (uu < hA && vv < wA) tA[uu][vv] = __ldcs(s + (ar + uu) * n + ac + vv);
      if (x != y && uu < wA && vv < hA) tB[uu][vv] = __ldcs(s + (ac + uu) * n + ar + vv);
    }
    __syncthreads();
    // B's place (rows ac.., cols ar..) receives A^T; A's place receives B^T
    for (int e = threadIdx.x; e < TS * TS; e += blockDim.x) {
      const int uu = e / TS, vv = e % TS;
      if (uu < wA && vv < hA) __stcs(s + (ac + uu) * n + ar + vv, tA[vv][uu]);
      if (x != y && uu < hA && vv < wA) __stcs(s + (ar + uu) * n + ac + vv, tB[vv][uu]);
    }
    __syncthreads();
  }
}

// Bands: contiguous R x C row-major blocks -> C x R.  Shared memory holds the
// band with row stride S = C + (C even) so the column-wise read is free of
// bank conflicts.
template <int EB>
__global__ void __launch_bounds__(kTileThreads)
    k_band_transpose(char *__restrict__ data, int64_t n_bands, uint32_t R, uint32_t C, uint32_t S,
                     FastDiv<uint32_t> cdiv, FastDiv<uint32_t> rdiv) {
  using E = typename ElemT<EB>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  E *sm = reinterpret_cast<E *>(smem_raw);
  const uint32_t nel = R * C;
  for (int64_t b = blockIdx.x; b < n_bands; b += gridDim.x) {
    E *g = reinterpret_cast<E *>(data) + b * (int64_t)nel;
    for (uint32_t e = threadIdx.x; e < nel; e += blockDim.x) {
      uint32_t r = cdiv.div(e);
      uint32_t c = e - r * C;
      sm[r * S + c] = __ldcs(g + e);
    }
    __syncthreads();
    for (uint32_t o = threadIdx.x; o < nel; o += blockDim.x) {
      uint32_t c = rdiv.div(o);
      uint32_t r = o - c * R;
      __stcs(g + o, sm[r * S + c]);
    }
    __syncthreads();
  }
}

}  // namespace t213
