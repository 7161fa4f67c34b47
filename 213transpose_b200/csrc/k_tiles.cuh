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
#include "tma.cuh"

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

// 32-bit variant for pair counts below 2^31: float square root, then the
// same exact +-1 corrections.
__device__ __forceinline__ void tri_decode32(uint32_t p, uint32_t nt, uint32_t &x, uint32_t &y) {
  const float b = 2.0f * (float)nt + 1.0f;
  int r = (int)((b - sqrtf(fmaxf(b * b - 8.0f * (float)p, 0.0f))) * 0.5f);
  if (r < 0) r = 0;
  if (r > (int)nt - 1) r = (int)nt - 1;
  auto start = [&](int64_t q) { return q * (int64_t)nt - q * (q - 1) / 2; };
  while (r > 0 && start(r) > (int64_t)p) r--;
  while (r + 1 < (int)nt && start(r + 1) <= (int64_t)p) r++;
  x = (uint32_t)r;
  y = (uint32_t)(r + ((int64_t)p - start(r)));
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

// Vectorised tile swap for 4-, 8- and 16-byte elements and blocks whose side
// is a multiple of 32: tiles are 32 x 32 elements, every global access is a
// 16-byte vector (a tile row is RV = 2*EB vectors), shared memory rows have a
// stride of 33 elements so both the row-wise fill and the column-wise drain
// are free of bank conflicts, and the vectors of the next tile pair are loaded
// into registers before the current pair is written back, so each thread
// keeps two pairs of loads in flight.
template <int EB>
struct TileVec {
  static constexpr int RV = 2 * EB;            // 16-byte vectors per tile row
  static constexpr int PE = 16 / EB;           // elements per vector
  static constexpr int VPT = (32 * RV) / kTileThreads;  // vectors per thread per tile
};

template <int EB>
__global__ void __launch_bounds__(kTileThreads)
    k_tile_swap_vec(char *__restrict__ data, int64_t n, int64_t slice_elems, uint32_t total, int64_t t,
                    FastDiv<uint32_t> fd_per_slice, FastDiv<uint32_t> fd_pairs, FastDiv<uint32_t> fd_Bn, uint32_t nt) {
  using E = typename ElemT<EB>::type;
  constexpr int RV = TileVec<EB>::RV, PE = TileVec<EB>::PE, VPT = TileVec<EB>::VPT;
  constexpr int S = 33;
  __shared__ E tA[32 * S];
  __shared__ E tB[32 * S];
  union V {
    uint4 v;
    E e[PE];
  };
  E *d = reinterpret_cast<E *>(data);

  auto origin = [&](uint32_t u, int64_t &ar, int64_t &ac, bool &diag) -> E * {
    const uint32_t k = fd_per_slice.div(u);
    const uint32_t r = u - k * fd_per_slice.get();
    const uint32_t blk = fd_pairs.div(r);
    const uint32_t p = r - blk * fd_pairs.get();
    const uint32_t I = fd_Bn.div(blk), J = blk - I * fd_Bn.get();
    uint32_t x, y;
    tri_decode32(p, nt, x, y);
    ar = (int64_t)x * 32;
    ac = (int64_t)y * 32;
    diag = (x == y);
    return d + (int64_t)k * slice_elems + ((int64_t)I * t) * n + (int64_t)J * t;
  };
  auto load = [&](E *s, int64_t ar, int64_t ac, bool diag, V (&ra)[VPT], V (&rb)[VPT]) {
#pragma unroll
    for (int q = 0; q < VPT; q++) {
      const int v = threadIdx.x + q * kTileThreads;
      const int r = v / RV, ch = v % RV;
      ra[q].v = __ldcs(reinterpret_cast<const uint4 *>(s + (ar + r) * n + ac) + ch);
      if (!diag) rb[q].v = __ldcs(reinterpret_cast<const uint4 *>(s + (ac + r) * n + ar) + ch);
    }
  };

  uint32_t u = blockIdx.x;
  if (u >= total) return;
  V na[VPT], nb[VPT];
  int64_t ar, ac;
  bool diag;
  E *s = origin(u, ar, ac, diag);
  load(s, ar, ac, diag, na, nb);
  for (; u < total; u += gridDim.x) {
    V ca[VPT], cb[VPT];
#pragma unroll
    for (int q = 0; q < VPT; q++) {
      ca[q] = na[q];
      cb[q] = nb[q];
    }
    E *cs = s;
    const int64_t car = ar, cac = ac;
    const bool cdiag = diag;
    if (u + gridDim.x < total) {
      s = origin(u + gridDim.x, ar, ac, diag);
      load(s, ar, ac, diag, na, nb);  // in flight while this pair is written back
    }
#pragma unroll
    for (int q = 0; q < VPT; q++) {
      const int v = threadIdx.x + q * kTileThreads;
      const int r = v / RV, ch = v % RV;
#pragma unroll
      for (int e = 0; e < PE; e++) {
        tA[r * S + ch * PE + e] = ca[q].e[e];
        if (!cdiag) tB[r * S + ch * PE + e] = cb[q].e[e];
      }
    }
    __syncthreads();
    // row w of A^T (column w of A) goes to B's place and vice versa
#pragma unroll
    for (int q = 0; q < VPT; q++) {
      const int v = threadIdx.x + q * kTileThreads;
      const int w = v / RV, ch = v % RV;
      V oa, ob;
#pragma unroll
      for (int e = 0; e < PE; e++) {
        oa.e[e] = tA[(ch * PE + e) * S + w];
        if (!cdiag) ob.e[e] = tB[(ch * PE + e) * S + w];
      }
      __stcs(reinterpret_cast<uint4 *>(cs + (cac + w) * n + car) + ch, oa.v);
      if (!cdiag) __stcs(reinterpret_cast<uint4 *>(cs + (car + w) * n + cac) + ch, ob.v);
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

// ---------------------------------------------------------------------------
// Band transpose fed by TMA: each CTA keeps a ring of NBUF band buffers; lane 0
// of warp 0 loads whole bands (one contiguous bulk copy each) NBUF-1 bands
// ahead, and all threads write the current band back transposed.  With VEC the
// write-back reads 16-byte chunks of QxQ element blocks (Q = 16/EB) row-wise
// from shared memory (conflict-free), transposes them in registers and stores
// 16-byte vectors; otherwise one element per thread, consecutive threads on
// consecutive output elements.  A buffer is reloaded only after every thread
// has finished reading it (barrier, then a proxy fence before the bulk copy).
// ---------------------------------------------------------------------------
template <int EB, bool VEC>
__global__ void __launch_bounds__(kTileThreads)
    k_band_bulk(char *__restrict__ data, int64_t n_bands, uint32_t R, uint32_t C, int nbuf,
                FastDiv<uint32_t> cdiv, FastDiv<uint32_t> rdiv, FastDiv<uint32_t> cqdiv, int *status) {
  using E = typename ElemT<EB>::type;
  constexpr int Q = 16 / EB;  // elements per 16-byte vector
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
  const uint32_t nel = R * C;
  const uint32_t bbytes = nel * EB;
  const uint32_t stride_bytes = (bbytes + 127) / 128 * 128;
  char *bufs = reinterpret_cast<char *>(smem_raw) + 128;
  __shared__ int s_fail;
  if (threadIdx.x == 0) {
    s_fail = 0;
    for (int i = 0; i < nbuf; i++) mbar_init(&bars[i], 1);
    fence_barrier_init();
    for (int i = 0; i < nbuf; i++) {
      const int64_t b = blockIdx.x + (int64_t)i * gridDim.x;
      if (b >= n_bands) break;
      mbar_expect_tx(&bars[i], bbytes);
      bulk_g2s(bufs + (int64_t)i * stride_bytes, data + b * (int64_t)bbytes, bbytes, &bars[i]);
    }
  }
  __syncthreads();
  int it = 0;
  for (int64_t b = blockIdx.x; b < n_bands; b += gridDim.x, it++) {
    const int slot = it % nbuf;
    if (!mbar_wait(&bars[slot], (uint32_t)((it / nbuf) & 1))) s_fail = 1;
    __syncthreads();
    if (s_fail) break;
    const E *sm = reinterpret_cast<const E *>(bufs + (int64_t)slot * stride_bytes);
    E *g = reinterpret_cast<E *>(data + b * (int64_t)bbytes);
    if constexpr (VEC) {
      // QxQ blocks: block (rb, cb) covers rows rb*Q.., columns cb*Q..
      const uint32_t cq = C / Q, nblk = (R / Q) * cq;
      for (uint32_t q = threadIdx.x; q < nblk; q += blockDim.x) {
        const uint32_t rb = cqdiv.div(q), cb = q - rb * cq;
        union {
          uint4 v;
          E e[Q];
        } in[Q], out[Q];
#pragma unroll
        for (int i = 0; i < Q; i++) in[i].v = *reinterpret_cast<const uint4 *>(sm + (rb * Q + i) * C + cb * Q);
#pragma unroll
        for (int i = 0; i < Q; i++)
#pragma unroll
          for (int j = 0; j < Q; j++) out[j].e[i] = in[i].e[j];
#pragma unroll
        for (int j = 0; j < Q; j++) __stcs(reinterpret_cast<uint4 *>(g + (cb * Q + j) * R + rb * Q), out[j].v);
      }
    } else {
      for (uint32_t o = threadIdx.x; o < nel; o += blockDim.x) {
        const uint32_t c = rdiv.div(o);
        const uint32_t r = o - c * R;
        __stcs(g + o, sm[r * C + c]);
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      const int64_t nb = b + (int64_t)nbuf * gridDim.x;
      if (nb < n_bands) {
        fence_proxy_async();
        mbar_expect_tx(&bars[slot], bbytes);
        bulk_g2s(bufs + (int64_t)slot * stride_bytes, data + nb * (int64_t)bbytes, bbytes, &bars[slot]);
      }
    }
  }
  (void)cdiv;
  if (threadIdx.x == 0 && s_fail) {
    // loads of iterations [it, it + nbuf) may still be in flight: wait for
    // them (each wait bounded again) so none lands after the CTA has exited
    for (int j = it; j < it + nbuf; j++) {
      if ((int64_t)blockIdx.x + (int64_t)j * gridDim.x >= n_bands) break;
      if (!mbar_wait(&bars[j % nbuf], (uint32_t)((j / nbuf) & 1))) break;
    }
    atomicExch(status, 5 /* T213_ERR_TIMEOUT */);
  }
}

}  // namespace t213
