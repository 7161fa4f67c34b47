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

#include <cuda.h>

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

// ---------------------------------------------------------------------------
// Tile swap fed by TMA.  Persistent CTAs of NCW consumer warps plus one
// producer warp (the last).  The producer's lane 0 loads tile pairs with tiled
// TMA copies (3-D boxes of TS rows x 128 bytes, 128-byte swizzle) into a ring
// of NS stages, up to NS pairs ahead of the consumers.  All consumer warps
// work on the same stage: each thread takes Q x Q blocks (Q = 16 / EB
// elements, one 16-byte chunk wide) of the pair, reads the block's Q rows,
// swaps it in registers and stores Q 16-byte vectors into the partner tile's
// place.  The eight lanes of each quarter-warp read eight different chunks of
// one row, which the swizzle puts in eight different bank groups, and each
// store instruction of a warp writes 64 contiguous bytes in each of eight
// output rows.  Every consumer waits on every stage in order and each warp
// releases it once (the empty barrier counts NCW arrivals), so each parity
// wait is at most one phase ahead.
//
// The data map views every slice as an m x (n * EB) byte matrix (dims
// {n*EB, m, d3}).  A pair is read completely before either of its tiles is
// written and no two CTAs share a pair, so the pass is in place.  Every wait
// is bounded; on timeout the CTA records T213_ERR_TIMEOUT, waits for its own
// loads in flight and returns.
// ---------------------------------------------------------------------------
// Pair p of a block's nt x nt tile grid (p < nt*(nt+1)/2) -> tiles (x, y),
// x <= y, ordered by super-tiles of grp x grp tiles (grp divides nt): first
// the grp*grp pairs of each off-diagonal super-tile pair (X < Y, row-major
// over the super-grid's strict upper triangle), then the grp*(grp+1)/2 pairs
// inside each diagonal super-tile.  Consecutive pairs -- the ones concurrent
// CTAs take -- then cover a grp-tile-wide region on both sides of the
// diagonal, so the rows read and written on either side are grp tiles long.
__device__ __forceinline__ void tile_pair_decode(uint32_t p, uint32_t nt, uint32_t grp, uint32_t &x, uint32_t &y) {
  const uint32_t nsup = nt / grp, gsq = grp * grp;
  const uint32_t off = nsup * (nsup - 1) / 2 * gsq;
  if (p < off) {
    const uint32_t sp = p / gsq, r = p - sp * gsq;
    uint32_t X, Yp;
    tri_decode32(sp, nsup - 1, X, Yp);
    const uint32_t xi = r / grp, yi = r - xi * grp;
    x = X * grp + xi;
    y = (Yp + 1) * grp + yi;
  } else {
    const uint32_t p2 = p - off, gd = grp * (grp + 1) / 2;
    const uint32_t D = p2 / gd, r = p2 - D * gd;
    uint32_t xi, yi;
    tri_decode32(r, grp, xi, yi);
    x = D * grp + xi;
    y = D * grp + yi;
  }
}

template <int EB, int TS_>
struct TileTma {
  static constexpr int TS = TS_;                    // tile side in elements
  static constexpr int NBOX = TS * EB / 128;        // 128-byte boxes per tile row
  static constexpr int BOX_BYTES = TS * 128;        // one box: TS rows of 128 bytes
  static constexpr int TILE_BYTES = TS * TS * EB;
  static constexpr int Q = 16 / EB;                 // elements per 16-byte chunk
  static constexpr int NQ = TS / Q;                 // Q x Q blocks per tile side
  static constexpr int BLOCKS = NQ * NQ;
  static_assert(NBOX >= 1 && TS * EB % 128 == 0, "a tile row is whole 128-byte boxes");
  static_assert(NQ % 8 == 0 && BLOCKS % 32 == 0, "block mapping needs 8 | NQ");
};

template <int EB, int TS>
__global__ void __launch_bounds__(1024)
    k_tile_swap_tma(const __grid_constant__ CUtensorMap tmap, char *__restrict__ data, int64_t n,
                    int64_t slice_elems, uint32_t total, int64_t t, FastDiv<uint32_t> fd_per_slice,
                    FastDiv<uint32_t> fd_pairs, FastDiv<uint32_t> fd_Bn, uint32_t nt, uint32_t grp, int ns,
                    int *status) {
  using E = typename ElemT<EB>::type;
  using TT = TileTma<EB, TS>;
  constexpr int Q = TT::Q, NQ = TT::NQ;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // barriers first, then the 1024-byte aligned stages (swizzle atoms)
  uint64_t *full = reinterpret_cast<uint64_t *>(smem_raw);
  uint64_t *empty = full + ns;
  const uint32_t base_u = smem_u32(smem_raw);
  unsigned char *stages = smem_raw + (((base_u + 16 * ns + 1023) & ~1023u) - base_u);
  __shared__ int s_fail, s_issued;
  const int ncw = (int)(blockDim.x >> 5) - 1;  // consumer warps
  const int nct = ncw * 32;                     // consumer threads
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    s_fail = 0;
    s_issued = 0;
    for (int i = 0; i < ns; i++) {
      mbar_init(&full[i], 1);
      mbar_init(&empty[i], (uint32_t)ncw);
    }
    fence_barrier_init();
  }
  __syncthreads();

  // pair u -> slice k, block (I, J), tiles (x, y) and (y, x)
  auto decode = [&](uint32_t u, uint32_t &k, uint32_t &I, uint32_t &J, uint32_t &x, uint32_t &y) {
    k = fd_per_slice.div(u);
    const uint32_t r = u - k * fd_per_slice.get();
    const uint32_t blk = fd_pairs.div(r);
    const uint32_t p = r - blk * fd_pairs.get();
    I = fd_Bn.div(blk);
    J = blk - I * fd_Bn.get();
    tile_pair_decode(p, nt, grp, x, y);
  };

  if (warp == ncw) {
    // ---------------------------------------------------------- producer --
    if (lane == 0) {
      prefetch_tmap(&tmap);
      int li = 0;  // pairs issued so far
      for (uint32_t u = blockIdx.x; u < total; u += gridDim.x, li++) {
        const int s = li % ns;
        if (li >= ns && !mbar_wait(&empty[s], (uint32_t)(((li / ns) - 1) & 1))) {
          s_fail = 1;
          break;
        }
        if (*(volatile int *)&s_fail) break;
        uint32_t k, I, J, x, y;
        decode(u, k, I, J, x, y);
        const bool diag = (x == y);
        unsigned char *sA = stages + (size_t)s * 2 * TT::TILE_BYTES;
        mbar_expect_tx(&full[s], diag ? TT::TILE_BYTES : 2 * TT::TILE_BYTES);
        const int32_t rowA = (int32_t)(I * (uint32_t)t + x * TS), colA = (int32_t)(J * (uint32_t)t + y * TS);
        const int32_t rowB = (int32_t)(I * (uint32_t)t + y * TS), colB = (int32_t)(J * (uint32_t)t + x * TS);
#pragma unroll
        for (int b = 0; b < TT::NBOX; b++)
          tma_load_3d(sA + b * TT::BOX_BYTES, &tmap, colA * EB + b * 128, rowA, (int32_t)k, &full[s]);
        if (!diag) {
#pragma unroll
          for (int b = 0; b < TT::NBOX; b++)
            tma_load_3d(sA + TT::TILE_BYTES + b * TT::BOX_BYTES, &tmap, colB * EB + b * 128, rowB, (int32_t)k,
                        &full[s]);
        }
      }
      s_issued = li;
    }
  } else {
    // --------------------------------------------------------- consumers --
    E *d = reinterpret_cast<E *>(data);
    int li = 0;
    for (uint32_t u = blockIdx.x; u < total; u += gridDim.x, li++) {
      const int s = li % ns;
      // every lane waits (each gets the barrier's acquire); the warp leaves
      // together if any lane's bounded wait ran out
      const bool ok = __all_sync(0xffffffffu, mbar_wait(&full[s], (uint32_t)((li / ns) & 1)));
      if (!ok) {
        if (lane == 0) s_fail = 1;
        break;
      }
      uint32_t k, I, J, x, y;
      decode(u, k, I, J, x, y);
      const bool diag = (x == y);
      E *blk0 = d + (int64_t)k * slice_elems + ((int64_t)I * t) * n + (int64_t)J * t;
      const unsigned char *sA = stages + (size_t)s * 2 * TT::TILE_BYTES;
      const int nblk = (diag ? 1 : 2) * TT::BLOCKS;
      // block g of the pair: tile h = g / BLOCKS (0: A at (x, y), 1: B at
      // (y, x)); source tile (sx, sy) is written transposed to tile (sy, sx)
#pragma unroll 2
      for (int g = threadIdx.x; g < nblk; g += nct) {
        const int h = g >= TT::BLOCKS;
        const int q = g - h * TT::BLOCKS;
        const unsigned char *src = sA + h * TT::TILE_BYTES;
        const uint32_t sx = h ? y : x, sy = h ? x : y;
        E *dst = blk0 + (int64_t)(sy * TS) * n + sx * TS;  // rows sy*TS.., cols sx*TS..
        const int cbl = q & 7, rbl = (q >> 3) & 3, rest = q >> 5;
        const int cb = (rest % (NQ / 8)) * 8 + cbl;
        const int rb = (rest / (NQ / 8)) * 4 + rbl;
        union V {
          uint4 v;
          E e[Q];
        } in[Q], out[Q];
#pragma unroll
        for (int i = 0; i < Q; i++) {
          const int r = rb * Q + i;
          const int bx = cb >> 3, cc = cb & 7;
          in[i].v = *reinterpret_cast<const uint4 *>(src + bx * TT::BOX_BYTES + r * 128 + ((cc ^ (r & 7)) << 4));
        }
#pragma unroll
        for (int i = 0; i < Q; i++)
#pragma unroll
          for (int j = 0; j < Q; j++) out[j].e[i] = in[i].e[j];
#pragma unroll
        for (int j = 0; j < Q; j++)
          __stcs(reinterpret_cast<uint4 *>(dst + (int64_t)(cb * Q + j) * n) + rb, out[j].v);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
  }
  __syncthreads();
  if (s_fail && threadIdx.x == nct) {
    // wait for every load this CTA issued (each wait bounded again) so none
    // lands in shared memory after the CTA has exited
    const int issued = s_issued;
    for (int s = 0; s < ns && s < issued; s++) {
      const int last = s + ((issued - 1 - s) / ns) * ns;  // last use of stage s that was issued
      if (!mbar_wait(&full[s], (uint32_t)((last / ns) & 1))) break;
    }
    atomicExch(status, 5 /* T213_ERR_TIMEOUT */);
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
