// Persistent executor of the batched form: one launch transposes many tensors
// of uneven shape and element size.
//
// The host flattens every tensor's plan into passes (BPass) and cuts each pass
// into items (BItem: a range of the pass's independent units).  Items are
// queued level by level — all first passes, then all second passes, ... —
// with the tensors in the same order on every level.  A CTA claims the next
// item with an atomic queue head, waits until the previous pass of the same
// tensor has completed all its items (a per-pass counter), runs the item, and
// counts it done.  Every item an item waits on sits earlier in the queue and
// was claimed by a running CTA, so the waits always end; they are bounded
// anyway (wait_ns of the global timer, 2 s unless a test lowers it; then
// T213_ERR_TIMEOUT in *status and the CTA leaves).
//
// Unit executors:
//   TILE   tile pairs of t x t block transposes (16-byte vectors when possible)
//   BAND   one R x C band: cp.async staging, 4x4 register transposes
//   COL    one column strip in shared memory, gathered
//   ROW    a group of rows in shared memory, gathered
//   CARRY  saves chunk-start segments of a cycle pass
//   SEG    cycle-walker items; each warp walks one item with a ring of bulk
//          asynchronous copies (TMA), or with 16-byte registers when the
//          segment is not 16-byte aligned
#pragma once

#include <string.h>

#include "../../include/t213.h"
#include "functors.cuh"
#include "k_cycles.cuh"
#include "k_gather.cuh"
#include "k_tiles.cuh"
#include "tma.cuh"

namespace t213 {

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

constexpr int kBatchThreads = 512;
constexpr int kBatchWarps = kBatchThreads / 32;
constexpr int kBatchRing = 6;                 // TMA buffers per walker warp
constexpr int64_t kBatchPiece = 2048;         // bytes per TMA walker piece
constexpr int64_t kBatchSmem = 192 * 1024;    // dynamic shared memory per CTA
constexpr int64_t kBatchBarBytes = 2048;      // mbarriers (first KB) and per-strip column offsets (second KB)
constexpr int kBatchAuxInts = 256;            // column offsets of one strip (W <= 256)

enum BKind { BK_TILE = 1, BK_BAND = 2, BK_COL = 3, BK_ROW = 4, BK_CARRY = 5, BK_SEG = 6 };

// A functor of any kind stored as raw bytes (the host copies the typed
// functor in; the device switches on the kind).
template <typename U>
struct AnyFn {
  int32_t kind = 0, pad = 0;
  alignas(16) unsigned char raw[112];
  template <typename F>
  __host__ void set(int k, const F &f) {
    static_assert(sizeof(F) <= sizeof(raw), "functor too large");
    kind = k;
    memcpy(raw, &f, sizeof(F));
  }
  template <typename F>
  __device__ __forceinline__ const F &as() const {
    return *reinterpret_cast<const F *>(raw);
  }
  __device__ __forceinline__ U col(U i, U j) const {
    switch (kind) {
      case T213_FN_C2R_PREROTATOR:
        return as<RotGather<U, RotC2RPre<U>>>()(i, j);
      case T213_FN_C2R_POSTROTATOR:
        return as<RotGather<U, RotC2RPost<U>>>()(i, j);
      case T213_FN_R2C_PREROTATOR:
        return as<RotGather<U, RotR2CPre<U>>>()(i, j);
      case T213_FN_R2C_POSTROTATOR:
        return as<RotGather<U, RotR2CPost<U>>>()(i, j);
      case T213_FN_C2R_FUSED_PREOP:
        return as<ColC2RFusedPre<U>>()(i, j);
      case T213_FN_C2R_FUSED_POSTOP:
        return as<ColC2RFusedPost<U>>()(i, j);
      case T213_FN_R2C_FUSED_PREOP:
        return as<ColR2CFusedPre<U>>()(i, j);
      default:
        return as<ColR2CFusedPost<U>>()(i, j);
    }
  }
  __device__ __forceinline__ U row(U i, U j) const {
    if (kind == T213_FN_R2C_SHUFFLE) return as<RowR2CShuffle<U>>()(i, j);
    return as<RowC2RShuffle<U>>()(i, j);
  }
  __device__ __forceinline__ U perm(U p) const {
    if (kind == 0) return as<SegPerm3<U>>()(p);
    if (kind == T213_FN_C2R_POSTPERMUTER) return as<PermC2RPost<U>>()(p);
    return as<PermR2CPre<U>>()(p);
  }
};

struct BPass {
  int32_t kind = 0, eb = 4, aw = 4, u64 = 0;
  char *data = nullptr;
  int64_t d3 = 0, m = 0, n = 0, slice_bytes = 0;
  int64_t W = 0, WS = 0, n_strips = 0;     // COL
  int64_t rows_per_unit = 0;               // ROW
  int64_t t = 0, Bm = 0, Bn = 0, nt = 0, pairs = 0;  // TILE
  int32_t tile_vec = 0, band_vec = 0;
  int32_t col_form = 0;                    // COL: cluster-local form 1-3 of the functor, 0 = evaluate it per element
  int32_t row_peel = 0;                    // ROW: 16-byte accesses over a pitch that is not a 16-byte multiple
  int64_t R = 0, C = 0;                    // BAND
  const Chunk *chunks = nullptr;           // SEG / CARRY
  const CarryItem *carries = nullptr;
  char *carry_buf = nullptr;
  int64_t n_chunks = 0, n_carry = 0, seg_bytes = 0, piece_bytes = 0, pieces = 0;
  int32_t seg_tma = 0, seg_aw = 16;
  int64_t n_units = 0;
  FastDiv<uint32_t> div_w, div_wl;  // COL: words per row of a full / the last strip; ROW: words per row
  FastDiv<uint64_t> div_m;          // ROW, COL: m
  FastDiv<uint32_t> div_m32;        // COL: m, for 32-bit indices
  int32_t done_ctr = 0, dep_ctr = -1;
  int64_t dep_target = 0;
  AnyFn<uint32_t> f32;
  AnyFn<uint64_t> f64;
};

struct BItem {
  int32_t pass, pad;
  int64_t u0, u1;
};

// ------------------------------------------------------------------ TILE ----
template <int EB>
__device__ __noinline__ void bx_tile_vec(const BPass &P, int64_t u0, int64_t u1, unsigned char *smem) {
  using E = typename ElemT<EB>::type;
  constexpr int RV = 2 * EB, PE = 16 / EB;
  constexpr int VPT = (32 * RV + kBatchThreads - 1) / kBatchThreads;  // vectors per thread per tile
  constexpr int S = 33;
  E *tA = reinterpret_cast<E *>(smem);
  E *tB = tA + 32 * S;
  union V {
    uint4 v;
    E e[PE];
  };
  const int64_t per_slice = P.Bm * P.Bn * P.pairs;
  E *d = reinterpret_cast<E *>(P.data);
  const int nvec = 32 * RV;
  auto origin = [&](int64_t u, int64_t &ar, int64_t &ac, bool &diag) -> E * {
    const int64_t k = u / per_slice, r = u - k * per_slice;
    const int64_t blk = r / P.pairs, p = r - blk * P.pairs;
    const int64_t I = blk / P.Bn, J = blk - I * P.Bn;
    int64_t x, y;
    tri_decode(p, P.nt, x, y);
    ar = x * 32;
    ac = y * 32;
    diag = x == y;
    return d + k * (P.m * P.n) + (I * P.t) * P.n + J * P.t;
  };
  auto load = [&](E *s, int64_t ar, int64_t ac, bool diag, V (&ra)[VPT], V (&rb)[VPT]) {
#pragma unroll
    for (int q = 0; q < VPT; q++) {
      const int v = threadIdx.x + q * kBatchThreads;
      if (v < nvec) {
        const int rr = v / RV, ch = v % RV;
        ra[q].v = __ldcs(reinterpret_cast<const uint4 *>(s + (ar + rr) * P.n + ac) + ch);
        if (!diag) rb[q].v = __ldcs(reinterpret_cast<const uint4 *>(s + (ac + rr) * P.n + ar) + ch);
      }
    }
  };
  V na[VPT], nb[VPT];
  int64_t ar, ac;
  bool diag;
  E *s = origin(u0, ar, ac, diag);
  load(s, ar, ac, diag, na, nb);
  for (int64_t u = u0; u < u1; u++) {
    V ca[VPT], cb[VPT];
#pragma unroll
    for (int q = 0; q < VPT; q++) {
      ca[q] = na[q];
      cb[q] = nb[q];
    }
    E *cs = s;
    const int64_t car = ar, cac = ac;
    const bool cdiag = diag;
    if (u + 1 < u1) {
      s = origin(u + 1, ar, ac, diag);
      load(s, ar, ac, diag, na, nb);
    }
#pragma unroll
    for (int q = 0; q < VPT; q++) {
      const int v = threadIdx.x + q * kBatchThreads;
      if (v < nvec) {
        const int rr = v / RV, ch = v % RV;
#pragma unroll
        for (int e = 0; e < PE; e++) {
          tA[rr * S + ch * PE + e] = ca[q].e[e];
          if (!cdiag) tB[rr * S + ch * PE + e] = cb[q].e[e];
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < VPT; q++) {
      const int v = threadIdx.x + q * kBatchThreads;
      if (v < nvec) {
        const int w = v / RV, ch = v % RV;
        V oa, ob;
#pragma unroll
        for (int e = 0; e < PE; e++) {
          oa.e[e] = tA[(ch * PE + e) * S + w];
          if (!cdiag) ob.e[e] = tB[(ch * PE + e) * S + w];
        }
        __stcs(reinterpret_cast<uint4 *>(cs + (cac + w) * P.n + car) + ch, oa.v);
        if (!cdiag) __stcs(reinterpret_cast<uint4 *>(cs + (car + w) * P.n + cac) + ch, ob.v);
      }
    }
    __syncthreads();
  }
}

template <int EB>
__device__ __noinline__ void bx_tile_scalar(const BPass &P, int64_t u0, int64_t u1, unsigned char *smem) {
  using E = typename ElemT<EB>::type;
  constexpr int TS = 32, S = TS + 1;
  E *tA = reinterpret_cast<E *>(smem);
  E *tB = tA + TS * S;
  const int64_t per_slice = P.Bm * P.Bn * P.pairs;
  E *d = reinterpret_cast<E *>(P.data);
  for (int64_t u = u0; u < u1; u++) {
    const int64_t k = u / per_slice, r = u - k * per_slice;
    const int64_t blk = r / P.pairs, p = r - blk * P.pairs;
    const int64_t I = blk / P.Bn, J = blk - I * P.Bn;
    int64_t x, y;
    tri_decode(p, P.nt, x, y);
    E *s = d + k * (P.m * P.n) + (I * P.t) * P.n + J * P.t;
    const int64_t ar = x * TS, ac = y * TS;
    const int64_t hA = min((int64_t)TS, P.t - ar), wA = min((int64_t)TS, P.t - ac);
    for (int e = threadIdx.x; e < TS * TS; e += blockDim.x) {
      const int uu = e / TS, vv = e % TS;
      if (uu < hA && vv < wA) tA[uu * S + vv] = s[(ar + uu) * P.n + ac + vv];
      if (x != y && uu < wA && vv < hA) tB[uu * S + vv] = s[(ac + uu) * P.n + ar + vv];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < TS * TS; e += blockDim.x) {
      const int uu = e / TS, vv = e % TS;
      if (uu < wA && vv < hA) s[(ac + uu) * P.n + ar + vv] = tA[vv * S + uu];
      if (x != y && uu < hA && vv < wA) s[(ar + uu) * P.n + ac + vv] = tB[vv * S + uu];
    }
    __syncthreads();
  }
}

// Double-buffered executors: the shared memory is split in two halves; the
// units of an item alternate between them, and unit u+1 is staged with
// cp.async (one commit group per unit) while unit u is written back.
constexpr int64_t kBatchHalf = kBatchSmem / 2;

// ------------------------------------------------------------------ BAND ----
template <int EB, bool VEC>
__device__ __noinline__ void bx_band(const BPass &P, int64_t u0, int64_t u1, unsigned char *smem) {
  using E = typename ElemT<EB>::type;
  constexpr int Q = 16 / EB;
  const uint32_t R = (uint32_t)P.R, C = (uint32_t)P.C, nel = R * C;
  const bool a16 = ((nel * EB) % 16 == 0) && (((uintptr_t)P.data) % 16 == 0);
  auto stage = [&](int64_t b, E *sm) {
    const E *g = reinterpret_cast<const E *>(P.data) + b * (int64_t)nel;
    if (a16) {
      const uint32_t nv = nel * EB / 16;
      for (uint32_t v = threadIdx.x; v < nv; v += blockDim.x)
        cp_async<16>(reinterpret_cast<uint4 *>(sm) + v, reinterpret_cast<const uint4 *>(g) + v);
    } else {
      for (uint32_t e = threadIdx.x; e < nel; e += blockDim.x) sm[e] = g[e];
    }
    cp_async_commit();
  };
  stage(u0, reinterpret_cast<E *>(smem));
  for (int64_t b = u0; b < u1; b++) {
    E *sm = reinterpret_cast<E *>(smem + ((b - u0) & 1) * kBatchHalf);
    if (b + 1 < u1) {
      stage(b + 1, reinterpret_cast<E *>(smem + ((b + 1 - u0) & 1) * kBatchHalf));
      cp_async_wait_group<1>();
    } else {
      cp_async_wait_group<0>();
    }
    __syncthreads();
    E *g = reinterpret_cast<E *>(P.data) + b * (int64_t)nel;
    if constexpr (VEC) {
      const uint32_t cq = C / Q, nblk = (R / Q) * cq;
      for (uint32_t q = threadIdx.x; q < nblk; q += blockDim.x) {
        const uint32_t rb = q / cq, cb = q - rb * cq;
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
        const uint32_t c = o / R, r = o - c * R;
        g[o] = sm[r * C + c];
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------- COL ----
// The functor type F is a template parameter (the dispatcher switches on the
// kind once per item), and every division by a per-pass constant goes
// through a FastDiv the host computed, so the per-element work is the
// functor's own arithmetic, one shared-memory read and the store.
template <typename T>
struct TypeTag {
  using type = T;
};

template <typename U>
__device__ __forceinline__ const AnyFn<U> &any_fn(const BPass &P);
template <>
__device__ __forceinline__ const AnyFn<uint32_t> &any_fn<uint32_t>(const BPass &P) {
  return P.f32;
}
template <>
__device__ __forceinline__ const AnyFn<uint64_t> &any_fn<uint64_t>(const BPass &P) {
  return P.f64;
}

template <typename U>
__device__ __forceinline__ FastDiv<U> pass_mdiv(const BPass &P);
template <>
__device__ __forceinline__ FastDiv<uint32_t> pass_mdiv<uint32_t>(const BPass &P) {
  return P.div_m32;
}
template <>
__device__ __forceinline__ FastDiv<uint64_t> pass_mdiv<uint64_t>(const BPass &P) {
  return P.div_m;
}

template <int EB, int AW, typename U, typename F>
__device__ __noinline__ void bx_col(const BPass &P, int64_t u0, int64_t u1, unsigned char *smem) {
  using E = typename ElemT<EB>::type;
  using Wd = typename WordT<AW>::type;
  using PK = Pack<AW, EB>;
  constexpr int PER = AW / EB;
  const F fn = any_fn<U>(P).template as<F>();
  const U m = (U)P.m, n = (U)P.n, W = (U)P.W, WS = (U)P.WS;
  const FastDiv<uint32_t> dfull = P.div_w, dlast = P.div_wl;  // words per row of a full / the last strip
  const int64_t pitch = P.n * EB;
  auto strip = [&](int64_t u, U &j0, FastDiv<uint32_t> &wd, char *&sbase) {
    const int64_t k = u / P.n_strips;
    const U s = (U)(u - k * P.n_strips);
    j0 = s * W;
    wd = j0 + W <= n ? dfull : dlast;
    sbase = P.data + (k * (int64_t)m * n + j0) * EB;
  };
  auto stage = [&](int64_t u, E *sm) {
    U j0;
    FastDiv<uint32_t> wd;
    char *sbase;
    strip(u, j0, wd, sbase);
    const uint32_t wpr = wd.get(), nw = (uint32_t)m * wpr;
    for (uint32_t t = threadIdx.x; t < nw; t += blockDim.x) {
      const uint32_t r = wd.div(t), w = t - r * wpr;
      const Wd *gp = reinterpret_cast<const Wd *>(sbase + (int64_t)r * pitch) + w;
      if constexpr (AW >= 4)
        cp_async<AW>(reinterpret_cast<Wd *>(sm + (int64_t)r * WS) + w, gp);
      else
        reinterpret_cast<Wd *>(sm + (int64_t)r * WS)[w] = *gp;
    }
    cp_async_commit();
  };
  stage(u0, reinterpret_cast<E *>(smem));
  for (int64_t u = u0; u < u1; u++) {
    E *sm = reinterpret_cast<E *>(smem + ((u - u0) & 1) * kBatchHalf);
    if (u + 1 < u1) {
      stage(u + 1, reinterpret_cast<E *>(smem + ((u + 1 - u0) & 1) * kBatchHalf));
      cp_async_wait_group<1>();
    } else {
      cp_async_wait_group<0>();
    }
    __syncthreads();
    U j0;
    FastDiv<uint32_t> wd;
    char *sbase;
    strip(u, j0, wd, sbase);
    const uint32_t wpr = wd.get(), nw = (uint32_t)m * wpr;
#pragma unroll 4
    for (uint32_t t = threadIdx.x; t < nw; t += blockDim.x) {
      const uint32_t r = wd.div(t), w = t - r * wpr;
      typename PK::U pk;
#pragma unroll
      for (int e = 0; e < PER; e++) {
        const U si = fn((U)r, j0 + w * PER + e);
        pk.e[e] = sm[(int64_t)si * WS + w * PER + e];
      }
      __stcs(reinterpret_cast<Wd *>(sbase + (int64_t)r * pitch) + w, pk.w);
    }
    __syncthreads();
  }
}

// COL items whose functor has a cluster-local form (the form k_col_local
// uses, with the whole strip in this CTA): column w of a strip has a key offset
// r_w, slot s of the staged strip holds source row Fm(s), and output row Gm(o)
// takes column w from slot (o + r_w) mod m.  The functor is evaluated once per
// column, the row maps once per row, and an element costs an add and a shared
// read.  A lane keeps one word of the rows it writes, so its offsets stay in
// registers.
template <int EB, int AW, typename U, typename Off, typename Fm, typename Gm>
__device__ __noinline__ void bx_col_local(const BPass &P, const Off off, const Fm F, const Gm G, int64_t u0, int64_t u1,
                                          unsigned char *smem, int *s_sh) {
  using E = typename ElemT<EB>::type;
  using Wd = typename WordT<AW>::type;
  using PK = Pack<AW, EB>;
  constexpr int PER = AW / EB;
  const U m = (U)P.m, n = (U)P.n, W = (U)P.W, WS = (U)P.WS;
  const FastDiv<uint32_t> dfull = P.div_w, dlast = P.div_wl;
  const int64_t pitch = P.n * EB;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  auto strip = [&](int64_t u, U &j0, FastDiv<uint32_t> &wd, char *&sbase) {
    const int64_t k = u / P.n_strips;
    const U s = (U)(u - k * P.n_strips);
    j0 = s * W;
    wd = j0 + W <= n ? dfull : dlast;
    sbase = P.data + (k * (int64_t)m * n + j0) * EB;
  };
  auto stage = [&](int64_t u, E *sm) {
    U j0;
    FastDiv<uint32_t> wd;
    char *sbase;
    strip(u, j0, wd, sbase);
    const uint32_t wpr = wd.get(), nw = (uint32_t)m * wpr;
    for (uint32_t t = threadIdx.x; t < nw; t += blockDim.x) {
      const uint32_t sl = wd.div(t), w = t - sl * wpr;
      const Wd *gp = reinterpret_cast<const Wd *>(sbase + (int64_t)F((U)sl) * pitch) + w;
      if constexpr (AW >= 4)
        cp_async<AW>(reinterpret_cast<Wd *>(sm + (int64_t)sl * WS) + w, gp);
      else
        reinterpret_cast<Wd *>(sm + (int64_t)sl * WS)[w] = *gp;
    }
    cp_async_commit();
  };
  stage(u0, reinterpret_cast<E *>(smem));
  for (int64_t u = u0; u < u1; u++) {
    E *sm = reinterpret_cast<E *>(smem + ((u - u0) & 1) * kBatchHalf);
    if (u + 1 < u1) {
      stage(u + 1, reinterpret_cast<E *>(smem + ((u + 1 - u0) & 1) * kBatchHalf));
      cp_async_wait_group<1>();
    } else {
      cp_async_wait_group<0>();
    }
    U j0;
    FastDiv<uint32_t> wd;
    char *sbase;
    strip(u, j0, wd, sbase);
    const uint32_t wpr = wd.get(), wn = wpr * PER;
    for (uint32_t w = threadIdx.x; w < wn; w += blockDim.x) s_sh[w] = (int)off(j0 + w);
    __syncthreads();  // the strip has landed and its offsets are in place
    auto slot = [&](U o, U r) -> U {
      const U v = o + r;
      return v >= m ? v - m : v;
    };
    if (32 % wpr == 0) {
      const uint32_t rpi = 32 / wpr, lr = lane / wpr, lw = lane - lr * wpr;
      U sh[PER];
#pragma unroll
      for (int e = 0; e < PER; e++) sh[e] = (U)s_sh[lw * PER + e];
      for (U ob = (U)warp * 32; ob < m; ob += (U)nwarps * 32) {
        const U myo = ob + lane;
        const U myrow = myo < m ? G(myo) : 0;
#pragma unroll 4
        for (uint32_t r = lr; r < 32; r += rpi) {
          const U row = __shfl_sync(0xffffffffu, myrow, r);
          const U o = ob + r;
          if (o < m) {
            typename PK::U pk;
#pragma unroll
            for (int e = 0; e < PER; e++) pk.e[e] = sm[(int64_t)slot(o, sh[e]) * WS + lw * PER + e];
            __stcs(reinterpret_cast<Wd *>(sbase + (int64_t)row * pitch) + lw, pk.w);
          }
        }
      }
    } else {
      const uint32_t nw = (uint32_t)m * wpr;
      for (uint32_t t = threadIdx.x; t < nw; t += blockDim.x) {
        const uint32_t o = wd.div(t), w = t - o * wpr;
        const U row = G((U)o);
        typename PK::U pk;
#pragma unroll
        for (int e = 0; e < PER; e++) {
          const uint32_t c = w * PER + e;
          pk.e[e] = sm[(int64_t)slot((U)o, (U)s_sh[c]) * WS + c];
        }
        __stcs(reinterpret_cast<Wd *>(sbase + (int64_t)row * pitch) + w, pk.w);
      }
    }
    __syncthreads();  // the buffer is restaged two strips on, the offsets by the next strip
  }
}

// ------------------------------------------------------------------- ROW ----
template <int EB, int AW, typename U, typename F>
__device__ __noinline__ void bx_row(const BPass &P, int64_t u0, int64_t u1, unsigned char *smem) {
  using E = typename ElemT<EB>::type;
  using Wd = typename WordT<AW>::type;
  using PK = Pack<AW, EB>;
  constexpr int PER = AW / EB;
  const F fn = any_fn<U>(P).template as<F>();
  const U m = (U)P.m, n = (U)P.n;
  const FastDiv<uint32_t> wd = P.div_w;  // words per row
  const FastDiv<uint64_t> md = P.div_m;  // m
  const uint32_t wpr = wd.get();
  const int64_t total_rows = P.d3 * P.m;
  auto stage = [&](int64_t u, E *sm) {
    const int64_t r0 = u * P.rows_per_unit;
    const int nr = (int)min((int64_t)P.rows_per_unit, total_rows - r0);
    const Wd *g = reinterpret_cast<const Wd *>(P.data + r0 * (int64_t)n * EB);
    const uint32_t nw = (uint32_t)nr * wpr;
    for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x) {
      if constexpr (AW >= 4)
        cp_async<AW>(reinterpret_cast<Wd *>(sm) + w, g + w);
      else
        reinterpret_cast<Wd *>(sm)[w] = g[w];
    }
    cp_async_commit();
  };
  stage(u0, reinterpret_cast<E *>(smem));
  for (int64_t u = u0; u < u1; u++) {
    E *sm = reinterpret_cast<E *>(smem + ((u - u0) & 1) * kBatchHalf);
    if (u + 1 < u1) {
      stage(u + 1, reinterpret_cast<E *>(smem + ((u + 1 - u0) & 1) * kBatchHalf));
      cp_async_wait_group<1>();
    } else {
      cp_async_wait_group<0>();
    }
    __syncthreads();
    const int64_t r0 = u * P.rows_per_unit;
    const int nr = (int)min((int64_t)P.rows_per_unit, total_rows - r0);
    Wd *g = reinterpret_cast<Wd *>(P.data + r0 * (int64_t)n * EB);
    const uint32_t nw = (uint32_t)nr * wpr;
    const uint64_t i_base = md.mod((uint64_t)r0);
#pragma unroll 4
    for (uint32_t w = threadIdx.x; w < nw; w += blockDim.x) {
      const uint32_t rr = wd.div(w);
      const U j0 = (U)(w - rr * wpr) * PER;
      const uint64_t ii = i_base + rr;
      const U i = (U)(ii < (uint64_t)m ? ii : md.mod(ii));
      typename PK::U pk;
      RowStepper<F, U> step(fn);
#pragma unroll
      for (int e = 0; e < PER; e++)
        pk.e[e] = sm[(int64_t)rr * n + (e == 0 ? step.first(i, j0) : step.next(i, j0 + e))];
      __stcs(g + w, pk.w);
    }
    __syncthreads();
  }
}

// ROW items whose pitch is not a 16-byte multiple, for elements of at most 4
// bytes: the unit (consecutive rows, one contiguous byte range [b0, b1)) is
// staged as the 16-byte blocks that cover it (bytes of the neighbouring units
// at both ends are read and never used) and written back with 16-byte stores
// between its first and last 16-byte boundary, single elements at the ends.
// A thread takes 16/EB consecutive elements and steps the shuffle along them.
template <int EB, typename U, typename F>
__device__ __noinline__ void bx_row_peel(const BPass &P, int64_t u0, int64_t u1, unsigned char *smem) {
  using E = typename ElemT<EB>::type;
  constexpr int PER = 16 / EB;
  const F fn = any_fn<U>(P).template as<F>();
  const U m = (U)P.m, n = (U)P.n;
  const FastDiv<uint32_t> nd = P.div_w;  // n (elements per row)
  const FastDiv<uint64_t> md = P.div_m;  // m
  const int64_t total_rows = P.d3 * P.m, row_bytes = P.n * EB;
  auto range = [&](int64_t u, uintptr_t &b0, uintptr_t &b1) {
    const int64_t r0 = u * P.rows_per_unit;
    const int64_t nr = min((int64_t)P.rows_per_unit, total_rows - r0);
    b0 = reinterpret_cast<uintptr_t>(P.data + r0 * row_bytes);
    b1 = b0 + (uintptr_t)(nr * row_bytes);
  };
  auto stage = [&](int64_t u, unsigned char *buf) {
    uintptr_t b0, b1;
    range(u, b0, b1);
    const uintptr_t a0 = b0 & ~(uintptr_t)15, a1 = (b1 + 15) & ~(uintptr_t)15;
    const uint32_t nv = (uint32_t)((a1 - a0) >> 4);
    const uint4 *g = reinterpret_cast<const uint4 *>(a0);
    for (uint32_t v = threadIdx.x; v < nv; v += blockDim.x) cp_async<16>(buf + 16 * (size_t)v, g + v);
    cp_async_commit();
  };
  stage(u0, smem);
  for (int64_t u = u0; u < u1; u++) {
    const E *sm = reinterpret_cast<const E *>(smem + ((u - u0) & 1) * kBatchHalf);
    if (u + 1 < u1) {
      stage(u + 1, smem + ((u + 1 - u0) & 1) * kBatchHalf);
      cp_async_wait_group<1>();
    } else {
      cp_async_wait_group<0>();
    }
    __syncthreads();
    uintptr_t b0, b1;
    range(u, b0, b1);
    const int64_t r0 = u * P.rows_per_unit;
    const U d0 = (U)((b0 - (b0 & ~(uintptr_t)15)) / EB);  // unit element 0 sits at sm[d0]
    const U i_base = (U)md.mod((uint64_t)r0);
    const U total = (U)((b1 - b0) / EB);
    auto locate = [&](U q, U &rr, U &j, U &i) {
      rr = (U)nd.div((uint32_t)q);
      j = q - rr * n;
      const uint64_t ii = (uint64_t)i_base + rr;
      i = (U)(ii < (uint64_t)m ? ii : md.mod(ii));
    };
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
          if (++j == n) {
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
    for (U t = threadIdx.x; t < qh + (total - qt); t += blockDim.x) {
      const U q = t < qh ? t : qt + (t - qh);
      U rr, j, i;
      locate(q, rr, j, i);
      reinterpret_cast<E *>(b0)[q] = sm[d0 + rr * n + fn(i, j)];
    }
    __syncthreads();
  }
}

// ----------------------------------------------------------------- CARRY ----
// unit = one (carry item, slice) segment.  The words of all the item's units
// are spread over every thread of the CTA (segments can be a few words long),
// with four loads in flight per thread before their stores.
template <int AW>
__device__ __forceinline__ void bx_carry_words(const BPass &P, int64_t u0, int64_t u1) {
  using W = typename WordT<AW>::type;
  const int64_t wps = P.seg_bytes / AW;
  const int64_t total = (u1 - u0) * wps;
  auto addr = [&](int64_t w, const W *&src, W *&dst) {
    const int64_t u = u0 + w / wps, word = w % wps;
    const int64_t ii = u / P.d3, k = u - ii * P.d3;
    const CarryItem ci = P.carries[ii];
    src = reinterpret_cast<const W *>(P.data + k * P.slice_bytes + ci.pos * P.seg_bytes) + word;
    dst = reinterpret_cast<W *>(P.carry_buf + (ci.slot * P.d3 + k) * P.seg_bytes) + word;
  };
  constexpr int UNR = 4;
  const int64_t step = (int64_t)blockDim.x * UNR;
  for (int64_t w0 = threadIdx.x; w0 < total; w0 += step) {
    const W *src[UNR];
    W *dst[UNR];
    W v[UNR];
#pragma unroll
    for (int q = 0; q < UNR; q++) {
      const int64_t w = w0 + (int64_t)q * blockDim.x;
      if (w < total) {
        addr(w, src[q], dst[q]);
        v[q] = __ldcg(src[q]);
      }
    }
#pragma unroll
    for (int q = 0; q < UNR; q++)
      if (w0 + (int64_t)q * blockDim.x < total) *dst[q] = v[q];
  }
}

__device__ __noinline__ void bx_carry(const BPass &P, int64_t u0, int64_t u1) {
  switch (P.seg_aw) {
    case 16: bx_carry_words<16>(P, u0, u1); break;
    case 8: bx_carry_words<8>(P, u0, u1); break;
    case 4: bx_carry_words<4>(P, u0, u1); break;
    case 2: bx_carry_words<2>(P, u0, u1); break;
    default: bx_carry_words<1>(P, u0, u1); break;
  }
}

// ------------------------------------------------------------------- SEG ----
// TMA ring walker run by lane 0 of one warp over one item (chunk, piece, slice).
template <typename U>
__device__ __noinline__ bool bx_seg_walk_tma(const BPass &P, const AnyFn<U> &f, int64_t it, uint64_t *bars, char *buf,
                                uint32_t &parity) {
  constexpr int NB = kBatchRing;
  const int64_t per_chunk = P.pieces * P.d3;
  const int64_t c = it / per_chunk, rest = it - c * per_chunk;
  const int64_t k = rest / P.pieces, pc = rest - k * P.pieces;
  const Chunk ch = P.chunks[c];
  const int64_t off = pc * P.piece_bytes;
  const uint32_t pb = (uint32_t)min(P.piece_bytes, P.seg_bytes - off);
  char *base = P.data + k * P.slice_bytes + off;
  const int64_t L = ch.len;
  U xi = (U)ch.start;
  U pos[NB];
  mbar_expect_tx(&bars[0], pb);
  if (ch.carry >= 0)
    bulk_g2s(buf, P.carry_buf + (ch.carry * P.d3 + k) * P.seg_bytes + off, pb, &bars[0]);
  else
    bulk_g2s(buf, base + (int64_t)xi * P.seg_bytes, pb, &bars[0]);
  pos[0] = xi;
  int64_t issued = 1;
  while (issued < L && issued <= NB - 2) {
    xi = f.perm(xi);
    const int b = (int)(issued % NB);
    pos[b] = xi;
    mbar_expect_tx(&bars[b], pb);
    bulk_g2s(buf + (int64_t)b * P.piece_bytes, base + (int64_t)xi * P.seg_bytes, pb, &bars[b]);
    issued++;
  }
  // on a timeout, wait (bounded) for the loads [waited, issued) still in
  // flight and drain the stores before giving up
  int64_t waited = 0;
  auto give_up = [&]() {
    for (int64_t j = waited; j < issued; j++) {
      const int b = (int)(j % NB);
      if (!mbar_wait(&bars[b], (parity >> b) & 1u)) break;
      parity ^= 1u << b;
    }
    bulk_wait_all<0>();
    return false;
  };
  if (!mbar_wait(&bars[0], parity & 1u)) return give_up();
  parity ^= 1u;
  waited = 1;
  U last = pos[0];
  for (int64_t s = 1; s <= L; s++) {
    const int bs = (int)(s % NB), bp = (int)((s - 1) % NB);
    U target;
    if (s < L) {
      if (!mbar_wait(&bars[bs], (parity >> bs) & 1u)) return give_up();
      parity ^= 1u << bs;
      waited = s + 1;
      target = pos[bs];
    } else {
      target = f.perm(last);
    }
    fence_proxy_async();
    bulk_s2g(base + (int64_t)target * P.seg_bytes, buf + (int64_t)bp * P.piece_bytes, pb);
    bulk_commit();
    last = target;
    if (issued < L) {
      bulk_wait_read<1>();
      xi = f.perm(xi);
      const int b = (int)(issued % NB);
      pos[b] = xi;
      mbar_expect_tx(&bars[b], pb);
      bulk_g2s(buf + (int64_t)b * P.piece_bytes, base + (int64_t)xi * P.seg_bytes, pb, &bars[b]);
      issued++;
    }
  }
  bulk_wait_read<0>();
  return true;
}

// Register walker: the warp walks one item, one 16-byte word per lane per
// segment piece (a piece is 32 words here).
template <int AW, typename U>
__device__ __noinline__ void bx_seg_walk_reg(const BPass &P, const AnyFn<U> &f, int64_t it, int lane) {
  using W = typename WordT<AW>::type;
  const int64_t per_chunk = P.pieces * P.d3;
  const int64_t c = it / per_chunk, rest = it - c * per_chunk;
  const int64_t k = rest / P.pieces, pc = rest - k * P.pieces;
  const int64_t off = (pc * 32 + lane) * AW;
  if (off >= P.seg_bytes) return;
  const Chunk ch = P.chunks[c];
  char *base = P.data + k * P.slice_bytes + off;
  U pos = (U)ch.start;
  W cur = (ch.carry >= 0) ? *reinterpret_cast<const W *>(P.carry_buf + (ch.carry * P.d3 + k) * P.seg_bytes + off)
                          : __ldcg(reinterpret_cast<const W *>(base + (int64_t)pos * P.seg_bytes));
  constexpr int UNR = 8;
  int64_t remaining = ch.len;
  while (remaining > 0) {
    const int cnt = remaining < UNR ? (int)remaining : UNR;
    const bool last_group = remaining == cnt;
    U ps[UNR];
    W nx[UNR];
#pragma unroll
    for (int u = 0; u < UNR; u++)
      if (u < cnt) {
        pos = f.perm(pos);
        ps[u] = pos;
      }
#pragma unroll
    for (int u = 0; u < UNR; u++)
      if (u < cnt && !(last_group && u == cnt - 1))
        nx[u] = __ldcg(reinterpret_cast<const W *>(base + (int64_t)ps[u] * P.seg_bytes));
#pragma unroll
    for (int u = 0; u < UNR; u++)
      if (u < cnt) __stcg(reinterpret_cast<W *>(base + (int64_t)ps[u] * P.seg_bytes), u == 0 ? cur : nx[u == 0 ? 0 : u - 1]);
    if (!last_group) cur = nx[UNR - 1];
    remaining -= cnt;
  }
}

// ---------------------------------------------------------------- kernel ----
template <typename U>
__device__ bool bx_dispatch(const BPass &P, const AnyFn<U> &f, int64_t u0, int64_t u1, unsigned char *dyn,
                            uint64_t *bars, uint32_t &parity) {
  unsigned char *smem = dyn;
  switch (P.kind) {
    case BK_TILE:
      if (P.tile_vec) {
        if (P.eb == 4) bx_tile_vec<4>(P, u0, u1, smem);
        else if (P.eb == 8) bx_tile_vec<8>(P, u0, u1, smem);
        else bx_tile_vec<16>(P, u0, u1, smem);
      } else {
        switch (P.eb) {
          case 1: bx_tile_scalar<1>(P, u0, u1, smem); break;
          case 2: bx_tile_scalar<2>(P, u0, u1, smem); break;
          case 4: bx_tile_scalar<4>(P, u0, u1, smem); break;
          case 8: bx_tile_scalar<8>(P, u0, u1, smem); break;
          default: bx_tile_scalar<16>(P, u0, u1, smem); break;
        }
      }
      return true;
    case BK_BAND:
      switch (P.eb) {
        case 1: bx_band<1, false>(P, u0, u1, smem); break;
        case 2: if (P.band_vec) bx_band<2, true>(P, u0, u1, smem); else bx_band<2, false>(P, u0, u1, smem); break;
        case 4: if (P.band_vec) bx_band<4, true>(P, u0, u1, smem); else bx_band<4, false>(P, u0, u1, smem); break;
        case 8: if (P.band_vec) bx_band<8, true>(P, u0, u1, smem); else bx_band<8, false>(P, u0, u1, smem); break;
        default: bx_band<16, false>(P, u0, u1, smem); break;
      }
      return true;
    case BK_COL: {
      if (P.col_form) {
        int *s_sh = reinterpret_cast<int *>(reinterpret_cast<unsigned char *>(bars) + 1024);
        auto loc = [&](auto off, auto F, auto G) {
          using Off = decltype(off);
          using Fm = decltype(F);
          using Gm = decltype(G);
          switch (P.eb * 100 + P.aw) {
            case 101: bx_col_local<1, 1, U, Off, Fm, Gm>(P, off, F, G, u0, u1, smem, s_sh); break;
            case 202: bx_col_local<2, 2, U, Off, Fm, Gm>(P, off, F, G, u0, u1, smem, s_sh); break;
            case 404: bx_col_local<4, 4, U, Off, Fm, Gm>(P, off, F, G, u0, u1, smem, s_sh); break;
            case 416: bx_col_local<4, 16, U, Off, Fm, Gm>(P, off, F, G, u0, u1, smem, s_sh); break;
            case 408: bx_col_local<4, 8, U, Off, Fm, Gm>(P, off, F, G, u0, u1, smem, s_sh); break;
            case 808: bx_col_local<8, 8, U, Off, Fm, Gm>(P, off, F, G, u0, u1, smem, s_sh); break;
            case 816: bx_col_local<8, 16, U, Off, Fm, Gm>(P, off, F, G, u0, u1, smem, s_sh); break;
            default: bx_col_local<16, 16, U, Off, Fm, Gm>(P, off, F, G, u0, u1, smem, s_sh); break;
          }
        };
        if (P.col_form == 2) {
          loc(OffAffine<U, false>{pass_mdiv<U>(P)}, MapId<U>{}, f.template as<PermR2CPre<U>>());
        } else if (P.col_form == 3) {
          loc(OffAffine<U, true>{pass_mdiv<U>(P)}, f.template as<PermR2CPre<U>>(), MapId<U>{});
        } else {
          switch (f.kind) {
            case T213_FN_C2R_PREROTATOR:
              loc(OffOfCol<U, RotGather<U, RotC2RPre<U>>>{f.template as<RotGather<U, RotC2RPre<U>>>()}, MapId<U>{}, MapId<U>{});
              break;
            case T213_FN_C2R_POSTROTATOR:
              loc(OffOfCol<U, RotGather<U, RotC2RPost<U>>>{f.template as<RotGather<U, RotC2RPost<U>>>()}, MapId<U>{}, MapId<U>{});
              break;
            case T213_FN_R2C_PREROTATOR:
              loc(OffOfCol<U, RotGather<U, RotR2CPre<U>>>{f.template as<RotGather<U, RotR2CPre<U>>>()}, MapId<U>{}, MapId<U>{});
              break;
            case T213_FN_R2C_POSTROTATOR:
              loc(OffOfCol<U, RotGather<U, RotR2CPost<U>>>{f.template as<RotGather<U, RotR2CPost<U>>>()}, MapId<U>{}, MapId<U>{});
              break;
            case T213_FN_C2R_FUSED_PREOP:
              loc(OffOfCol<U, ColC2RFusedPre<U>>{f.template as<ColC2RFusedPre<U>>()}, MapId<U>{}, MapId<U>{});
              break;
            default:
              loc(OffOfCol<U, ColR2CFusedPost<U>>{f.template as<ColR2CFusedPost<U>>()}, MapId<U>{}, MapId<U>{});
              break;
          }
        }
        return true;
      }
      auto go = [&](auto tag) {
        using F = typename decltype(tag)::type;
        switch (P.eb * 100 + P.aw) {
          case 101: bx_col<1, 1, U, F>(P, u0, u1, smem); break;
          case 202: bx_col<2, 2, U, F>(P, u0, u1, smem); break;
          case 404: bx_col<4, 4, U, F>(P, u0, u1, smem); break;
          case 416: bx_col<4, 16, U, F>(P, u0, u1, smem); break;
            case 408: bx_col<4, 8, U, F>(P, u0, u1, smem); break;
          case 808: bx_col<8, 8, U, F>(P, u0, u1, smem); break;
          case 816: bx_col<8, 16, U, F>(P, u0, u1, smem); break;
          default: bx_col<16, 16, U, F>(P, u0, u1, smem); break;
        }
      };
      switch (f.kind) {
        case T213_FN_C2R_PREROTATOR: go(TypeTag<RotGather<U, RotC2RPre<U>>>{}); break;
        case T213_FN_C2R_POSTROTATOR: go(TypeTag<RotGather<U, RotC2RPost<U>>>{}); break;
        case T213_FN_R2C_PREROTATOR: go(TypeTag<RotGather<U, RotR2CPre<U>>>{}); break;
        case T213_FN_R2C_POSTROTATOR: go(TypeTag<RotGather<U, RotR2CPost<U>>>{}); break;
        case T213_FN_C2R_FUSED_PREOP: go(TypeTag<ColC2RFusedPre<U>>{}); break;
        case T213_FN_C2R_FUSED_POSTOP: go(TypeTag<ColC2RFusedPost<U>>{}); break;
        case T213_FN_R2C_FUSED_PREOP: go(TypeTag<ColR2CFusedPre<U>>{}); break;
        default: go(TypeTag<ColR2CFusedPost<U>>{}); break;
      }
      return true;
    }
    case BK_ROW: {
      auto go = [&](auto tag) {
        using F = typename decltype(tag)::type;
        switch (P.eb * 100 + P.aw) {
          case 101: bx_row<1, 1, U, F>(P, u0, u1, smem); break;
          case 202: bx_row<2, 2, U, F>(P, u0, u1, smem); break;
          case 404: bx_row<4, 4, U, F>(P, u0, u1, smem); break;
          case 416: bx_row<4, 16, U, F>(P, u0, u1, smem); break;
            case 408: bx_row<4, 8, U, F>(P, u0, u1, smem); break;
          case 808: bx_row<8, 8, U, F>(P, u0, u1, smem); break;
          case 816: bx_row<8, 16, U, F>(P, u0, u1, smem); break;
          default: bx_row<16, 16, U, F>(P, u0, u1, smem); break;
        }
      };
      if (P.row_peel) {
        auto gp = [&](auto tag) {
          using F = typename decltype(tag)::type;
          switch (P.eb) {
            case 1: bx_row_peel<1, U, F>(P, u0, u1, smem); break;
            case 2: bx_row_peel<2, U, F>(P, u0, u1, smem); break;
            default: bx_row_peel<4, U, F>(P, u0, u1, smem); break;
          }
        };
        if (f.kind == T213_FN_R2C_SHUFFLE)
          gp(TypeTag<RowR2CShuffle<U>>{});
        else
          gp(TypeTag<RowC2RShuffle<U>>{});
        return true;
      }
      if (f.kind == T213_FN_R2C_SHUFFLE)
        go(TypeTag<RowR2CShuffle<U>>{});
      else
        go(TypeTag<RowC2RShuffle<U>>{});
      return true;
    }
    case BK_CARRY:
      bx_carry(P, u0, u1);
      return true;
    case BK_SEG: {
      const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
      bool ok = true;
      if (P.seg_tma) {
        if (lane == 0) {
          char *buf = reinterpret_cast<char *>(dyn) + (int64_t)warp * kBatchRing * kBatchPiece;
          for (int64_t it = u0 + warp; it < u1 && ok; it += kBatchWarps)
            ok = bx_seg_walk_tma<U>(P, f, it, bars + warp * kBatchRing, buf, parity);
          bulk_wait_all<0>();
          asm volatile("fence.proxy.async;" ::: "memory");
        }
      } else {
        for (int64_t it = u0 + warp; it < u1; it += kBatchWarps) {
          switch (P.seg_aw) {
            case 16: bx_seg_walk_reg<16, U>(P, f, it, lane); break;
            case 8: bx_seg_walk_reg<8, U>(P, f, it, lane); break;
            case 4: bx_seg_walk_reg<4, U>(P, f, it, lane); break;
            case 2: bx_seg_walk_reg<2, U>(P, f, it, lane); break;
            default: bx_seg_walk_reg<1, U>(P, f, it, lane); break;
          }
        }
      }
      return ok;
    }
  }
  return true;
}

__global__ void __launch_bounds__(kBatchThreads, 1)
    k_batch(const BPass *__restrict__ passes, const BItem *__restrict__ items, int64_t n_items,
            unsigned long long *ctrs, unsigned long long *head, int *status, uint64_t wait_ns) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
  unsigned char *dyn = smem_raw + kBatchBarBytes;
  __shared__ long long s_next;
  __shared__ int s_fail;
  // per-warp walker barriers (lane 0 of each warp owns kBatchRing of them)
  if (threadIdx.x % 32 == 0) {
    const int warp = threadIdx.x / 32;
    for (int i = 0; i < kBatchRing; i++) mbar_init(&bars[warp * kBatchRing + i], 1);
    fence_barrier_init();
  }
  if (threadIdx.x == 0) {
    s_fail = 0;
    s_next = (long long)atomicAdd(head, 1ull);
  }
  uint32_t parity = 0;  // owned by lane 0 of each warp
  __syncthreads();
  for (;;) {
    const long long it = s_next;
    if (it >= n_items) break;
    const BItem w = items[it];
    const BPass &P = passes[w.pass];
    if (P.dep_ctr >= 0 && threadIdx.x == 0) {
      volatile unsigned long long *dc = ctrs + P.dep_ctr;
      uint32_t polls = 0;
      uint64_t t0 = 0;
      while (*dc < (unsigned long long)P.dep_target) {
        if (polls == 0) t0 = global_ns();
        if (++polls > kWaitLimit || ((polls & 15) == 0 && global_ns() - t0 > wait_ns)) {
          s_fail = 1;
          break;
        }
        __nanosleep(polls < 64 ? 32 : 256);
      }
      __threadfence();
      asm volatile("fence.proxy.async;" ::: "memory");
    }
    __syncthreads();
    if (s_fail) break;
    // claim the following item now; its value is only needed after this one
    unsigned long long claimed = 0;
    if (threadIdx.x == 0) claimed = atomicAdd(head, 1ull);
    bool ok = P.u64 ? bx_dispatch<uint64_t>(P, P.f64, w.u0, w.u1, dyn, bars, parity)
                    : bx_dispatch<uint32_t>(P, P.f32, w.u0, w.u1, dyn, bars, parity);
    if (!ok) s_fail = 1;
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      atomicAdd(ctrs + P.done_ctr, 1ull);
      s_next = (long long)claimed;
    }
    __syncthreads();
    if (s_fail) break;
  }
  if (threadIdx.x == 0 && s_fail) atomicExch(status, 5 /* T213_ERR_TIMEOUT */);
}

}  // namespace t213
