/*
 * ORACLE — TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of kaihsin/213transpose's algorithm for the in-place 213
 * transpose.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load this file, and only as the checker; the product never links it.
 *
 * Contents
 *   - t213o_seq_tt:     the reference's out-of-place rank-N gather
 *                       (TensorUtil<T>::seq_tt, src/tensor_util.cpp:79-92), the
 *                       authoritative answer for every shape.
 *   - t213o_gather213:  the same answer specialised to the 213 permutation,
 *                       blocked and OpenMP-parallel (this project's own code).
 *   - t213o_ramp:       the known-answer input data[i] = i
 *                       (TensorUtil<T>::init_data, src/tensor_util.cpp:42-47).
 *   - the index functors of include/equations.h and include/skinny.h, in exact
 *     64-bit arithmetic (the reference computes several of them in 32-bit int,
 *     which wraps for large slices; wherever it does not wrap the values agree);
 *   - host executors of every pass (rotate, row shuffle, column shuffle, row
 *     scatter-permute) and of the C2R / R2C / skinny drivers and the public
 *     dispatcher (src/transpose.cu:18-124, src/skinny.cu:313-363), so the
 *     decomposition can be checked pass by pass against the GPU.
 *
 * Parity is pinned: t213o_seq_tt is checked byte for byte against outputs of
 * the reference's own gen_ans (built from its sources by oracle/Makefile) in
 * tests/golden/.
 *
 * Reference-bug emulation (flags of t213o_transpose / t213o_c2r / t213o_r2c),
 * used only to explain divergences of the reference's GPU build:
 *   T213O_REF_POSTOP_BUG  c2r::col_op's fused branch passes d2/c where the math
 *                         needs c (src/transpose.cu:22).
 *   T213O_REF_REG8_BUG    the 8-byte register row shuffles (C2R and R2C) launch
 *                         without a slice offset, so only slice 0 is shuffled,
 *                         and the R=57 variant covers only 57*512 columns
 *                         (src/shuffle.cu:40-49, include/register_ops.h:66-80).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/t213.h"

typedef int64_t i64;
typedef uint64_t u64;

#define T213O_REF_POSTOP_BUG 1
#define T213O_REF_REG8_BUG 2
#define T213O_SMEM_PER_BLOCK 49152 /* cudaDeviceProp::sharedMemPerBlock, src/introspect.cu:34-36 */

/* ------------------------------------------------------------------------- */
/* answer generators                                                         */
/* ------------------------------------------------------------------------- */

/* src/tensor_util.cpp:7-23 (strides) and :79-92 (gather).  For every source
 * linear index, the destination index is the sum over axes i of the source
 * coordinate along i times the destination stride of axis i, where that
 * stride is the product of the extents of the axes that precede i in the
 * permuted order. */
int t213o_seq_tt(void *ans, const void *data, int rank, const i64 *dim, const i64 *perm, i64 eb) {
  if (rank <= 0 || rank > 16 || eb <= 0) return -1;
  i64 stride[16], stride_d[16], vol = 1;
  for (int i = 0; i < rank; i++) {
    stride[i] = vol;
    vol *= dim[i];
  }
  for (int i = 0; i < rank; i++) {
    i64 s = 1;
    for (int j = 0; perm[j] != i; j++) s *= dim[perm[j]];
    stride_d[i] = s;
  }
  const char *src = (const char *)data;
  char *dst = (char *)ans;
  for (i64 idx_s = 0; idx_s < vol; idx_s++) {
    i64 idx_d = 0;
    for (int i = 0; i < rank; i++) idx_d += ((idx_s / stride[i]) % dim[i]) * stride_d[i];
    memcpy(dst + idx_d * eb, src + idx_s * eb, (size_t)eb);
  }
  return 0;
}

/* 213 answer: dst[i2 + d2*i1 + d1*d2*i3] = src[i1 + d1*i2 + d1*d2*i3].
 * Blocked over 32x32 tiles so that both sides stay cache friendly. */
void t213o_gather213(void *dst, const void *src, i64 d1, i64 d2, i64 d3, i64 eb) {
  const char *s = (const char *)src;
  char *d = (char *)dst;
  const i64 T = 32;
  const i64 nb1 = (d1 + T - 1) / T, nb2 = (d2 + T - 1) / T;
  const i64 total = d3 * nb1 * nb2;
#pragma omp parallel for schedule(static)
  for (i64 w = 0; w < total; w++) {
    i64 k = w / (nb1 * nb2), r = w % (nb1 * nb2);
    i64 b2 = r / nb1, b1 = r % nb1;
    const char *ss = s + k * d1 * d2 * eb;
    char *dd = d + k * d1 * d2 * eb;
    i64 e2 = (b2 + 1) * T < d2 ? (b2 + 1) * T : d2;
    i64 e1 = (b1 + 1) * T < d1 ? (b1 + 1) * T : d1;
    for (i64 i2 = b2 * T; i2 < e2; i2++)
      for (i64 i1 = b1 * T; i1 < e1; i1++)
        memcpy(dd + (i2 + d2 * i1) * eb, ss + (i1 + d1 * i2) * eb, (size_t)eb);
  }
}

/* data[i] = i as a little-endian integer of eb bytes (sign-extended for the
 * 16-byte case: low 8 bytes i, high 8 bytes ~i so both halves vary). */
void t213o_ramp(void *data, i64 n, i64 eb) {
  char *p = (char *)data;
#pragma omp parallel for schedule(static)
  for (i64 i = 0; i < n; i++) {
    if (eb == 4) {
      int32_t v = (int32_t)i;
      memcpy(p + i * 4, &v, 4);
    } else if (eb == 8) {
      int64_t v = i;
      memcpy(p + i * 8, &v, 8);
    } else if (eb == 16) {
      int64_t v[2] = {i, ~i};
      memcpy(p + i * 16, v, 16);
    } else {
      u64 v = (u64)i;
      memcpy(p + i * eb, &v, (size_t)eb);
    }
  }
}

/* ------------------------------------------------------------------------- */
/* integer helpers                                                           */
/* ------------------------------------------------------------------------- */

static i64 pmod(i64 x, i64 m) { /* mathematical modulus, result in [0,m) */
  i64 r = x % m;
  return r < 0 ? r + m : r;
}

/* gcd(a,b) and the inverse of a modulo b (0 if gcd != 1): src/gcd.cpp:3-30. */
i64 t213o_ext_gcd(i64 a, i64 b, i64 *mmi) {
  i64 x = 0, lastx = 1, origb = b;
  while (b != 0) {
    i64 q = a / b, nb = a % b;
    a = b;
    b = nb;
    i64 nx = lastx - q * x;
    lastx = x;
    x = nx;
  }
  if (mmi) *mmi = (a == 1) ? (lastx < 0 ? lastx + origb : lastx) : 0;
  return a;
}

/* (x*y) mod m for 0 <= x,y < m without overflow. */
static i64 mulmod(i64 x, i64 y, i64 m) { return (i64)(((__int128)x * (__int128)y) % (__int128)m); }

/* ------------------------------------------------------------------------- */
/* index functors (include/equations.h, include/skinny.h)                    */
/* ------------------------------------------------------------------------- */

typedef struct {
  int kind;
  i64 p[4];
} fn_t;

/* c2r::shuffle::f (equations.h:26-43) */
static i64 c2r_f(i64 m, i64 n, i64 c, i64 i, i64 j) {
  i64 r = j + i * (n - 1);
  return (i - (j % c) <= m - c) ? r : r + m;
}

/* column rotation amount r(j) of the four rotators */
static i64 rot_amount(const fn_t *f, i64 j) {
  switch (f->kind) {
    case T213_FN_C2R_PREROTATOR: /* (b) equations.h:78-94 */
      return j / f->p[0];
    case T213_FN_C2R_POSTROTATOR: /* (m) equations.h:97-113 */
      return j % f->p[0];
    case T213_FN_R2C_PREROTATOR: { /* (m) equations.h:159-176 */
      i64 jm = j % f->p[0];
      return jm == 0 ? 0 : f->p[0] - jm;
    }
    case T213_FN_R2C_POSTROTATOR: { /* (b, m) equations.h:196-222 */
      i64 bd = j / f->p[0], m = f->p[1];
      if (bd == 0) return 0;
      return bd < m ? m - bd : m + m - bd;
    }
  }
  return -1;
}

/* row shuffle s_i(j) */
static i64 row_src(const fn_t *f, i64 i, i64 j) {
  i64 m = f->p[0], n = f->p[1], c = f->p[2], k = f->p[3];
  switch (f->kind) {
    case T213_FN_C2R_SHUFFLE:      /* equations.h:45-53 */
    case T213_FN_C2R_LONG_SHUFFLE: /* skinny.h:57-66: the same map in 64-bit */
    {
      i64 b = n / c;
      i64 fij = c2r_f(m, n, c, i, j);
      i64 q = fij / c, rem = fij % c;
      return mulmod(pmod(k, b), q % b, b) + rem * b;
    }
    case T213_FN_R2C_SHUFFLE: { /* equations.h:187-193 */
      i64 b = n / c;
      i64 r = ((j / b + i) % m) + (i64)(((__int128)j * m) % n);
      return r % n;
    }
  }
  return -1;
}

/* column shuffle source row f(i,j) */
static i64 col_src(const fn_t *f, i64 i, i64 j) {
  switch (f->kind) {
    case T213_FN_C2R_FUSED_PREOP: { /* (m, b) skinny.h:19-22 */
      i64 m = f->p[0], b = f->p[1];
      return (i + j / b) % m;
    }
    case T213_FN_C2R_FUSED_POSTOP: { /* (m, n, c) skinny.h:74-77 */
      i64 m = f->p[0], n = f->p[1], c = f->p[2];
      i64 v = (i64)(((__int128)i * n) % m) - ((i * c) / m) % m + j % m;
      return pmod(v, m);
    }
    case T213_FN_R2C_FUSED_PREOP: { /* (a, c, m, q) skinny.h:94-106 */
      i64 a = f->p[0], c = f->p[1], m = f->p[2], q = f->p[3];
      i64 idx = (i + m - (j % m)) % m;
      i64 t1 = a * (((c - 1) * idx) % c);
      i64 t2 = mulmod(((c - 1 + idx) / c) % a, pmod(q, a), a);
      return t1 + t2;
    }
    case T213_FN_R2C_FUSED_POSTOP: { /* (m, b) skinny.h:113-116 */
      i64 m = f->p[0], b = f->p[1];
      return (i + m - (j / b) % m) % m;
    }
  }
  return -1;
}

/* row permutation destination p(i) (scatter) */
static i64 row_dst(const fn_t *f, i64 i) {
  i64 m = f->p[0], n = f->p[1], c = f->p[2];
  switch (f->kind) {
    case T213_FN_C2R_POSTPERMUTER: { /* equations.h:120-124: (i*n - i/a) mod m */
      i64 a = m / c;
      return pmod((i64)(((__int128)i * n) % m) - (i / a), m);
    }
    case T213_FN_R2C_PREPERMUTER: { /* equations.h:140-152 */
      i64 a = m / c, b = n / c, q;
      t213o_ext_gcd(b, a, &q);
      i64 kk = ((c - 1) * i) % c;
      i64 l = (c - 1 + i) / c;
      return kk * a + mulmod(l % a, pmod(q, a), a);
    }
  }
  return -1;
}

/* Evaluates one functor: rotators return r(j), shufflers s_i(j), column
 * shufflers f(i,j), permuters p(i).  Exposed for tests. */
i64 t213o_index(int kind, const i64 *prm, i64 i, i64 j) {
  fn_t f;
  f.kind = kind;
  for (int q = 0; q < 4; q++) f.p[q] = prm[q];
  if (kind >= 1 && kind <= 4) return rot_amount(&f, j);
  if (kind >= 10 && kind <= 12) return row_src(&f, i, j);
  if (kind >= 20 && kind <= 23) return col_src(&f, i, j);
  if (kind >= 30 && kind <= 31) return row_dst(&f, i);
  return -1;
}

/* ------------------------------------------------------------------------- */
/* pass executors on host buffers: d3 slices of m rows x n columns           */
/* ------------------------------------------------------------------------- */

static fn_t mkfn(int kind, const i64 *prm) {
  fn_t f;
  f.kind = kind;
  for (int q = 0; q < 4; q++) f.p[q] = prm ? prm[q] : 0;
  return f;
}

/* rotate: new[i][j] = old[(i + r(j)) mod m][j]   (src/rotate.cu:217-235 semantics) */
int t213o_rotate(int kind, const i64 *prm, void *data, i64 d3, i64 m, i64 n, i64 eb) {
  fn_t f = mkfn(kind, prm);
  if (kind < 1 || kind > 4) return -1;
  char *d = (char *)data;
  char *col = (char *)malloc((size_t)(m * eb));
  if (!col) return -2;
  for (i64 k = 0; k < d3; k++) {
    char *s = d + k * m * n * eb;
    for (i64 j = 0; j < n; j++) {
      i64 r = pmod(rot_amount(&f, j), m);
      for (i64 i = 0; i < m; i++) memcpy(col + i * eb, s + (i * n + j) * eb, (size_t)eb);
      for (i64 i = 0; i < m; i++) memcpy(s + (i * n + j) * eb, col + ((i + r) % m) * eb, (size_t)eb);
    }
  }
  free(col);
  return 0;
}

/* row shuffle: new[i][j] = old[i][s_i(j)]   (src/smem_ops.cu:77-100 semantics).
 * only_slice0 / max_cols emulate the 8-byte register-shuffle launch bug. */
static int row_shuffle_impl(const fn_t *f, char *d, i64 d3, i64 m, i64 n, i64 eb, i64 slices,
                            i64 max_cols) {
  char *row = (char *)malloc((size_t)(n * eb));
  if (!row) return -2;
  for (i64 k = 0; k < d3 && k < slices; k++) {
    char *s = d + k * m * n * eb;
    for (i64 i = 0; i < m; i++) {
      memcpy(row, s + i * n * eb, (size_t)(n * eb));
      for (i64 j = 0; j < n && j < max_cols; j++) {
        i64 sj = row_src(f, i, j);
        if (sj < 0 || sj >= n) {
          free(row);
          return -3;
        }
        memcpy(s + (i * n + j) * eb, row + sj * eb, (size_t)eb);
      }
    }
  }
  free(row);
  return 0;
}

int t213o_row_shuffle(int kind, const i64 *prm, void *data, i64 d3, i64 m, i64 n, i64 eb) {
  if (kind < 10 || kind > 12) return -1;
  fn_t f = mkfn(kind, prm);
  return row_shuffle_impl(&f, (char *)data, d3, m, n, eb, d3, n);
}

/* column shuffle: new[i][j] = old[f(i,j)][j]   (src/col_shuffle.cu:10-28 semantics) */
int t213o_col_shuffle(int kind, const i64 *prm, void *data, i64 d3, i64 m, i64 n, i64 eb) {
  if (kind < 20 || kind > 23) return -1;
  fn_t f = mkfn(kind, prm);
  char *d = (char *)data;
  char *col = (char *)malloc((size_t)(m * eb));
  if (!col) return -2;
  for (i64 k = 0; k < d3; k++) {
    char *s = d + k * m * n * eb;
    for (i64 j = 0; j < n; j++) {
      for (i64 i = 0; i < m; i++) memcpy(col + i * eb, s + (i * n + j) * eb, (size_t)eb);
      for (i64 i = 0; i < m; i++) {
        i64 si = col_src(&f, i, j);
        if (si < 0 || si >= m) {
          free(col);
          return -3;
        }
        memcpy(s + (i * n + j) * eb, col + si * eb, (size_t)eb);
      }
    }
  }
  free(col);
  return 0;
}

/* row scatter permutation: new[p(i)][*] = old[i][*]   (src/permute.cu:51-114 semantics) */
int t213o_scatter_permute(int kind, const i64 *prm, void *data, i64 d3, i64 m, i64 n, i64 eb) {
  if (kind < 30 || kind > 31) return -1;
  fn_t f = mkfn(kind, prm);
  char *d = (char *)data;
  i64 slice = m * n * eb;
  char *tmp = (char *)malloc((size_t)slice);
  if (!tmp) return -2;
  for (i64 k = 0; k < d3; k++) {
    char *s = d + k * slice;
    memcpy(tmp, s, (size_t)slice);
    for (i64 i = 0; i < m; i++) {
      i64 p = row_dst(&f, i);
      if (p < 0 || p >= m) {
        free(tmp);
        return -3;
      }
      memcpy(s + p * n * eb, tmp + i * n * eb, (size_t)(n * eb));
    }
  }
  free(tmp);
  return 0;
}

/* Cycle structure of a row permuter: writes the number of non-trivial cycles
 * and the longest cycle length (src/permute.cu:18-49 finds the same cycles). */
int t213o_permuter_cycles(int kind, const i64 *prm, i64 m, i64 *n_cycles, i64 *max_len) {
  fn_t f = mkfn(kind, prm);
  char *seen = (char *)calloc((size_t)m, 1);
  if (!seen) return -2;
  i64 nc = 0, ml = 0;
  for (i64 h = 0; h < m; h++) {
    if (seen[h]) continue;
    i64 len = 0, x = h;
    while (!seen[x]) {
      seen[x] = 1;
      x = row_dst(&f, x);
      len++;
    }
    if (len > 1) {
      nc++;
      if (len > ml) ml = len;
    }
  }
  free(seen);
  *n_cycles = nc;
  *max_len = ml;
  return 0;
}

/* ------------------------------------------------------------------------- */
/* drivers                                                                   */
/* ------------------------------------------------------------------------- */

/* c = gcd(m, n) and k = inverse of a = m/c modulo b = n/c
 * (src/transpose.cu:34-40; k = t when c == 1). */
static void c2r_consts(i64 m, i64 n, i64 *c, i64 *k) {
  i64 t;
  *c = t213o_ext_gcd(m, n, &t);
  if (*c > 1)
    t213o_ext_gcd(m / *c, n / *c, k);
  else
    *k = t;
}

/* c = gcd(m, n) and q = inverse of b = n/c modulo a = m/c (src/transpose.cu:76-82). */
static void r2c_consts(i64 m, i64 n, i64 *c, i64 *q) {
  i64 t;
  *c = t213o_ext_gcd(n, m, &t);
  if (*c > 1)
    t213o_ext_gcd(n / *c, m / *c, q);
  else
    *q = t;
}

/* The reference's row-shuffle dispatch (src/shuffle.cu:12-64) for both
 * shufflers.  Every variant computes the same gather, except that with
 * T213O_REF_REG8_BUG the 8-byte register variants (rows over 48 KB and under
 * 29696 columns) are launched without a slice offset, so only slice 0 is
 * shuffled, and R = 57 registers of 512 threads cover 57 * 512 columns
 * (src/shuffle.cu:40-49, include/register_ops.h:66-80). */
static int ref_row_shuffle(const fn_t *f, char *data, i64 d3, i64 m, i64 n, i64 eb, int flags) {
  i64 slices = d3, maxc = n;
  if ((flags & T213O_REF_REG8_BUG) && eb == 8) {
    int compress = 2 * n * eb <= T213O_SMEM_PER_BLOCK / 32;
    int smem = n * eb <= T213O_SMEM_PER_BLOCK;
    if (!compress && !smem && n < 29696) {
      slices = 1;
      maxc = (n < 6918) ? 18 * 512 : 57 * 512;
    }
  }
  return row_shuffle_impl(f, data, d3, m, n, eb, slices, maxc);
}

/* C2R: the slice is m = d2 rows x n = d1 columns (src/transpose.cu:18-47).
 * The column op is the fused column shuffle when a 32-column strip of the
 * slice fits the reference's 48 KB shared-memory limit, else a post-rotation
 * and a row scatter; both give the same permutation. */
int t213o_c2r(void *data, i64 d1, i64 d2, i64 d3, i64 eb, int flags) {
  i64 m = d2, n = d1, c, k;
  if (m <= 0 || n <= 0 || d3 <= 0) return 0;
  c2r_consts(m, n, &c, &k);
  int rc;
  if (c > 1) {
    i64 p[4] = {n / c, 0, 0, 0};
    if ((rc = t213o_rotate(T213_FN_C2R_PREROTATOR, p, data, d3, m, n, eb))) return rc;
  }
  {
    fn_t f = mkfn(T213_FN_C2R_SHUFFLE, (i64[4]){m, n, c, k});
    if ((rc = ref_row_shuffle(&f, (char *)data, d3, m, n, eb, flags))) return rc;
  }
  if (T213O_SMEM_PER_BLOCK / (eb * m) >= 32) {
    i64 third = (flags & T213O_REF_POSTOP_BUG) ? m / c : c;
    i64 p[4] = {m, n, third, 0};
    return t213o_col_shuffle(T213_FN_C2R_FUSED_POSTOP, p, data, d3, m, n, eb);
  }
  {
    i64 p[4] = {m, 0, 0, 0};
    if ((rc = t213o_rotate(T213_FN_C2R_POSTROTATOR, p, data, d3, m, n, eb))) return rc;
    i64 q[4] = {m, n, c, 0};
    return t213o_scatter_permute(T213_FN_R2C_PREPERMUTER, q, data, d3, m, n, eb);
  }
}

/* R2C with the reference's argument convention (src/transpose.cu:70-89): the
 * passes view the slice as m = d2 rows x n = d1 columns, which is the OUTPUT
 * shape; the input is the n x m matrix. */
int t213o_r2c(void *data, i64 d1, i64 d2, i64 d3, i64 eb, int flags) {
  i64 m = d2, n = d1, c, q;
  if (m <= 0 || n <= 0 || d3 <= 0) return 0;
  r2c_consts(m, n, &c, &q);
  int rc;
  if (T213O_SMEM_PER_BLOCK / (eb * m) >= 32) {
    i64 p[4] = {m / c, c, m, q};
    if ((rc = t213o_col_shuffle(T213_FN_R2C_FUSED_PREOP, p, data, d3, m, n, eb))) return rc;
  } else {
    i64 p[4] = {m, n, c, 0};
    if ((rc = t213o_scatter_permute(T213_FN_C2R_POSTPERMUTER, p, data, d3, m, n, eb))) return rc;
    i64 r[4] = {m, 0, 0, 0};
    if ((rc = t213o_rotate(T213_FN_R2C_PREROTATOR, r, data, d3, m, n, eb))) return rc;
  }
  {
    fn_t f = mkfn(T213_FN_R2C_SHUFFLE, (i64[4]){m, n, c, q});
    if ((rc = ref_row_shuffle(&f, (char *)data, d3, m, n, eb, flags))) return rc;
  }
  if (c > 1) {
    i64 p[4] = {n / c, m, 0, 0};
    return t213o_rotate(T213_FN_R2C_POSTROTATOR, p, data, d3, m, n, eb);
  }
  return 0;
}

/* skinny C2R, m = d2 <= 32 rows (src/skinny.cu:313-333) */
int t213o_skinny_c2r(void *data, i64 d1, i64 d2, i64 d3, i64 eb) {
  i64 m = d2, n = d1, c, k;
  if (m <= 0 || n <= 0 || d3 <= 0) return 0;
  c2r_consts(m, n, &c, &k);
  int rc;
  if (c > 1) {
    i64 p[4] = {m, n / c, 0, 0};
    if ((rc = t213o_col_shuffle(T213_FN_C2R_FUSED_PREOP, p, data, d3, m, n, eb))) return rc;
  }
  {
    i64 p[4] = {m, n, c, k};
    if ((rc = t213o_row_shuffle(T213_FN_C2R_LONG_SHUFFLE, p, data, d3, m, n, eb))) return rc;
  }
  i64 p[4] = {m, n, c, 0};
  return t213o_col_shuffle(T213_FN_C2R_FUSED_POSTOP, p, data, d3, m, n, eb);
}

/* skinny R2C, m = d2 <= 32 rows of the output view (src/skinny.cu:344-363) */
int t213o_skinny_r2c(void *data, i64 d1, i64 d2, i64 d3, i64 eb) {
  i64 m = d2, n = d1, c, q;
  if (m <= 0 || n <= 0 || d3 <= 0) return 0;
  r2c_consts(m, n, &c, &q);
  int rc;
  {
    i64 p[4] = {m / c, c, m, q};
    if ((rc = t213o_col_shuffle(T213_FN_R2C_FUSED_PREOP, p, data, d3, m, n, eb))) return rc;
  }
  {
    i64 p[4] = {m, n, c, 0};
    if ((rc = t213o_row_shuffle(T213_FN_R2C_SHUFFLE, p, data, d3, m, n, eb))) return rc;
  }
  if (c > 1) {
    i64 p[4] = {m, n / c, 0, 0};
    return t213o_col_shuffle(T213_FN_R2C_FUSED_POSTOP, p, data, d3, m, n, eb);
  }
  return 0;
}

/* public dispatcher (src/transpose.cu:99-124) */
int t213o_transpose(void *data, i64 d1, i64 d2, i64 d3, i64 eb, int flags) {
  if (d2 <= 32 || d1 <= 32) {
    if (d2 < d1) return t213o_skinny_c2r(data, d1, d2, d3, eb);
    return t213o_skinny_r2c(data, d2, d1, d3, eb);
  }
  if (d1 >= d2) return t213o_c2r(data, d1, d2, d3, eb, flags);
  return t213o_r2c(data, d2, d1, d3, eb, flags);
}
