/*
 * inplace_detail.h — reference-compatible detail API (the pass entry points of
 * kaihsin/213transpose: include/rotate.h, shuffle.h, col_shuffle.h, permute.h,
 * skinny.h, equations.h).  The functors here are host-side descriptors with
 * the reference constructors' signatures; the passes themselves run in the
 * CUDA library through the C ABI of t213.h.  Each pass runs on the legacy
 * default stream and returns when it is done; failures throw
 * std::runtime_error.
 */
#pragma once

#include <stdint.h>

#include <stdexcept>
#include <string>

#include "t213.h"

namespace inplace {

namespace detail {

struct functor_desc {
  int kind;
  int64_t p[4];  /* the constructor's arguments, in the reference's order */
  int np;
};

inline void t213_throw_on(int status, const char *what) {
  if (status != T213_OK)
    throw std::runtime_error(std::string(what) + ": " + t213_status_string(status) + ": " + t213_last_error());
}

int t213_sync_default_stream();

namespace c2r {

struct prerotator : functor_desc {       /* equations.h:78-94 */
  explicit prerotator(int b) : functor_desc{T213_FN_C2R_PREROTATOR, {b, 0, 0, 0}, 1} {}
};
struct postrotator : functor_desc {      /* equations.h:97-113 */
  explicit postrotator(int m) : functor_desc{T213_FN_C2R_POSTROTATOR, {m, 0, 0, 0}, 1} {}
};
struct shuffle : functor_desc {          /* equations.h:12-54 */
  shuffle(int m, int n, int c, int k) : functor_desc{T213_FN_C2R_SHUFFLE, {m, n, c, k}, 4} {}
};
struct long_shuffle : functor_desc {     /* skinny.h:29-67 */
  long_shuffle(int m, int n, int c, int k) : functor_desc{T213_FN_C2R_LONG_SHUFFLE, {m, n, c, k}, 4} {}
};
struct postpermuter : functor_desc {     /* equations.h:115-128 */
  postpermuter(int m, int n, int c) : functor_desc{T213_FN_C2R_POSTPERMUTER, {m, n, c, 0}, 3} {}
};
struct fused_preop : functor_desc {      /* skinny.h:12-26 */
  fused_preop(int m, int b) : functor_desc{T213_FN_C2R_FUSED_PREOP, {m, b, 0, 0}, 2} {}
};
struct fused_postop : functor_desc {     /* skinny.h:69-78 */
  fused_postop(int m, int n, int c) : functor_desc{T213_FN_C2R_FUSED_POSTOP, {m, n, c, 0}, 3} {}
};
template <typename T> void skinny_transpose(T *data, int d1, int d2, int d3);

}  // namespace c2r

namespace r2c {

struct prepermuter : functor_desc {      /* equations.h:134-157 */
  prepermuter(int m, int n, int c) : functor_desc{T213_FN_R2C_PREPERMUTER, {m, n, c, 0}, 3} {}
};
struct prerotator : functor_desc {       /* equations.h:159-176 */
  explicit prerotator(int m) : functor_desc{T213_FN_R2C_PREROTATOR, {m, 0, 0, 0}, 1} {}
};
struct shuffle : functor_desc {          /* equations.h:178-194 */
  shuffle(int m, int n, int c, int k) : functor_desc{T213_FN_R2C_SHUFFLE, {m, n, c, k}, 4} {}
};
struct postrotator : functor_desc {      /* equations.h:196-222 */
  postrotator(int b, int m) : functor_desc{T213_FN_R2C_POSTROTATOR, {b, m, 0, 0}, 2} {}
};
struct fused_preop : functor_desc {      /* skinny.h:87-107 */
  fused_preop(int a, int c, int m, int q) : functor_desc{T213_FN_R2C_FUSED_PREOP, {a, c, m, q}, 4} {}
};
struct fused_postop : functor_desc {     /* skinny.h:109-117 */
  fused_postop(int m, int b) : functor_desc{T213_FN_R2C_FUSED_POSTOP, {m, b, 0, 0}, 2} {}
};
template <typename T> void skinny_transpose(T *data, int d1, int d2, int d3);

}  // namespace r2c

namespace c2r {
typedef r2c::prepermuter scatter_postpermuter;   /* equations.h:226-236 */
}
namespace r2c {
typedef c2r::postpermuter scatter_prepermuter;
}

/* include/rotate.h:6-7 */
template <typename F, typename T>
void rotate(F f, int d3, int d2, int d1, T *data) {
  t213_throw_on(t213_rotate(f.kind, f.p, f.np, data, d3, d2, d1, (int)sizeof(T), 0),
                "inplace::detail::rotate");
  t213_throw_on(t213_sync_default_stream(), "inplace::detail::rotate");
}

/* include/shuffle.h:5-6 */
template <typename T, typename F>
void shuffle_fn(T *data, int d3, int d2, int d1, F s) {
  t213_throw_on(t213_row_shuffle(s.kind, s.p, s.np, data, d3, d2, d1, (int)sizeof(T), 0),
                "inplace::detail::shuffle_fn");
  t213_throw_on(t213_sync_default_stream(), "inplace::detail::shuffle_fn");
}

/* include/col_shuffle.h:8-9 */
template <typename F, typename T>
void col_shuffle_fn(F fn, int d3, int d2, int d1, T *data) {
  t213_throw_on(t213_col_shuffle(fn.kind, fn.p, fn.np, data, d3, d2, d1, (int)sizeof(T), 0),
                "inplace::detail::col_shuffle_fn");
  t213_throw_on(t213_sync_default_stream(), "inplace::detail::col_shuffle_fn");
}

/* include/permute.h:6-7 */
template <typename T, typename F>
void scatter_permute(F f, int d3, int d2, int d1, T *data) {
  t213_throw_on(t213_scatter_permute(f.kind, f.p, f.np, data, d3, d2, d1, (int)sizeof(T), 0),
                "inplace::detail::scatter_permute");
  t213_throw_on(t213_sync_default_stream(), "inplace::detail::scatter_permute");
}

}  // namespace detail
}  // namespace inplace
