// Index functors of the C2R / R2C decomposition (Catanzaro, Keller & Garland,
// "A Decomposition for In-place Matrix Transposition", PPoPP 2014, as extended
// by kaihsin/213transpose with a batch axis) and of the segment permutations
// used by the block and band plans.
//
// Inside a slice the matrix has m rows and n columns, c = gcd(m,n), a = m/c,
// b = n/c.  Every functor is templated on its index word U (uint32_t when the
// host has checked that all intermediate values stay below 2^31, otherwise
// uint64_t with values below 2^63) and is usable on host and device, so the
// host computes cycle tables with exactly the device's arithmetic.
//
// Three shapes of functor:
//   column gathers  src(i,j): new[i][j] = old[src(i,j)][j]
//   row gathers     src(i,j): new[i][j] = old[i][src(i,j)]
//   scatters        dst(p):   new[dst(p)] = old[p]   (p indexes whole segments)
// Every gather result is reduced into range, so a functor built from
// inconsistent parameters can only give a wrong permutation, never an
// out-of-bounds access.
#pragma once

#include "common.cuh"

namespace t213 {

// ---------------------------------------------------------------- rotators --
// Amounts r(j) of the four rotators of include/equations.h, each a function of
// its own constructor parameters only.  RotGather turns one into the column
// gather new[i][j] = old[(i + r(j)) mod m][j] of an m-row slice, reducing the
// amount modulo m the way the reference's (i - r + d2) % d2 does.

template <typename U>
struct RotC2RPre {  // r = j / b                      equations.h:78-94
  FastDiv<U> b;
  RotC2RPre() = default;
  __host__ explicit RotC2RPre(int64_t b_) : b(b_) {}
  T213_HD U amount(U j) const { return b.div(j); }
};

template <typename U>
struct RotC2RPost {  // r = j mod m                   equations.h:97-113
  FastDiv<U> m;
  RotC2RPost() = default;
  __host__ explicit RotC2RPost(int64_t m_) : m(m_) {}
  T213_HD U amount(U j) const { return m.mod(j); }
};

template <typename U>
struct RotR2CPre {  // r = (m - j mod m) mod m        equations.h:159-176
  FastDiv<U> m;
  RotR2CPre() = default;
  __host__ explicit RotR2CPre(int64_t m_) : m(m_) {}
  T213_HD U amount(U j) const {
    U jm = m.mod(j);
    return jm ? m.get() - jm : 0;
  }
};

template <typename U>
struct RotR2CPost {  // r = 0 if j < b, m - j/b if j/b < m, else 2m - j/b   equations.h:196-222
  FastDiv<U> b;
  U m;
  RotR2CPost() = default;
  __host__ RotR2CPost(int64_t b_, int64_t m_) : b(b_), m((U)m_) {}
  T213_HD U amount(U j) const {
    U bd = b.div(j);
    if (bd == 0) return 0;
    if (bd < m) return m - bd;
    return bd < m + m ? m + m - bd : 0;
  }
};

template <typename U, typename R>
struct RotGather {
  R r;
  FastDiv<U> m;
  RotGather() = default;
  __host__ RotGather(R r_, int64_t m_) : r(r_), m(m_) {}
  T213_HD U operator()(U i, U j) const {
    U a = r.amount(j);
    if (a >= m.get()) a = m.mod(a);
    U s = i + a;
    return s >= m.get() ? s - m.get() : s;
  }
};

// ------------------------------------------------------- column shufflers --

template <typename U>
struct ColC2RFusedPre {  // (i + j/b) mod m           skinny.h:12-26
  FastDiv<U> m, b;
  ColC2RFusedPre() = default;
  __host__ ColC2RFusedPre(int64_t m_, int64_t b_) : m(m_), b(b_) {}
  T213_HD U operator()(U i, U j) const { return m.mod(i + b.div(j)); }
};

template <typename U>
struct ColC2RFusedPost {  // (i*n - i*c/m + j) mod m   skinny.h:69-78
  FastDiv<U> m;
  U n, c;
  ColC2RFusedPost() = default;
  __host__ ColC2RFusedPost(int64_t m_, int64_t n_, int64_t c_) : m(m_), n((U)n_), c((U)c_) {}
  T213_HD U operator()(U i, U j) const {
    U mm = m.get();
    U t1 = m.mod(i * n);
    U t2 = m.mod(m.div(i * c));
    U v = t1 + (mm - t2) + m.mod(j);  // < 3m
    return m.mod(v);
  }
};

template <typename U>
struct ColR2CFusedPre {  // p((i - j) mod m)           skinny.h:87-107
  FastDiv<U> a, c, m;
  U q;
  ColR2CFusedPre() = default;
  __host__ ColR2CFusedPre(int64_t a_, int64_t c_, int64_t m_, int64_t q_)
      : a(a_), c(c_), m(m_), q((U)(q_ % (a_ > 0 ? a_ : 1))) {}
  T213_HD U p(U idx) const {
    U cm1 = c.get() - 1;
    U t1 = a.get() * c.mod(cm1 * idx);
    U t2 = a.mod(a.mod(c.div(cm1 + idx)) * q);
    return t1 + t2;
  }
  T213_HD U operator()(U i, U j) const {
    U mm = m.get();
    U idx = m.mod(i + mm - m.mod(j));
    U s = p(idx);
    return s < mm ? s : m.mod(s);
  }
};

template <typename U>
struct ColR2CFusedPost {  // (i + m - j/b) mod m       skinny.h:109-117
  FastDiv<U> m, b;
  ColR2CFusedPost() = default;
  __host__ ColR2CFusedPost(int64_t m_, int64_t b_) : m(m_), b(b_) {}
  T213_HD U operator()(U i, U j) const { return m.mod(i + m.get() - m.mod(b.div(j))); }
};

// ----------------------------------------------------------- row shufflers --

template <typename U>
struct RowC2RShuffle {  // equations.h:12-54 (and the 64-bit long_shuffle, skinny.h:29-67)
  FastDiv<U> c, b, n;
  U m, k;
  RowC2RShuffle() = default;
  __host__ RowC2RShuffle(int64_t m_, int64_t n_, int64_t c_, int64_t k_)
      : c(c_), b(n_ / (c_ > 0 ? c_ : 1)), n(n_), m((U)m_) {
    int64_t bb = n_ / (c_ > 0 ? c_ : 1);
    int64_t kk = bb > 0 ? k_ % bb : 0;
    if (kk < 0) kk += bb;
    k = (U)kk;
  }
  T213_HD U operator()(U i, U j) const {
    if (c.get() == 1) {
      // coprime m, n: f = j + i(n-1) (i < m always satisfies the low test), so
      // f mod n = (j - i) mod n and s = k * (j - i) mod n, with k < b = n
      const U nn = n.get();
      const U im = i < nn ? i : n.mod(i);
      const U d = j >= im ? j - im : j + nn - im;
      return n.mod(k * d);
    }
    U jc = c.mod(j);
    // i - (j mod c) <= m - c, evaluated without unsigned wrap
    bool low = i + c.get() <= m + jc;
    U f = j + i * (n.get() - 1) + (low ? 0 : m);
    U qq = c.div(f);
    U rem = f - qq * c.get();
    U s = b.mod(k * b.mod(qq)) + rem * b.get();
    return s < n.get() ? s : n.mod(s);
  }
};

template <typename U>
struct RowR2CShuffle {  // equations.h:178-194
  FastDiv<U> m, n, b;
  RowR2CShuffle() = default;
  __host__ RowR2CShuffle(int64_t m_, int64_t n_, int64_t c_) : m(m_), n(n_), b(n_ / (c_ > 0 ? c_ : 1)) {}
  T213_HD U operator()(U i, U j) const {
    if (b.get() == n.get()) return n.mod(i + j * m.get());  // c = 1: j / b = 0 and i < m
    U r = m.mod(b.div(j) + i) + j * m.get();
    return n.mod(r);
  }
};

// Row shufflers evaluated along a row: first(i, j), then next(i, j + 1),
// next(i, j + 2), ... carry the functor's intermediate values from one column
// to the next.  Any other row functor is evaluated anew at every column.
template <typename F, typename U>
struct RowStepper {
  const F &f;
  T213_HD explicit RowStepper(const F &f_) : f(f_) {}
  T213_HD U first(U i, U j) { return f(i, j); }
  T213_HD U next(U i, U j) { return f(i, j); }
};

// C2R shuffle.  Coprime m, n: s = k (j - i) mod n grows by k.  Otherwise, with
// jc = j mod c, f = j + i (n - 1) (+ m when i - jc > m - c), q = f / c, r =
// f mod c and s = (k (q mod b)) mod b + r b: while the +m term stays put, f
// grows by one, so r does, carrying into q, whose term (k q) mod b then grows
// by k mod b; when the +m term flips (jc wrapping, or reaching the bound),
// everything is evaluated anew.
template <typename U>
struct RowStepper<RowC2RShuffle<U>, U> {
  const RowC2RShuffle<U> &f;
  U n, b, c, k, i = 0, jc = 0, rem = 0, bq = 0, kb = 0, s = 0;
  bool low = false;
  T213_HD explicit RowStepper(const RowC2RShuffle<U> &f_)
      : f(f_), n(f_.n.get()), b(f_.b.get()), c(f_.c.get()), k(f_.k) {}
  T213_HD U first(U i_, U j) {
    if (c == 1) return s = f(i_, j);
    i = i_;
    jc = f.c.mod(j);
    low = i + c <= f.m + jc;
    const U ff = j + i * (n - 1) + (low ? 0 : f.m);
    const U qq = f.c.div(ff);
    rem = ff - qq * c;
    bq = f.b.mod(qq);
    kb = f.b.mod(k * bq);
    return s = kb + rem * b;
  }
  T213_HD U next(U i_, U j) {
    if (c == 1) {
      const U t = s + k;
      return s = t >= n ? t - n : t;
    }
    if (++jc == c) jc = 0;
    if ((i + c <= f.m + jc) != low) return first(i_, j);
    if (++rem == c) {
      rem = 0;
      if (++bq == b) bq = 0;
      kb += k;
      if (kb >= b) kb -= b;
    }
    return s = kb + rem * b;
  }
};

// R2C shuffle: s = ((j / b + i) mod m + j m) mod n grows by m mod n while j / b
// stays put (always, when m and n are coprime: b = n); at a multiple of b it
// is evaluated anew.
template <typename U>
struct RowStepper<RowR2CShuffle<U>, U> {
  const RowR2CShuffle<U> &f;
  U inc, n, b, jb = 0, s = 0;
  T213_HD explicit RowStepper(const RowR2CShuffle<U> &f_)
      : f(f_), inc(f_.n.mod(f_.m.get())), n(f_.n.get()), b(f_.b.get()) {}
  T213_HD U first(U i, U j) {
    jb = b == n ? 0 : f.b.mod(j);
    return s = f(i, j);
  }
  T213_HD U next(U i, U j) {
    if (b != n && ++jb == b) {
      jb = 0;
      return s = f(i, j);
    }
    const U t = s + inc;
    return s = t >= n ? t - n : t;
  }
};

// ------------------------------------------------------------ row scatters --
// new[dst(i)][*] = old[i][*]

template <typename U>
struct PermC2RPost {  // (i*n - i/a) mod m            equations.h:115-128
  FastDiv<U> m, a;
  U n;
  PermC2RPost() = default;
  __host__ PermC2RPost(int64_t m_, int64_t n_, int64_t c_)
      : m(m_), a(m_ / (c_ > 0 ? c_ : 1)), n((U)n_) {}
  T213_HD U operator()(U i) const {
    U mm = m.get();
    U t = m.mod(i * n) + mm - m.mod(a.div(i));
    return m.mod(t);
  }
};

template <typename U>
struct PermR2CPre {  // equations.h:134-157
  FastDiv<U> c, a, m;
  U q;
  PermR2CPre() = default;
  // q = inverse of b modulo a, computed by the host (extended Euclid).
  __host__ PermR2CPre(int64_t m_, int64_t c_, int64_t q_)
      : c(c_), a(m_ / (c_ > 0 ? c_ : 1)), m(m_), q((U)q_) {}
  T213_HD U operator()(U i) const {
    U cm1 = c.get() - 1;
    U kk = c.mod(cm1 * i);
    U l = c.div(cm1 + i);
    U s = kk * a.get() + a.mod(a.mod(l) * q);
    return s < m.get() ? s : m.mod(s);
  }
};

// ------------------------------------------------------ segment permutation --
// An [A][Mid][C] array of segments rearranged to [C][Mid][A]:
//   p = (x*Mid + s)*C + y  ->  (y*Mid + s)*A + x.
// Mid == 1 is the transposition of an A x C matrix of segments.
template <typename U>
struct SegPerm3 {
  FastDiv<U> C, Mid;
  U A, mid, cc;
  SegPerm3() = default;
  __host__ SegPerm3(int64_t A_, int64_t Mid_, int64_t C_) : C(C_), Mid(Mid_), A((U)A_), mid((U)Mid_), cc((U)C_) {}
  T213_HD U operator()(U p) const {
    U y = C.mod(p);
    U t = C.div(p);
    U s = Mid.mod(t);
    U x = Mid.div(t);
    return (y * mid + s) * A + x;
  }
};

}  // namespace t213
