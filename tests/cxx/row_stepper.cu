// Host check of the row steppers: along every row of many (m, n, c, k), the
// values first(i, 0), next(i, 1), next(i, 2), ... equal the row shuffle
// functors evaluated at every column, for the C2R and the R2C shuffle, both
// index widths, coprime and non-coprime shapes.  Prints "ok <cases>" or the
// first mismatch, and exits non-zero on a mismatch.
#include <cstdint>
#include <cstdio>
#include <random>

#include "functors.cuh"

using namespace t213;

static int64_t gcd64(int64_t a, int64_t b) {
  while (b) {
    const int64_t t = a % b;
    a = b;
    b = t;
  }
  return a;
}

template <typename F, typename U>
static bool check_rows(const F &f, int64_t m, int64_t n, const char *what, std::mt19937_64 &rng) {
  RowStepper<F, U> st(f);
  const int64_t rows[] = {0, 1, m / 2, m - 2, m - 1, (int64_t)(rng() % (uint64_t)m)};
  for (int64_t i : rows) {
    if (i < 0 || i >= m) continue;
    // start at column 0 and at a random column, as a word inside a row does
    const int64_t j0s[] = {0, (int64_t)(rng() % (uint64_t)n)};
    for (int64_t j0 : j0s) {
      U got = st.first((U)i, (U)j0);
      for (int64_t j = j0; j < n; j++) {
        if (j > j0) got = st.next((U)i, (U)j);
        const U want = f((U)i, (U)j);
        if (got != want) {
          std::printf("%s mismatch m=%lld n=%lld i=%lld j=%lld (start %lld): %llu != %llu\n", what, (long long)m,
                      (long long)n, (long long)i, (long long)j, (long long)j0, (unsigned long long)got,
                      (unsigned long long)want);
          return false;
        }
      }
    }
  }
  return true;
}

template <typename U>
static bool one(int64_t m, int64_t n, std::mt19937_64 &rng) {
  const int64_t c = gcd64(m, n), b = n / c;
  const int64_t k = b > 1 ? (int64_t)(rng() % (uint64_t)b) : 0;
  if (!check_rows<RowC2RShuffle<U>, U>(RowC2RShuffle<U>(m, n, c, k), m, n, "c2r", rng)) return false;
  return check_rows<RowR2CShuffle<U>, U>(RowR2CShuffle<U>(m, n, c), m, n, "r2c", rng);
}

int main() {
  std::mt19937_64 rng(12345);
  int cases = 0;
  // chosen shapes: coprime, small and large gcds, c == n, c == m
  const int64_t shapes[][2] = {{7, 5},    {12, 18},   {18, 12},   {64, 48},  {48, 64},   {3, 3},     {1, 9},
                               {9, 1},    {2, 1000},  {1000, 2},  {96, 3000}, {3951, 3210}, {7918, 6150},
                               {6150, 7918}, {4096, 4096}, {30, 1002}, {1002, 334}, {5, 15}, {15, 5}};
  for (auto &s : shapes) {
    if (!one<uint32_t>(s[0], s[1], rng) || !one<uint64_t>(s[0], s[1], rng)) return 1;
    cases += 2;
  }
  // random shapes with a common factor
  for (int t = 0; t < 300; t++) {
    const int64_t g = 1 + (int64_t)(rng() % 24);
    const int64_t m = g * (1 + (int64_t)(rng() % 300)), n = g * (1 + (int64_t)(rng() % 300));
    if (!one<uint32_t>(m, n, rng)) return 1;
    cases++;
  }
  std::printf("ok %d\n", cases);
  return 0;
}
