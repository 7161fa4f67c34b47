// Shared device/host helpers of the in-place 213 transpose: exact division by
// run-time invariant divisors, raw element types, vector access helpers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#ifndef T213_HD
#define T213_HD __host__ __device__ __forceinline__
#endif

namespace t213 {

// ---------------------------------------------------------------------------
// Division by a run-time invariant divisor, after Granlund & Montgomery,
// "Division by Invariant Integers using Multiplication" (PLDI 1994), in the
// round-up form.  For a divisor d >= 2 let l = ceil(log2 d) and, for N-bit
// words, mul = ceil(2^(N-1+l) / d).  mul fits in N bits, and for every
// dividend 0 <= x < 2^(N-1)
//     floor(x / d) = mulhi_N(x, mul) >> (l - 1)
// because the rounding error of mul contributes less than x / 2^(N-1+l) <
// 2^-l <= 1/d to the quotient.  d == 1 is stored as mul == 0.
// ---------------------------------------------------------------------------

T213_HD uint32_t mulhi32(uint32_t x, uint32_t y) {
#ifdef __CUDA_ARCH__
  return __umulhi(x, y);
#else
  return (uint32_t)(((uint64_t)x * (uint64_t)y) >> 32);
#endif
}

T213_HD uint64_t mulhi64(uint64_t x, uint64_t y) {
#ifdef __CUDA_ARCH__
  return __umul64hi(x, y);
#else
  return (uint64_t)(((unsigned __int128)x * (unsigned __int128)y) >> 64);
#endif
}

template <typename U>
struct FastDiv;

template <>
struct FastDiv<uint32_t> {
  uint32_t d = 1, mul = 0, sh = 0;
  FastDiv() = default;
  __host__ explicit FastDiv(uint64_t divisor) : d((uint32_t)divisor) {
    if (d <= 1) {
      d = 1;
      mul = 0;
      sh = 0;
      return;
    }
    uint32_t l = 0;
    while ((1ull << l) < d) l++;
    mul = (uint32_t)((((uint64_t)1 << (31 + l)) + d - 1) / d);
    sh = l - 1;
  }
  T213_HD uint32_t div(uint32_t x) const { return mul ? (mulhi32(x, mul) >> sh) : x; }
  T213_HD uint32_t mod(uint32_t x) const { return x - div(x) * d; }
  T213_HD uint32_t get() const { return d; }
};

template <>
struct FastDiv<uint64_t> {
  uint64_t d = 1, mul = 0;
  uint32_t sh = 0;
  FastDiv() = default;
  __host__ explicit FastDiv(uint64_t divisor) : d(divisor) {
    if (d <= 1) {
      d = 1;
      mul = 0;
      sh = 0;
      return;
    }
    uint32_t l = 0;
    while (l < 64 && (((unsigned __int128)1) << l) < d) l++;
    unsigned __int128 num = ((unsigned __int128)1) << (63 + l);
    mul = (uint64_t)((num + d - 1) / d);
    sh = l - 1;
  }
  T213_HD uint64_t div(uint64_t x) const { return mul ? (mulhi64(x, mul) >> sh) : x; }
  T213_HD uint64_t mod(uint64_t x) const { return x - div(x) * d; }
  T213_HD uint64_t get() const { return d; }
};

// ---------------------------------------------------------------------------
// Raw element types: the transpose moves bits, so each element size maps to
// an unsigned type (uint4 for 16 bytes) of that size.
// ---------------------------------------------------------------------------
template <int EB>
struct ElemT;
template <>
struct ElemT<1> {
  using type = uint8_t;
};
template <>
struct ElemT<2> {
  using type = uint16_t;
};
template <>
struct ElemT<4> {
  using type = uint32_t;
};
template <>
struct ElemT<8> {
  using type = unsigned long long;
};
template <>
struct ElemT<16> {
  using type = uint4;
};

// Access word of AW bytes (1..16).
template <int AW>
struct WordT;
template <>
struct WordT<1> {
  using type = uint8_t;
};
template <>
struct WordT<2> {
  using type = uint16_t;
};
template <>
struct WordT<4> {
  using type = uint32_t;
};
template <>
struct WordT<8> {
  using type = uint2;
};
template <>
struct WordT<16> {
  using type = uint4;
};

// Packs AW/EB elements into one access word and back.
template <int AW, int EB>
struct Pack {
  using W = typename WordT<AW>::type;
  using E = typename ElemT<EB>::type;
  static constexpr int N = AW / EB;
  union U {
    W w;
    E e[N];
  };
};

}  // namespace t213
