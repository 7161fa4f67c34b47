// ORACLE SUPPORT — TEST INFRASTRUCTURE ONLY.
// Exposes the reference's own CPU answer generator, TensorUtil<T>::seq_tt
// (src/tensor_util.cpp:79-92, compiled from the reference's sources by
// oracle/Makefile into oracle/_ref/), through a C entry point for ctypes.
// 4-byte elements use TensorUtil<int>, 8-byte ones TensorUtil<long long>,
// exactly as the reference's drivers do (src/gen_ans.cpp:29-38); the gather
// copies whole elements, so the bytes of any 4- or 8-byte type move unchanged.
#include <cstdio>
#include "tensor_util.h"

extern "C" int ref_seq_tt(void *ans, void *data, int d1, int d2, int d3, int type_size) {
  int dim[3] = {d1, d2, d3};
  int perm[3] = {1, 0, 2};
  if (type_size == 4) {
    TensorUtil<int> tu(nullptr, 3, dim, perm);
    tu.seq_tt(static_cast<int *>(ans), static_cast<int *>(data));
  } else if (type_size == 8) {
    TensorUtil<long long> tu(nullptr, 3, dim, perm);
    tu.seq_tt(static_cast<long long *>(ans), static_cast<long long *>(data));
  } else {
    return -1;
  }
  return 0;
}

// The reference's known-answer input (src/tensor_util.cpp:42-47).
extern "C" int ref_init_data(void *data, int d1, int d2, int d3, int type_size) {
  int dim[3] = {d1, d2, d3};
  int perm[3] = {1, 0, 2};
  if (type_size == 4) {
    TensorUtil<int> tu(nullptr, 3, dim, perm);
    tu.init_data(static_cast<int *>(data));
  } else if (type_size == 8) {
    TensorUtil<long long> tu(nullptr, 3, dim, perm);
    tu.init_data(static_cast<long long *>(data));
  } else {
    return -1;
  }
  return 0;
}
