// ORACLE SUPPORT — TEST INFRASTRUCTURE ONLY.
// C entry points around the reference's own GPU library (compiled unmodified
// from its sources by oracle/Makefile into oracle/_ref/libref_inplace.so), so
// GPU tests can compare this project's output with the reference's output on
// the shapes where the reference is correct and in bounds.
// The reference prefetches its argument as managed memory
// (src/transpose.cu:104), so callers must pass memory from ref_alloc_managed.
#include <cuda_runtime.h>
#include "transpose.h"

// type codes of ref_inplace_transpose_typed: the four instantiations of the
// reference's dispatcher (src/transpose.cu:126-129)
enum { REF_INT32 = 0, REF_FLOAT = 1, REF_INT64 = 2, REF_DOUBLE = 3 };

extern "C" int ref_inplace_transpose_typed(void *data, int d1, int d2, int d3, int code) {
  switch (code) {
    case REF_INT32: inplace::transpose(static_cast<int *>(data), d1, d2, d3); break;
    case REF_FLOAT: inplace::transpose(static_cast<float *>(data), d1, d2, d3); break;
    case REF_INT64: inplace::transpose(static_cast<long long *>(data), d1, d2, d3); break;
    case REF_DOUBLE: inplace::transpose(static_cast<double *>(data), d1, d2, d3); break;
    default: return -1;
  }
  cudaError_t e = cudaDeviceSynchronize();
  return e == cudaSuccess ? 0 : (int)e;
}

extern "C" int ref_inplace_transpose(void *data, int d1, int d2, int d3, int type_size) {
  if (type_size == 4) return ref_inplace_transpose_typed(data, d1, d2, d3, REF_INT32);
  if (type_size == 8) return ref_inplace_transpose_typed(data, d1, d2, d3, REF_INT64);
  return -1;
}

extern "C" void *ref_alloc_managed(size_t bytes) {
  void *p = nullptr;
  if (cudaMallocManaged(&p, bytes) != cudaSuccess) return nullptr;
  return p;
}

extern "C" int ref_free_managed(void *p) { return (int)cudaFree(p); }
