// ORACLE SUPPORT — TEST INFRASTRUCTURE ONLY.
// C entry points around the reference's own GPU library (compiled unmodified
// from its sources by oracle/Makefile into oracle/_ref/libref_inplace.so), so
// GPU tests can compare this project's output with the reference's output on
// the shapes where the reference is correct and in bounds.
// The reference prefetches its argument as managed memory
// (src/transpose.cu:104), so callers must pass memory from ref_alloc_managed.
#include <cuda_runtime.h>
#include "transpose.h"

extern "C" int ref_inplace_transpose(void *data, int d1, int d2, int d3, int type_size) {
  if (type_size == 4)
    inplace::transpose(static_cast<int *>(data), d1, d2, d3);
  else if (type_size == 8)
    inplace::transpose(static_cast<long long *>(data), d1, d2, d3);
  else
    return -1;
  cudaError_t e = cudaDeviceSynchronize();
  return e == cudaSuccess ? 0 : (int)e;
}

extern "C" void *ref_alloc_managed(size_t bytes) {
  void *p = nullptr;
  if (cudaMallocManaged(&p, bytes) != cudaSuccess) return nullptr;
  return p;
}

extern "C" int ref_free_managed(void *p) { return (int)cudaFree(p); }
