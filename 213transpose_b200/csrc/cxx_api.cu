// Reference-compatible C++ API (include/transpose.h, include/inplace_detail.h)
// over the C ABI.  Compiled into lib/libinplacett.a together with the library.
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>

#include "../../include/inplace_detail.h"
#include "../../include/t213.h"
#include "../../include/transpose.h"

namespace inplace {

namespace detail {

int t213_sync_default_stream() {
  cudaError_t e = cudaStreamSynchronize(0);
  return e == cudaSuccess ? T213_OK : T213_ERR_CUDA;
}

namespace c2r {
template <typename T>
void skinny_transpose(T *data, int d1, int d2, int d3) {  // src/skinny.cu:313-333
  t213_throw_on(t213_skinny_c2r_transpose(data, d1, d2, d3, (int)sizeof(T), 0), "inplace::detail::c2r::skinny_transpose");
  t213_throw_on(t213_sync_default_stream(), "inplace::detail::c2r::skinny_transpose");
}
}  // namespace c2r

namespace r2c {
template <typename T>
void skinny_transpose(T *data, int d1, int d2, int d3) {  // src/skinny.cu:344-363
  t213_throw_on(t213_skinny_r2c_transpose(data, d1, d2, d3, (int)sizeof(T), 0), "inplace::detail::r2c::skinny_transpose");
  t213_throw_on(t213_sync_default_stream(), "inplace::detail::r2c::skinny_transpose");
}
}  // namespace r2c

}  // namespace detail

namespace c2r {
template <typename T>
void transpose(T *data, int d1, int d2, int d3) {  // src/transpose.cu:30-47
  detail::t213_throw_on(t213_c2r_transpose(data, d1, d2, d3, (int)sizeof(T), 0), "inplace::c2r::transpose");
  detail::t213_throw_on(detail::t213_sync_default_stream(), "inplace::c2r::transpose");
}
}  // namespace c2r

namespace r2c {
template <typename T>
void transpose(T *data, int d1, int d2, int d3) {  // src/transpose.cu:70-89
  detail::t213_throw_on(t213_r2c_transpose(data, d1, d2, d3, (int)sizeof(T), 0), "inplace::r2c::transpose");
  detail::t213_throw_on(detail::t213_sync_default_stream(), "inplace::r2c::transpose");
}
}  // namespace r2c

template <typename T>
void transpose(T *data, int d1, int d2, int d3) {  // src/transpose.cu:99-124
  detail::t213_throw_on(t213_transpose(data, d1, d2, d3, (int)sizeof(T), 0), "inplace::transpose");
  detail::t213_throw_on(detail::t213_sync_default_stream(), "inplace::transpose");
}

#define T213_INSTANTIATE(T)                                              \
  template void transpose<T>(T *, int, int, int);                       \
  template void c2r::transpose<T>(T *, int, int, int);                  \
  template void r2c::transpose<T>(T *, int, int, int);                  \
  template void detail::c2r::skinny_transpose<T>(T *, int, int, int);   \
  template void detail::r2c::skinny_transpose<T>(T *, int, int, int);

T213_INSTANTIATE(int)
T213_INSTANTIATE(long long)
T213_INSTANTIATE(float)
T213_INSTANTIATE(double)
T213_INSTANTIATE(int4)
T213_INSTANTIATE(float4)
T213_INSTANTIATE(longlong2)
T213_INSTANTIATE(double2)

}  // namespace inplace
