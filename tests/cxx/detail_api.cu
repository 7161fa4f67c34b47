// A caller of the reference's C++ interface, written against this project's
// headers exactly as it would be written against the reference's
// (include/transpose.h:3-19, include/rotate.h:6-7, include/shuffle.h:5-6,
// include/col_shuffle.h:8-9, include/permute.h:6-7, include/skinny.h:9-10,84-85,
// include/equations.h), and linked against lib/libinplacett.a.
//
// Test infrastructure: tests/test_cxx_api.py builds it with nvcc and runs it.
//
//   detail_api <call> <type> d1 d2 d3 in.bin out.bin [functor args...]
//
// reads d1*d2*d3 elements of <type> from in.bin into managed memory (what the
// reference requires), makes ONE call of the reference's interface and writes
// the result to out.bin.  For the detail calls the slice is m = d2 rows by
// n = d1 columns, as in the reference.
//
//   call:  transpose | c2r | r2c | skinny_c2r | skinny_r2c
//          rotate <functor> | shuffle <functor> | col_shuffle <functor>
//          | scatter_permute <functor>
//   type:  int | longlong | float | double | int4 | float4 | longlong2 | double2
//   functor (with its constructor's arguments): c2r_prerotator b,
//          c2r_postrotator m, r2c_prerotator m, r2c_postrotator b m,
//          c2r_shuffle m n c k, c2r_long_shuffle m n c k, r2c_shuffle m n c k,
//          c2r_fused_preop m b, c2r_fused_postop m n c, r2c_fused_preop a c m q,
//          r2c_fused_postop m b, c2r_scatter_postpermuter m n c,
//          r2c_scatter_prepermuter m n c
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>

#include "col_shuffle.h"
#include "equations.h"
#include "permute.h"
#include "rotate.h"
#include "shuffle.h"
#include "skinny.h"
#include "transpose.h"

namespace d = inplace::detail;

static int arg(char **argv, int argc, int i) {
  if (i >= argc) throw std::runtime_error("missing functor argument");
  return atoi(argv[i]);
}

template <typename T>
static void call(const std::string &what, T *data, int d1, int d2, int d3, int argc, char **argv) {
  if (what == "transpose") return inplace::transpose(data, d1, d2, d3);
  if (what == "c2r") return inplace::c2r::transpose(data, d1, d2, d3);
  if (what == "r2c") return inplace::r2c::transpose(data, d1, d2, d3);
  if (what == "skinny_c2r") return d::c2r::skinny_transpose(data, d1, d2, d3);
  if (what == "skinny_r2c") return d::r2c::skinny_transpose(data, d1, d2, d3);
  if (argc < 9) throw std::runtime_error("missing functor");
  const std::string f = argv[8];
  auto a = [&](int i) { return arg(argv, argc, 9 + i); };
  if (what == "rotate") {
    if (f == "c2r_prerotator") return d::rotate(d::c2r::prerotator(a(0)), d3, d2, d1, data);
    if (f == "c2r_postrotator") return d::rotate(d::c2r::postrotator(a(0)), d3, d2, d1, data);
    if (f == "r2c_prerotator") return d::rotate(d::r2c::prerotator(a(0)), d3, d2, d1, data);
    if (f == "r2c_postrotator") return d::rotate(d::r2c::postrotator(a(0), a(1)), d3, d2, d1, data);
  } else if (what == "shuffle") {
    if (f == "c2r_shuffle") return d::shuffle_fn(data, d3, d2, d1, d::c2r::shuffle(a(0), a(1), a(2), a(3)));
    if (f == "c2r_long_shuffle")
      return d::shuffle_fn(data, d3, d2, d1, d::c2r::long_shuffle(a(0), a(1), a(2), a(3)));
    if (f == "r2c_shuffle") return d::shuffle_fn(data, d3, d2, d1, d::r2c::shuffle(a(0), a(1), a(2), a(3)));
  } else if (what == "col_shuffle") {
    if (f == "c2r_fused_preop") return d::col_shuffle_fn(d::c2r::fused_preop(a(0), a(1)), d3, d2, d1, data);
    if (f == "c2r_fused_postop")
      return d::col_shuffle_fn(d::c2r::fused_postop(a(0), a(1), a(2)), d3, d2, d1, data);
    if (f == "r2c_fused_preop")
      return d::col_shuffle_fn(d::r2c::fused_preop(a(0), a(1), a(2), a(3)), d3, d2, d1, data);
    if (f == "r2c_fused_postop") return d::col_shuffle_fn(d::r2c::fused_postop(a(0), a(1)), d3, d2, d1, data);
  } else if (what == "scatter_permute") {
    if (f == "c2r_scatter_postpermuter")
      return d::scatter_permute(d::c2r::scatter_postpermuter(a(0), a(1), a(2)), d3, d2, d1, data);
    if (f == "r2c_scatter_prepermuter")
      return d::scatter_permute(d::r2c::scatter_prepermuter(a(0), a(1), a(2)), d3, d2, d1, data);
  }
  throw std::runtime_error("unknown call " + what + " " + f);
}

template <typename T>
static int run(const std::string &what, int d1, int d2, int d3, const char *in, const char *out, int argc,
               char **argv) {
  const size_t vol = (size_t)d1 * d2 * d3;
  T *data = nullptr;
  if (cudaMallocManaged(&data, vol * sizeof(T)) != cudaSuccess) return 3;
  FILE *fi = fopen(in, "rb");
  if (!fi || fread(data, sizeof(T), vol, fi) != vol) return 4;
  fclose(fi);
  try {
    call<T>(what, data, d1, d2, d3, argc, argv);
  } catch (const std::exception &e) {
    fprintf(stderr, "detail_api: %s\n", e.what());
    return 5;
  }
  FILE *fo = fopen(out, "wb");
  if (!fo || fwrite(data, sizeof(T), vol, fo) != vol) return 6;
  fclose(fo);
  cudaFree(data);
  return 0;
}

int main(int argc, char **argv) {
  if (argc < 8) {
    fprintf(stderr, "usage: detail_api <call> <type> d1 d2 d3 in.bin out.bin [functor args...]\n");
    return 2;
  }
  const std::string what = argv[1], type = argv[2];
  const int d1 = atoi(argv[3]), d2 = atoi(argv[4]), d3 = atoi(argv[5]);
  const char *in = argv[6], *out = argv[7];
  if (type == "int") return run<int>(what, d1, d2, d3, in, out, argc, argv);
  if (type == "longlong") return run<long long>(what, d1, d2, d3, in, out, argc, argv);
  if (type == "float") return run<float>(what, d1, d2, d3, in, out, argc, argv);
  if (type == "double") return run<double>(what, d1, d2, d3, in, out, argc, argv);
  if (type == "int4") return run<int4>(what, d1, d2, d3, in, out, argc, argv);
  if (type == "float4") return run<float4>(what, d1, d2, d3, in, out, argc, argv);
  if (type == "longlong2") return run<longlong2>(what, d1, d2, d3, in, out, argc, argv);
  if (type == "double2") return run<double2>(what, d1, d2, d3, in, out, argc, argv);
  fprintf(stderr, "detail_api: unknown type %s\n", type.c_str());
  return 2;
}
