// gen_ans d1 d2 d3 type_size [outfile]
// The reference's answer generator (src/gen_ans.cpp:21-43), same arguments
// and output: the 213 transpose of data[i] = i (TensorUtil::init_data,
// src/tensor_util.cpp:42-47) as raw int (type_size 4) or long long
// (otherwise) values, to outfile or stdout.
//
// Like the reference's, this answer is computed on the host by an
// out-of-place gather (the semantics of TensorUtil::seq_tt,
// src/tensor_util.cpp:79-92), independently of the GPU library, so that
// `cmp` of test_213inplace's output with this file checks the GPU path
// against a separate computation.  The gather runs over 64 x 64 tiles of each
// slice instead of element by element.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

template <typename T>
static int gen(long long d1, long long d2, long long d3, FILE *fp) {
  const size_t vol = (size_t)d1 * (size_t)d2 * (size_t)d3;
  std::vector<T> out(vol);
  // input element (i1, i2, i3) is data[(i3 * d2 + i2) * d1 + i1] = that index;
  // it lands at (i3 * d1 + i1) * d2 + i2
  const long long B = 64;
  for (long long i3 = 0; i3 < d3; i3++)
    for (long long b2 = 0; b2 < d2; b2 += B)
      for (long long b1 = 0; b1 < d1; b1 += B) {
        const long long e2 = std::min(d2, b2 + B), e1 = std::min(d1, b1 + B);
        for (long long i1 = b1; i1 < e1; i1++)
          for (long long i2 = b2; i2 < e2; i2++)
            out[(size_t)((i3 * d1 + i1) * d2 + i2)] = (T)((i3 * d2 + i2) * d1 + i1);
      }
  return fwrite(out.data(), sizeof(T), vol, fp) == vol ? 0 : 1;
}

int main(int argc, char **argv) {
  if (argc != 5 && argc != 6) {
    fprintf(stderr, "Usage: gen_ans d1 d2 d3 type_size [outfile]\n");
    return 1;
  }
  const long long d1 = atoll(argv[1]), d2 = atoll(argv[2]), d3 = atoll(argv[3]);
  const int ts = atoi(argv[4]);
  if (d1 < 0 || d2 < 0 || d3 < 0) {
    fprintf(stderr, "gen_ans: negative dimension\n");
    return 1;
  }
  FILE *fp = (argc == 6) ? fopen(argv[5], "wb") : stdout;
  if (!fp) {
    perror("gen_ans");
    return 1;
  }
  const int rc = (ts == 4) ? gen<int>(d1, d2, d3, fp) : gen<long long>(d1, d2, d3, fp);
  if (fp != stdout) fclose(fp);
  return rc;
}
