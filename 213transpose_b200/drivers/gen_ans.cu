// gen_ans d1 d2 d3 type_size [outfile]
// Same arguments and output as the reference's answer generator
// (src/gen_ans.cpp:21-43): the 213 transpose of data[i] = i as raw int
// (type_size 4) or long long (otherwise) bytes, to outfile or stdout.  Here the
// answer is computed on the GPU through t213_transpose_host.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "t213.h"

template <typename T>
static int gen(int d1, int d2, int d3, FILE *fp) {
  size_t vol = (size_t)d1 * (size_t)d2 * (size_t)d3;
  std::vector<T> h(vol);
  for (size_t i = 0; i < vol; i++) h[i] = (T)i;
  int rc = t213_transpose_host(h.data(), d1, d2, d3, (int)sizeof(T), nullptr);
  if (rc) {
    fprintf(stderr, "t213_transpose_host: %s: %s\n", t213_status_string(rc), t213_last_error());
    return 1;
  }
  fwrite(h.data(), sizeof(T), vol, fp);
  return 0;
}

int main(int argc, char **argv) {
  if (argc != 5 && argc != 6) {
    fprintf(stderr, "Usage: gen_ans d1 d2 d3 type_size [outfile]\n");
    return 1;
  }
  int d1 = atoi(argv[1]), d2 = atoi(argv[2]), d3 = atoi(argv[3]), ts = atoi(argv[4]);
  FILE *fp = (argc == 6) ? fopen(argv[5], "wb") : stdout;
  int rc = (ts == 4) ? gen<int>(d1, d2, d3, fp) : gen<long long>(d1, d2, d3, fp);
  if (fp != stdout) fclose(fp);
  return rc;
}
