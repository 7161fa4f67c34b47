// test_213inplace d1 d2 d3 type_size [outfile]
// Same arguments and output file as the reference's driver
// (src/test_213inplace.cu:66-90): fills managed memory with data[i] = i
// (int for type_size 4, long long otherwise), transposes it in place with
// inplace::transpose, prints the time and the effective bandwidth, and dumps
// the result as raw bytes.  The bandwidth printed here is 2*bytes/time (the
// reference multiplies by sizeof(T) once more).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <exception>

#include "transpose.h"

template <typename T>
static int run(int d1, int d2, int d3, FILE *fp) {
  size_t vol = (size_t)d1 * (size_t)d2 * (size_t)d3;
  size_t bytes = vol * sizeof(T);
  printf("Data size = %.5f GB\n", (double)bytes / 1e9);
  T *d = nullptr;
  if (cudaMallocManaged(&d, bytes) != cudaSuccess) {
    fprintf(stderr, "cudaMallocManaged failed\n");
    return 1;
  }
  for (size_t i = 0; i < vol; i++) d[i] = (T)i;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, 0);
  try {
    inplace::transpose(d, d1, d2, d3);
  } catch (const std::exception &e) {
    fprintf(stderr, "%s\n", e.what());
    return 1;
  }
  cudaDeviceSynchronize();
  cudaEventRecord(b, 0);
  cudaEventSynchronize(b);
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  printf("Execution Time: %.5fms\nEffective Bandwidth: %.5fGB/s\n", ms, (double)bytes * 2 / 1e6 / ms);
  if (fp) fwrite(d, sizeof(T), vol, fp);
  cudaFree(d);
  return 0;
}

int main(int argc, char **argv) {
  if (argc != 5 && argc != 6) {
    printf("Usage: [d1][d2][d3][Size of data type in byte][Output file]\nOutput file could be ignored\n");
    return 0;
  }
  int d1 = atoi(argv[1]), d2 = atoi(argv[2]), d3 = atoi(argv[3]), ts = atoi(argv[4]);
  FILE *fp = (argc == 6) ? fopen(argv[5], "wb") : nullptr;
  int rc = (ts == 4) ? run<int>(d1, d2, d3, fp) : run<long long>(d1, d2, d3, fp);
  if (fp) fclose(fp);
  return rc;
}
