// t213_row_shuffle_noalloc (include/t213_noalloc.h): the row shuffle staged
// through a fixed file-scope device array instead of an allocated workspace.
//
// Rows are copied group by group (as many whole rows as fit the scratch) with
// one device-to-device copy, then k_row_gather_staged gathers each row of the
// group back from the copy: new[i][j] = old[i][fn(i, j)].  The copy and the
// kernel are stream-ordered, so the next group's copy cannot overwrite the
// scratch before the previous gather has read it.
//
// No device memory is allocated by a call: the scratch lives in this file's
// module, whose 32 MiB the CUDA driver reserves on a device when it loads the
// module there.  With CUDA's default lazy module loading that happens at the
// first use on the device -- in set-up, where the scratch address is looked
// up -- so the first call on a device (an empty call is enough) must come
// before the caller's own allocator has filled the device.  After that the
// launch needs no dynamic shared memory and no cached occupancy query.
#include <mutex>

#include "../../include/t213_noalloc.h"
#include "internal.h"
#include "k_gather.cuh"

namespace t213 {
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[T213_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;

struct NoallocDevice {
  bool ready = false;
  char *scratch = nullptr;
  int sms = 0;
};

std::mutex g_setup_mu;
NoallocDevice g_dev[kMaxDevices];

// First call on a device: the scratch address and the SM count.
int setup(int dev, NoallocDevice **out) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  NoallocDevice &d = g_dev[dev];
  if (!d.ready) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(no-alloc scratch)");
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_status(e, "cudaDeviceGetAttribute");
    d.scratch = static_cast<char *>(p);
    d.sms = sms;
    d.ready = true;
  }
  *out = &d;
  return T213_OK;
}

// One group of rows gathered back from its copy in the scratch: thread t
// takes word t of the group (row t / words_per_row), so short rows keep the
// whole grid busy too.  The scratch copy is at most 32 MiB and stays in L2.
template <int EB, int AW, typename F, typename U>
__global__ void __launch_bounds__(kGatherThreads)
    k_row_gather_staged(char *__restrict__ data, const char *__restrict__ scratch, int64_t row0, uint32_t n_words,
                        U n, FastDiv<uint32_t> words_per_row, FastDiv<uint64_t> mdiv, F fn) {
  using E = typename ElemT<EB>::type;
  using W = typename WordT<AW>::type;
  using P = Pack<AW, EB>;
  constexpr int PER = AW / EB;
  const E *src = reinterpret_cast<const E *>(scratch);
  W *dst = reinterpret_cast<W *>(data + row0 * (int64_t)n * EB);
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n_words; t += gridDim.x * blockDim.x) {
    const uint32_t r = words_per_row.div(t);
    const U j0 = (U)(t - r * words_per_row.get()) * PER;
    const U i = (U)mdiv.mod((uint64_t)(row0 + r));
    const E *srow = src + (int64_t)r * n;
    typename P::U pk;
#pragma unroll
    for (int e = 0; e < PER; e++) pk.e[e] = __ldcg(srow + fn(i, j0 + e));
    __stcs(dst + t, pk.w);
  }
}

template <typename U, typename Fn>
bool with_row_shuffle(const FnSpec &f, Fn &&fn) {
  switch (f.kind) {
    case T213_FN_C2R_SHUFFLE:
    case T213_FN_C2R_LONG_SHUFFLE:
      return fn(RowC2RShuffle<U>(f.p[0], f.p[1], f.p[2], f.p[3]));
    case T213_FN_R2C_SHUFFLE:
      return fn(RowR2CShuffle<U>(f.p[0], f.p[1], f.p[2]));
  }
  return false;
}

}  // namespace
}  // namespace t213

using namespace t213;

extern "C" int t213_row_shuffle_noalloc(int32_t fn_kind, const int64_t *fn_params, int32_t n_params, void *data,
                                        int64_t d3, int64_t d2, int64_t d1, int32_t eb, t213_stream_t stream) {
  if (d1 < 0 || d2 < 0 || d3 < 0) {
    set_error("negative dimension");
    return T213_ERR_INVALID_ARGUMENT;
  }
  if (eb != 1 && eb != 2 && eb != 4 && eb != 8 && eb != 16) {
    set_error("element size must be 1, 2, 4, 8 or 16 bytes");
    return T213_ERR_UNSUPPORTED;
  }
  if (n_params < 0 || n_params > 4 || (n_params > 0 && !fn_params)) {
    set_error("functor parameters: 0..4 values");
    return T213_ERR_INVALID_ARGUMENT;
  }
  if (fn_kind != T213_FN_C2R_SHUFFLE && fn_kind != T213_FN_C2R_LONG_SHUFFLE && fn_kind != T213_FN_R2C_SHUFFLE) {
    set_error("functor kind is not a row shuffler");
    return T213_ERR_INVALID_ARGUMENT;
  }
  FnSpec f;
  f.kind = fn_kind;
  for (int q = 0; q < n_params; q++) f.p[q] = fn_params[q];
  const int64_t m = d2, n = d1;
  if (f.p[0] != m || f.p[1] != n || f.p[2] <= 0 || f.p[3] < 0) {
    set_error("row shuffler parameters must be (m=d2, n=d1, c>0, k)");
    return T213_ERR_INVALID_ARGUMENT;
  }
  const int64_t row_bytes = n * eb;
  if (row_bytes > T213_NOALLOC_SCRATCH_BYTES) {
    set_error("a row is longer than the 32 MiB no-alloc scratch (d1 * elem_bytes > T213_NOALLOC_SCRATCH_BYTES)");
    return T213_ERR_UNSUPPORTED;
  }
  // set-up first, so that an empty call reserves the scratch on this device
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("device ordinal out of range for the no-alloc scratch table");
    return T213_ERR_UNSUPPORTED;
  }
  NoallocDevice *D = nullptr;
  int rc = setup(dev, &D);
  if (rc) return rc;
  if (d1 == 0 || d2 == 0 || d3 == 0) return T213_OK;
  if (!data) {
    set_error("data is NULL");
    return T213_ERR_INVALID_ARGUMENT;
  }
  if (((uintptr_t)data) % (uintptr_t)std::min(eb, 16)) {
    set_error("data is not aligned to its element size");
    return T213_ERR_INVALID_ARGUMENT;
  }

  cudaStream_t st = (cudaStream_t)stream;
  const int aw = (eb >= 16 || (eb >= 4 && (((uintptr_t)data | (uint64_t)row_bytes) & 15) == 0)) ? 16 : eb;
  const int64_t total_rows = d3 * m;
  const int64_t group_rows = std::max<int64_t>(1, T213_NOALLOC_SCRATCH_BYTES / row_bytes);
  const bool u32 = fits32(f, m, n);
  int status = T213_OK;
  bool known = false;
  auto run = [&](auto EBc, auto AWc) -> bool {
    constexpr int EB = decltype(EBc)::value;
    constexpr int AW = decltype(AWc)::value;
    constexpr int PER = AW / EB;
    auto go = [&](auto UT) -> bool {
      using U = decltype(UT);
      return with_row_shuffle<U>(f, [&](auto fn) -> bool {
        using F = decltype(fn);
        known = true;
        const int64_t words = n / PER;
        const FastDiv<uint32_t> wpr((uint64_t)words);
        const FastDiv<uint64_t> md((uint64_t)m);
        for (int64_t r0 = 0; r0 < total_rows; r0 += group_rows) {
          const int64_t nr = std::min<int64_t>(group_rows, total_rows - r0);
          cudaError_t ce = cudaMemcpyAsync(D->scratch, (char *)data + r0 * row_bytes, (size_t)(nr * row_bytes),
                                           cudaMemcpyDeviceToDevice, st);
          if (ce != cudaSuccess) {
            status = cuda_status(ce, "cudaMemcpyAsync (no-alloc scratch)");
            return true;
          }
          const int64_t n_words = nr * words;  // below 2^25: the group fits 32 MiB
          const unsigned grid = (unsigned)std::max<int64_t>(
              1, std::min<int64_t>((int64_t)D->sms * 8, (n_words + kGatherThreads - 1) / kGatherThreads));
          k_row_gather_staged<EB, AW, F, U><<<grid, kGatherThreads, 0, st>>>(
              (char *)data, (const char *)D->scratch, r0, (uint32_t)n_words, (U)n, wpr, md, fn);
          ce = cudaGetLastError();
          if (ce != cudaSuccess) {
            status = cuda_status(ce, "k_row_gather_staged launch");
            return true;
          }
        }
        return true;
      });
    };
    return u32 ? go(uint32_t{}) : go(uint64_t{});
  };
  if (!dispatch_eb_aw(eb, aw, run) || !known) {
    set_error("unsupported element size or functor");
    return T213_ERR_UNSUPPORTED;
  }
  return status;
}
