// t213_transpose_host: end-to-end transpose of a tensor that lives in host
// memory.  Slices are grouped into chunks; chunk g+1 is copied in while chunk g
// is transposed and chunk g-1 is copied out, on three internal streams, so the
// two copy directions overlap each other and the kernels.
#include <algorithm>
#include <map>

#include "plan.h"

namespace t213 {
namespace {

struct HostIo {
  cudaStream_t s_in = nullptr, s_comp = nullptr, s_out = nullptr;
  char *buf = nullptr;
  size_t cap = 0;
  std::vector<cudaEvent_t> ev;
};

std::mutex g_mu;
std::map<int, HostIo> g_io;

int ensure(HostIo &io, size_t bytes, size_t n_events) {
  cudaError_t e;
  if (!io.s_in) {
    if ((e = cudaStreamCreateWithFlags(&io.s_in, cudaStreamNonBlocking)) ||
        (e = cudaStreamCreateWithFlags(&io.s_comp, cudaStreamNonBlocking)) ||
        (e = cudaStreamCreateWithFlags(&io.s_out, cudaStreamNonBlocking)))
      return cuda_status(e, "cudaStreamCreate");
  }
  if (io.cap < bytes) {
    if (io.buf) cudaFree(io.buf);
    io.buf = nullptr;
    io.cap = 0;
    if ((e = cudaMalloc(&io.buf, bytes))) return cuda_status(e, "staging cudaMalloc");
    io.cap = bytes;
  }
  while (io.ev.size() < n_events) {
    cudaEvent_t v;
    if ((e = cudaEventCreateWithFlags(&v, cudaEventDisableTiming))) return cuda_status(e, "cudaEventCreate");
    io.ev.push_back(v);
  }
  return T213_OK;
}

}  // namespace
}  // namespace t213

using namespace t213;

extern "C" int t213_transpose_host(void *host_data, int64_t d1, int64_t d2, int64_t d3, int32_t elem_bytes,
                                   t213_stream_t stream) {
  if (d1 < 0 || d2 < 0 || d3 < 0) {
    set_error("negative dimension");
    return T213_ERR_INVALID_ARGUMENT;
  }
  if (elem_bytes != 1 && elem_bytes != 2 && elem_bytes != 4 && elem_bytes != 8 && elem_bytes != 16) {
    set_error("element size must be 1, 2, 4, 8 or 16 bytes");
    return T213_ERR_UNSUPPORTED;
  }
  const int64_t slice = d1 * d2 * elem_bytes;
  const int64_t total = slice * d3;
  if (total == 0) return T213_OK;
  if (!host_data) {
    set_error("data is NULL");
    return T213_ERR_INVALID_ARGUMENT;
  }
  cudaStream_t user = (cudaStream_t)stream;
  const int64_t group = std::max<int64_t>(1, std::min<int64_t>(d3, ((int64_t)96 << 20) / std::max<int64_t>(1, slice)));
  const int64_t n_groups = (d3 + group - 1) / group;
  const int dev = dev_info().id;
  std::lock_guard<std::mutex> lk(g_mu);
  HostIo &io = g_io[dev];
  int rc = ensure(io, (size_t)total, (size_t)(2 * n_groups + 2));
  if (rc) return rc;
  cudaError_t e;
  // order after the caller's stream
  if ((e = cudaEventRecord(io.ev[0], user))) return cuda_status(e, "cudaEventRecord");
  cudaStreamWaitEvent(io.s_in, io.ev[0], 0);
  char *h = (char *)host_data;
  for (int64_t g = 0; g < n_groups; g++) {
    const int64_t k0 = g * group, nk = std::min<int64_t>(group, d3 - k0);
    const size_t off = (size_t)(k0 * slice), bytes = (size_t)(nk * slice);
    cudaEvent_t ein = io.ev[2 + 2 * g], ec = io.ev[3 + 2 * g];
    if ((e = cudaMemcpyAsync(io.buf + off, h + off, bytes, cudaMemcpyHostToDevice, io.s_in)))
      return cuda_status(e, "cudaMemcpyAsync H2D");
    cudaEventRecord(ein, io.s_in);
    cudaStreamWaitEvent(io.s_comp, ein, 0);
    std::shared_ptr<Plan> P = get_plan(d1, d2, nk, elem_bytes, T213_PLAN_AUTO, 0, &rc);
    if (!P) return rc;
    if ((rc = run_plan(*P, io.buf + off, io.s_comp, nullptr))) return rc;
    cudaEventRecord(ec, io.s_comp);
    cudaStreamWaitEvent(io.s_out, ec, 0);
    if ((e = cudaMemcpyAsync(h + off, io.buf + off, bytes, cudaMemcpyDeviceToHost, io.s_out)))
      return cuda_status(e, "cudaMemcpyAsync D2H");
  }
  cudaEventRecord(io.ev[1], io.s_out);
  cudaStreamWaitEvent(user, io.ev[1], 0);
  if ((e = cudaStreamSynchronize(io.s_out))) return cuda_status(e, "cudaStreamSynchronize");
  return T213_OK;
}
