// Batched form (persistent executor) — first build: the looped baseline only.
#include "plan.h"

using namespace t213;

struct t213_batch_st {
  int dummy;
};

extern "C" {

int t213_transpose_looped(const t213_tensor_desc *tensors, int32_t count, t213_stream_t stream) {
  if (count < 0 || (count > 0 && !tensors)) return T213_ERR_INVALID_ARGUMENT;
  for (int32_t i = 0; i < count; i++) {
    const t213_tensor_desc &d = tensors[i];
    int rc = d.plan_kind == T213_PLAN_AUTO
                 ? t213_transpose(d.data, d.d1, d.d2, d.d3, d.elem_bytes, stream)
                 : t213_transpose_with_plan(d.data, d.d1, d.d2, d.d3, d.elem_bytes, d.plan_kind, 0, stream);
    if (rc) return rc;
  }
  return T213_OK;
}

int t213_batch_create(const t213_tensor_desc *, int32_t, t213_batch *) { return T213_ERR_UNSUPPORTED; }
int t213_batch_execute(t213_batch, t213_stream_t) { return T213_ERR_UNSUPPORTED; }
int t213_batch_status(t213_batch, t213_stream_t) { return T213_ERR_UNSUPPORTED; }
int t213_batch_describe(t213_batch, char *, size_t) { return T213_ERR_UNSUPPORTED; }
int t213_batch_destroy(t213_batch) { return T213_OK; }

}  // extern "C"
