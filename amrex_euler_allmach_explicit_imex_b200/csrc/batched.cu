// Batched independent explicit solves (placeholder until the batched kernels land).
#include <string>

#include "ctx.h"

struct ecg_batch {
  std::string err;
};

extern "C" {
ecg_status ecg_batch_create(ecg_batch** out, int32_t, const ecg_run_config*, const ecg_gpu_options*)
{
  if (out) *out = nullptr;
  return ECG_ERR_UNSUPPORTED;
}
void ecg_batch_destroy(ecg_batch* b) { delete b; }
ecg_status ecg_batch_upload(ecg_batch*, int32_t, const double*, int32_t, int32_t, int64_t, int64_t) { return ECG_ERR_UNSUPPORTED; }
ecg_status ecg_batch_download(ecg_batch*, int32_t, double*, int32_t, int32_t, int64_t, int64_t) { return ECG_ERR_UNSUPPORTED; }
ecg_status ecg_batch_run(ecg_batch*, int32_t, ecg_batch_result*) { return ECG_ERR_UNSUPPORTED; }
const char* ecg_batch_last_error(const ecg_batch* b) { return b ? b->err.c_str() : "null batch"; }
}
