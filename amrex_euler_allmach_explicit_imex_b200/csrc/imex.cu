// IMEX T1/S2 BDLTV20 source-map step (placeholder until the IMEX kernels land).
#include "ctx.h"

struct EcgImexState {};

void imex_free(ecg_ctx* c)
{
  delete c->imex;
  c->imex = nullptr;
}

ecg_status imex_run(ecg_ctx*, int32_t, double, ecg_run_result*) { return ECG_ERR_UNSUPPORTED; }

extern "C" ecg_status ecg_imex_step(ecg_ctx* c, double, ecg_imex_diag*)
{
  if (!c) return ECG_ERR_BAD_ARG;
  return ECG_ERR_UNSUPPORTED;
}
