// Adjoint of the explicit step (placeholder until the adjoint kernels land).
#include "ctx.h"

extern "C" {
ecg_status ecg_explicit_step_vjp_device(ecg_ctx*, const double*, double, const double*, double*) { return ECG_ERR_UNSUPPORTED; }
ecg_status ecg_explicit_step_device(ecg_ctx*, const double*, double, double*) { return ECG_ERR_UNSUPPORTED; }
}
