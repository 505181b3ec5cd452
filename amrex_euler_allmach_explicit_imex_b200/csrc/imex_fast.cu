// IMEX stencil kernels built with -fmad=true (default arithmetic mode).
#include <string>
#define ECG_NS ecg_fast
#define ECG_IMEX_FAST_DIV 1
#include "imex_kernels.cuh"

const EcgImexOps ecg_imex_fast_ops = {ecg_fast::imex_star,     ecg_fast::imex_faces, ecg_fast::imex_matrix,
                                      ecg_fast::imex_closeout, ecg_fast::imex_eq78,  ecg_fast::imex_assemble,
                                      ecg_fast::imex_refresh};
