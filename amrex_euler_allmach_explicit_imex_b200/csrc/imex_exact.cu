// IMEX stencil kernels built with -fmad=false (bit-identical arithmetic mode).
#include <string>
#define ECG_NS ecg_exact
#include "imex_kernels.cuh"

const EcgImexOps ecg_imex_exact_ops = {ecg_exact::imex_star,     ecg_exact::imex_faces, ecg_exact::imex_matrix,
                                      ecg_exact::imex_closeout, ecg_exact::imex_eq78,  ecg_exact::imex_assemble,
                                      ecg_exact::imex_refresh};
