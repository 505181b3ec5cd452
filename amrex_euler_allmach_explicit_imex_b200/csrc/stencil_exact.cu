// Stencil kernels built with -fmad=false: no FMA contraction, IEEE division
// and square root, the reference's operand order -> bit-identical to the
// reference CPU build (ECG_ARITH_EXACT).
#define ECG_NS ecg_exact
#include "stencil.cuh"

const EcgStencilOps ecg_exact_ops = {ecg_exact::launch_fv_step,   ecg_exact::launch_state_reduce,
                                     ecg_exact::launch_ghost_box, ecg_exact::launch_init_stats,
                                     ecg_exact::launch_init_state_stats, ecg_exact::launch_seed_stats,
                                     ecg_exact::launch_init_state};
