// Stencil kernels built with -fmad=true (ECG_ARITH_FAST, the default): FMA
// contraction; within 1e-12 relative per step of the reference CPU build.
#define ECG_NS ecg_fast
#define ECG_FAST_KERNEL 1
#include "stencil.cuh"

const EcgStencilOps ecg_fast_ops = {ecg_fast::launch_fv_step,   ecg_fast::launch_state_reduce,
                                    ecg_fast::launch_ghost_box, ecg_fast::launch_init_stats,
                                    ecg_fast::launch_init_state_stats, ecg_fast::launch_seed_stats,
                                    ecg_fast::launch_init_state};
