// FP32-arithmetic step kernels, StoreF32S storage (FP32 deviations).
#define AEROSIM_FAST_STORE StoreF32S
#define AEROSIM_FAST_FN launch_step_fast_f32
#define AEROSIM_BATCH_FN launch_batch_fast_f32
#include "lbm_fast_impl.cuh"
