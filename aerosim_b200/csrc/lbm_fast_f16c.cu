// FP32-arithmetic step kernels, StoreF16C storage (FP16 with mass-compensated rounding).
#define AEROSIM_FAST_STORE StoreF16C
#define AEROSIM_FAST_FN launch_step_fast_f16c
#define AEROSIM_BATCH_FN launch_batch_fast_f16c
#include "lbm_fast_impl.cuh"
