// FP32-arithmetic step kernels, StoreF16S storage.
#define AEROSIM_FAST_STORE StoreF16S
#define AEROSIM_FAST_FN launch_step_fast_f16s
#define AEROSIM_BATCH_FN launch_batch_fast_f16s
#include "lbm_fast_impl.cuh"
