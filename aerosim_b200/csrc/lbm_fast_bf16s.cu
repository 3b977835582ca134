// FP32-arithmetic step kernels, StoreBF16S storage.
#define AEROSIM_FAST_STORE StoreBF16S
#define AEROSIM_FAST_FN launch_step_fast_bf16s
#define AEROSIM_BATCH_FN launch_batch_fast_bf16s
#include "lbm_fast_impl.cuh"
