// Fixed device scratch used by xs_run_path_device_noalloc (see xs_noalloc.cu).
#pragma once
#include <cuda_runtime.h>

#define XS_NOALLOC_SCRATCH_DOUBLE2 (1u << 20) /* 16 MiB of complex FP64 */
#define XS_NOALLOC_MAX_DEVICES 64

cudaError_t xs_noalloc_scratch_address(void** out);
