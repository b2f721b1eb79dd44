/*
 * pb_band.cu -- learned-band global alignment kernels (see pb_cuda.h).
 */
#include <cuda_runtime.h>
#include "pb_cuda.h"
