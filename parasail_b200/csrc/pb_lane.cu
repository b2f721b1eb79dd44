/*
 * pb_lane.cu -- lane-exact striped kernels (see pb_cuda.h).
 */
#include <cuda_runtime.h>
#include "pb_cuda.h"
