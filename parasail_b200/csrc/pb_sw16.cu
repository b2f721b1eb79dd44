/*
 * pb_sw16.cu -- fast Smith-Waterman score-only kernel (int16x2 lanes).
 */
#include <cstdio>
#include <cuda_runtime.h>

#include "pb_cuda.h"
#include "pb_kernels.cuh"

extern "C" int pb_cuda_align_sw16(const pb_batch *b)
{
    (void)b;
    return -1;
}
