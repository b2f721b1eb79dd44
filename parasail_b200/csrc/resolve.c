/*
 * resolve.c -- host helpers around pb_resolve.h (flag bits of each width).
 */
#include "pb_internal.h"

volatile long pb_ambiguous_count = 0;

int pb_flag_bits(int bits)
{
    return bits == 8 ? PARASAIL_FLAG_BITS_8 : bits == 16 ? PARASAIL_FLAG_BITS_16 : PARASAIL_FLAG_BITS_32;
}

/* The AVX2 lane count of each width, which the reference reports. */
int pb_flag_lanes(int bits)
{
    return bits == 8 ? PARASAIL_FLAG_LANES_32 : bits == 16 ? PARASAIL_FLAG_LANES_16 : PARASAIL_FLAG_LANES_8;
}
