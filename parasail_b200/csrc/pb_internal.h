/*
 * pb_internal.h -- declarations shared by the host C files of parasail-b200.
 */
#ifndef PARASAIL_B200_PB_INTERNAL_H
#define PARASAIL_B200_PB_INTERNAL_H

#include <stdio.h>
#include <stdint.h>

#include "parasail.h"
#include "pb_cuda.h"
#include "pb_resolve.h"

/* Validation macros with the reference's messages and return contract
 * (parasail/memory.h:46-80): print "<func>: ..." to stderr, return 0/NULL. */
#define PB_CHECK_NULL(var) do {                                  \
    if (!(var)) {                                                \
        fprintf(stderr, "%s: missing %s\n", __func__, #var);     \
        return 0;                                                \
    }                                                            \
} while (0)

#define PB_CHECK_GT0(var) do {                                   \
    if ((var) <= 0) {                                            \
        fprintf(stderr, "%s: %s must be > 0\n", __func__, #var); \
        return 0;                                                \
    }                                                            \
} while (0)

#define PB_CHECK_GE0(var) do {                                    \
    if ((var) < 0) {                                              \
        fprintf(stderr, "%s: %s must be >= 0\n", __func__, #var); \
        return 0;                                                 \
    }                                                             \
} while (0)

/* Host handle behind parasail_profile_t.profileN.{score,matches,similar}. */
typedef struct pb_host_profile {
    pb_device_profile dev;
    int refs;          /* members of the parasail_profile_t that point here */
    int stats;         /* built by a _stats creator */
    int widths;        /* bit 0: 8, bit 1: 16, bit 2: 32 */
} pb_host_profile;

/* result.c */
parasail_result_t *pb_result_new(int with_stats);

/* trace.c: releases the path of a trace result */
void pb_trace_free(parasail_result_t *r);

/* profile.c */
parasail_profile_t *pb_profile_create(const char *s1, int s1Len,
                                      const parasail_matrix_t *matrix,
                                      int widths, int stats, int serial_orientation);
const pb_device_profile *pb_profile_device(const parasail_profile_t *profile);

/* align.c */
int pb_gpu_ready(const char *func);
int pb_run_job_pair(const pb_device_profile *dp, const pb_job *job, const uint8_t *codes,
                    int tlen, pb_record *rec);
parasail_result_t *pb_record_to_result(const pb_record *rec);

/* tier resolution helpers (resolve.c) */
int pb_flag_lanes(int bits);
int pb_flag_bits(int bits);
extern volatile long pb_ambiguous_count;

#endif
