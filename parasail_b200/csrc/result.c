/*
 * result.c -- parasail_result_t allocation, release and accessors, plus
 * parasail_version and parasail_time.
 *
 * Reference: src/memory.c:140-166 (new / new_stats), :277-327 (free),
 * :777-1028 (accessors), src/time.c:19-70 (timer).
 */
#include <stdlib.h>
#include <time.h>

#include "pb_internal.h"

parasail_result_t *pb_result_new(int with_stats)
{
    parasail_result_t *r = (parasail_result_t *)calloc(1, sizeof *r);
    if (!r) {
        fprintf(stderr, "%s: failed to malloc %zu bytes\n", __func__, sizeof *r);
        return NULL;
    }
    if (with_stats) {
        r->stats = (parasail_result_extra_stats_t *)calloc(1, sizeof *r->stats);
        if (!r->stats) {
            fprintf(stderr, "%s: failed to malloc %zu bytes\n", __func__, sizeof *r->stats);
            free(r);
            return NULL;
        }
    }
    return r;
}

void parasail_result_free(parasail_result_t *result)
{
    if (!result) {
        fprintf(stderr, "%s: attempted free of NULL result pointer\n", __func__);
        return;
    }
    if ((result->flag & PARASAIL_FLAG_STATS) && result->stats) free(result->stats);
    if (result->flag & PARASAIL_FLAG_TRACE) pb_trace_free(result);
    free(result);
}

void parasail_version(int *major, int *minor, int *patch)
{
    *major = PARASAIL_VERSION_MAJOR;
    *minor = PARASAIL_VERSION_MINOR;
    *patch = PARASAIL_VERSION_PATCH;
}

double parasail_time(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + (double)ts.tv_nsec * 1e-9;
}

#define FLAG_ACCESSOR(fn, expr)                                      \
    int fn(const parasail_result_t *const restrict result)           \
    {                                                                \
        PB_CHECK_NULL(result);                                       \
        return (expr);                                               \
    }

FLAG_ACCESSOR(parasail_result_is_nw, result->flag & PARASAIL_FLAG_NW)
FLAG_ACCESSOR(parasail_result_is_sg, result->flag & PARASAIL_FLAG_SG)
FLAG_ACCESSOR(parasail_result_is_sw, result->flag & PARASAIL_FLAG_SW)
FLAG_ACCESSOR(parasail_result_is_saturated, result->flag & PARASAIL_FLAG_SATURATED)
FLAG_ACCESSOR(parasail_result_is_banded, result->flag & PARASAIL_FLAG_BANDED)
FLAG_ACCESSOR(parasail_result_is_scan, result->flag & PARASAIL_FLAG_SCAN)
FLAG_ACCESSOR(parasail_result_is_striped, result->flag & PARASAIL_FLAG_STRIPED)
FLAG_ACCESSOR(parasail_result_is_diag, result->flag & PARASAIL_FLAG_DIAG)
FLAG_ACCESSOR(parasail_result_is_blocked, result->flag & PARASAIL_FLAG_BLOCKED)
FLAG_ACCESSOR(parasail_result_is_stats, result->flag & PARASAIL_FLAG_STATS)
FLAG_ACCESSOR(parasail_result_is_stats_table,
              (result->flag & PARASAIL_FLAG_STATS) && (result->flag & PARASAIL_FLAG_TABLE))
FLAG_ACCESSOR(parasail_result_is_stats_rowcol,
              (result->flag & PARASAIL_FLAG_STATS) && (result->flag & PARASAIL_FLAG_ROWCOL))
FLAG_ACCESSOR(parasail_result_is_table, result->flag & PARASAIL_FLAG_TABLE)
FLAG_ACCESSOR(parasail_result_is_rowcol, result->flag & PARASAIL_FLAG_ROWCOL)
FLAG_ACCESSOR(parasail_result_is_trace, result->flag & PARASAIL_FLAG_TRACE)
FLAG_ACCESSOR(parasail_result_get_score, result->score)
FLAG_ACCESSOR(parasail_result_get_end_query, result->end_query)
FLAG_ACCESSOR(parasail_result_get_end_ref, result->end_ref)

/* src/memory.c:885-905: stats accessors assert the STATS flag */
#define STATS_ACCESSOR(fn, field)                                               \
    int fn(const parasail_result_t *const restrict result)                      \
    {                                                                           \
        PB_CHECK_NULL(result);                                                  \
        if (!(result->flag & PARASAIL_FLAG_STATS)) {                            \
            fprintf(stderr, "%s: assert(%s) failed\n", __func__,                \
                    "parasail_result_is_stats(result)");                        \
            return 0;                                                           \
        }                                                                       \
        return result->stats->field;                                            \
    }

STATS_ACCESSOR(parasail_result_get_matches, matches)
STATS_ACCESSOR(parasail_result_get_similar, similar)
STATS_ACCESSOR(parasail_result_get_length, length)
