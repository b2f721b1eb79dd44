/*
 * filter.c -- parasail_b200_candidate_pairs: the candidate pairs of the
 * reference aligner's exact-match filter (apps/parasail_aligner.cpp:
 * 1316-1420, :1816-1904), computed on the GPU (pb_filter.cu).
 */
#include <stdlib.h>
#include <string.h>

#include "pb_internal.h"
#include "parasail_b200.h"

/* pair keys held on the device at once while the pairs are emitted */
#define PB_FILTER_BUDGET (1LL << 27)

int pb_cuda_candidate_pairs(const uint8_t *h_text, long long n, uint8_t sep, int cutoff, int cross,
                            long long budget, unsigned long long **h_pairs, long long *count);

int parasail_b200_candidate_pairs(const char *text, size_t size, char sentinel, int cutoff, long db_chars,
                                  int **pairs, size_t *count)
{
    unsigned long long *keys = NULL;
    long long n = 0, k;
    int cross = -1;
    size_t i;
    if (!text || !pairs || !count) {
        fprintf(stderr, "%s: missing text, pairs or count\n", __func__);
        return -1;
    }
    *pairs = NULL;
    *count = 0;
    if (cutoff < 1) {
        fprintf(stderr, "%s: cutoff must be > 0\n", __func__);
        return -1;
    }
    if (size == 0) return 0;
    if (text[size - 1] != sentinel) {
        fprintf(stderr, "%s: the text must end with the sentinel '%c'\n", __func__, sentinel);
        return -1;
    }
    if (size > 0x7fffffffULL) {
        fprintf(stderr, "%s: text of %zu characters is past 2^31 - 1\n", __func__, size);
        return -1;
    }
    if (db_chars >= 0) {
        /* a sequence belongs to the database when its sentinel lies in the
         * first db_chars characters (parasail_aligner.cpp:1231-1241) */
        cross = 0;
        for (i = 0; i < (size_t)db_chars && i < size; ++i) cross += text[i] == sentinel;
    }
    if (!pb_gpu_ready(__func__)) return -1;
    if (pb_cuda_candidate_pairs((const uint8_t *)text, (long long)size, (uint8_t)sentinel, cutoff, cross,
                                PB_FILTER_BUDGET, &keys, &n) != 0) {
        fprintf(stderr, "%s: CUDA failure\n", __func__);
        return -1;
    }
    *pairs = (int *)malloc(sizeof(int) * 2 * (size_t)(n ? n : 1));
    if (!*pairs) {
        free(keys);
        return -1;
    }
    for (k = 0; k < n; ++k) {
        (*pairs)[2 * k] = (int)(keys[k] >> 32);
        (*pairs)[2 * k + 1] = (int)(unsigned)keys[k];
    }
    free(keys);
    *count = (size_t)n;
    return 0;
}
