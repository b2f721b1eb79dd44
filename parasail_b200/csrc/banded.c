/*
 * banded.c -- parasail_nw_banded (reference src/nw_banded.c:29-189).
 */
#include <stdlib.h>

#include "pb_internal.h"
#include "parasail_b200.h"

int pb_nw_banded_fits_wave(const parasail_matrix_t *matrix);

parasail_result_t *parasail_nw_banded(const char *const restrict s1, const int s1Len,
                                      const char *const restrict s2, const int s2Len,
                                      const int open, const int gap, const int k,
                                      const parasail_matrix_t *matrix)
{
    parasail_profile_t *profile;
    parasail_result_t *r;
    uint8_t *codes;
    int j, score = 0;
    PB_CHECK_NULL(s1);
    PB_CHECK_GT0(s1Len);
    PB_CHECK_NULL(s2);
    PB_CHECK_GT0(s2Len);
    PB_CHECK_GE0(open);
    PB_CHECK_GE0(gap);
    PB_CHECK_GT0(k);
    PB_CHECK_NULL(matrix);
    if (!pb_gpu_ready(__func__)) return NULL;
    if (pb_nw_banded_fits_wave(matrix)) {
        /* the band as diagonals on the wavefront kernel (pb_nwlong.cu) */
        const int64_t zero = 0;
        if (parasail_b200_nw_banded_batch(matrix, s1, &zero, &s1Len, s2, &zero, &s2Len, 1, open, gap, k, &score) != 0) {
            fprintf(stderr, "%s: GPU alignment failed\n", __func__);
            return NULL;
        }
        r = pb_result_new(0);
        if (!r) return NULL;
        r->score = score;
        r->end_query = s1Len - 1;
        r->end_ref = s2Len - 1;
        r->flag = PARASAIL_FLAG_NW | PARASAIL_FLAG_NOVEC | PARASAIL_FLAG_BANDED
                | PARASAIL_FLAG_BITS_32 | PARASAIL_FLAG_LANES_1;
        return r;
    }
    /* other matrices (PSSM, wider alphabets or scores): one pair on the
     * column recurrence of src/nw_banded.c */
    profile = pb_profile_create(s1, s1Len, matrix, 4, 0, 1);
    if (!profile) return NULL;
    codes = (uint8_t *)malloc((size_t)s2Len);
    if (!codes) { parasail_profile_free(profile); return NULL; }
    for (j = 0; j < s2Len; ++j) codes[j] = (uint8_t)matrix->mapper[(unsigned char)s2[j]];
    if (pb_cuda_nw_banded(pb_profile_device(profile), codes, s2Len, open, gap, k, &score) != 0) {
        fprintf(stderr, "%s: GPU alignment failed\n", __func__);
        free(codes);
        parasail_profile_free(profile);
        return NULL;
    }
    free(codes);
    parasail_profile_free(profile);
    r = pb_result_new(0);
    if (!r) return NULL;
    r->score = score;
    r->end_query = s1Len - 1;
    r->end_ref = s2Len - 1;
    /* src/nw_banded.c:74-76 */
    r->flag = PARASAIL_FLAG_NW | PARASAIL_FLAG_NOVEC | PARASAIL_FLAG_BANDED
            | PARASAIL_FLAG_BITS_32 | PARASAIL_FLAG_LANES_1;
    return r;
}
