/*
 * profile.c -- query profiles (parasail_profile_create*, parasail_profile_free).
 *
 * The reference builds one striped SIMD profile per lane width
 * (src/memory_avx2.c:28-528) and stores it in profileN.score (plus
 * matches/similar planes for stats). Here every creator builds ONE
 * device-resident profile (pb_device_profile, built on the GPU by
 * k_build_profile) and every member the reference would set points to the
 * same refcounted handle, so parasail_profile_free's per-member calls to
 * profile->free (src/memory.c:698-746) release it exactly once.
 *
 * As in the reference, s1 and matrix are borrowed, not copied
 * (src/memory.c:660-696): callers keep them alive while the profile is used.
 */
#include <stdlib.h>
#include <string.h>

#include "pb_internal.h"

static void pb_profile_member_free(void *p)
{
    pb_host_profile *h = (pb_host_profile *)p;
    if (!h) return;
    if (--h->refs <= 0) {
        pb_cuda_profile_destroy(&h->dev);
        free(h);
    }
}

/* widths: bit0 8, bit1 16, bit2 32. serial_orientation: score(query letter,
 * target letter) = matrix[query][target] as the serial kernels read it
 * (src/sw.c:121-125); otherwise matrix[target][query] as the reference's
 * profile builders do (src/memory_avx2.c:113-116). */
parasail_profile_t *pb_profile_create(const char *s1, int s1Len,
                                      const parasail_matrix_t *matrix,
                                      int widths, int stats, int serial_orientation)
{
    parasail_profile_t *profile;
    pb_host_profile *h;
    uint8_t *codes;
    int *table = NULL;
    const int *tab;
    int qlen, size, i, k;

    PB_CHECK_NULL(matrix);
    if (matrix->type == PARASAIL_MATRIX_TYPE_SQUARE || stats) PB_CHECK_NULL(s1);
    qlen = matrix->type == PARASAIL_MATRIX_TYPE_SQUARE ? s1Len : matrix->length;
    PB_CHECK_GT0(qlen);
    if (!pb_gpu_ready(__func__)) return NULL;
    size = matrix->size;
    if (size > 255) {
        fprintf(stderr, "%s: alphabet of %d letters exceeds 255\n", __func__, size);
        return NULL;
    }
    codes = (uint8_t *)malloc((size_t)qlen);
    if (!codes) return NULL;
    for (i = 0; i < qlen; ++i)
        codes[i] = s1 ? (uint8_t)matrix->mapper[(unsigned char)s1[i]] : 0;
    if (matrix->type == PARASAIL_MATRIX_TYPE_PSSM) {
        /* row i, letter k: matrix[size*i + mapper[alphabet[k]]] (src/memory_avx2.c:118-120) */
        table = (int *)malloc(sizeof(int) * (size_t)qlen * size);
        if (!table) { free(codes); return NULL; }
        for (i = 0; i < qlen; ++i)
            for (k = 0; k < size; ++k)
                table[(size_t)i * size + k] =
                    matrix->matrix[(size_t)size * i + matrix->mapper[(unsigned char)matrix->alphabet[k]]];
        tab = table;
    } else if (serial_orientation) {
        table = (int *)malloc(sizeof(int) * (size_t)size * size);
        if (!table) { free(codes); return NULL; }
        for (k = 0; k < size; ++k)
            for (i = 0; i < size; ++i) table[(size_t)k * size + i] = matrix->matrix[(size_t)i * size + k];
        tab = table;
    } else {
        tab = matrix->matrix;
    }
    h = (pb_host_profile *)calloc(1, sizeof *h);
    profile = (parasail_profile_t *)calloc(1, sizeof *profile);
    if (!h || !profile) {
        free(h); free(profile); free(table); free(codes);
        return NULL;
    }
    if (pb_cuda_profile_create(tab, matrix->type == PARASAIL_MATRIX_TYPE_PSSM, size, codes, qlen,
                               matrix->max, matrix->min, &h->dev) != 0) {
        fprintf(stderr, "%s: %s\n", __func__, pb_cuda_last_error());
        free(h); free(profile); free(table); free(codes);
        return NULL;
    }
    free(table);
    free(codes);
    h->stats = stats;
    h->widths = widths;
    profile->s1 = s1;
    profile->s1Len = qlen;
    profile->matrix = matrix;
    profile->free = pb_profile_member_free;
    profile->stop = INT32_MAX;
#define SET_MEMBERS(bit, member)                                             \
    if (widths & (bit)) {                                                    \
        profile->member.score = h; h->refs++;                                \
        if (stats) {                                                         \
            profile->member.matches = h; profile->member.similar = h;        \
            h->refs += 2;                                                    \
        }                                                                    \
    }
    SET_MEMBERS(1, profile8)
    SET_MEMBERS(2, profile16)
    SET_MEMBERS(4, profile32)
#undef SET_MEMBERS
    return profile;
}

const pb_device_profile *pb_profile_device(const parasail_profile_t *profile)
{
    const pb_host_profile *h = NULL;
    if (profile->profile16.score) h = (const pb_host_profile *)profile->profile16.score;
    else if (profile->profile8.score) h = (const pb_host_profile *)profile->profile8.score;
    else if (profile->profile32.score) h = (const pb_host_profile *)profile->profile32.score;
    return h ? &h->dev : NULL;
}

void parasail_profile_free(parasail_profile_t *profile)
{
    if (!profile) {
        fprintf(stderr, "%s: attempted free of NULL profile pointer\n", __func__);
        return;
    }
#define FREE_MEMBER(member)                                           \
    if (profile->member.score) profile->free(profile->member.score);  \
    if (profile->member.matches) profile->free(profile->member.matches); \
    if (profile->member.similar) profile->free(profile->member.similar);
    FREE_MEMBER(profile8)
    FREE_MEMBER(profile16)
    FREE_MEMBER(profile32)
    FREE_MEMBER(profile64)
#undef FREE_MEMBER
    free(profile);
}

#define CREATOR(name, widths, stats)                                               \
    parasail_profile_t *name(const char *const restrict s1, const int s1Len,       \
                             const parasail_matrix_t *matrix)                      \
    {                                                                              \
        return pb_profile_create(s1, s1Len, matrix, widths, stats, 0);            \
    }

CREATOR(parasail_profile_create_8, 1, 0)
CREATOR(parasail_profile_create_16, 2, 0)
CREATOR(parasail_profile_create_32, 4, 0)
CREATOR(parasail_profile_create_sat, 7, 0)
CREATOR(parasail_profile_create_stats_8, 1, 1)
CREATOR(parasail_profile_create_stats_16, 2, 1)
CREATOR(parasail_profile_create_stats_32, 4, 1)
CREATOR(parasail_profile_create_stats_sat, 7, 1)
