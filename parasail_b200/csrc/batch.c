/*
 * batch.c -- parasail-b200 batch API (include/parasail_b200.h).
 *
 * Parses the parasail function name into a job (algorithm, semi-global ends,
 * stats, striped/scan, width or the _sat chain), validates the arguments with
 * the reference's checks, and runs the device pipeline of pb_batch.cu.
 */
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#include "pb_internal.h"
#include "parasail_b200.h"

static const struct { const char *name; int alg, sgflags; } g_algs[] = {
    {"sw", PB_SW, 0}, {"nw", PB_NW, 0},
    {"sg_qb_de", PB_SG, PB_S1_BEG | PB_S2_END}, {"sg_qe_db", PB_SG, PB_S1_END | PB_S2_BEG},
    {"sg_qb_db", PB_SG, PB_S1_BEG | PB_S2_BEG}, {"sg_qe_de", PB_SG, PB_S1_END | PB_S2_END},
    {"sg_qb", PB_SG, PB_S1_BEG}, {"sg_qe", PB_SG, PB_S1_END},
    {"sg_qx", PB_SG, PB_S1_BEG | PB_S1_END}, {"sg_db", PB_SG, PB_S2_BEG},
    {"sg_de", PB_SG, PB_S2_END}, {"sg_dx", PB_SG, PB_S2_BEG | PB_S2_END},
    {"sg", PB_SG, PB_S1_BEG | PB_S1_END | PB_S2_BEG | PB_S2_END},
};

/* "[parasail_]ALG[_stats]_{striped,scan}[_profile]_{8,16,32,sat}" -> job.
 * want_profile: 1 profile form required, 0 direct form required, -1 either
 * (both forms of one function return the same results). */
static int parse_job(const char *funcname, int want_profile, int open, int gap,
                     const parasail_matrix_t *matrix, pb_job *job)
{
    const char *s = funcname;
    size_t k, n;
    int alg = -1, sgf = 0, stats = 0, striped = -1, bits = -1, prof = 0;
    if (!s) return -1;
    if (0 == strncmp(s, "parasail_", 9)) s += 9;
    for (k = 0; k < sizeof g_algs / sizeof g_algs[0]; ++k) {
        n = strlen(g_algs[k].name);
        if (0 == strncmp(s, g_algs[k].name, n) && s[n] == '_') {
            alg = g_algs[k].alg; sgf = g_algs[k].sgflags; s += n; break;
        }
    }
    if (alg < 0) return -1;
    if (0 == strncmp(s, "_stats", 6)) { stats = 1; s += 6; }
    if (0 == strncmp(s, "_striped", 8)) { striped = 1; s += 8; }
    else if (0 == strncmp(s, "_scan", 5)) { striped = 0; s += 5; }
    else return -1;
    if (0 == strncmp(s, "_profile", 8)) { prof = 1; s += 8; }
    if (0 == strcmp(s, "_8")) bits = 8;
    else if (0 == strcmp(s, "_16")) bits = 16;
    else if (0 == strcmp(s, "_32")) bits = 32;
    else if (0 == strcmp(s, "_sat")) bits = 0;
    else return -1;
    if (want_profile >= 0 && prof != want_profile) return -1;
    memset(job, 0, sizeof *job);
    job->mode.alg = alg; job->mode.sgflags = sgf; job->mode.stats = stats;
    job->mode.striped = striped; job->mode.open = open; job->mode.gap = gap;
    job->mode.mmax = matrix->max; job->mode.mmin = matrix->min;
    job->bits = bits;
    job->base_flags = (alg == PB_SW ? PARASAIL_FLAG_SW : alg == PB_NW ? PARASAIL_FLAG_NW : PARASAIL_FLAG_SG)
                    | (striped ? PARASAIL_FLAG_STRIPED : PARASAIL_FLAG_SCAN);
    if (alg == PB_SG) {
        if (sgf & PB_S1_BEG) job->base_flags |= PARASAIL_FLAG_SG_S1_BEG;
        if (sgf & PB_S1_END) job->base_flags |= PARASAIL_FLAG_SG_S1_END;
        if (sgf & PB_S2_BEG) job->base_flags |= PARASAIL_FLAG_SG_S2_BEG;
        if (sgf & PB_S2_END) job->base_flags |= PARASAIL_FLAG_SG_S2_END;
    }
    return 0;
}

static void mapper_bytes(const parasail_matrix_t *m, uint8_t *out)
{
    int c;
    for (c = 0; c < 256; ++c) out[c] = (uint8_t)m->mapper[c];
}

/* The device writes records in the public layout (the resolution leaves
 * the last field, reserved, at 0), so results are copied straight into the
 * caller's array. */
_Static_assert(sizeof(pb_record) == sizeof(parasail_b200_record_t), "record layout");
_Static_assert(offsetof(pb_record, score) == offsetof(parasail_b200_record_t, score), "record layout");
_Static_assert(offsetof(pb_record, end_query) == offsetof(parasail_b200_record_t, end_query), "record layout");
_Static_assert(offsetof(pb_record, end_ref) == offsetof(parasail_b200_record_t, end_ref), "record layout");
_Static_assert(offsetof(pb_record, flag) == offsetof(parasail_b200_record_t, flag), "record layout");
_Static_assert(offsetof(pb_record, matches) == offsetof(parasail_b200_record_t, matches), "record layout");
_Static_assert(offsetof(pb_record, similar) == offsetof(parasail_b200_record_t, similar), "record layout");
_Static_assert(offsetof(pb_record, length) == offsetof(parasail_b200_record_t, length), "record layout");
_Static_assert(offsetof(pb_record, ambig) == offsetof(parasail_b200_record_t, reserved), "record layout");

static int check_common(const char *func, const parasail_profile_t *profile, int n, int open, int gap)
{
    if (!profile) { fprintf(stderr, "%s: missing %s\n", func, "profile"); return -1; }
    if (!profile->matrix) { fprintf(stderr, "%s: missing %s\n", func, "profile->matrix"); return -1; }
    if (!pb_profile_device(profile)) { fprintf(stderr, "%s: missing %s\n", func, "profile->profile.score"); return -1; }
    if (n < 0) { fprintf(stderr, "%s: %s must be >= 0\n", func, "n"); return -1; }
    if (open < 0) { fprintf(stderr, "%s: %s must be >= 0\n", func, "open"); return -1; }
    if (gap < 0) { fprintf(stderr, "%s: %s must be >= 0\n", func, "gap"); return -1; }
    return 0;
}

int parasail_b200_batch_profile(const char *funcname, const parasail_profile_t *profile,
                                const char *targets, const int64_t *offsets, const int *lengths,
                                int n, int open, int gap, parasail_b200_record_t *records)
{
    pb_job job;
    pb_batch b;
    const pb_device_profile *profs[1];
    uint8_t map[256];
    int i, rc;
    if (check_common(__func__, profile, n, open, gap) != 0) return -1;
    if (n == 0) return 0;
    if (!targets || !offsets || !lengths || !records) { fprintf(stderr, "%s: missing arrays\n", __func__); return -1; }
    for (i = 0; i < n; ++i)
        if (lengths[i] <= 0) { fprintf(stderr, "%s: lengths[%d] must be > 0\n", __func__, i); return -1; }
    if (parse_job(funcname, 1, open, gap, profile->matrix, &job) != 0) {
        fprintf(stderr, "%s: unknown profile function '%s'\n", __func__, funcname ? funcname : "(null)");
        return -1;
    }
    if (!pb_gpu_ready(__func__)) return -1;
    memset(&b, 0, sizeof b);
    profs[0] = pb_profile_device(profile);
    b.alg = job.mode.alg; b.sgflags = job.mode.sgflags; b.stats = job.mode.stats;
    b.open = open; b.gap = gap; b.profs = profs; b.nprofs = 1; b.npairs = n;
    mapper_bytes(profile->matrix, map);
    rc = pb_cuda_batch_host(&job, &b, map, targets, offsets, lengths, NULL, NULL, NULL, n, (pb_record *)records);
    if (rc != 0) fprintf(stderr, "%s: GPU alignment failed: %s\n", __func__, pb_cuda_last_error());
    return rc;
}

int parasail_b200_batch_profile_device(const char *funcname, const parasail_profile_t *profile,
                                       const uint8_t *d_codes, const int64_t *d_offsets,
                                       const int *d_lengths, int n, int open, int gap,
                                       parasail_b200_record_t *d_records)
{
    pb_job job;
    pb_batch b;
    const pb_device_profile *profs[1];
    if (check_common(__func__, profile, n, open, gap) != 0) return -1;
    if (n == 0) return 0;
    if (!d_codes || !d_offsets || !d_lengths || !d_records) { fprintf(stderr, "%s: missing arrays\n", __func__); return -1; }
    if (parse_job(funcname, 1, open, gap, profile->matrix, &job) != 0) {
        fprintf(stderr, "%s: unknown profile function '%s'\n", __func__, funcname ? funcname : "(null)");
        return -1;
    }
    if (!pb_gpu_ready(__func__)) return -1;
    memset(&b, 0, sizeof b);
    profs[0] = pb_profile_device(profile);
    b.alg = job.mode.alg; b.sgflags = job.mode.sgflags; b.stats = job.mode.stats;
    b.open = open; b.gap = gap; b.profs = profs; b.nprofs = 1; b.npairs = n;
    b.d_targets = d_codes; b.d_toff = d_offsets; b.d_tlen = d_lengths;
    /* parasail_b200_record_t and pb_record share one layout of 8 ints */
    return pb_cuda_batch_run(&job, &b, (pb_record *)d_records);
}

int parasail_b200_batch_profile_device_noalloc(const char *funcname, const parasail_profile_t *profile,
                                               const uint8_t *d_codes, const int64_t *d_offsets,
                                               const int *d_lengths, int n, int open, int gap,
                                               parasail_b200_record_t *d_records)
{
    pb_job job;
    pb_batch b;
    const pb_device_profile *profs[1];
    if (check_common(__func__, profile, n, open, gap) != 0) return -1;
    if (n == 0) return 0;
    if (!d_codes || !d_offsets || !d_lengths || !d_records) { fprintf(stderr, "%s: missing arrays\n", __func__); return -1; }
    if (parse_job(funcname, 1, open, gap, profile->matrix, &job) != 0) {
        fprintf(stderr, "%s: unknown profile function '%s'\n", __func__, funcname ? funcname : "(null)");
        return -1;
    }
    if (pb_job_is_faststats(&job)) {
        fprintf(stderr, "%s: '%s' needs the two-pass statistics pipeline, which this entry point does not run\n",
                __func__, funcname);
        return -1;
    }
    if (n > pb_cuda_noalloc_max_pairs()) {
        fprintf(stderr, "%s: %d pairs exceed the limit of %d\n", __func__, n, pb_cuda_noalloc_max_pairs());
        return -1;
    }
    if (!pb_gpu_ready(__func__)) return -1;
    memset(&b, 0, sizeof b);
    profs[0] = pb_profile_device(profile);
    b.alg = job.mode.alg; b.sgflags = job.mode.sgflags; b.stats = job.mode.stats;
    b.open = open; b.gap = gap; b.profs = profs; b.nprofs = 1; b.npairs = n;
    /* padded rows of the width whose saturation checks the records carry
     * (serial forms and Smith-Waterman score-only need none) */
    b.pad_rows = (job.bits < 0 || (job.mode.alg == PB_SW && !job.mode.stats)) ? 0
               : (job.bits == 0 || job.bits == 8) ? 32 : job.bits == 16 ? 16 : 8;
    b.d_targets = d_codes; b.d_toff = d_offsets; b.d_tlen = d_lengths;
    if (pb_cuda_noalloc_run(&job, &b, (pb_record *)d_records) != 0) {
        fprintf(stderr, "%s: %s\n", __func__, pb_cuda_noalloc_last_error());
        return -1;
    }
    return 0;
}

size_t parasail_b200_noalloc_scratch_bytes(void) { return pb_cuda_noalloc_capacity(); }

int parasail_b200_batch_pairs(const char *funcname, const parasail_matrix_t *matrix,
                              const char *queries, const int64_t *qoffsets, const int *qlengths,
                              const char *targets, const int64_t *toffsets, const int *tlengths,
                              int n, int open, int gap, parasail_b200_record_t *records)
{
    pb_job job;
    pb_batch b;
    uint8_t map[256];
    int32_t *d_mat = NULL;
    int i, rc;
    if (!matrix) { fprintf(stderr, "%s: missing %s\n", __func__, "matrix"); return -1; }
    if (matrix->type != PARASAIL_MATRIX_TYPE_SQUARE) {
        fprintf(stderr, "%s: pairs batches need a square matrix\n", __func__);
        return -1;
    }
    if (n < 0 || open < 0 || gap < 0) { fprintf(stderr, "%s: invalid n/open/gap\n", __func__); return -1; }
    if (n == 0) return 0;
    if (!queries || !qoffsets || !qlengths || !targets || !toffsets || !tlengths || !records) {
        fprintf(stderr, "%s: missing arrays\n", __func__);
        return -1;
    }
    for (i = 0; i < n; ++i)
        if (qlengths[i] <= 0 || tlengths[i] <= 0) { fprintf(stderr, "%s: pair %d has an empty sequence\n", __func__, i); return -1; }
    if (parse_job(funcname, 0, open, gap, matrix, &job) != 0) {
        fprintf(stderr, "%s: unknown function '%s'\n", __func__, funcname ? funcname : "(null)");
        return -1;
    }
    if (!pb_gpu_ready(__func__)) return -1;
    d_mat = (int32_t *)pb_cuda_malloc(sizeof(int32_t) * (size_t)matrix->size * matrix->size);
    if (!d_mat) return -1;
    /* vector-kernel orientation: row = target letter (src/memory_avx2.c:113-116) */
    if (pb_cuda_h2d(d_mat, matrix->matrix, sizeof(int32_t) * (size_t)matrix->size * matrix->size) != 0) {
        pb_cuda_free(d_mat);
        return -1;
    }
    pb_cuda_sync();
    memset(&b, 0, sizeof b);
    b.alg = job.mode.alg; b.sgflags = job.mode.sgflags; b.stats = job.mode.stats;
    b.open = open; b.gap = gap; b.nprofs = 0; b.npairs = n;
    b.d_mat = d_mat; b.msize = matrix->size; b.mmax = matrix->max; b.mmin = matrix->min;
    mapper_bytes(matrix, map);
    rc = pb_cuda_batch_host(&job, &b, map, targets, toffsets, tlengths, queries, qoffsets, qlengths, n,
                            (pb_record *)records);
    if (rc != 0) fprintf(stderr, "%s: GPU alignment failed: %s\n", __func__, pb_cuda_last_error());
    pb_cuda_free(d_mat);
    pb_cuda_sync();
    return rc;
}

/* Database search: nq profiles x n targets in one pipeline (all queries of
 * a Smith-Waterman score batch share one kernel launch). records[q * n + i]. */
static int db_common(const char *func, const char *funcname, const parasail_profile_t *const *profiles,
                     int nq, int n, int open, int gap, pb_job *job, const pb_device_profile **profs)
{
    int q;
    if (!profiles || nq <= 0) { fprintf(stderr, "%s: missing %s\n", func, "profiles"); return -1; }
    for (q = 0; q < nq; ++q) {
        if (check_common(func, profiles[q], n, open, gap) != 0) return -1;
        if (profiles[q]->matrix != profiles[0]->matrix) {
            fprintf(stderr, "%s: all profiles must share one matrix\n", func);
            return -1;
        }
        profs[q] = pb_profile_device(profiles[q]);
    }
    if (parse_job(funcname, 1, open, gap, profiles[0]->matrix, job) != 0) {
        fprintf(stderr, "%s: unknown profile function '%s'\n", func, funcname ? funcname : "(null)");
        return -1;
    }
    return pb_gpu_ready(func) ? 0 : -1;
}

int parasail_b200_batch_db(const char *funcname, const parasail_profile_t *const *profiles, int nq,
                           const char *targets, const int64_t *offsets, const int *lengths, int n,
                           int open, int gap, parasail_b200_record_t *records)
{
    pb_job job;
    pb_batch b;
    const pb_device_profile **profs;
    uint8_t map[256];
    int i, rc;
    if (n == 0) return 0;
    if (!targets || !offsets || !lengths || !records) { fprintf(stderr, "%s: missing arrays\n", __func__); return -1; }
    for (i = 0; i < n; ++i)
        if (lengths[i] <= 0) { fprintf(stderr, "%s: lengths[%d] must be > 0\n", __func__, i); return -1; }
    profs = (const pb_device_profile **)malloc(sizeof(*profs) * (size_t)(nq > 0 ? nq : 1));
    if (!profs) return -1;
    if (db_common(__func__, funcname, profiles, nq, n, open, gap, &job, profs) != 0) { free(profs); return -1; }
    memset(&b, 0, sizeof b);
    b.alg = job.mode.alg; b.sgflags = job.mode.sgflags; b.stats = job.mode.stats;
    b.open = open; b.gap = gap; b.profs = profs; b.nprofs = nq; b.npairs = n;
    mapper_bytes(profiles[0]->matrix, map);
    rc = pb_cuda_batch_host(&job, &b, map, targets, offsets, lengths, NULL, NULL, NULL, n, (pb_record *)records);
    if (rc != 0) fprintf(stderr, "%s: GPU alignment failed: %s\n", __func__, pb_cuda_last_error());
    free(profs);
    return rc;
}

int parasail_b200_batch_db_device(const char *funcname, const parasail_profile_t *const *profiles, int nq,
                                  const uint8_t *d_codes, const int64_t *d_offsets, const int *d_lengths,
                                  int n, int open, int gap, parasail_b200_record_t *d_records)
{
    pb_job job;
    pb_batch b;
    const pb_device_profile **profs;
    int rc;
    if (n == 0) return 0;
    if (!d_codes || !d_offsets || !d_lengths || !d_records) { fprintf(stderr, "%s: missing arrays\n", __func__); return -1; }
    profs = (const pb_device_profile **)malloc(sizeof(*profs) * (size_t)(nq > 0 ? nq : 1));
    if (!profs) return -1;
    if (db_common(__func__, funcname, profiles, nq, n, open, gap, &job, profs) != 0) { free(profs); return -1; }
    memset(&b, 0, sizeof b);
    b.alg = job.mode.alg; b.sgflags = job.mode.sgflags; b.stats = job.mode.stats;
    b.open = open; b.gap = gap; b.profs = profs; b.nprofs = nq; b.npairs = n;
    b.d_targets = d_codes; b.d_toff = d_offsets; b.d_tlen = d_lengths;
    rc = pb_cuda_batch_run(&job, &b, (pb_record *)d_records);
    free(profs);
    return rc;
}

/* Matrix table on the device for the pairs and all-vs-all batches: vector
 * orientation, row = target letter (src/memory_avx2.c:113-116). */
static int32_t *matrix_to_device(const parasail_matrix_t *matrix)
{
    int32_t *d_mat = (int32_t *)pb_cuda_malloc(sizeof(int32_t) * (size_t)matrix->size * matrix->size);
    if (!d_mat) return NULL;
    if (pb_cuda_h2d(d_mat, matrix->matrix, sizeof(int32_t) * (size_t)matrix->size * matrix->size) != 0) {
        pb_cuda_free(d_mat);
        return NULL;
    }
    pb_cuda_sync();
    return d_mat;
}

static int check_square(const char *func, const parasail_matrix_t *matrix, int n, int open, int gap)
{
    if (!matrix) { fprintf(stderr, "%s: missing %s\n", func, "matrix"); return -1; }
    if (matrix->type != PARASAIL_MATRIX_TYPE_SQUARE) {
        fprintf(stderr, "%s: this batch needs a square matrix\n", func);
        return -1;
    }
    if (n < 0 || open < 0 || gap < 0) { fprintf(stderr, "%s: invalid n/open/gap\n", func); return -1; }
    return 0;
}

int parasail_b200_batch_pairs_device(const char *funcname, const parasail_matrix_t *matrix,
                                     const uint8_t *d_qcodes, const int64_t *d_qoffsets, const int *d_qlengths,
                                     const uint8_t *d_tcodes, const int64_t *d_toffsets, const int *d_tlengths,
                                     int n, int open, int gap, parasail_b200_record_t *d_records)
{
    pb_job job;
    pb_batch b;
    int32_t *d_mat;
    int rc;
    if (check_square(__func__, matrix, n, open, gap) != 0) return -1;
    if (n == 0) return 0;
    if (!d_qcodes || !d_qoffsets || !d_qlengths || !d_tcodes || !d_toffsets || !d_tlengths || !d_records) {
        fprintf(stderr, "%s: missing arrays\n", __func__);
        return -1;
    }
    if (parse_job(funcname, 0, open, gap, matrix, &job) != 0) {
        fprintf(stderr, "%s: unknown function '%s'\n", __func__, funcname ? funcname : "(null)");
        return -1;
    }
    if (!pb_gpu_ready(__func__)) return -1;
    if (!(d_mat = matrix_to_device(matrix))) return -1;
    memset(&b, 0, sizeof b);
    b.alg = job.mode.alg; b.sgflags = job.mode.sgflags; b.stats = job.mode.stats;
    b.open = open; b.gap = gap; b.nprofs = 0; b.npairs = n;
    b.d_mat = d_mat; b.msize = matrix->size; b.mmax = matrix->max; b.mmin = matrix->min;
    b.d_qall = d_qcodes; b.d_qoff = d_qoffsets; b.d_qlen = d_qlengths;
    b.d_targets = d_tcodes; b.d_toff = d_toffsets; b.d_tlen = d_tlengths;
    rc = pb_cuda_batch_run(&job, &b, (pb_record *)d_records);
    if (rc != 0) fprintf(stderr, "%s: GPU alignment failed: %s\n", __func__, pb_cuda_last_error());
    pb_cuda_free(d_mat);
    pb_cuda_sync();
    return rc;
}

/* All-vs-all: the upper triangle of n sequences, pair p = (i, j), i < j,
 * in row-major order, query i (the profile side) against target j. */
static int all_common(const char *func, const char *funcname, const parasail_matrix_t *matrix, int n,
                      int open, int gap, pb_job *job, pb_batch *b, int32_t **d_mat)
{
    if (check_square(func, matrix, n, open, gap) != 0) return -1;
    if ((long long)n * (n - 1) / 2 > 0x7fffffffLL) {
        fprintf(stderr, "%s: %d sequences give more than 2^31 - 1 pairs\n", func, n);
        return -1;
    }
    if (parse_job(funcname, -1, open, gap, matrix, job) != 0) {
        fprintf(stderr, "%s: unknown function '%s'\n", func, funcname ? funcname : "(null)");
        return -1;
    }
    if (!pb_gpu_ready(func)) return -1;
    if (!(*d_mat = matrix_to_device(matrix))) return -1;
    memset(b, 0, sizeof *b);
    b->alg = job->mode.alg; b->sgflags = job->mode.sgflags; b->stats = job->mode.stats;
    b->open = open; b->gap = gap; b->nprofs = 0;
    b->d_mat = *d_mat; b->msize = matrix->size; b->mmax = matrix->max; b->mmin = matrix->min;
    return 0;
}

int parasail_b200_batch_all(const char *funcname, const parasail_matrix_t *matrix,
                            const char *seqs, const int64_t *offsets, const int *lengths, int n,
                            int open, int gap, parasail_b200_record_t *records)
{
    pb_job job;
    pb_batch b;
    int32_t *d_mat = NULL;
    uint8_t map[256];
    int i, rc;
    if (n < 2) return 0;
    if (!seqs || !offsets || !lengths || !records) { fprintf(stderr, "%s: missing arrays\n", __func__); return -1; }
    for (i = 0; i < n; ++i)
        if (lengths[i] <= 0) { fprintf(stderr, "%s: lengths[%d] must be > 0\n", __func__, i); return -1; }
    if (all_common(__func__, funcname, matrix, n, open, gap, &job, &b, &d_mat) != 0) return -1;
    mapper_bytes(matrix, map);
    rc = pb_cuda_batch_all_host(&job, &b, map, seqs, offsets, lengths, n, (pb_record *)records);
    if (rc != 0) fprintf(stderr, "%s: GPU alignment failed: %s\n", __func__, pb_cuda_last_error());
    pb_cuda_free(d_mat);
    pb_cuda_sync();
    return rc;
}

int parasail_b200_batch_all_device(const char *funcname, const parasail_matrix_t *matrix,
                                   const uint8_t *d_codes, const int64_t *d_offsets, const int *d_lengths,
                                   int n, int open, int gap, parasail_b200_record_t *d_records)
{
    pb_job job;
    pb_batch b;
    int32_t *d_mat = NULL;
    int rc;
    if (n < 2) return 0;
    if (!d_codes || !d_offsets || !d_lengths || !d_records) { fprintf(stderr, "%s: missing arrays\n", __func__); return -1; }
    if (all_common(__func__, funcname, matrix, n, open, gap, &job, &b, &d_mat) != 0) return -1;
    rc = pb_cuda_batch_all(&job, &b, d_codes, d_offsets, d_lengths, n, (pb_record *)d_records);
    if (rc != 0) fprintf(stderr, "%s: GPU alignment failed: %s\n", __func__, pb_cuda_last_error());
    pb_cuda_free(d_mat);
    pb_cuda_sync();
    return rc;
}

/* ---- database-search plans ---------------------------------------------- */

struct parasail_b200_db_plan {
    void *plan;
    uint8_t *d_codes;       /* the caller's target buffer the plan reads */
    uint8_t mapper[256];    /* the profiles' matrix mapper, for runs from host memory */
};

parasail_b200_db_plan_t *parasail_b200_db_plan_create(const char *funcname, const parasail_profile_t *const *profiles,
                                                      int nq, const uint8_t *d_codes, const int64_t *d_offsets,
                                                      const int *d_lengths, int n, int open, int gap,
                                                      parasail_b200_record_t *d_records)
{
    pb_job job;
    pb_batch b;
    const pb_device_profile **profs;
    parasail_b200_db_plan_t *pl;
    if (n <= 0 || !d_codes || !d_offsets || !d_lengths || !d_records) {
        fprintf(stderr, "%s: missing arrays or n <= 0\n", __func__);
        return NULL;
    }
    profs = (const pb_device_profile **)malloc(sizeof(*profs) * (size_t)(nq > 0 ? nq : 1));
    pl = (parasail_b200_db_plan_t *)calloc(1, sizeof *pl);
    if (!profs || !pl) { free(profs); free(pl); return NULL; }
    if (db_common(__func__, funcname, profiles, nq, n, open, gap, &job, profs) != 0) {
        free(profs); free(pl); return NULL;
    }
    memset(&b, 0, sizeof b);
    b.alg = job.mode.alg; b.sgflags = job.mode.sgflags; b.stats = job.mode.stats;
    b.open = open; b.gap = gap; b.profs = profs; b.nprofs = nq; b.npairs = n;
    b.d_targets = d_codes; b.d_toff = d_offsets; b.d_tlen = d_lengths;
    pl->d_codes = (uint8_t *)d_codes;
    mapper_bytes(profiles[0]->matrix, pl->mapper);
    if (pb_cuda_db_plan_create(&job, &b, (pb_record *)d_records, &pl->plan) != 0) {
        fprintf(stderr, "%s: '%s' cannot be planned (plans hold Smith-Waterman score-only searches with "
                "open > gap and int8 profiles)\n", __func__, funcname ? funcname : "(null)");
        free(profs); free(pl); return NULL;
    }
    free(profs);
    return pl;
}

int parasail_b200_db_plan_run(parasail_b200_db_plan_t *plan)
{
    if (!plan) { fprintf(stderr, "%s: missing %s\n", __func__, "plan"); return -1; }
    return pb_cuda_db_plan_run(plan->plan);
}

int parasail_b200_db_plan_run_host(parasail_b200_db_plan_t *plan, const char *targets, size_t nbytes,
                                   parasail_b200_record_t *records)
{
    if (!plan || !records || (nbytes && !targets)) {
        fprintf(stderr, "%s: missing plan, targets or records\n", __func__);
        return -1;
    }
    return pb_cuda_db_plan_run_host(plan->plan, targets, nbytes, plan->d_codes, plan->mapper, (pb_record *)records);
}

void parasail_b200_db_plan_free(parasail_b200_db_plan_t *plan)
{
    if (!plan) return;
    pb_cuda_db_plan_free(plan->plan);
    free(plan);
}
