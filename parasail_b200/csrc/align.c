/*
 * align.c -- the parasail.h alignment entry points of parasail-b200.
 *
 * Every entry point validates its arguments with the reference's checks and
 * messages (e.g. src/sw_striped_avx2_256_16.c:178-185), maps the target
 * through matrix->mapper, runs the pair on the GPU and builds a
 * parasail_result_t with the reference's flags and sentinel values:
 *
 *   profile forms  parasail_{alg}[_stats]_{striped,scan}_profile_{8,16,32,sat}
 *   direct forms   parasail_{alg}[_stats]_{striped,scan}_{8,16,32,sat}
 *                  (build a profile, align, free it: src/sw_striped_avx2_256_16.c:110-138)
 *   serial forms   parasail_{alg}[_stats], parasail_{alg}[_stats]_scan
 *                  (src/sw.c etc.: flags NOVEC / NOVEC_SCAN, 32-bit, 1 lane)
 *
 * The `_sat` chains try 8, then 16, then 32 bits (src/satcheck.c); the
 * verdict of each width comes from resolve.c. SW stats striped follows the
 * reference's two-pass FASTSTATS wrapper (src/sw_stats_striped_avx2_256_16.c:694-730).
 */
#include <stdlib.h>
#include <string.h>

#include "pb_internal.h"

int pb_gpu_ready(const char *func)
{
    if (pb_cuda_init() != 0) {
        fprintf(stderr, "%s: no usable CUDA device: %s\n", func, pb_cuda_last_error());
        return 0;
    }
    return 1;
}

static int alg_flag(int alg)
{
    return alg == PB_SW ? PARASAIL_FLAG_SW : alg == PB_NW ? PARASAIL_FLAG_NW : PARASAIL_FLAG_SG;
}

static int sg_bits(int alg, int sgflags)
{
    int f = 0;
    if (alg != PB_SG) return 0;
    if (sgflags & PB_S1_BEG) f |= PARASAIL_FLAG_SG_S1_BEG;
    if (sgflags & PB_S1_END) f |= PARASAIL_FLAG_SG_S1_END;
    if (sgflags & PB_S2_BEG) f |= PARASAIL_FLAG_SG_S2_BEG;
    if (sgflags & PB_S2_END) f |= PARASAIL_FLAG_SG_S2_END;
    return f;
}

/* Runs one pair. kernel 1 = the int16x2 Smith-Waterman score kernel, which
 * reruns out-of-range pairs on the exact kernel itself; 0 = exact kernel. */
static int run_pair(int kernel, const pb_device_profile *dp, const pb_mode *m, int stats,
                    int pad_rows, const uint8_t *codes, int tlen, int qlim, int tlim,
                    int scan_vgap, pb_pair_out *out)
{
    pb_batch b;
    const pb_device_profile *profs[1];
    int64_t off = 0;
    memset(&b, 0, sizeof b);
    profs[0] = dp;
    b.alg = m->alg; b.sgflags = m->sgflags; b.stats = stats;
    b.open = m->open; b.gap = m->gap; b.pad_rows = pad_rows;
    b.profs = profs; b.nprofs = 1;
    b.scan_vgap = scan_vgap;
    /* one pair: the single-pair paths (one upload, one launch, one
     * download); the batch pipeline for what they do not take */
    if (kernel == 1 && qlim <= 0 && tlim <= 0) {
        const int rc = pb_cuda_sw_single(dp, m->open, m->gap, codes, tlen, out);
        if (rc != -2) return rc;
    } else if (kernel == 0) {
        return pb_cuda_exact_single(&b, codes, tlen, qlim, tlim, out);
    }
    return pb_cuda_align_host(kernel, &b, codes, &off, &tlen, qlim > 0 ? &qlim : NULL,
                              tlim > 0 ? &tlim : NULL, NULL, 1, out);
}

parasail_result_t *pb_record_to_result(const pb_record *rec)
{
    const int stats = (rec->flag & PARASAIL_FLAG_STATS) != 0;
    parasail_result_t *r = pb_result_new(stats);
    if (!r) return NULL;
    r->score = rec->score;
    r->end_query = rec->end_query;
    r->end_ref = rec->end_ref;
    r->flag = rec->flag;
    if (stats) {
        r->stats->matches = rec->matches;
        r->stats->similar = rec->similar;
        r->stats->length = rec->length;
    }
    if (rec->ambig) pb_ambiguous_count += rec->ambig;
    return r;
}

/* One pair through the job's passes and the reference's width chain
 * (pb_chain_resolve). */
int pb_run_job_pair(const pb_device_profile *dp, const pb_job *job, const uint8_t *codes,
                    int tlen, pb_record *rec)
{
    const pb_mode *m = &job->mode;
    pb_pair_out o1, o2;
    const int score_only_sw = m->alg == PB_SW && (!m->stats || pb_job_is_faststats(job));
    const int pad = (job->bits < 0 || (m->alg == PB_SW && !m->stats)) ? 0
                  : (job->bits == 0 || job->bits == 8) ? 32 : job->bits == 16 ? 16 : 8;
    /* the serial scan forms at open < gap, where their vertical gap departs
     * from the serial DP's (with or without statistics) */
    const int scan_vgap = job->bits < 0 && (job->base_flags & PARASAIL_FLAG_NOVEC_SCAN) && m->open < m->gap;
    int rc;
    memset(&o2, 0, sizeof o2);
    if (score_only_sw && job->bits >= 0)
        rc = run_pair(1, dp, m, 0, 0, codes, tlen, 0, 0, 0, &o1);
    else
        rc = run_pair(0, dp, m, m->stats, pad, codes, tlen, 0, 0, scan_vgap, &o1);
    if (rc != 0) return rc;
    if (pb_needs_pass2(job, &o1)) {
        rc = run_pair(0, dp, m, 1, 32, codes, tlen, o1.end_query + 1, o1.end_ref + 1, 0, &o2);
        if (rc != 0) return rc;
    }
    {
        pb_lane_res e[3];
        int round;
        memset(e, 0, sizeof e);
        *rec = pb_chain_resolve(job, &o1, &o2, dp->qlen, tlen, &e[0], &e[1], &e[2]);
        /* striped widths the exact values do not give: the lane-exact
         * kernel of that width, then resolve again */
        for (round = 0; round < 3 && (rec->ambig == 8 || rec->ambig == 16 || rec->ambig == 32); ++round) {
            pb_lane_res *x = &e[rec->ambig == 8 ? 0 : rec->ambig == 16 ? 1 : 2];
            if (pb_cuda_lane_pair(rec->ambig, dp, &job->mode, codes, tlen, &o1, x) != 0) return -1;
            *rec = pb_chain_resolve(job, &o1, &o2, dp->qlen, tlen, &e[0], &e[1], &e[2]);
        }
        if (rec->ambig == 8 || rec->ambig == 16 || rec->ambig == 32) return -1;
    }
    return 0;
}

/* bits: 8/16/32, or 0 for the 8->16->32 chain. scheme_flag: STRIPED/SCAN. */
static parasail_result_t *align_vector(const pb_device_profile *dp, const pb_mode *m,
                                       const uint8_t *codes, int tlen, int bits,
                                       int scheme_flag)
{
    pb_job job;
    pb_record rec;
    job.mode = *m;
    job.bits = bits;
    job.base_flags = alg_flag(m->alg) | sg_bits(m->alg, m->sgflags) | scheme_flag;
    if (pb_run_job_pair(dp, &job, codes, tlen, &rec) != 0) {
        fprintf(stderr, "parasail-b200: GPU alignment failed: %s\n", pb_cuda_last_error());
        return NULL;
    }
    return pb_record_to_result(&rec);
}

static uint8_t *map_target(const parasail_matrix_t *matrix, const char *s2, int s2Len)
{
    int j;
    uint8_t *c = (uint8_t *)malloc((size_t)s2Len + 16);
    if (!c) return NULL;
    for (j = 0; j < s2Len; ++j) c[j] = (uint8_t)matrix->mapper[(unsigned char)s2[j]];
    return c;
}

/* Profile-form entry point body. */
static parasail_result_t *profile_entry(const char *func, const parasail_profile_t *profile,
                                        const char *s2, int s2Len, int open, int gap,
                                        int alg, int sgflags, int stats, int striped, int bits)
{
    const void *member;
    const pb_device_profile *dp;
    uint8_t *codes;
    parasail_result_t *r;
    pb_mode m;
    if (!profile) { fprintf(stderr, "%s: missing %s\n", func, "profile"); return NULL; }
    /* the first width that runs must have its profile (src/satcheck.c calls _8 first) */
    member = (bits == 16) ? profile->profile16.score
           : (bits == 32) ? profile->profile32.score : profile->profile8.score;
    if (!member) {
        fprintf(stderr, "%s: missing %s\n", func,
                bits == 16 ? "profile->profile16.score" : bits == 32 ? "profile->profile32.score"
                                                                     : "profile->profile8.score");
        return NULL;
    }
    if (stats) {
        const void *mm = (bits == 16) ? profile->profile16.matches
                       : (bits == 32) ? profile->profile32.matches : profile->profile8.matches;
        if (!mm) {
            fprintf(stderr, "%s: missing %s\n", func, "profile->profile.matches");
            return NULL;
        }
    }
    if (!profile->matrix) { fprintf(stderr, "%s: missing %s\n", func, "profile->matrix"); return NULL; }
    if (profile->s1Len <= 0) { fprintf(stderr, "%s: %s must be > 0\n", func, "profile->s1Len"); return NULL; }
    if (!s2) { fprintf(stderr, "%s: missing %s\n", func, "s2"); return NULL; }
    if (s2Len <= 0) { fprintf(stderr, "%s: %s must be > 0\n", func, "s2Len"); return NULL; }
    if (open < 0) { fprintf(stderr, "%s: %s must be >= 0\n", func, "open"); return NULL; }
    if (gap < 0) { fprintf(stderr, "%s: %s must be >= 0\n", func, "gap"); return NULL; }
    if (!pb_gpu_ready(func)) return NULL;
    dp = pb_profile_device(profile);
    codes = map_target(profile->matrix, s2, s2Len);
    if (!dp || !codes) { free(codes); return NULL; }
    m.alg = alg; m.sgflags = sgflags; m.stats = stats; m.striped = striped;
    m.open = open; m.gap = gap; m.mmax = profile->matrix->max; m.mmin = profile->matrix->min;
    r = align_vector(dp, &m, codes, s2Len, bits, striped ? PARASAIL_FLAG_STRIPED : PARASAIL_FLAG_SCAN);
    free(codes);
    return r;
}

/* Direct-form entry point: build a profile for the call, then as above. */
static parasail_result_t *direct_entry(const char *func, const char *s1, int s1Len,
                                       const char *s2, int s2Len, int open, int gap,
                                       const parasail_matrix_t *matrix, int alg, int sgflags,
                                       int stats, int striped, int bits)
{
    parasail_profile_t *profile;
    parasail_result_t *r;
    if (!s2) { fprintf(stderr, "%s: missing %s\n", func, "s2"); return NULL; }
    if (s2Len <= 0) { fprintf(stderr, "%s: %s must be > 0\n", func, "s2Len"); return NULL; }
    if (open < 0) { fprintf(stderr, "%s: %s must be >= 0\n", func, "open"); return NULL; }
    if (gap < 0) { fprintf(stderr, "%s: %s must be >= 0\n", func, "gap"); return NULL; }
    if (!matrix) { fprintf(stderr, "%s: missing %s\n", func, "matrix"); return NULL; }
    if (matrix->type == PARASAIL_MATRIX_TYPE_SQUARE) {
        if (!s1) { fprintf(stderr, "%s: missing %s\n", func, "s1"); return NULL; }
        if (s1Len <= 0) { fprintf(stderr, "%s: %s must be > 0\n", func, "s1Len"); return NULL; }
    }
    profile = pb_profile_create(s1, s1Len, matrix, 7, stats, 0);
    if (!profile) return NULL;
    r = profile_entry(func, profile, s2, s2Len, open, gap, alg, sgflags, stats, striped, bits);
    parasail_profile_free(profile);
    return r;
}

/* Serial-form entry point (reference src/sw.c etc.): exact 32-bit DP, flags
 * NOVEC or NOVEC_SCAN, BITS_INT, LANES_1. */
static parasail_result_t *serial_entry(const char *func, const char *s1, int s1Len,
                                       const char *s2, int s2Len, int open, int gap,
                                       const parasail_matrix_t *matrix, int alg, int sgflags,
                                       int stats, int scan)
{
    parasail_profile_t *profile;
    const pb_device_profile *dp;
    uint8_t *codes;
    pb_mode m;
    pb_job job;
    pb_record rec;
    int rc;
    if (!s2) { fprintf(stderr, "%s: missing %s\n", func, "_s2"); return NULL; }
    if (s2Len <= 0) { fprintf(stderr, "%s: %s must be > 0\n", func, "s2Len"); return NULL; }
    if (open < 0) { fprintf(stderr, "%s: %s must be >= 0\n", func, "open"); return NULL; }
    if (gap < 0) { fprintf(stderr, "%s: %s must be >= 0\n", func, "gap"); return NULL; }
    if (!matrix) { fprintf(stderr, "%s: missing %s\n", func, "matrix"); return NULL; }
    if (matrix->type == PARASAIL_MATRIX_TYPE_SQUARE || stats) {
        if (!s1) { fprintf(stderr, "%s: missing %s\n", func, "_s1"); return NULL; }
    }
    if (matrix->type == PARASAIL_MATRIX_TYPE_SQUARE && s1Len <= 0) {
        fprintf(stderr, "%s: %s must be > 0\n", func, "_s1Len");
        return NULL;
    }
    profile = pb_profile_create(s1, s1Len, matrix, 4, stats, 1);
    if (!profile) return NULL;
    dp = pb_profile_device(profile);
    codes = map_target(matrix, s2, s2Len);
    if (!codes) { parasail_profile_free(profile); return NULL; }
    m.alg = alg; m.sgflags = sgflags; m.stats = stats; m.striped = 0;
    m.open = open; m.gap = gap; m.mmax = matrix->max; m.mmin = matrix->min;
    job.mode = m;
    job.bits = -1;
    job.base_flags = alg_flag(alg) | sg_bits(alg, sgflags)
                   | (scan ? PARASAIL_FLAG_NOVEC_SCAN : PARASAIL_FLAG_NOVEC)
                   | PARASAIL_FLAG_BITS_32 | PARASAIL_FLAG_LANES_1;
    rc = pb_run_job_pair(dp, &job, codes, s2Len, &rec);
    free(codes);
    parasail_profile_free(profile);
    if (rc != 0) {
        fprintf(stderr, "%s: GPU alignment failed: %s\n", func, pb_cuda_last_error());
        return NULL;
    }
    return pb_record_to_result(&rec);
}

/* ---- generated entry points -------------------------------------------- */

#define PFN(name, alg, sgf, st, striped, bits)                                         \
    parasail_result_t *name(const parasail_profile_t *const restrict profile,          \
                            const char *const restrict s2, const int s2Len,            \
                            const int open, const int gap)                             \
    {                                                                                  \
        return profile_entry(#name, profile, s2, s2Len, open, gap, alg, sgf, st,       \
                             striped, bits);                                           \
    }

#define DFN(name, alg, sgf, st, striped, bits)                                         \
    parasail_result_t *name(const char *const restrict s1, const int s1Len,            \
                            const char *const restrict s2, const int s2Len,            \
                            const int open, const int gap,                             \
                            const parasail_matrix_t *matrix)                           \
    {                                                                                  \
        return direct_entry(#name, s1, s1Len, s2, s2Len, open, gap, matrix, alg, sgf,  \
                            st, striped, bits);                                        \
    }

#define SFN(name, alg, sgf, st, scan)                                                  \
    parasail_result_t *name(const char *const restrict s1, const int s1Len,            \
                            const char *const restrict s2, const int s2Len,            \
                            const int open, const int gap,                             \
                            const parasail_matrix_t *matrix)                           \
    {                                                                                  \
        return serial_entry(#name, s1, s1Len, s2, s2Len, open, gap, matrix, alg, sgf,  \
                            st, scan);                                                 \
    }

#define WIDTHS(P, D, base, alg, sgf, st, striped, scheme)                              \
    P(base##_##scheme##_profile_8, alg, sgf, st, striped, 8)                           \
    P(base##_##scheme##_profile_16, alg, sgf, st, striped, 16)                         \
    P(base##_##scheme##_profile_32, alg, sgf, st, striped, 32)                         \
    P(base##_##scheme##_profile_sat, alg, sgf, st, striped, 0)                         \
    D(base##_##scheme##_8, alg, sgf, st, striped, 8)                                   \
    D(base##_##scheme##_16, alg, sgf, st, striped, 16)                                 \
    D(base##_##scheme##_32, alg, sgf, st, striped, 32)                                 \
    D(base##_##scheme##_sat, alg, sgf, st, striped, 0)

#define FAMILY(base, alg, sgf, st)                                                     \
    SFN(base, alg, sgf, st, 0)                                                         \
    SFN(base##_scan, alg, sgf, st, 1)                                                  \
    WIDTHS(PFN, DFN, base, alg, sgf, st, 1, striped)                                   \
    WIDTHS(PFN, DFN, base, alg, sgf, st, 0, scan)

#define BOTH(name, alg, sgf)                                                           \
    FAMILY(name, alg, sgf, 0)                                                          \
    FAMILY(name##_stats, alg, sgf, 1)

/* semi-global cases: src/sg_helper.h:53-63 (s1_beg, s1_end, s2_beg, s2_end) */
BOTH(parasail_sw, PB_SW, 0)
BOTH(parasail_nw, PB_NW, 0)
BOTH(parasail_sg, PB_SG, PB_S1_BEG | PB_S1_END | PB_S2_BEG | PB_S2_END)
BOTH(parasail_sg_qb, PB_SG, PB_S1_BEG)
BOTH(parasail_sg_qe, PB_SG, PB_S1_END)
BOTH(parasail_sg_qx, PB_SG, PB_S1_BEG | PB_S1_END)
BOTH(parasail_sg_db, PB_SG, PB_S2_BEG)
BOTH(parasail_sg_de, PB_SG, PB_S2_END)
BOTH(parasail_sg_dx, PB_SG, PB_S2_BEG | PB_S2_END)
BOTH(parasail_sg_qb_de, PB_SG, PB_S1_BEG | PB_S2_END)
BOTH(parasail_sg_qe_db, PB_SG, PB_S1_END | PB_S2_BEG)
BOTH(parasail_sg_qb_db, PB_SG, PB_S1_BEG | PB_S2_BEG)
BOTH(parasail_sg_qe_de, PB_SG, PB_S1_END | PB_S2_END)
