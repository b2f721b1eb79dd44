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

/* Runs one pair through the exact kernel. */
static int run_pair(const pb_device_profile *dp, const pb_mode *m, int pad_rows,
                    const uint8_t *codes, int tlen, int qlim, int tlim, pb_pair_out *out)
{
    pb_batch b;
    const pb_device_profile *profs[1];
    int64_t off = 0;
    memset(&b, 0, sizeof b);
    profs[0] = dp;
    b.alg = m->alg; b.sgflags = m->sgflags; b.stats = m->stats;
    b.open = m->open; b.gap = m->gap; b.pad_rows = pad_rows;
    b.profs = profs; b.nprofs = 1;
    return pb_cuda_align_host(0, &b, codes, &off, &tlen, qlim > 0 ? &qlim : NULL,
                              tlim > 0 ? &tlim : NULL, NULL, 1, out);
}

static parasail_result_t *make_result(int flags, int stats, int score, int eq, int er,
                                      int matches, int similar, int length)
{
    parasail_result_t *r = pb_result_new(stats);
    if (!r) return NULL;
    r->score = score;
    r->end_query = eq;
    r->end_ref = er;
    r->flag = flags | (stats ? PARASAIL_FLAG_STATS : 0);
    if (stats) {
        r->stats->matches = matches;
        r->stats->similar = similar;
        r->stats->length = length;
    }
    return r;
}

/* Saturated values of the reference's kernels: biased SW striped kernels
 * report INT_MAX_w - INT_MIN_w (src/sw_striped_avx2_256_16.c:379-382, :412),
 * the 32-bit one INT32_MAX (src/sw_striped_avx2_256_32.c:356), all others 0
 * (src/nw_scan_avx2_256_16.c:386-392). */
static int sat_score_sw_striped(int bits)
{
    return bits == 8 ? 255 : bits == 16 ? 65535 : INT32_MAX;
}

/* bits: 8/16/32, or 0 for the 8->16->32 chain. scheme_flag: STRIPED/SCAN. */
static parasail_result_t *align_vector(const pb_device_profile *dp, const pb_mode *m,
                                       const uint8_t *codes, int tlen, int bits,
                                       int scheme_flag)
{
    static const int chain[3] = {8, 16, 32};
    const int first = bits == 0 ? 0 : (bits == 8 ? 0 : bits == 16 ? 1 : 2);
    const int last = bits == 0 ? 2 : first;
    const int qlen = dp->qlen;
    const int base = alg_flag(m->alg) | sg_bits(m->alg, m->sgflags) | scheme_flag;
    pb_pair_out o, o2;
    int t, have2 = 0;
    int v = PB_CLEAN;

    if (m->alg == PB_SW && m->stats && m->striped) {
        /* FASTSTATS: score pass, then a stats pass on the prefix */
        pb_mode m1 = *m;
        m1.stats = 0;
        if (run_pair(dp, &m1, 0, codes, tlen, 0, 0, &o) != 0) goto gpu_error;
        for (t = first; t <= last; ++t) {
            const int w = chain[t];
            const int fl = base | pb_flag_bits(w) | pb_flag_lanes(w);
            if (pb_resolve_faststats_pass1(m, w, &o) == PB_SAT) {
                if (t < last) continue;
                return make_result(fl | PARASAIL_FLAG_SATURATED, 0, sat_score_sw_striped(w), 0, 0, 0, 0, 0);
            }
            if (!have2) {
                if (run_pair(dp, m, 32, codes, tlen, o.end_query + 1, o.end_ref + 1, &o2) != 0) goto gpu_error;
                have2 = 1;
            }
            v = pb_resolve_tier(m, w, &o2, o.end_query + 1, o.end_ref + 1);
            if (v == PB_SAT) {
                if (t < last) continue;
                return make_result(fl | PARASAIL_FLAG_SATURATED, 1, 0, o.end_query, o.end_ref, 0, 0, 0);
            }
            return make_result(fl, 1, o.score, o.end_query, o.end_ref, o2.matches, o2.similar, o2.length);
        }
        return NULL;
    }

    {
        const int need_pad = !(m->alg == PB_SW && !m->stats);
        const int pad = need_pad ? (bits == 0 || bits == 8 ? 32 : bits == 16 ? 16 : 8) : 0;
        if (run_pair(dp, m, pad, codes, tlen, 0, 0, &o) != 0) goto gpu_error;
        for (t = first; t <= last; ++t) {
            const int w = chain[t];
            const int fl = base | pb_flag_bits(w) | pb_flag_lanes(w);
            v = pb_resolve_tier(m, w, &o, qlen, tlen);
            if (v == PB_SAT) {
                if (t < last) continue;
                if (m->alg == PB_SW && m->striped && !m->stats)
                    return make_result(fl | PARASAIL_FLAG_SATURATED, 0, sat_score_sw_striped(w), 0, 0, 0, 0, 0);
                return make_result(fl | PARASAIL_FLAG_SATURATED, m->stats, 0, 0, 0, 0, 0, 0);
            }
            return make_result(fl, m->stats, o.score, o.end_query, o.end_ref, o.matches, o.similar, o.length);
        }
    }
    return NULL;
gpu_error:
    fprintf(stderr, "parasail-b200: GPU alignment failed: %s\n", pb_cuda_last_error());
    return NULL;
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
    pb_pair_out o;
    pb_mode m;
    int flags;
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
    if (run_pair(dp, &m, 0, codes, s2Len, 0, 0, &o) != 0) {
        fprintf(stderr, "%s: GPU alignment failed: %s\n", func, pb_cuda_last_error());
        free(codes);
        parasail_profile_free(profile);
        return NULL;
    }
    free(codes);
    parasail_profile_free(profile);
    flags = alg_flag(alg) | sg_bits(alg, sgflags) | (scan ? PARASAIL_FLAG_NOVEC_SCAN : PARASAIL_FLAG_NOVEC)
          | PARASAIL_FLAG_BITS_32 | PARASAIL_FLAG_LANES_1;
    return make_result(flags, stats, o.score, o.end_query, o.end_ref, o.matches, o.similar, o.length);
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
