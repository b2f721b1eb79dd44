/*
 * ref_driver.c -- CPU baseline and per-pair parity source: runs the
 * reference's own AVX2 striped/scan profile functions
 * (oracle/_ref/libparasail_ref.so) with OpenMP across pairs, the pattern of
 * the reference's tests/test_openmp.c:353-378 and
 * apps/parasail_aligner.cpp:1606-1622 (one profile per query, guided
 * schedule over pairs). TEST/BASELINE INFRASTRUCTURE ONLY.
 *
 *   ref_driver FAMILY WIDTH MATRIX OPEN GAP MODE QFILE TFILE THREADS [LIMIT]
 *              [-s STRIDE] [-r REPS] [-w WARMUP] [-o RECORDS]
 *
 *   FAMILY  e.g. sw_striped, nw_stats_scan, sg_qx_stats_striped
 *   WIDTH   8 | 16 | 32 | sat (sat = 8 -> 16 -> 32 retry, src/satcheck.c)
 *   MATRIX  a built-in name (blosum62) or ALPHABET:MATCH:MISMATCH
 *   MODE    db    every query of QFILE against every target of TFILE
 *                 (pair p = query p / nt, target p % nt)
 *           pairs line i of QFILE against line i of TFILE (a profile per
 *                 pair, as the reference's non-profile functions build)
 *           all   upper triangle of QFILE, row-major: pair p = (i, j), i < j,
 *                 query i against target j (TFILE ignored)
 *   LIMIT   cap on the number of pairs run (a bounded sample)
 *   STRIDE  run only pairs p = 0, STRIDE, 2*STRIDE, ... (a seeded-free,
 *           evenly spread sample of the same length distribution)
 *   REPS    timed repetitions of the whole pair loop (default 1), after
 *           WARMUP untimed ones (default 0); profiles are built inside each
 *           repetition, as a caller would
 *   RECORDS binary file receiving one record per sampled pair, in sample
 *           order: int32 score, end_query, end_ref, flag, matches, similar,
 *           length, 0 (the layout of parasail_b200_record_t)
 *
 * Prints: "pairs cells seconds checksum nsaturated" for the timed
 * repetitions (seconds summed over them, pairs and cells of one), then a
 * line "reps t1 t2 ..." with each repetition's seconds.
 */
#include <dlfcn.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "parasail.h"

typedef parasail_result_t *(*pfn_t)(const parasail_profile_t *, const char *, int, int, int);
typedef parasail_profile_t *(*pcr_t)(const char *, int, const parasail_matrix_t *);

static char **read_lines(const char *path, int *n, int **lens)
{
    FILE *f = fopen(path, "r");
    char **v = NULL;
    size_t cap = 0, len = 0;
    char *line = NULL;
    size_t lcap = 0;
    ssize_t r;
    int *L = NULL;
    *n = 0;
    if (!f) { perror(path); exit(2); }
    while ((r = getline(&line, &lcap, f)) > 0) {
        while (r > 0 && (line[r - 1] == '\n' || line[r - 1] == '\r')) line[--r] = 0;
        if (r == 0) continue;
        if (len == cap) {
            cap = cap ? 2 * cap : 1024;
            v = realloc(v, cap * sizeof *v);
            L = realloc(L, cap * sizeof *L);
        }
        L[len] = (int)r;
        v[len++] = strdup(line);
    }
    free(line);
    fclose(f);
    *n = (int)len;
    *lens = L;
    return v;
}

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + ts.tv_nsec * 1e-9;
}

int main(int argc, char **argv)
{
    const char *family, *width, *mspec, *mode, *recpath = NULL;
    int open, gap, threads, nq = 0, nt = 0, k, a;
    long limit = -1, stride = 1;
    int reps = 1, warm = 0;
    char **Q, **T = NULL;
    int *QL = NULL, *TL = NULL;
    const parasail_matrix_t *matrix;
    pfn_t fn[3] = {0};
    pcr_t creator;
    int widths[3], nw = 0, stats, is_db, is_pairs;
    char name[256];
    void *self = dlopen(NULL, RTLD_NOW);
    if (argc < 10) { fprintf(stderr, "usage: see ref_driver.c\n"); return 2; }
    family = argv[1]; width = argv[2]; mspec = argv[3];
    open = atoi(argv[4]); gap = atoi(argv[5]); mode = argv[6];
    threads = atoi(argv[9]);
    for (a = 10; a < argc; ++a) {
        if (!strcmp(argv[a], "-s") && a + 1 < argc) stride = atol(argv[++a]);
        else if (!strcmp(argv[a], "-r") && a + 1 < argc) reps = atoi(argv[++a]);
        else if (!strcmp(argv[a], "-w") && a + 1 < argc) warm = atoi(argv[++a]);
        else if (!strcmp(argv[a], "-o") && a + 1 < argc) recpath = argv[++a];
        else if (argv[a][0] != '-') limit = atol(argv[a]);
        else { fprintf(stderr, "unknown option %s\n", argv[a]); return 2; }
    }
    if (stride < 1) stride = 1;
    if (reps < 1) reps = 1;
    stats = strstr(family, "_stats") != NULL;
    is_db = !strcmp(mode, "db");
    is_pairs = !strcmp(mode, "pairs");
    if (strchr(mspec, ':')) {
        char alpha[64];
        int mt, mm;
        sscanf(mspec, "%63[^:]:%d:%d", alpha, &mt, &mm);
        matrix = parasail_matrix_create(alpha, mt, mm);
    } else {
        matrix = parasail_matrix_lookup(mspec);
    }
    if (!matrix) { fprintf(stderr, "unknown matrix %s\n", mspec); return 2; }
    if (0 == strcmp(width, "sat")) { widths[0] = 8; widths[1] = 16; widths[2] = 32; nw = 3; }
    else { widths[0] = atoi(width); nw = 1; }
    for (k = 0; k < nw; ++k) {
        snprintf(name, sizeof name, "parasail_%s_profile_avx2_256_%d", family, widths[k]);
        fn[k] = (pfn_t)dlsym(self, name);
        if (!fn[k]) { fprintf(stderr, "missing %s\n", name); return 2; }
    }
    snprintf(name, sizeof name, "parasail_profile_create%s_avx_256_%s", stats ? "_stats" : "", width);
    creator = (pcr_t)dlsym(self, name);
    if (!creator) { fprintf(stderr, "missing %s\n", name); return 2; }
    Q = read_lines(argv[7], &nq, &QL);
    if (strcmp(mode, "all")) T = read_lines(argv[8], &nt, &TL);
    omp_set_num_threads(threads);

    {
        long npairs_all, nsamp;
        int64_t *rowstart = NULL;     /* all mode: first pair index of row i */
        int32_t *rec = NULL;
        double total = 0, *rep_s = calloc(reps, sizeof(double));
        double cells = 0;
        long long checksum = 0, nsat = 0;
        long done = 0;
        int nprof = is_pairs ? 0 : nq;
        parasail_profile_t **profs = calloc(nprof ? nprof : 1, sizeof *profs);
        if (is_db) npairs_all = (long)nq * nt;
        else if (is_pairs) npairs_all = nq < nt ? nq : nt;
        else npairs_all = (long)nq * (nq - 1) / 2;
        nsamp = (npairs_all + stride - 1) / stride;
        if (limit >= 0 && limit < nsamp) nsamp = limit;
        if (!is_db && !is_pairs) {
            rowstart = malloc(sizeof(int64_t) * (nq + 1));
            rowstart[0] = 0;
            for (k = 0; k < nq; ++k) rowstart[k + 1] = rowstart[k] + (nq - 1 - k);
        }
        if (recpath) rec = calloc((size_t)nsamp * 8, sizeof(int32_t));
        for (int rep = 0; rep < warm + reps; ++rep) {
            double t0 = now_s(), t1;
            double c = 0;
            long long chk = 0, ns = 0;
            long dn = 0;
            /* profiles once per query, as the aligner does (apps/parasail_aligner.cpp:1559-1567) */
#pragma omp parallel for schedule(dynamic, 1)
            for (k = 0; k < nprof; ++k) profs[k] = creator(Q[k], QL[k], matrix);
#pragma omp parallel for schedule(guided) reduction(+ : c, chk, ns, dn)
            for (long s = 0; s < nsamp; ++s) {
                const long p = s * stride;
                const char *q, *t;
                int ql, tl;
                parasail_profile_t *prof = NULL, *own = NULL;
                parasail_result_t *r = NULL;
                int w;
                if (is_db) {
                    prof = profs[p / nt];
                    q = Q[p / nt]; ql = QL[p / nt];
                    t = T[p % nt]; tl = TL[p % nt];
                } else if (is_pairs) {
                    q = Q[p]; ql = QL[p];
                    t = T[p]; tl = TL[p];
                    own = prof = creator(q, ql, matrix);
                } else {
                    /* p -> (i, j), i < j, row-major upper triangle */
                    long lo = 0, hi = nq - 1;
                    while (lo < hi) {       /* last row i with rowstart[i] <= p */
                        long mid = (lo + hi + 1) / 2;
                        if (rowstart[mid] <= p) lo = mid; else hi = mid - 1;
                    }
                    prof = profs[lo];
                    q = Q[lo]; ql = QL[lo];
                    t = Q[lo + 1 + (p - rowstart[lo])]; tl = QL[lo + 1 + (p - rowstart[lo])];
                }
                for (w = 0; w < nw; ++w) {
                    if (r) parasail_result_free(r);
                    r = fn[w](prof, t, tl, open, gap);
                    if (!(r->flag & PARASAIL_FLAG_SATURATED)) break;
                }
                if (r->flag & PARASAIL_FLAG_SATURATED) ns += 1;
                chk += r->score;
                c += (double)ql * (double)tl;
                dn += 1;
                if (rec) {
                    int32_t *o = rec + (size_t)s * 8;
                    o[0] = r->score; o[1] = r->end_query; o[2] = r->end_ref; o[3] = r->flag;
                    if (r->flag & PARASAIL_FLAG_STATS) {
                        o[4] = parasail_result_get_matches(r);
                        o[5] = parasail_result_get_similar(r);
                        o[6] = parasail_result_get_length(r);
                    } else {
                        o[4] = o[5] = o[6] = 0;
                    }
                    o[7] = 0;
                }
                parasail_result_free(r);
                if (own) parasail_profile_free(own);
            }
            for (k = 0; k < nprof; ++k) parasail_profile_free(profs[k]);
            t1 = now_s();
            if (rep >= warm) {
                rep_s[rep - warm] = t1 - t0;
                total += t1 - t0;
                cells = c; checksum = chk; nsat = ns; done = dn;
            }
        }
        printf("%ld %.0f %.6f %lld %lld\n", done, cells, total, checksum, nsat);
        printf("reps");
        for (k = 0; k < reps; ++k) printf(" %.6f", rep_s[k]);
        printf("\n");
        if (rec) {
            FILE *f = fopen(recpath, "wb");
            if (!f || fwrite(rec, sizeof(int32_t) * 8, (size_t)nsamp, f) != (size_t)nsamp) {
                perror(recpath);
                return 2;
            }
            fclose(f);
        }
    }
    return 0;
}
