/*
 * ref_driver.c -- CPU baseline: times the reference's own AVX2 striped/scan
 * profile functions (oracle/_ref/libparasail_ref.so) with OpenMP across
 * pairs, the pattern of the reference's tests/test_openmp.c:353-378 and
 * apps/parasail_aligner.cpp:1606-1622 (one profile per query, guided
 * schedule over targets). TEST/BASELINE INFRASTRUCTURE ONLY.
 *
 *   ref_driver FAMILY WIDTH MATRIX OPEN GAP MODE QFILE TFILE THREADS [LIMIT]
 *
 *   FAMILY  e.g. sw_striped, nw_stats_scan, sg_qx_stats_striped
 *   WIDTH   8 | 16 | 32 | sat (sat = 8 -> 16 -> 32 retry, src/satcheck.c)
 *   MATRIX  a built-in name (blosum62) or ALPHABET:MATCH:MISMATCH
 *   MODE    db    every query of QFILE against every target of TFILE
 *           pairs line i of QFILE against line i of TFILE
 *           all   upper triangle of QFILE (TFILE ignored)
 *   LIMIT   optional cap on the number of pairs run (a bounded sample)
 *
 * Prints one line: pairs cells seconds checksum(sum of scores) nsaturated.
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

static char **read_lines(const char *path, int *n)
{
    FILE *f = fopen(path, "r");
    char **v = NULL;
    size_t cap = 0, len = 0;
    char *line = NULL;
    size_t lcap = 0;
    ssize_t r;
    *n = 0;
    if (!f) { perror(path); exit(2); }
    while ((r = getline(&line, &lcap, f)) > 0) {
        while (r > 0 && (line[r - 1] == '\n' || line[r - 1] == '\r')) line[--r] = 0;
        if (r == 0) continue;
        if (len == cap) { cap = cap ? 2 * cap : 1024; v = realloc(v, cap * sizeof *v); }
        v[len++] = strdup(line);
    }
    free(line);
    fclose(f);
    *n = (int)len;
    return v;
}

int main(int argc, char **argv)
{
    const char *family, *width, *mspec, *mode;
    int open, gap, threads, nq = 0, nt = 0, k;
    long limit = -1;
    char **Q, **T = NULL;
    const parasail_matrix_t *matrix;
    pfn_t fn[3] = {0};
    pcr_t creator;
    int widths[3], nw = 0, stats;
    char name[256];
    void *self = dlopen(NULL, RTLD_NOW);
    if (argc < 10) { fprintf(stderr, "usage: see ref_driver.c\n"); return 2; }
    family = argv[1]; width = argv[2]; mspec = argv[3];
    open = atoi(argv[4]); gap = atoi(argv[5]); mode = argv[6];
    threads = atoi(argv[9]);
    if (argc > 10) limit = atol(argv[10]);
    stats = strstr(family, "_stats") != NULL;
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
    Q = read_lines(argv[7], &nq);
    if (strcmp(mode, "all")) T = read_lines(argv[8], &nt);
    omp_set_num_threads(threads);

    {
        long npairs = 0, done = 0;
        double cells = 0, t0, t1;
        long long checksum = 0, nsat = 0;
        int nprof = 0;
        parasail_profile_t **profs;
        struct timespec ts;
        if (!strcmp(mode, "db")) npairs = (long)nq * nt;
        else if (!strcmp(mode, "pairs")) npairs = nq < nt ? nq : nt;
        else npairs = (long)nq * (nq - 1) / 2;
        if (limit >= 0 && limit < npairs) npairs = limit;
        nprof = !strcmp(mode, "pairs") ? 0 : nq;
        profs = calloc(nprof ? nprof : 1, sizeof *profs);
        clock_gettime(CLOCK_MONOTONIC, &ts);
        t0 = ts.tv_sec + ts.tv_nsec * 1e-9;
        /* profiles once per query, as the aligner does (apps/parasail_aligner.cpp:1559-1567) */
#pragma omp parallel for schedule(dynamic, 1)
        for (k = 0; k < nprof; ++k) profs[k] = creator(Q[k], (int)strlen(Q[k]), matrix);
#pragma omp parallel for schedule(guided) reduction(+ : cells, checksum, nsat, done)
        for (long p = 0; p < npairs; ++p) {
            const char *q, *t;
            parasail_profile_t *prof = NULL, *own = NULL;
            parasail_result_t *r = NULL;
            int w;
            if (!strcmp(mode, "db")) {
                prof = profs[p / nt];
                q = Q[p / nt];
                t = T[p % nt];
            } else if (!strcmp(mode, "pairs")) {
                q = Q[p];
                t = T[p];
                own = prof = creator(q, (int)strlen(q), matrix);
            } else {
                /* p -> (i, j), i < j, row-major upper triangle */
                long i = 0, rem = p;
                while (rem >= nq - 1 - i) { rem -= nq - 1 - i; ++i; }
                prof = profs[i];
                q = Q[i];
                t = Q[i + 1 + rem];
            }
            for (w = 0; w < nw; ++w) {
                if (r) parasail_result_free(r);
                r = fn[w](prof, t, (int)strlen(t), open, gap);
                if (!(r->flag & PARASAIL_FLAG_SATURATED)) break;
            }
            if (r->flag & PARASAIL_FLAG_SATURATED) nsat += 1;
            checksum += r->score;
            cells += (double)strlen(q) * (double)strlen(t);
            done += 1;
            parasail_result_free(r);
            if (own) parasail_profile_free(own);
        }
        clock_gettime(CLOCK_MONOTONIC, &ts);
        t1 = ts.tv_sec + ts.tv_nsec * 1e-9;
        printf("%ld %.0f %.6f %lld %lld\n", done, cells, t1 - t0, checksum, nsat);
    }
    return 0;
}
