/*
 * oracle.h -- CPU oracle for parasail-b200. TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's serial algorithms for the hot path
 * (jeffdaily/parasail v2.6.2: src/sw.c, src/nw.c, src/sg.c, src/sw_stats.c,
 * src/nw_stats.c, src/sg_stats.c, src/nw_banded.c), plus the statistics of the
 * padded striped/scan layout that the vector kernels' saturation checks read.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * it, and only as the checker. The product library never links it.
 *
 * Parity pin: tests/test_oracle.py checks this restatement against the
 * reference's own known answers (tests/test_basic.c:22-80) and against the
 * reference library compiled from source (oracle/_ref/libparasail_ref.so).
 *
 * Sequences are passed already mapped to matrix indices (matrix->mapper).
 */
#ifndef PARASAIL_B200_ORACLE_H
#define PARASAIL_B200_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORACLE_SW = 0, ORACLE_NW = 1, ORACLE_SG = 2 };
/* semi-global free-end bits, reference src/sg_helper.h:53-63 order */
enum { ORACLE_S1_BEG = 1, ORACLE_S1_END = 2, ORACLE_S2_BEG = 4, ORACLE_S2_END = 8 };

typedef struct {
    int size;           /* alphabet size (includes the trailing '*') */
    const int *matrix;  /* square: size*size, row = query code; pssm: length*size */
    int is_pssm;        /* 1: row index is the query position */
    int max, min;
} oracle_matrix_t;

typedef struct {
    int score, end_query, end_ref;
    int matches, similar, length;
} oracle_result_t;

/* Statistics of the DP extended with padded query rows [s1Len, padLen)
 * (profile score 0, match 0, similar 0), which is what the striped/scan
 * kernels compute. All values exact (64-bit). */
typedef struct {
    int64_t max_h;        /* max H over all cells, real and padded */
    int64_t min_h_real;   /* min H over real rows */
    int64_t min_h_pad;    /* min H over padded rows (INT64_MAX if none) */
    int64_t min_f;        /* min vertical-gap F over all cells (F(-1,j) = -inf) */
    int64_t max_stat;     /* max of matches/similar/length over all cells */
    int64_t max_stat_real;/* the same over real rows only */
} oracle_padstats_t;

/* Serial Gotoh DP with the reference's tie-breaks. Returns 0 on success. */
int oracle_align(int alg, int sgflags, int stats,
                 const int *s1, int s1Len, const int *s2, int s2Len,
                 int open, int gap, const oracle_matrix_t *m,
                 oracle_result_t *r);

/* The reference's serial scan forms, score only (src/nw_scan.c,
 * src/sg_scan.c, src/sw_scan.c): F extends from Ht = max(diagonal, E), so
 * they differ from oracle_align at open < gap. Returns 0 on success. */
int oracle_align_scan(int alg, int sgflags,
                      const int *s1, int s1Len, const int *s2, int s2Len,
                      int open, int gap, const oracle_matrix_t *m,
                      oracle_result_t *r);

/* The reference's serial scan forms with statistics (src/nw_stats_scan.c,
 * src/sg_stats_scan.c, src/sw_stats_scan.c): the recurrence of
 * oracle_align_scan with the counts of the chosen cell. Returns 0 on
 * success. */
int oracle_align_scan_stats(int alg, int sgflags,
                            const int *s1, int s1Len, const int *s2, int s2Len,
                            int open, int gap, const oracle_matrix_t *m,
                            oracle_result_t *r);

/* Same recurrence over padLen >= s1Len query rows; fills *ps. */
int oracle_padstats(int alg, int sgflags, int stats,
                    const int *s1, int s1Len, int padLen,
                    const int *s2, int s2Len,
                    int open, int gap, const oracle_matrix_t *m,
                    oracle_padstats_t *ps);

/* Banded global alignment, reference src/nw_banded.c:29-189. */
int oracle_nw_banded(const int *s1, int s1Len, const int *s2, int s2Len,
                     int open, int gap, int k, const oracle_matrix_t *m,
                     oracle_result_t *r);

/* Many pairs at once (OpenMP over pairs); pair p aligns
 * s1[s1off[p] .. +s1len[p]) against s2[s2off[p] .. +s2len[p]). */
int oracle_align_batch(int alg, int sgflags, int stats, int npairs,
                       const int *s1, const int64_t *s1off, const int *s1len,
                       const int *s2, const int64_t *s2off, const int *s2len,
                       int open, int gap, const oracle_matrix_t *m,
                       oracle_result_t *r, int nthreads);

/* Optimal-path diagonal range of a global alignment: the min and max of
 * (i - j) over every cell that lies on at least one optimal path, computed
 * from a forward and a reverse pass (used to check band labels). */
int oracle_nw_diag_range(const int *s1, int s1Len, const int *s2, int s2Len,
                         int open, int gap, const oracle_matrix_t *m,
                         int *dmin, int *dmax, int *score);

/* Global alignment restricted to diagonals lo <= i - j <= hi. */
int oracle_nw_band(const int *s1, int s1Len, const int *s2, int s2Len,
                   int open, int gap, int lo, int hi, const oracle_matrix_t *m, int64_t *score);

#ifdef __cplusplus
}
#endif
#endif
