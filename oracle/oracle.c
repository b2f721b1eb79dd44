/*
 * oracle.c -- CPU oracle for parasail-b200. TEST INFRASTRUCTURE ONLY.
 *
 * Restates the reference's serial dynamic programs (jeffdaily/parasail
 * v2.6.2) in plain C over mapped residue codes. Each function cites the
 * reference lines it follows. Arithmetic is 64-bit so that the values are the
 * exact mathematical DP values; the reference's serial code uses `int` with
 * NEG_INF = INT32_MIN/2, which gives the same values for all inputs whose
 * scores fit in 32 bits.
 *
 * Loaded only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg, as the checker; never by the product library.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>

#define NEG_INF (INT64_MIN / 4)
#define MAX2(a, b) ((a) > (b) ? (a) : (b))

static inline int64_t subst(const oracle_matrix_t *m, const int *s1, int i,
                            int t)
{
    /* serial kernels index matrow = matrix[size * s1[i]] (square) or
     * matrix[size * i] (pssm), then matrow[s2[j]]: src/sw.c:121-125 */
    return m->is_pssm ? m->matrix[(int64_t)m->size * i + t]
                      : m->matrix[(int64_t)m->size * s1[i] + t];
}

/* One DP over rows [0, nrows) of which [0, s1Len) are real. Rows past s1Len
 * are the padded rows of the striped/scan layout: substitution score 0,
 * match 0, similar 0 (src/memory_avx2.c:111-127, :360-370), and boundary
 * column values continued by the same formula (src/nw_striped_avx2_256_16.c
 * H/E initialisation). When r != NULL the reference's score/end rules are
 * applied (SW: src/sw.c:150-158, src/sw_stats.c:249-262; NW: src/nw.c:156-158;
 * SG: src/sg.c:171-240). */
static int run_dp(int alg, int sgflags, int stats,
                  const int *s1, int s1Len, int nrows,
                  const int *s2, int s2Len, int64_t open, int64_t gap,
                  const oracle_matrix_t *m, oracle_result_t *r,
                  oracle_padstats_t *ps)
{
    const int s1_beg = (alg == ORACLE_SG) && (sgflags & ORACLE_S1_BEG);
    const int s1_end = (alg == ORACLE_SG) && (sgflags & ORACLE_S1_END);
    const int s2_beg = (alg == ORACLE_SG) && (sgflags & ORACLE_S2_BEG);
    const int s2_end = (alg == ORACLE_SG) && (sgflags & ORACLE_S2_END);
    int64_t *H = malloc(sizeof(int64_t) * (s2Len + 1));
    int64_t *F = malloc(sizeof(int64_t) * (s2Len + 1));
    int64_t *HM = calloc(s2Len + 1, sizeof(int64_t));
    int64_t *HS = calloc(s2Len + 1, sizeof(int64_t));
    int64_t *HL = calloc(s2Len + 1, sizeof(int64_t));
    int64_t *FM = calloc(s2Len + 1, sizeof(int64_t));
    int64_t *FS = calloc(s2Len + 1, sizeof(int64_t));
    int64_t *FL = calloc(s2Len + 1, sizeof(int64_t));
    int64_t score = NEG_INF, matches = 0, similar = 0, length = 0;
    int end_query = s1Len, end_ref = s2Len;
    int i, j;
    if (!H || !F || !HM || !HS || !HL || !FM || !FS || !FL) {
        free(H); free(F); free(HM); free(HS); free(HL); free(FM); free(FS); free(FL);
        return -1;
    }
    if (ps) {
        ps->max_h = INT64_MIN;
        ps->min_h_real = INT64_MAX;
        ps->min_h_pad = INT64_MAX;
        ps->min_f = INT64_MAX;
        ps->max_stat = INT64_MIN;
        ps->max_stat_real = INT64_MIN;
    }
    if (alg == ORACLE_SW) score = NEG_INF;
    /* first row: src/sw.c:112-119, src/nw.c:112-119, src/sg.c:117-130 */
    H[0] = 0;
    F[0] = NEG_INF;
    for (j = 1; j <= s2Len; ++j) {
        if (alg == ORACLE_SW || (alg == ORACLE_SG && s2_beg)) H[j] = 0;
        else H[j] = -open - (int64_t)(j - 1) * gap;
        F[j] = NEG_INF;
    }
    for (i = 1; i <= nrows; ++i) {
        const int real = i <= s1Len;
        int64_t NH = H[0], NHM = HM[0], NHS = HS[0], NHL = HL[0];
        int64_t WH, WHM = 0, WHS = 0, WHL = 0;
        int64_t E = NEG_INF, EM = 0, ES = 0, EL = 0;
        if (alg == ORACLE_SW || (alg == ORACLE_SG && s1_beg)) WH = 0;
        else WH = -open - (int64_t)(i - 1) * gap;
        H[0] = WH; HM[0] = 0; HS[0] = 0; HL[0] = 0;
        for (j = 1; j <= s2Len; ++j) {
            const int t = s2[j - 1];
            const int64_t sc = real ? subst(m, s1, i - 1, t) : 0;
            const int64_t mt = real ? (!m->is_pssm ? (s1[i - 1] == t) : (s1[i - 1] == t)) : 0;
            int64_t NWH = NH, NWM = NHM, NWS = NHS, NWL = NHL;
            int64_t F_opn, F_ext, E_opn, E_ext, H_dag;
            NH = H[j]; NHM = HM[j]; NHS = HS[j]; NHL = HL[j];
            /* src/sw_stats.c:191-229 */
            F_opn = NH - open;
            F_ext = F[j] - gap;
            F[j] = MAX2(F_opn, F_ext);
            E_opn = WH - open;
            E_ext = E - gap;
            E = MAX2(E_opn, E_ext);
            H_dag = NWH + sc;
            WH = MAX2(H_dag, E);
            WH = MAX2(WH, F[j]);
            if (alg == ORACLE_SW) WH = MAX2(WH, 0);
            if (stats) {
                if (F_opn > F_ext) { FM[j] = NHM; FS[j] = NHS; FL[j] = NHL; }
                FL[j] += 1;
                if (E_opn > E_ext) { EM = WHM; ES = WHS; EL = WHL; }
                EL += 1;
                if (WH == H_dag) {
                    WHM = NWM + mt;
                    WHS = NWS + (sc > 0);
                    WHL = NWL + 1;
                } else if (WH == F[j]) {
                    WHM = FM[j]; WHS = FS[j]; WHL = FL[j];
                } else {
                    WHM = EM; WHS = ES; WHL = EL;
                }
                if (alg == ORACLE_SW && WH <= 0) { WHM = 0; WHS = 0; WHL = 0; }
            }
            H[j] = WH; HM[j] = WHM; HS[j] = WHS; HL[j] = WHL;
            if (ps) {
                int64_t st = MAX2(WHM, MAX2(WHS, WHL));
                if (WH > ps->max_h) ps->max_h = WH;
                if (real) { if (WH < ps->min_h_real) ps->min_h_real = WH; }
                else { if (WH < ps->min_h_pad) ps->min_h_pad = WH; }
                if (F[j] < ps->min_f) ps->min_f = F[j];
                if (stats) {
                    if (st > ps->max_stat) ps->max_stat = st;
                    if (real && st > ps->max_stat_real) ps->max_stat_real = st;
                }
            }
            if (r && real && alg == ORACLE_SW) {
                /* src/sw.c:150-158 */
                if (WH > score || (WH == score && j - 1 < end_ref)) {
                    score = WH; end_query = i - 1; end_ref = j - 1;
                    matches = WHM; similar = WHS; length = WHL;
                }
            }
            if (r && alg == ORACLE_SG && i == s1Len) {
                /* last row, src/sg.c:219-237 */
                if (s1_end && s2_end) {
                    if (WH > score || (WH == score && j - 1 < end_ref)) {
                        score = WH; end_query = s1Len - 1; end_ref = j - 1;
                        matches = WHM; similar = WHS; length = WHL;
                    }
                } else if (s2_end) {
                    if (WH > score) {
                        score = WH; end_query = s1Len - 1; end_ref = j - 1;
                        matches = WHM; similar = WHS; length = WHL;
                    }
                }
            }
        }
        if (r && alg == ORACLE_SG && real) {
            if (i < s1Len) {
                /* last column, src/sg.c:160-164 */
                if (s1_end && WH > score) {
                    score = WH; end_query = i - 1; end_ref = s2Len - 1;
                    matches = WHM; similar = WHS; length = WHL;
                }
            } else {
                /* src/sg.c:238-242 */
                if ((s1_end && WH > score) || (!s1_end && !s2_end)) {
                    score = WH; end_query = s1Len - 1; end_ref = s2Len - 1;
                    matches = WHM; similar = WHS; length = WHL;
                }
            }
        }
        if (r && alg == ORACLE_NW && i == s1Len) {
            /* src/nw.c:156-158 / src/nw_stats.c:241-247 */
            score = H[s2Len]; end_query = s1Len - 1; end_ref = s2Len - 1;
            matches = HM[s2Len]; similar = HS[s2Len]; length = HL[s2Len];
        }
    }
    if (r) {
        r->score = (int)score;
        r->end_query = end_query;
        r->end_ref = end_ref;
        r->matches = (int)matches;
        r->similar = (int)similar;
        r->length = (int)length;
    }
    free(H); free(F); free(HM); free(HS); free(HL); free(FM); free(FS); free(FL);
    return 0;
}

int oracle_align(int alg, int sgflags, int stats,
                 const int *s1, int s1Len, const int *s2, int s2Len,
                 int open, int gap, const oracle_matrix_t *m,
                 oracle_result_t *r)
{
    if (!s2 || s2Len <= 0 || !s1 || s1Len <= 0 || open < 0 || gap < 0 || !m || !r)
        return -1;
    return run_dp(alg, sgflags, stats, s1, s1Len, s1Len, s2, s2Len, open, gap,
                  m, r, NULL);
}

int oracle_padstats(int alg, int sgflags, int stats,
                    const int *s1, int s1Len, int padLen,
                    const int *s2, int s2Len,
                    int open, int gap, const oracle_matrix_t *m,
                    oracle_padstats_t *ps)
{
    if (!s2 || s2Len <= 0 || !s1 || s1Len <= 0 || padLen < s1Len || !m || !ps)
        return -1;
    return run_dp(alg, sgflags, stats, s1, s1Len, padLen, s2, s2Len, open, gap,
                  m, NULL, ps);
}

/* src/nw_banded.c:29-189, restated with the band stored as a column of
 * colLen = k - low + 1 query positions that slides down one row per target
 * column. */
int oracle_nw_banded(const int *s1, int s1Len, const int *s2, int s2Len,
                     int open, int gap, int k, const oracle_matrix_t *m,
                     oracle_result_t *r)
{
    int64_t *HB, *EB, *H, *E;
    int low, colLen, colOff, i, j;
    if (!s1 || s1Len <= 0 || !s2 || s2Len <= 0 || open < 0 || gap < 0 || k <= 0 || !m || !r)
        return -1;
    low = s1Len - s2Len - k;                 /* :92-96 */
    if (s1Len > s2Len) low = s2Len - s1Len - k;
    colLen = k - low + 1;
    colOff = s1Len > s2Len ? -k : low;
    HB = calloc(colLen + 2, sizeof(int64_t));
    EB = calloc(colLen + 2, sizeof(int64_t));
    if (!HB || !EB) { free(HB); free(EB); return -1; }
    H = HB + 1;
    E = EB + 1;
    /* :113-125 -- the initial column; indices below -colOff-1 stay 0 as the
     * reference's memset leaves them. */
    for (i = -colOff + 1, j = 0; i < colLen; ++i, ++j) {
        H[i] = -(int64_t)open - (int64_t)j * gap;
        E[i] = NEG_INF;
    }
    if (-colOff - 1 >= -1 && -colOff - 1 <= colLen) { H[-colOff - 1] = -open; E[-colOff - 1] = NEG_INF; }
    if (-colOff >= -1 && -colOff <= colLen) { H[-colOff] = 0; E[-colOff] = NEG_INF; }
    H[-1] = NEG_INF; E[-1] = NEG_INF;
    H[colLen] = NEG_INF; E[colLen] = NEG_INF;
    for (j = 0; j < s2Len; ++j) {
        int64_t F = NEG_INF;
        if (colOff < 0 && -colOff - 1 <= colLen) H[-colOff - 1] = -(int64_t)open - (int64_t)j * gap;
        for (i = 0; i < colLen; ++i) {
            int pos = colOff + i;
            int64_t H_dag, E_opn, E_ext, F_opn, F_ext, mv;
            if (pos < 0 || pos >= s1Len) continue;
            mv = subst(m, s1, pos, s2[j]);
            H_dag = H[i] + mv;
            E_opn = H[i + 1] - open;
            E_ext = E[i + 1] - gap;
            F_opn = H[i - 1] - open;
            F_ext = F - gap;
            E[i] = MAX2(E_opn, E_ext);
            F = MAX2(F_opn, F_ext);
            H[i] = MAX2(E[i], F);
            H[i] = MAX2(H[i], H_dag);
        }
        colOff += 1;
    }
    r->score = (int)(s1Len > s2Len ? H[-low] : H[k]);   /* :179 */
    r->end_query = s1Len - 1;
    r->end_ref = s2Len - 1;
    r->matches = r->similar = r->length = 0;
    free(HB);
    free(EB);
    return 0;
}

int oracle_align_batch(int alg, int sgflags, int stats, int npairs,
                       const int *s1, const int64_t *s1off, const int *s1len,
                       const int *s2, const int64_t *s2off, const int *s2len,
                       int open, int gap, const oracle_matrix_t *m,
                       oracle_result_t *r, int nthreads)
{
    int p, bad = 0;
    (void)nthreads;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1) reduction(+:bad)
    for (p = 0; p < npairs; ++p) {
        if (oracle_align(alg, sgflags, stats, s1 + s1off[p], s1len[p],
                         s2 + s2off[p], s2len[p], open, gap, m, &r[p]) != 0)
            bad += 1;
    }
    return bad ? -1 : 0;
}

/* Forward and reverse global DPs. A cell (i, j) lies on an optimal path in
 * the H state iff fwdH(i,j) + revH(i,j) - s(i,j) == opt, where revH is the
 * reverse DP on reversed sequences ending with (i, j)'s own substitution;
 * gap cells are covered through the E/F states: fwdE(i,j) + revE'(i,j) with
 * one open penalty replaced by an extension. The min/max of i - j over those
 * cells bounds every optimal path's diagonal excursion. */
int oracle_nw_diag_range(const int *s1, int s1Len, const int *s2, int s2Len,
                         int open, int gap, const oracle_matrix_t *m,
                         int *dmin, int *dmax, int *score)
{
    const int64_t n = s1Len, mm = s2Len;
    int64_t *fH, *fE, *fF, *bH, *bE, *bF;
    int64_t i, j, opt;
    int lo = 1 << 30, hi = -(1 << 30);
    const size_t cells = (size_t)(n + 2) * (size_t)(mm + 2);
    fH = malloc(cells * sizeof(int64_t)); fE = malloc(cells * sizeof(int64_t));
    fF = malloc(cells * sizeof(int64_t)); bH = malloc(cells * sizeof(int64_t));
    bE = malloc(cells * sizeof(int64_t)); bF = malloc(cells * sizeof(int64_t));
    if (!fH || !fE || !fF || !bH || !bE || !bF) {
        free(fH); free(fE); free(fF); free(bH); free(bE); free(bF);
        return -1;
    }
#define IX(a, b) ((size_t)(a) * (size_t)(mm + 2) + (size_t)(b))
    /* forward, 1-based cells; row/col 0 are the boundary */
    for (i = 0; i <= n; ++i) {
        for (j = 0; j <= mm; ++j) {
            if (i == 0 && j == 0) { fH[IX(0,0)] = 0; fE[IX(0,0)] = fF[IX(0,0)] = NEG_INF; continue; }
            if (i == 0) { fH[IX(0,j)] = -open - (j - 1) * gap; fE[IX(0,j)] = fH[IX(0,j)]; fF[IX(0,j)] = NEG_INF; continue; }
            if (j == 0) { fH[IX(i,0)] = -open - (i - 1) * gap; fF[IX(i,0)] = fH[IX(i,0)]; fE[IX(i,0)] = NEG_INF; continue; }
            fE[IX(i,j)] = MAX2(fH[IX(i,j-1)] - open, fE[IX(i,j-1)] - gap);
            fF[IX(i,j)] = MAX2(fH[IX(i-1,j)] - open, fF[IX(i-1,j)] - gap);
            fH[IX(i,j)] = MAX2(fH[IX(i-1,j-1)] + subst(m, s1, (int)i - 1, s2[j - 1]),
                               MAX2(fE[IX(i,j)], fF[IX(i,j)]));
        }
    }
    opt = fH[IX(n, mm)];
    /* reverse: bH(i,j) = best score of a path from the state "about to
     * leave cell (i,j) in H" to the corner; bE/bF = the same having just
     * entered (i,j) through a horizontal/vertical gap that may extend. */
    for (i = n; i >= 0; --i) {
        for (j = mm; j >= 0; --j) {
            int64_t h = NEG_INF, e = NEG_INF, f = NEG_INF;
            if (i == n && j == mm) { bH[IX(i,j)] = 0; bE[IX(i,j)] = 0; bF[IX(i,j)] = 0; continue; }
            if (i < n && j < mm) h = MAX2(h, bH[IX(i+1,j+1)] + subst(m, s1, (int)i, s2[j]));
            if (j < mm) { h = MAX2(h, bE[IX(i,j+1)] - open); e = MAX2(e, bE[IX(i,j+1)] - gap); }
            if (i < n) { h = MAX2(h, bF[IX(i+1,j)] - open); f = MAX2(f, bF[IX(i+1,j)] - gap); }
            /* a gap state may also close into H at this cell */
            e = MAX2(e, h);
            f = MAX2(f, h);
            bH[IX(i,j)] = h; bE[IX(i,j)] = e; bF[IX(i,j)] = f;
        }
    }
    for (i = 0; i <= n; ++i) {
        for (j = 0; j <= mm; ++j) {
            int on = 0;
            if (i > 0 && j > 0 && fH[IX(i,j)] + bH[IX(i,j)] == opt) on = 1;
            if (!on && j > 0 && fE[IX(i,j)] > NEG_INF / 2 && fE[IX(i,j)] + bE[IX(i,j)] == opt) on = 1;
            if (!on && i > 0 && fF[IX(i,j)] > NEG_INF / 2 && fF[IX(i,j)] + bF[IX(i,j)] == opt) on = 1;
            if (on) {
                int d = (int)(i - j);
                if (d < lo) lo = d;
                if (d > hi) hi = d;
            }
        }
    }
#undef IX
    *dmin = lo;
    *dmax = hi;
    *score = (int)opt;
    free(fH); free(fE); free(fF); free(bH); free(bE); free(bF);
    return 0;
}

/* Global alignment restricted to the band of diagonals lo <= i - j <= hi
 * (i, j: 1-based grid points, (0,0) the start): grid points outside the
 * band, boundary points included, are unreachable. The full-matrix case
 * (lo <= -s2Len, hi >= s1Len) equals oracle_align(ORACLE_NW). Used to check
 * the learned-band kernels; the reference has no such function (its
 * parasail_nw_banded, restated above, uses its own band layout). */
int oracle_nw_band(const int *s1, int s1Len, const int *s2, int s2Len,
                   int open, int gap, int lo, int hi, const oracle_matrix_t *m, int64_t *score)
{
    int64_t *H = malloc(sizeof(int64_t) * (s2Len + 1));
    int64_t *F = malloc(sizeof(int64_t) * (s2Len + 1));
    int i, j;
    if (!H || !F) { free(H); free(F); return -1; }
#define INB(a, b) ((a) - (b) >= lo && (a) - (b) <= hi)
    H[0] = 0;
    F[0] = NEG_INF;
    for (j = 1; j <= s2Len; ++j) {
        H[j] = INB(0, j) ? -(int64_t)open - (int64_t)(j - 1) * gap : NEG_INF;
        F[j] = NEG_INF;
    }
    for (i = 1; i <= s1Len; ++i) {
        int64_t NH = H[0];
        int64_t WH = INB(i, 0) ? -(int64_t)open - (int64_t)(i - 1) * gap : NEG_INF;
        int64_t E = NEG_INF;
        H[0] = WH;
        for (j = 1; j <= s2Len; ++j) {
            int64_t NWH = NH, f, e, h;
            NH = H[j];
            f = MAX2(NH - open, F[j] - gap);
            e = MAX2(WH - open, E - gap);
            h = MAX2(NWH + subst(m, s1, i - 1, s2[j - 1]), MAX2(e, f));
            if (!INB(i, j)) { h = NEG_INF; e = NEG_INF; f = NEG_INF; }
            F[j] = f;
            E = e;
            WH = h;
            H[j] = h;
        }
    }
#undef INB
    *score = H[s2Len];
    free(H);
    free(F);
    return 0;
}

/* The reference's serial scan forms, score only (src/nw_scan.c:116-168,
 * src/sg_scan.c:142-238, src/sw_scan.c:123-172): per target column, E from
 * the previous column's H, Ht = max(H(i-1, j-1) + s, E), then a running
 * Ft(i) = max(Ht(i-1), Ft(i-1) - gap) with Ht(-1) the column's top boundary,
 * and H = max(Ht, Ft - open) (SW also 0). Ft extends from Ht, not from H, so
 * at open < gap these forms do not reopen a vertical gap from a vertical gap
 * and differ from the serial DP; at open >= gap they equal it. End rules:
 * SW the first maximum in column-major order; SG the last row's maximum over
 * columns < s2Len - 1 (s2_end), then the last column over all rows
 * (s1_end), then the corner (s2_end), each by a strict >. */
int oracle_align_scan(int alg, int sgflags,
                      const int *s1, int s1Len, const int *s2, int s2Len,
                      int open, int gap, const oracle_matrix_t *m,
                      oracle_result_t *r)
{
    const int s1_beg = (alg == ORACLE_SG) && (sgflags & ORACLE_S1_BEG);
    const int s1_end = (alg == ORACLE_SG) && (sgflags & ORACLE_S1_END);
    const int s2_beg = (alg == ORACLE_SG) && (sgflags & ORACLE_S2_BEG);
    const int s2_end = (alg == ORACLE_SG) && (sgflags & ORACLE_S2_END);
    int64_t *HB, *H, *E, *HtB, *Ht;
    int64_t score = NEG_INF;
    int end_query = s1Len, end_ref = s2Len, i, j;
    if (!s2 || s2Len <= 0 || !s1 || s1Len <= 0 || open < 0 || gap < 0 || !m || !r)
        return -1;
    HB = malloc((size_t)(s1Len + 1) * sizeof(int64_t));
    HtB = malloc((size_t)(s1Len + 1) * sizeof(int64_t));
    E = malloc((size_t)s1Len * sizeof(int64_t));
    if (!HB || !HtB || !E) { free(HB); free(HtB); free(E); return -1; }
    H = HB + 1;
    Ht = HtB + 1;
    H[-1] = 0;
    for (i = 0; i < s1Len; ++i) {
        H[i] = (alg == ORACLE_SW || s1_beg) ? 0 : -(int64_t)open - (int64_t)i * gap;
        E[i] = NEG_INF;
    }
    for (j = 0; j < s2Len; ++j) {
        int64_t Ft = NEG_INF;
        const int64_t top = (alg == ORACLE_SW || s2_beg) ? 0 : -(int64_t)open - (int64_t)j * gap;
        for (i = 0; i < s1Len; ++i) {
            const int64_t eo = H[i] - open, ee = E[i] - gap;
            E[i] = eo > ee ? eo : ee;
        }
        for (i = 0; i < s1Len; ++i) {
            const int64_t hd = H[i - 1] + subst(m, s1, i, s2[j]);
            Ht[i] = hd > E[i] ? hd : E[i];
        }
        Ht[-1] = top;
        for (i = 0; i < s1Len; ++i) {
            const int64_t fe = Ft - gap;
            int64_t h;
            Ft = Ht[i - 1] >= fe ? Ht[i - 1] : fe;
            h = Ht[i] > Ft - open ? Ht[i] : Ft - open;
            if (alg == ORACLE_SW) {
                if (h < 0) h = 0;
                if (h > score) { score = h; end_query = i; end_ref = j; }
            }
            H[i] = h;
            if (s1_end && j == s2Len - 1 && h > score) { score = h; end_query = i; end_ref = j; }
        }
        H[-1] = top;
        if (s2_end && j < s2Len - 1 && H[s1Len - 1] > score) {
            score = H[s1Len - 1]; end_query = s1Len - 1; end_ref = j;
        }
    }
    if (alg == ORACLE_SG && s2_end && H[s1Len - 1] > score) {
        score = H[s1Len - 1]; end_query = s1Len - 1; end_ref = s2Len - 1;
    }
    if (alg == ORACLE_NW || (alg == ORACLE_SG && !s1_end && !s2_end)) {
        score = H[s1Len - 1]; end_query = s1Len - 1; end_ref = s2Len - 1;
    }
    memset(r, 0, sizeof *r);
    r->score = (int)score;
    r->end_query = end_query;
    r->end_ref = end_ref;
    free(HB); free(HtB); free(E);
    return 0;
}

/* The reference's serial scan forms with statistics (src/nw_stats_scan.c:
 * 162-279, src/sg_stats_scan.c:186-364, src/sw_stats_scan.c:159-283): the
 * scan recurrence of oracle_align_scan with the counts of the chosen cell.
 * E's counts come from H (strict >) or extend; Ht takes the diagonal's
 * counts when diagonal >= E; the running Ft takes H(i-1)'s counts when
 * H(i-1) > Ft(i-1) - gap (H(i-1) of this column; row -1 reads the previous
 * column's top boundary, counts 0), else extends; H takes Ht's counts when
 * Ht > Ft - open, on a tie F's when E beat the diagonal, else Ft's. SW
 * clamps H at 0 with counts 0 and keeps the first maximum in column-major
 * order; SG keeps the last row's maximum over columns (s2_end) and then the
 * last column's rows (s1_end; with s2_end a tie in a lower row moves the
 * end there). */
int oracle_align_scan_stats(int alg, int sgflags,
                            const int *s1, int s1Len, const int *s2, int s2Len,
                            int open, int gap, const oracle_matrix_t *m,
                            oracle_result_t *r)
{
    const int s1_beg = (alg == ORACLE_SG) && (sgflags & ORACLE_S1_BEG);
    const int s1_end = (alg == ORACLE_SG) && (sgflags & ORACLE_S1_END);
    const int s2_beg = (alg == ORACLE_SG) && (sgflags & ORACLE_S2_BEG);
    const int s2_end = (alg == ORACLE_SG) && (sgflags & ORACLE_S2_END);
    const int sw = alg == ORACLE_SW;
    int64_t *buf, *H, *HM, *HS, *HL, *E, *EM, *ES, *EL, *Ht, *HtM, *HtS, *HtL;
    char *Ex;
    int64_t score = NEG_INF, matches = 0, similar = 0, length = 0;
    int end_query = s1Len, end_ref = s2Len, i, j;
    if (!s2 || s2Len <= 0 || !s1 || s1Len <= 0 || open < 0 || gap < 0 || !m || !r)
        return -1;
    buf = calloc((size_t)(s1Len + 1) * 12, sizeof(int64_t));
    Ex = calloc((size_t)s1Len, 1);
    if (!buf || !Ex) { free(buf); free(Ex); return -1; }
    /* H, HM, HS, HL, Ht, HtM, HtS, HtL with a row -1; E, EM, ES, EL */
    H = buf + 1; HM = H + (s1Len + 1); HS = HM + (s1Len + 1); HL = HS + (s1Len + 1);
    Ht = HL + (s1Len + 1); HtM = Ht + (s1Len + 1); HtS = HtM + (s1Len + 1); HtL = HtS + (s1Len + 1);
    E = HtL + s1Len; EM = E + (s1Len + 1); ES = EM + (s1Len + 1); EL = ES + (s1Len + 1);
    H[-1] = 0;
    for (i = 0; i < s1Len; ++i) {
        H[i] = (sw || s1_beg) ? 0 : -(int64_t)open - (int64_t)i * gap;
        E[i] = NEG_INF;
    }
    for (j = 0; j < s2Len; ++j) {
        int64_t Ft = NEG_INF, FtM = 0, FtS = 0, FtL = 0;
        const int64_t top = (sw || s2_beg) ? 0 : -(int64_t)open - (int64_t)j * gap;
        for (i = 0; i < s1Len; ++i) {
            const int64_t eo = H[i] - open, ee = E[i] - gap;
            if (eo > ee) { E[i] = eo; EM[i] = HM[i]; ES[i] = HS[i]; EL[i] = HL[i]; }
            else E[i] = ee;
            EL[i] += 1;
        }
        Ht[-1] = top;
        for (i = 0; i < s1Len; ++i) {
            const int64_t sc = subst(m, s1, i, s2[j]);
            const int64_t hd = H[i - 1] + sc;
            Ex[i] = E[i] > hd;
            if (hd >= E[i]) {
                Ht[i] = hd; HtM[i] = HM[i - 1] + (s1[i] == s2[j]); HtS[i] = HS[i - 1] + (sc > 0);
                HtL[i] = HL[i - 1] + 1;
            } else {
                Ht[i] = E[i]; HtM[i] = EM[i]; HtS[i] = ES[i]; HtL[i] = EL[i];
            }
        }
        for (i = 0; i < s1Len; ++i) {
            const int64_t fe = Ft - gap;
            int64_t fo;
            Ft = Ht[i - 1] >= fe ? Ht[i - 1] : fe;
            fo = Ft - open;
            if (H[i - 1] > fe) { FtM = HM[i - 1]; FtS = HS[i - 1]; FtL = HL[i - 1]; }
            FtL += 1;
            if (Ht[i] > fo || (Ht[i] == fo && !Ex[i])) {
                H[i] = Ht[i] > fo ? Ht[i] : fo; HM[i] = HtM[i]; HS[i] = HtS[i]; HL[i] = HtL[i];
            } else {
                H[i] = fo; HM[i] = FtM; HS[i] = FtS; HL[i] = FtL;
            }
            if (sw) {
                if (H[i] <= 0) { H[i] = 0; HM[i] = HS[i] = HL[i] = 0; }
                if (H[i] > score) {
                    score = H[i]; matches = HM[i]; similar = HS[i]; length = HL[i];
                    end_query = i; end_ref = j;
                }
            }
        }
        H[-1] = top;
        if (s2_end && H[s1Len - 1] > score) {
            score = H[s1Len - 1]; matches = HM[s1Len - 1]; similar = HS[s1Len - 1]; length = HL[s1Len - 1];
            end_query = s1Len - 1; end_ref = j;
        }
    }
    if (s1_end) {
        for (i = 0; i < s1Len; ++i) {
            if (H[i] > score || (s2_end && H[i] == score && end_ref == s2Len - 1 && i < end_query)) {
                score = H[i]; matches = HM[i]; similar = HS[i]; length = HL[i];
                end_query = i; end_ref = s2Len - 1;
            }
        }
    }
    if (!sw && !s1_end && !s2_end) {
        score = H[s1Len - 1]; matches = HM[s1Len - 1]; similar = HS[s1Len - 1]; length = HL[s1Len - 1];
        end_query = s1Len - 1; end_ref = s2Len - 1;
    }
    memset(r, 0, sizeof *r);
    r->score = (int)score; r->end_query = end_query; r->end_ref = end_ref;
    r->matches = (int)matches; r->similar = (int)similar; r->length = (int)length;
    free(buf); free(Ex);
    return 0;
}
