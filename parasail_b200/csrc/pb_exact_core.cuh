/*
 * pb_exact_core.cuh -- the per-pair dynamic program of the exact kernel,
 * callable from device code (k_exact) and from host test harnesses.
 *
 * Semantics follow the reference's serial dynamic programs exactly
 * (jeffdaily/parasail v2.6.2 src/sw.c:131-158, src/nw.c:131-156,
 * src/sg.c:142-242 and the _stats twins src/sw_stats.c:183-262,
 * src/nw_stats.c:165-228, src/sg_stats.c), which the reference's striped and
 * scan kernels reproduce for every non-saturated result.
 */
#ifndef PARASAIL_B200_PB_EXACT_CORE_CUH
#define PARASAIL_B200_PB_EXACT_CORE_CUH

#include <cstdint>
#include <climits>

#include "pb_cuda.h"
#include "pb_kernels.cuh"

#ifndef PB_RESTRICT
#define PB_RESTRICT __restrict__
#endif

namespace pb {


static constexpr int NEG_INF = INT32_MIN / 2;   /* src/sw.c:16 */

struct Cell {
    int h, m, s, l;
};

template <int ALG>
__host__ __device__ __forceinline__ int top_h(int j, int open, int gap, int sgflags)
{
    /* row -1: src/sw.c:112-119, src/nw.c:112-119, src/sg.c:117-130 */
    if (ALG == PB_SW) return 0;
    if (ALG == PB_SG && (sgflags & PB_S2_BEG)) return 0;
    return -open - j * gap;
}

template <int ALG>
__host__ __device__ __forceinline__ int left_h(int i, int open, int gap, int sgflags)
{
    /* column -1: src/sw.c:129, src/nw.c:129, src/sg.c:146 */
    if (ALG == PB_SW) return 0;
    if (ALG == PB_SG && (sgflags & PB_S1_BEG)) return 0;
    return -open - i * gap;
}

/* SCANF: the vertical gap of the reference's serial scan forms
 * (src/nw_scan.c:128-146, src/sg_scan.c:155-173, src/sw_scan.c:146-152),
 * F(i) = max(Ht(i-1) - open, F(i-1) - gap) with Ht = max(diagonal, E): a
 * vertical gap is not reopened from a vertical gap, which differs from the
 * serial DP at open < gap. The kernel then carries in fu the F of the next
 * row instead of the F of the row above.
 * With statistics (src/nw_stats_scan.c:215-228) F takes H(i-1)'s counts
 * when H(i-1) - open > F(i-1) - gap. Given fu = F(i), that test is
 * H(i-1) - open > fu, except on a tie, where it holds exactly when F(i)
 * came from Ht(i-1) - open strictly; that one bit travels with the carried
 * F length as its complement (~len < 0), so strip buffers keep their size.
 * Row 0 reads the bit set (the reference's F starts at -infinity). */
template <int ALG, bool STATS, int R, bool SCANF = false>
__host__ __device__ __forceinline__ void exact_pair(const ExactParams &p, const int k)
{
    const int pid = p.order ? p.order[k] : k;          /* output slot */
    const int ti = p.nt ? pid % p.nt : pid;            /* target (and per-pair query) index */

    const bool matmode = p.mat != nullptr;
    ProfDesc pd;
    if (matmode) {
        pd.prof = nullptr; pd.prof8 = nullptr; pd.qcodes = p.qall + p.qoff[ti];
        pd.qlen = p.qlen[ti]; pd.lp = 0; pd.size = p.msize; pd.pad_ = 0;
    } else {
        pd = p.profs[p.nt ? pid / p.nt : (p.prof_index ? p.prof_index[pid] : 0)];
    }
    const uint8_t *PB_RESTRICT tseq = p.targets + p.toff[ti];
    const int ql = p.qlim ? p.qlim[pid] : pd.qlen;
    const int tl = p.tlim ? p.tlim[pid] : p.tlen[ti];
    const int open = p.open, gap = p.gap, sgf = p.sgflags;
    const int c8 = (ql + 7) & ~7, c16 = (ql + 15) & ~15, c32 = (ql + 31) & ~31;
    const int nrows = p.pad_rows == 0 ? ql
                    : (p.pad_rows == 8 ? c8 : (p.pad_rows == 16 ? c16 : c32));
    const int NV = STATS ? 8 : 2;
    int *PB_RESTRICT buf = p.scratch + p.soff[pid];

    /* outputs and predicate accumulators */
    int max_h = INT32_MIN, min_h_real = INT32_MAX, max_st_real = INT32_MIN;
    int min_f_real = INT32_MAX;
    int min_h_pad0 = INT32_MAX, min_h_pad1 = INT32_MAX, min_h_pad2 = INT32_MAX;
    int max_st_pad0 = INT32_MIN, max_st_pad1 = INT32_MIN, max_st_pad2 = INT32_MIN;
    int min_f_pad0 = INT32_MAX, min_f_pad1 = INT32_MAX, min_f_pad2 = INT32_MAX;
    int status = 0;

    /* SW best cell: (score desc, j asc, i asc), src/sw.c:150-158 */
    Cell best = {NEG_INF, 0, 0, 0};
    int best_i = ql, best_j = tl;
    /* SG: last column over rows < ql-1, last row over all j, corner */
    Cell lc = {NEG_INF, 0, 0, 0};
    int lc_i = -1;
    Cell lr = {NEG_INF, 0, 0, 0};
    int lr_j = -1;
    Cell corner = {0, 0, 0, 0};

    for (int r0 = 0; r0 < nrows; r0 += R) {
        int Hl[R], E[R];
        int HlM[R], HlS[R], HlL[R], EM[R], ES[R], EL[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            Hl[r] = left_h<ALG>(r0 + r, open, gap, sgf);
            E[r] = NEG_INF;
            if (STATS) { HlM[r] = HlS[r] = HlL[r] = 0; EM[r] = ES[r] = EL[r] = 0; }
        }
        /* diagonal of row r0 at column 0: H(r0-1, -1) */
        int dg = r0 == 0 ? 0 : left_h<ALG>(r0 - 1, open, gap, sgf);
        int dgM = 0, dgS = 0, dgL = 0;

        for (int j = 0; j < tl; ++j) {
            const int code = tseq[j];
            if (code >= pd.size) status |= PB_ST_BADCODE;
            const int csafe = code < pd.size ? code : 0;
            const int32_t *PB_RESTRICT prow = matmode ? p.mat + (size_t)csafe * p.msize
                                                      : pd.prof + (size_t)csafe * pd.lp;
            int hu, fu, huM = 0, huS = 0, huL = 0, fuM = 0, fuS = 0, fuL = 0;
            int *bj = buf + (size_t)j * NV;
            if (r0 == 0) {
                hu = top_h<ALG>(j, open, gap, sgf);
                fu = SCANF ? hu - open : NEG_INF;
                if (SCANF && STATS) fuL = ~0;
            } else {
                hu = bj[0];
                fu = bj[1];
                if (STATS) { huM = bj[2]; huS = bj[3]; huL = bj[4]; fuM = bj[5]; fuS = bj[6]; fuL = bj[7]; }
            }
            /* diagonal of every row of the strip: row r reads H(i-1, j-1),
             * i.e. row r-1 of the previous column (row 0: the row above the
             * strip, carried in dg) */
            int Dg[R], DgM[R], DgS[R], DgL[R];
#pragma unroll
            for (int r = R - 1; r >= 1; --r) {
                Dg[r] = Hl[r - 1];
                if (STATS) { DgM[r] = HlM[r - 1]; DgS[r] = HlS[r - 1]; DgL[r] = HlL[r - 1]; }
            }
            Dg[0] = dg;
            if (STATS) { DgM[0] = dgM; DgS[0] = dgS; DgL[0] = dgL; }
            dg = hu; dgM = huM; dgS = huS; dgL = huL;
            /* Rows are fully unrolled for score-only runs. With statistics
             * the row loop stays rolled: unrolled, the sm_100a build of this
             * loop lost the diagonal's statistics in on-device tests (CUDA
             * 12.9, ptxas -O1..-O3; correct at -O0 and in the host build). */
#pragma unroll (STATS ? 1 : R)
            for (int r = 0; r < R; ++r) {
                const int i = r0 + r;
                const bool real = i < ql;
                const int sc = real ? (matmode ? prow[pd.qcodes[i]] : prow[i]) : 0;
                /* F: vertical gap (along the query), E: horizontal gap */
                const int f_opn = hu - open, f_ext = fu - gap;
                const int fn = SCANF ? fu : max(f_opn, f_ext);
                const int e_opn = Hl[r] - open, e_ext = E[r] - gap;
                const int en = max(e_opn, e_ext);
                const int hdag = Dg[r] + sc;
                const int ht = max(hdag, en);
                int hn = max(ht, fn);
                if (ALG == PB_SW) hn = max(hn, 0);
                int hM = 0, hS = 0, hL = 0, fM = 0, fS = 0, fL = 0;
                if (STATS) {
                    /* src/sw_stats.c:205-237: gap-source choice by strict >,
                     * then cell choice diagonal > F > E, SW resets at H <= 0 */
                    const bool fb = SCANF && fuL < 0;
                    const bool fo = SCANF ? (f_opn > fu || (f_opn == fu && fb)) : f_opn > f_ext;
                    fM = fo ? huM : fuM;
                    fS = fo ? huS : fuS;
                    fL = (fo ? huL : (fb ? ~fuL : fuL)) + 1;
                    const bool eo = e_opn > e_ext;
                    const int eM = eo ? HlM[r] : EM[r];
                    const int eS = eo ? HlS[r] : ES[r];
                    const int eL = (eo ? HlL[r] : EL[r]) + 1;
                    EM[r] = eM; ES[r] = eS; EL[r] = eL;
                    const bool isd = hn == hdag, isf = hn == fn;
                    const int mt = real ? (pd.qcodes[i] == code) : 0;
                    hM = isd ? DgM[r] + mt : (isf ? fM : eM);
                    hS = isd ? DgS[r] + (sc > 0) : (isf ? fS : eS);
                    hL = isd ? DgL[r] + 1 : (isf ? fL : eL);
                    if (ALG == PB_SW) {
                        const bool z = hn <= 0;
                        hM = z ? 0 : hM;
                        hS = z ? 0 : hS;
                        hL = z ? 0 : hL;
                    }
                }
                E[r] = en;

                /* predicate statistics */
                if (i < nrows) {
                    max_h = max(max_h, hn);
                    if (real) {
                        min_h_real = min(min_h_real, hn);
                        min_f_real = min(min_f_real, fn);
                        if (STATS) max_st_real = max(max_st_real, hL);
                    } else if (i < c8) {
                        min_h_pad0 = min(min_h_pad0, hn);
                        min_f_pad0 = min(min_f_pad0, fn);
                        if (STATS) max_st_pad0 = max(max_st_pad0, hL);
                    } else if (i < c16) {
                        min_h_pad1 = min(min_h_pad1, hn);
                        min_f_pad1 = min(min_f_pad1, fn);
                        if (STATS) max_st_pad1 = max(max_st_pad1, hL);
                    } else {
                        min_h_pad2 = min(min_h_pad2, hn);
                        min_f_pad2 = min(min_f_pad2, fn);
                        if (STATS) max_st_pad2 = max(max_st_pad2, hL);
                    }
                }
                /* end-position rules */
                if (real) {
                    if (ALG == PB_SW) {
                        if (hn > best.h || (hn == best.h && (j < best_j || (j == best_j && i < best_i)))) {
                            best.h = hn; best.m = hM; best.s = hS; best.l = hL;
                            best_i = i; best_j = j;
                        }
                    } else {
                        if (i == ql - 1) {
                            if (hn > lr.h) { lr.h = hn; lr.m = hM; lr.s = hS; lr.l = hL; lr_j = j; }
                            if (j == tl - 1) { corner.h = hn; corner.m = hM; corner.s = hS; corner.l = hL; }
                        } else if (ALG == PB_SG && j == tl - 1) {
                            if (hn > lc.h) { lc.h = hn; lc.m = hM; lc.s = hS; lc.l = hL; lc_i = i; }
                        }
                    }
                }
                Hl[r] = hn;
                if (STATS) { HlM[r] = hM; HlS[r] = hS; HlL[r] = hL; }
                hu = hn; fu = SCANF ? max(ht - open, fn - gap) : fn;
                if (STATS) {
                    huM = hM; huS = hS; huL = hL; fuM = fM; fuS = fS;
                    fuL = (SCANF && ht - open > fn - gap) ? ~fL : fL;
                }
            }
            if (r0 + R < nrows) {
                bj[0] = hu; bj[1] = fu;
                if (STATS) { bj[2] = huM; bj[3] = huS; bj[4] = huL; bj[5] = fuM; bj[6] = fuS; bj[7] = fuL; }
            }
        }
    }

    Cell res;
    int eq, er;
    if (ALG == PB_SW) {
        res = best; eq = best_i; er = best_j;
    } else if (ALG == PB_NW) {
        res = corner; eq = ql - 1; er = tl - 1;
    } else {
        /* src/sg.c:160-242 */
        const bool s1e = sgf & PB_S1_END, s2e = sgf & PB_S2_END;
        res.h = NEG_INF; res.m = res.s = res.l = 0;
        eq = ql; er = tl;
        if (s1e && lc_i >= 0) { res = lc; eq = lc_i; er = tl - 1; }
        if (s1e && s2e) {
            if (lr.h > res.h || (lr.h == res.h && lr_j < er)) { res = lr; eq = ql - 1; er = lr_j; }
        } else if (s2e) {
            if (lr.h > res.h) { res = lr; eq = ql - 1; er = lr_j; }
        }
        if ((s1e && corner.h > res.h) || (!s1e && !s2e)) { res = corner; eq = ql - 1; er = tl - 1; }
    }

    pb_pair_out o;
    o.score = res.h; o.end_query = eq; o.end_ref = er;
    o.matches = res.m; o.similar = res.s; o.length = res.l;
    o.max_h = max_h; o.min_h_real = min_h_real; o.max_stat_real = max_st_real;
    o.min_f_real = min_f_real;
    o.min_h_pad[0] = min_h_pad0; o.min_h_pad[1] = min_h_pad1; o.min_h_pad[2] = min_h_pad2;
    o.max_stat_pad[0] = max_st_pad0; o.max_stat_pad[1] = max_st_pad1; o.max_stat_pad[2] = max_st_pad2;
    o.min_f_pad[0] = min_f_pad0; o.min_f_pad[1] = min_f_pad1; o.min_f_pad[2] = min_f_pad2;
    o.status = status;
    p.out[pid] = o;
}

}  // namespace pb

#endif
