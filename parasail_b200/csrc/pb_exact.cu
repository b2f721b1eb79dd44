/*
 * pb_exact.cu -- exact 32-bit alignment kernel (any mode, optional stats).
 *
 * One thread aligns one pair. The query rows are processed in strips of R
 * rows held in registers; the thread sweeps the whole target for each strip
 * and hands the strip's bottom row (H, F and their statistics) to the next
 * strip through a per-pair buffer in global memory.
 *
 * Semantics follow the reference's serial dynamic programs exactly
 * (jeffdaily/parasail v2.6.2 src/sw.c:131-158, src/nw.c:131-156,
 * src/sg.c:142-242 and the _stats twins src/sw_stats.c:183-262,
 * src/nw_stats.c:165-228, src/sg_stats.c), which the reference's striped and
 * scan kernels reproduce for every non-saturated result. The kernel also
 * records the statistics that the reference's vector kernels use to decide
 * saturation: extreme values over the real query rows and over the padded
 * rows of the 8-, 16- and 32-lane layouts.
 */
#include <cstdint>
#include <climits>

#include "pb_cuda.h"
#include "pb_kernels.cuh"

namespace pb {

static constexpr int NEG_INF = INT32_MIN / 2;   /* src/sw.c:16 */

struct Cell {
    int h, m, s, l;
};

template <int ALG>
__device__ __forceinline__ int top_h(int j, int open, int gap, int sgflags)
{
    /* row -1: src/sw.c:112-119, src/nw.c:112-119, src/sg.c:117-130 */
    if (ALG == PB_SW) return 0;
    if (ALG == PB_SG && (sgflags & PB_S2_BEG)) return 0;
    return -open - j * gap;
}

template <int ALG>
__device__ __forceinline__ int left_h(int i, int open, int gap, int sgflags)
{
    /* column -1: src/sw.c:129, src/nw.c:129, src/sg.c:146 */
    if (ALG == PB_SW) return 0;
    if (ALG == PB_SG && (sgflags & PB_S1_BEG)) return 0;
    return -open - i * gap;
}

template <int ALG, bool STATS, int R>
__global__ void __launch_bounds__(128)
k_exact(ExactParams p)
{
    const int pid = blockIdx.x * blockDim.x + threadIdx.x;
    if (pid >= p.npairs) return;

    const ProfDesc pd = p.profs[p.prof_index ? p.prof_index[pid] : 0];
    const uint8_t *__restrict__ tseq = p.targets + p.toff[pid];
    const int ql = p.qlim ? p.qlim[pid] : pd.qlen;
    const int tl = p.tlim ? p.tlim[pid] : p.tlen[pid];
    const int open = p.open, gap = p.gap, sgf = p.sgflags;
    const int c8 = (ql + 7) & ~7, c16 = (ql + 15) & ~15, c32 = (ql + 31) & ~31;
    const int nrows = p.pad_rows == 0 ? ql
                    : (p.pad_rows == 8 ? c8 : (p.pad_rows == 16 ? c16 : c32));
    const int NV = STATS ? 8 : 2;
    int *__restrict__ buf = p.scratch + p.soff[pid];

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
            const int32_t *__restrict__ prow = pd.prof + (size_t)(code < pd.size ? code : 0) * pd.lp;
            int hu, fu, huM = 0, huS = 0, huL = 0, fuM = 0, fuS = 0, fuL = 0;
            int *bj = buf + (size_t)j * NV;
            if (r0 == 0) {
                hu = top_h<ALG>(j, open, gap, sgf);
                fu = NEG_INF;
            } else {
                hu = bj[0];
                fu = bj[1];
                if (STATS) { huM = bj[2]; huS = bj[3]; huL = bj[4]; fuM = bj[5]; fuS = bj[6]; fuL = bj[7]; }
            }
            int hd = dg, hdM = dgM, hdS = dgS, hdL = dgL;
            dg = hu; dgM = huM; dgS = huS; dgL = huL;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int i = r0 + r;
                const bool real = i < ql;
                const int sc = real ? prow[i] : 0;
                /* F: vertical gap (along the query), E: horizontal gap */
                const int f_opn = hu - open, f_ext = fu - gap;
                const int fn = max(f_opn, f_ext);
                const int e_opn = Hl[r] - open, e_ext = E[r] - gap;
                const int en = max(e_opn, e_ext);
                const int hdag = hd + sc;
                int hn = max(max(hdag, en), fn);
                if (ALG == PB_SW) hn = max(hn, 0);
                int hM = 0, hS = 0, hL = 0, fM = 0, fS = 0, fL = 0;
                if (STATS) {
                    /* src/sw_stats.c:205-237 */
                    if (f_opn > f_ext) { fM = huM; fS = huS; fL = huL; }
                    else { fM = fuM; fS = fuS; fL = fuL; }
                    fL += 1;
                    if (e_opn > e_ext) { EM[r] = HlM[r]; ES[r] = HlS[r]; EL[r] = HlL[r]; }
                    EL[r] += 1;
                    if (hn == hdag) {
                        const int mt = real ? (pd.qcodes[i] == code) : 0;
                        hM = hdM + mt; hS = hdS + (sc > 0); hL = hdL + 1;
                    } else if (hn == fn) {
                        hM = fM; hS = fS; hL = fL;
                    } else {
                        hM = EM[r]; hS = ES[r]; hL = EL[r];
                    }
                    if (ALG == PB_SW && hn <= 0) { hM = hS = hL = 0; }
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
                /* shift: this cell's left value becomes the next row's diagonal */
                hd = Hl[r];
                if (STATS) { hdM = HlM[r]; hdS = HlS[r]; hdL = HlL[r]; }
                Hl[r] = hn;
                if (STATS) { HlM[r] = hM; HlS[r] = hS; HlL[r] = hL; }
                hu = hn; fu = fn;
                if (STATS) { huM = hM; huS = hS; huL = hL; fuM = fM; fuS = fS; fuL = fL; }
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

template <int ALG, bool STATS>
static void launch_alg(const ExactParams &p, cudaStream_t st)
{
    constexpr int R = STATS ? 8 : 16;
    const int threads = 128;
    const int blocks = (p.npairs + threads - 1) / threads;
    k_exact<ALG, STATS, R><<<blocks, threads, 0, st>>>(p);
}

void launch_exact(const ExactParams &p, int alg, bool stats, cudaStream_t st)
{
    if (p.npairs <= 0) return;
    if (alg == PB_SW) { if (stats) launch_alg<PB_SW, true>(p, st); else launch_alg<PB_SW, false>(p, st); }
    else if (alg == PB_NW) { if (stats) launch_alg<PB_NW, true>(p, st); else launch_alg<PB_NW, false>(p, st); }
    else { if (stats) launch_alg<PB_SG, true>(p, st); else launch_alg<PB_SG, false>(p, st); }
}

}  // namespace pb
