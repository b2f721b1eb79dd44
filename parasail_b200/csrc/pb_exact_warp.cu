/*
 * pb_exact_warp.cu -- the exact 32-bit kernel for long pairs: one warp per
 * pair instead of one thread, score only or with statistics.
 *
 * The thread-per-pair kernel (pb_exact.cu) runs a pair's strips one after
 * another on one thread, so a launch lasts as long as its largest pair
 * (2000 x 5000 residues took about 0.9 s). Here a pass covers 32 x R query
 * rows (R = 16 score-only, 8 with statistics): lane k holds rows
 * r0 + kR .. r0 + kR + R - 1 and at iteration t
 * computes target column t - k, so the row above its first row is lane
 * k-1's last row at the same column, computed one iteration earlier and
 * passed by one warp shuffle. Passes run one after another on the warp;
 * lane 31 leaves its bottom row in the pair's buffer for the next pass's
 * lane 0 (the buffer is overwritten 31 columns behind the reads).
 *
 * Every cell follows exact_pair (pb_exact_core.cuh) exactly: the same
 * recurrence and boundaries (src/sw.c:131-158, src/nw.c:131-156,
 * src/sg.c:142-242), the same extremes per row region for the width
 * verdicts, and the same end rules. Each lane keeps its own partial ends
 * and extremes, merged across the warp at the end: SW best by score, then
 * column, then row; SG last column by score, then row; the last row and
 * the corner come from the lane that holds row ql - 1.
 */
#include "pb_exact_core.cuh"

namespace pb {

static constexpr int EW_WARPS = 4;         /* warps per block */

/* rows per lane */
template <bool STATS> struct EwRows { static constexpr int value = STATS ? 8 : 16; };

/* a cell's score with its statistics (matches, similar, length) */
struct EwCell { int h, m, s, l; };

__device__ __forceinline__ bool ew_better(int h, int j, int i, int bh, int bj, int bi)
{
    return h > bh || (h == bh && (j < bj || (j == bj && i < bi)));
}

__device__ __forceinline__ EwCell ew_shfl_xor(const EwCell &c, int o)
{
    return EwCell{__shfl_xor_sync(0xffffffffu, c.h, o), __shfl_xor_sync(0xffffffffu, c.m, o),
                  __shfl_xor_sync(0xffffffffu, c.s, o), __shfl_xor_sync(0xffffffffu, c.l, o)};
}

__device__ __forceinline__ EwCell ew_shfl(const EwCell &c, int src)
{
    return EwCell{__shfl_sync(0xffffffffu, c.h, src), __shfl_sync(0xffffffffu, c.m, src),
                  __shfl_sync(0xffffffffu, c.s, src), __shfl_sync(0xffffffffu, c.l, src)};
}

/* PAIRS: pair k has its own query codes (qall + qoff[k], qlen[k]) scored
 * through the square matrix mat[target letter * msize + query letter];
 * else profiles: every query of profs against the same nt targets, or
 * (nt = 0) pair k's profile profs[prof_index[k]] against target k */
template <int ALG, bool STATS, bool PAIRS, bool SCANF>
__global__ void __launch_bounds__(EW_WARPS * 32)
k_exact_warp(ExactParams p, int nitems)
{
    constexpr int EW_R = EwRows<STATS>::value;
    const int lane = threadIdx.x & 31;
    const int item = blockIdx.x * EW_WARPS + (threadIdx.x >> 5);
    if (item >= nitems) return;
    const int pid = p.order[item];
    const int ti = PAIRS || !p.nt ? pid : pid % p.nt;
    ProfDesc pd;
    const uint8_t *qseq = nullptr;
    if (PAIRS) {
        qseq = p.qall + p.qoff[pid];
        pd.prof = nullptr; pd.qcodes = nullptr; pd.lp = 0; pd.qlen = p.qlen[pid]; pd.size = p.msize;
    } else {
        /* every query against nt targets, or one profile per pair */
        pd = p.profs[p.nt ? pid / p.nt : (p.prof_index ? p.prof_index[pid] : 0)];
    }
    const uint8_t *tseq = p.targets + p.toff[ti];
    const int ql = p.qlim ? p.qlim[pid] : pd.qlen;       /* a prefix of the pair when limited */
    const int tl = p.tlim ? p.tlim[pid] : p.tlen[ti];
    const int open = p.open, gap = p.gap, sgf = p.sgflags;
    const int c8 = (ql + 7) & ~7, c16 = (ql + 15) & ~15, c32 = (ql + 31) & ~31;
    const int nrows = p.pad_rows == 0 ? ql : (p.pad_rows == 8 ? c8 : (p.pad_rows == 16 ? c16 : c32));
    /* the pass hand-off, per column: (H, F), or with statistics
     * (H, F, HM, HS) and (HL, FM, FS, FL) */
    int2 *buf = reinterpret_cast<int2 *>(p.scratch + p.soff[pid]);
    int4 *buf4 = reinterpret_cast<int4 *>(p.scratch + p.soff[pid]);

    int max_h = INT32_MIN, min_h_real = INT32_MAX, min_f_real = INT32_MAX;
    int min_h_pad0 = INT32_MAX, min_h_pad1 = INT32_MAX, min_h_pad2 = INT32_MAX;
    int min_f_pad0 = INT32_MAX, min_f_pad1 = INT32_MAX, min_f_pad2 = INT32_MAX;
    int max_st_real = INT32_MIN, max_st_pad0 = INT32_MIN, max_st_pad1 = INT32_MIN, max_st_pad2 = INT32_MIN;
    int status = 0;
    EwCell best = {NEG_INF, 0, 0, 0};                   /* SW */
    int best_i = ql, best_j = tl;
    EwCell lc = {NEG_INF, 0, 0, 0};                     /* SG last column, rows < ql - 1 */
    int lc_i = -1;
    EwCell lr = {NEG_INF, 0, 0, 0};                     /* last row (owner lane) */
    int lr_j = -1;
    EwCell corner = {0, 0, 0, 0};                       /* owner lane */

    const int pass_rows = 32 * EW_R;
    for (int r0 = 0; r0 < nrows; r0 += pass_rows) {
        const int R0 = r0 + lane * EW_R;
        int qc[PAIRS ? EW_R : 1];
        if (PAIRS) {
#pragma unroll
            for (int r = 0; r < EW_R; ++r) {
                int c = R0 + r < ql ? qseq[R0 + r] : 0;
                if (c >= p.msize) { status |= PB_ST_BADCODE; c = 0; }
                qc[r] = c;
            }
        }
        int Hl[EW_R], E[EW_R];
        int HlM[EW_R], HlS[EW_R], HlL[EW_R], EM[EW_R], ES[EW_R], EL[EW_R];
#pragma unroll
        for (int r = 0; r < EW_R; ++r) {
            Hl[r] = left_h<ALG>(R0 + r, open, gap, sgf);
            E[r] = NEG_INF;
            if (STATS) { HlM[r] = HlS[r] = HlL[r] = 0; EM[r] = ES[r] = EL[r] = 0; }
        }
        /* H(R0 - 1, j - 1), starting at column -1 */
        int dg = R0 == 0 ? 0 : left_h<ALG>(R0 - 1, open, gap, sgf);
        int dgM = 0, dgS = 0, dgL = 0;
        /* this lane's last row at its previous column */
        int sh_h = NEG_INF, sh_f = NEG_INF, sh_hM = 0, sh_hS = 0, sh_hL = 0, sh_fM = 0, sh_fS = 0, sh_fL = 0;
        const bool more = r0 + pass_rows < nrows;
        for (int it = 0; it < tl + 31; ++it) {
            const int j = it - lane;
            int up_h = __shfl_up_sync(0xffffffffu, sh_h, 1);
            int up_f = __shfl_up_sync(0xffffffffu, sh_f, 1);
            int huM = 0, huS = 0, huL = 0, fuM = 0, fuS = 0, fuL = 0;
            if (STATS) {
                huM = __shfl_up_sync(0xffffffffu, sh_hM, 1);
                huS = __shfl_up_sync(0xffffffffu, sh_hS, 1);
                huL = __shfl_up_sync(0xffffffffu, sh_hL, 1);
                fuM = __shfl_up_sync(0xffffffffu, sh_fM, 1);
                fuS = __shfl_up_sync(0xffffffffu, sh_fS, 1);
                fuL = __shfl_up_sync(0xffffffffu, sh_fL, 1);
            }
            if (j < 0 || j >= tl) continue;
            if (lane == 0) {
                if (r0 == 0) {
                    up_h = top_h<ALG>(j, open, gap, sgf); up_f = SCANF ? up_h - open : NEG_INF;
                    huM = huS = huL = fuM = fuS = fuL = 0;
                    if (SCANF && STATS) fuL = ~0;   /* F of row 0 from the top (exact_pair's SCANF) */
                } else if (STATS) {
                    const int4 a = buf4[2 * j], b = buf4[2 * j + 1];
                    up_h = a.x; up_f = a.y; huM = a.z; huS = a.w; huL = b.x; fuM = b.y; fuS = b.z; fuL = b.w;
                } else {
                    const int2 v = buf[j]; up_h = v.x; up_f = v.y;
                }
            }
            const int code = tseq[j];
            if (code >= pd.size) status |= PB_ST_BADCODE;
            const int csafe = code < pd.size ? code : 0;
            const int32_t *prow = PAIRS ? p.mat + (size_t)csafe * p.msize : pd.prof + (size_t)csafe * pd.lp;
            int hu = up_h, fu = up_f;
            int hd = dg, hdM = dgM, hdS = dgS, hdL = dgL;
            dg = up_h;
            if (STATS) { dgM = huM; dgS = huS; dgL = huL; }
#pragma unroll
            for (int r = 0; r < EW_R; ++r) {
                const int i = R0 + r;
                const bool real = i < ql;
                const int sc = real ? (PAIRS ? __ldg(&prow[qc[r]]) : prow[i]) : 0;
                const int f_opn = hu - open, f_ext = fu - gap;
                const int fn = SCANF ? fu : max(f_opn, f_ext);
                const int e_opn = Hl[r] - open, e_ext = E[r] - gap;
                const int en = max(e_opn, e_ext);
                const int hdag = hd + sc;
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
                    const int mt = real ? ((PAIRS ? qc[r] : (int)pd.qcodes[i]) == code) : 0;
                    hM = isd ? hdM + mt : (isf ? fM : eM);
                    hS = isd ? hdS + (sc > 0) : (isf ? fS : eS);
                    hL = isd ? hdL + 1 : (isf ? fL : eL);
                    if (ALG == PB_SW) {
                        const bool z = hn <= 0;
                        hM = z ? 0 : hM;
                        hS = z ? 0 : hS;
                        hL = z ? 0 : hL;
                    }
                }
                E[r] = en;
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
                if (real) {
                    if (ALG == PB_SW) {
                        if (ew_better(hn, j, i, best.h, best_j, best_i)) {
                            best = EwCell{hn, hM, hS, hL}; best_i = i; best_j = j;
                        }
                    } else if (i == ql - 1) {
                        if (hn > lr.h) { lr = EwCell{hn, hM, hS, hL}; lr_j = j; }
                        if (j == tl - 1) corner = EwCell{hn, hM, hS, hL};
                    } else if (ALG == PB_SG && j == tl - 1) {
                        if (hn > lc.h) { lc = EwCell{hn, hM, hS, hL}; lc_i = i; }
                    }
                }
                hd = Hl[r];
                Hl[r] = hn;
                hu = hn;
                fu = SCANF ? max(ht - open, fn - gap) : fn;
                if (STATS) {
                    hdM = HlM[r]; hdS = HlS[r]; hdL = HlL[r];
                    HlM[r] = hM; HlS[r] = hS; HlL[r] = hL;
                    huM = hM; huS = hS; huL = hL; fuM = fM; fuS = fS;
                    fuL = (SCANF && ht - open > fn - gap) ? ~fL : fL;
                }
            }
            sh_h = hu;
            sh_f = fu;
            if (STATS) { sh_hM = huM; sh_hS = huS; sh_hL = huL; sh_fM = fuM; sh_fS = fuS; sh_fL = fuL; }
            /* the next pass's lane 0 reads column j; this pass's lane 0 has
             * read it 31 iterations ago */
            if (lane == 31 && more) {
                if (STATS) {
                    buf4[2 * j] = make_int4(hu, fu, huM, huS);
                    buf4[2 * j + 1] = make_int4(huL, fuM, fuS, fuL);
                } else {
                    buf[j] = make_int2(hu, fu);
                }
            }
        }
        __syncwarp();
    }

    /* merge the lanes */
    for (int o = 16; o; o >>= 1) {
        max_h = max(max_h, __shfl_xor_sync(0xffffffffu, max_h, o));
        min_h_real = min(min_h_real, __shfl_xor_sync(0xffffffffu, min_h_real, o));
        min_f_real = min(min_f_real, __shfl_xor_sync(0xffffffffu, min_f_real, o));
        min_h_pad0 = min(min_h_pad0, __shfl_xor_sync(0xffffffffu, min_h_pad0, o));
        min_h_pad1 = min(min_h_pad1, __shfl_xor_sync(0xffffffffu, min_h_pad1, o));
        min_h_pad2 = min(min_h_pad2, __shfl_xor_sync(0xffffffffu, min_h_pad2, o));
        min_f_pad0 = min(min_f_pad0, __shfl_xor_sync(0xffffffffu, min_f_pad0, o));
        min_f_pad1 = min(min_f_pad1, __shfl_xor_sync(0xffffffffu, min_f_pad1, o));
        min_f_pad2 = min(min_f_pad2, __shfl_xor_sync(0xffffffffu, min_f_pad2, o));
        status |= __shfl_xor_sync(0xffffffffu, status, o);
        max_st_real = max(max_st_real, __shfl_xor_sync(0xffffffffu, max_st_real, o));
        max_st_pad0 = max(max_st_pad0, __shfl_xor_sync(0xffffffffu, max_st_pad0, o));
        max_st_pad1 = max(max_st_pad1, __shfl_xor_sync(0xffffffffu, max_st_pad1, o));
        max_st_pad2 = max(max_st_pad2, __shfl_xor_sync(0xffffffffu, max_st_pad2, o));
        const EwCell bc = ew_shfl_xor(best, o);
        const int bi = __shfl_xor_sync(0xffffffffu, best_i, o);
        const int bj = __shfl_xor_sync(0xffffffffu, best_j, o);
        if (ew_better(bc.h, bj, bi, best.h, best_j, best_i)) { best = bc; best_i = bi; best_j = bj; }
        const EwCell cc = ew_shfl_xor(lc, o);
        const int ci = __shfl_xor_sync(0xffffffffu, lc_i, o);
        if (ci >= 0 && (lc_i < 0 || cc.h > lc.h || (cc.h == lc.h && ci < lc_i))) { lc = cc; lc_i = ci; }
    }
    /* the last row and the corner: the lane holding row ql - 1 */
    const int owner = ((ql - 1) % pass_rows) / EW_R;
    lr = ew_shfl(lr, owner);
    lr_j = __shfl_sync(0xffffffffu, lr_j, owner);
    corner = ew_shfl(corner, owner);
    if (lane != 0) return;

    EwCell res;
    int eq, er;
    if (ALG == PB_SW) {
        res = best; eq = best_i; er = best_j;
    } else if (ALG == PB_NW) {
        res = corner; eq = ql - 1; er = tl - 1;
    } else {
        /* src/sg.c:160-242 */
        const bool s1e = sgf & PB_S1_END, s2e = sgf & PB_S2_END;
        res = EwCell{NEG_INF, 0, 0, 0};
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

template <bool STATS, bool PAIRS, bool SCANF = false>
static void launch_ew(const ExactParams &p, int alg, int nitems, cudaStream_t st)
{
    const int blocks = (nitems + EW_WARPS - 1) / EW_WARPS;
    if (alg == PB_SW) k_exact_warp<PB_SW, STATS, PAIRS, SCANF><<<blocks, EW_WARPS * 32, 0, st>>>(p, nitems);
    else if (alg == PB_NW) k_exact_warp<PB_NW, STATS, PAIRS, SCANF><<<blocks, EW_WARPS * 32, 0, st>>>(p, nitems);
    else k_exact_warp<PB_SG, STATS, PAIRS, SCANF><<<blocks, EW_WARPS * 32, 0, st>>>(p, nitems);
}

void launch_exact_warp(const ExactParams &p, int alg, bool stats, int nitems, cudaStream_t st)
{
    if (nitems <= 0) return;
    const bool pairs = p.mat != nullptr;
    if (p.scan_vgap) {
        /* the serial scan forms' vertical gap, one query per call */
        if (stats) launch_ew<true, false, true>(p, alg, nitems, st); else launch_ew<false, false, true>(p, alg, nitems, st);
    } else if (stats) {
        if (pairs) launch_ew<true, true>(p, alg, nitems, st); else launch_ew<true, false>(p, alg, nitems, st);
    } else {
        if (pairs) launch_ew<false, true>(p, alg, nitems, st); else launch_ew<false, false>(p, alg, nitems, st);
    }
}

int exact_warp_pass_rows(bool stats) { return 32 * (stats ? EwRows<true>::value : EwRows<false>::value); }

}  // namespace pb
