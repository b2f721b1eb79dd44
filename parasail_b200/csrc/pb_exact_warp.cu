/*
 * pb_exact_warp.cu -- the exact 32-bit kernel for long queries, score only:
 * one warp per pair instead of one thread.
 *
 * The thread-per-pair kernel (pb_exact.cu) runs a pair's strips one after
 * another on one thread, so a launch lasts as long as its largest pair
 * (2000 x 5000 residues took about 0.9 s). Here a pass covers 32 x R query
 * rows: lane k holds rows r0 + kR .. r0 + kR + R - 1 and at iteration t
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

static constexpr int EW_R = 16;            /* query rows per lane */
static constexpr int EW_WARPS = 4;         /* warps per block */

__device__ __forceinline__ bool ew_better(int h, int j, int i, int bh, int bj, int bi)
{
    return h > bh || (h == bh && (j < bj || (j == bj && i < bi)));
}

template <int ALG>
__global__ void __launch_bounds__(EW_WARPS * 32)
k_exact_warp(ExactParams p, int nitems)
{
    const int lane = threadIdx.x & 31;
    const int item = blockIdx.x * EW_WARPS + (threadIdx.x >> 5);
    if (item >= nitems) return;
    const int pid = p.order[item];
    const int ti = pid % p.nt;
    const ProfDesc pd = p.profs[pid / p.nt];
    const uint8_t *tseq = p.targets + p.toff[ti];
    const int ql = pd.qlen;
    const int tl = p.tlen[ti];
    const int open = p.open, gap = p.gap, sgf = p.sgflags;
    const int c8 = (ql + 7) & ~7, c16 = (ql + 15) & ~15, c32 = (ql + 31) & ~31;
    const int nrows = p.pad_rows == 0 ? ql : (p.pad_rows == 8 ? c8 : (p.pad_rows == 16 ? c16 : c32));
    int2 *buf = reinterpret_cast<int2 *>(p.scratch + p.soff[pid]);   /* tl x (H, F) */

    int max_h = INT32_MIN, min_h_real = INT32_MAX, min_f_real = INT32_MAX;
    int min_h_pad0 = INT32_MAX, min_h_pad1 = INT32_MAX, min_h_pad2 = INT32_MAX;
    int min_f_pad0 = INT32_MAX, min_f_pad1 = INT32_MAX, min_f_pad2 = INT32_MAX;
    int status = 0;
    int best_h = NEG_INF, best_i = ql, best_j = tl;     /* SW */
    int lc_h = NEG_INF, lc_i = -1;                      /* SG last column, rows < ql - 1 */
    int lr_h = NEG_INF, lr_j = -1;                      /* last row (owner lane) */
    int corner_h = 0;                                   /* owner lane */

    const int pass_rows = 32 * EW_R;
    for (int r0 = 0; r0 < nrows; r0 += pass_rows) {
        const int R0 = r0 + lane * EW_R;
        int Hl[EW_R], E[EW_R];
#pragma unroll
        for (int r = 0; r < EW_R; ++r) {
            Hl[r] = left_h<ALG>(R0 + r, open, gap, sgf);
            E[r] = NEG_INF;
        }
        /* H(R0 - 1, j - 1), starting at column -1 */
        int dg = R0 == 0 ? 0 : left_h<ALG>(R0 - 1, open, gap, sgf);
        int sh_h = NEG_INF, sh_f = NEG_INF;       /* this lane's last row at its previous column */
        const bool more = r0 + pass_rows < nrows;
        for (int it = 0; it < tl + 31; ++it) {
            const int j = it - lane;
            int up_h = __shfl_up_sync(0xffffffffu, sh_h, 1);
            int up_f = __shfl_up_sync(0xffffffffu, sh_f, 1);
            if (j < 0 || j >= tl) continue;
            if (lane == 0) {
                if (r0 == 0) { up_h = top_h<ALG>(j, open, gap, sgf); up_f = NEG_INF; }
                else { const int2 v = buf[j]; up_h = v.x; up_f = v.y; }
            }
            const int code = tseq[j];
            if (code >= pd.size) status |= PB_ST_BADCODE;
            const int csafe = code < pd.size ? code : 0;
            const int32_t *prow = pd.prof + (size_t)csafe * pd.lp;
            int hu = up_h, fu = up_f;
            int hd = dg;
            dg = up_h;
#pragma unroll
            for (int r = 0; r < EW_R; ++r) {
                const int i = R0 + r;
                const bool real = i < ql;
                const int sc = real ? prow[i] : 0;
                const int fn = max(hu - open, fu - gap);
                const int en = max(Hl[r] - open, E[r] - gap);
                int hn = max(max(hd + sc, en), fn);
                if (ALG == PB_SW) hn = max(hn, 0);
                E[r] = en;
                if (i < nrows) {
                    max_h = max(max_h, hn);
                    if (real) {
                        min_h_real = min(min_h_real, hn);
                        min_f_real = min(min_f_real, fn);
                    } else if (i < c8) {
                        min_h_pad0 = min(min_h_pad0, hn);
                        min_f_pad0 = min(min_f_pad0, fn);
                    } else if (i < c16) {
                        min_h_pad1 = min(min_h_pad1, hn);
                        min_f_pad1 = min(min_f_pad1, fn);
                    } else {
                        min_h_pad2 = min(min_h_pad2, hn);
                        min_f_pad2 = min(min_f_pad2, fn);
                    }
                }
                if (real) {
                    if (ALG == PB_SW) {
                        if (ew_better(hn, j, i, best_h, best_j, best_i)) { best_h = hn; best_i = i; best_j = j; }
                    } else if (i == ql - 1) {
                        if (hn > lr_h) { lr_h = hn; lr_j = j; }
                        if (j == tl - 1) corner_h = hn;
                    } else if (ALG == PB_SG && j == tl - 1) {
                        if (hn > lc_h) { lc_h = hn; lc_i = i; }
                    }
                }
                hd = Hl[r];
                Hl[r] = hn;
                hu = hn;
                fu = fn;
            }
            sh_h = hu;
            sh_f = fu;
            /* the next pass's lane 0 reads column j; this pass's lane 0 has
             * read it 31 iterations ago */
            if (lane == 31 && more) buf[j] = make_int2(hu, fu);
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
        const int bh = __shfl_xor_sync(0xffffffffu, best_h, o);
        const int bi = __shfl_xor_sync(0xffffffffu, best_i, o);
        const int bj = __shfl_xor_sync(0xffffffffu, best_j, o);
        if (ew_better(bh, bj, bi, best_h, best_j, best_i)) { best_h = bh; best_i = bi; best_j = bj; }
        const int ch = __shfl_xor_sync(0xffffffffu, lc_h, o);
        const int ci = __shfl_xor_sync(0xffffffffu, lc_i, o);
        if (ci >= 0 && (lc_i < 0 || ch > lc_h || (ch == lc_h && ci < lc_i))) { lc_h = ch; lc_i = ci; }
    }
    /* the last row and the corner: the lane holding row ql - 1 */
    const int owner = ((ql - 1) % pass_rows) / EW_R;
    lr_h = __shfl_sync(0xffffffffu, lr_h, owner);
    lr_j = __shfl_sync(0xffffffffu, lr_j, owner);
    corner_h = __shfl_sync(0xffffffffu, corner_h, owner);
    if (lane != 0) return;

    int res, eq, er;
    if (ALG == PB_SW) {
        res = best_h; eq = best_i; er = best_j;
    } else if (ALG == PB_NW) {
        res = corner_h; eq = ql - 1; er = tl - 1;
    } else {
        /* src/sg.c:160-242 */
        const bool s1e = sgf & PB_S1_END, s2e = sgf & PB_S2_END;
        res = NEG_INF;
        eq = ql; er = tl;
        if (s1e && lc_i >= 0) { res = lc_h; eq = lc_i; er = tl - 1; }
        if (s1e && s2e) {
            if (lr_h > res || (lr_h == res && lr_j < er)) { res = lr_h; eq = ql - 1; er = lr_j; }
        } else if (s2e) {
            if (lr_h > res) { res = lr_h; eq = ql - 1; er = lr_j; }
        }
        if ((s1e && corner_h > res) || (!s1e && !s2e)) { res = corner_h; eq = ql - 1; er = tl - 1; }
    }
    pb_pair_out o;
    o.score = res; o.end_query = eq; o.end_ref = er;
    o.matches = 0; o.similar = 0; o.length = 0;
    o.max_h = max_h; o.min_h_real = min_h_real; o.max_stat_real = INT32_MIN;
    o.min_f_real = min_f_real;
    o.min_h_pad[0] = min_h_pad0; o.min_h_pad[1] = min_h_pad1; o.min_h_pad[2] = min_h_pad2;
    o.max_stat_pad[0] = INT32_MIN; o.max_stat_pad[1] = INT32_MIN; o.max_stat_pad[2] = INT32_MIN;
    o.min_f_pad[0] = min_f_pad0; o.min_f_pad[1] = min_f_pad1; o.min_f_pad[2] = min_f_pad2;
    o.status = status;
    p.out[pid] = o;
}

void launch_exact_warp(const ExactParams &p, int alg, int nitems, cudaStream_t st)
{
    if (nitems <= 0) return;
    const int blocks = (nitems + EW_WARPS - 1) / EW_WARPS;
    if (alg == PB_SW) k_exact_warp<PB_SW><<<blocks, EW_WARPS * 32, 0, st>>>(p, nitems);
    else if (alg == PB_NW) k_exact_warp<PB_NW><<<blocks, EW_WARPS * 32, 0, st>>>(p, nitems);
    else k_exact_warp<PB_SG><<<blocks, EW_WARPS * 32, 0, st>>>(p, nitems);
}

}  // namespace pb
