/*
 * pb_pair16.cu -- global (NW), semi-global (SG) and local (SW) alignment of
 * batches of independent pairs in packed int16x2 lanes, with statistics
 * (matches, similar, length) from a traceback walk over direction bits.
 *
 * Inter-task schedule: one thread aligns one pair; a warp takes a task of
 * 32 pairs of like size (items sorted by passes and columns); a persistent
 * grid pulls tasks in order of cost. The query is processed in passes of
 * 2 x 16 rows lag-packed in int16x2 words, as in the Smith-Waterman
 * database kernel (pb_sw16.cu): the low half of every register holds strip
 * A (rows r0..r0+15) at column j, the high half strip B (rows r0+16..r0+31)
 * at column j-1, so strip B reads strip A's bottom row from the previous
 * iteration. A pass hands its bottom row (H and F) to the next pass through
 * the warp's buffer laid out [column][lane] (one 256-byte transaction per
 * warp access). Each lane (pairs mode) or each warp (all 32 pairs of the
 * task share a query) stages the scores of the pass's 32 rows against every
 * alphabet letter in shared memory as int8 (a column's 16 + 16 scores are
 * two 16-byte loads expanded by sign-extending byte permutes).
 *
 * Semantics are the reference's serial dynamic programs (src/sw.c:102-158,
 * src/nw.c:102-156, src/sg.c:117-242 and the _stats twins), which its
 * striped and scan kernels reproduce for every non-saturated result:
 *   F(i,j) = max(H(i-1,j) - open, F(i-1,j) - gap)    vertical gap
 *   E(i,j) = max(H(i,j-1) - open, E(i,j-1) - gap)    horizontal gap
 *   H(i,j) = max(H(i-1,j-1) + s(i,j), E(i,j), F(i,j)) (SW: and 0)
 * with the boundaries of src/nw.c:102-120 and src/sg.c:117-143, and the end
 * rules of src/sw.c:150-158 (first maximum in column-major order) and
 * src/sg.c:160-242.
 *
 * Exactness in 16 bits. An item runs here only when sound bounds keep
 * every value it computes, padded rows included, inside int16 with the
 * differences below as well: every H is at most max(matrix) x (min(rows,
 * cols) + 1), and at least -(3 open + (rows32 + cols + 2) gap) + min(matrix)
 * (a path of two gaps reaches any cell); E and F are at least H - open.
 * "-inf" is a per-lane value NEG = LB - open - 1, which no gap opened from
 * a real cell can tie. Items outside the bounds run on the exact 32-bit
 * kernel instead.
 *
 * Statistics. The reference's statistics recurrence (src/sw_stats.c:
 * 204-264, src/nw_stats.c:190-218, src/sg_stats.c:227-265) carries, with
 * every H, E and F, the counts of the one path its tie rules select: the
 * gap source by strict > (open only when H - open > E - gap), the cell
 * source diagonal, then F, then E; SW restarts at H <= 0 and the boundary
 * cells carry 0. Those counts are the counts along that path. With
 * statistics the kernel stores, per cell, the four decisions that define
 * the path: not-diagonal (H > H_diag + s), not-F (H > F), E opened and F
 * opened -- each the sign bit of an int16 difference, shifted into per-row
 * bit accumulators: bit r (low half, strip A) and 16 + r (high half, strip
 * B) of four words stored as one uint4 per lane per iteration. The walk
 * (k_p16_walk) then follows the path back from the end cell, adding 1 to
 * length per step and, on diagonal steps, the match and positive-score
 * indicators; in SW it stops where the running H value (the end score
 * minus the steps walked) reaches 0, in NW/SG at the boundary.
 */
#include <cstdio>
#include <cstdint>
#include <climits>
#include <cstring>
#include <algorithm>
#include <vector>

#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <dlfcn.h>
#include <mutex>
#include <string>

#include "pb_cuda.h"
#include "pb_kernels.cuh"
#include "pb_resolve.h"

namespace pb {

static constexpr int P16_R = 16;              /* rows per strip; two strips per pass */
static constexpr int P16_PASS = 2 * P16_R;

__device__ __forceinline__ uint32_t p16_prmt(uint32_t a, uint32_t b, uint32_t sel)
{
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
    return d;
}

/* byte K of a (low half) and of b (high half), sign-extended to int16x2 */
template <int K>
__device__ __forceinline__ uint32_t p16_pair(uint32_t a, uint32_t b)
{
    constexpr uint32_t sel = (K) | ((K | 8) << 4) | ((4 + K) << 8) | (((4 + K) | 8) << 12);
    return p16_prmt(a, b, sel);
}

__device__ __forceinline__ uint32_t p16_splat(int v) { return ((uint32_t)(uint16_t)v) | ((uint32_t)(uint16_t)v << 16); }
__device__ __forceinline__ int p16_lo(uint32_t x) { return (int)(int16_t)(x & 0xffffu); }
__device__ __forceinline__ int p16_hi(uint32_t x) { return (int)(int16_t)(x >> 16); }

/* The bounds of one item (see the file comment). */
struct P16Bounds {
    int lb, ub;
};

__host__ __device__ __forceinline__ P16Bounds p16_bounds(int alg, int rows, int cols, int open, int gap,
                                                         int mmax, int mmin)
{
    P16Bounds b;
    const long long r32 = ((long long)rows + 31) / 32 * 32;
    const long long mn = mmin < 0 ? mmin : 0, mx = mmax > 0 ? mmax : 0;
    const long long ub = mx * ((rows < cols ? rows : cols) + 1);
    long long lb = alg == PB_SW ? mn : -(3LL * open + (r32 + cols + 2) * (long long)gap) + mn;
    b.lb = lb < INT_MIN / 2 ? INT_MIN / 2 : (int)lb;
    b.ub = ub > INT_MAX / 2 ? INT_MAX / 2 : (int)ub;
    return b;
}

__host__ __device__ __forceinline__ bool p16_fits(const P16Bounds &b, int open, int gap)
{
    return (long long)b.ub - b.lb + open + gap + 1 <= 32000;
}

/* boundary H of row -1 (column j) and column -1 (row i); H(-1,-1) = 0 */
__device__ __forceinline__ int p16_top(int alg, int sgf, int j, int open, int gap)
{
    if (alg == PB_SW || (alg == PB_SG && (sgf & PB_S2_BEG))) return 0;
    return -open - j * gap;
}

__device__ __forceinline__ int p16_left(int alg, int sgf, int i, int open, int gap)
{
    if (i < 0) return 0;
    if (alg == PB_SW || (alg == PB_SG && (sgf & PB_S1_BEG))) return 0;
    return -open - i * gap;
}

struct P16Best {
    int score, i, j;
};

/*
 * One task (32 items) per warp at a time. SHARED: every lane of a task has
 * the same query (its scores are staged once per warp); else every lane
 * stages its own. BITS: store the direction bits. ENDS: compute score and
 * ends (off for the FASTSTATS prefix pass, whose ends are known).
 */
template <int ALG, bool BITS, bool ENDS, bool SHARED, int WARPS>
__global__ void __launch_bounds__(WARPS * 32, (WARPS == 8 ? 2 : 4))
k_p16(P16Params p, const int *__restrict__ tlist, int ntl, int *counter)
{
    extern __shared__ __align__(16) int8_t s_mem[];
    const int L = p.nletters;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    /* shared memory: [matrix L x L int8, padded to 16] [per-warp score slices] */
    const int mat_bytes = p.mat8 ? ((L * L + 15) & ~15) : 0;
    const int lane_stride = SHARED ? 0 : L * P16_PASS + 16;
    const int warp_bytes = SHARED ? L * P16_PASS : 32 * lane_stride;
    int8_t *s_mat = s_mem;
    int8_t *wslice = s_mem + mat_bytes + wid * warp_bytes;
    int8_t *myslice = wslice + lane * lane_stride;
    if (p.mat8)
        for (int k = threadIdx.x; k < L * L; k += blockDim.x) s_mat[k] = p.mat8[k];
    __syncthreads();

    /* pass boundary: strip B's bottom row per column, H low and F high */
    uint32_t *buf = p.scratch + (size_t)(blockIdx.x * WARPS + wid) * (size_t)(p.maxlen + 1) * 32;
    /* SW ends: this thread's copies of its strips' best columns */
    uint4 *save = ENDS && ALG == PB_SW ? p.colsave + ((size_t)blockIdx.x * blockDim.x + threadIdx.x) * (P16_R / 2)
                                       : nullptr;
    const int open = p.open, gap = p.gap, sgf = p.sgflags;
    const uint32_t gO = p16_splat(-open), gE = p16_splat(-gap);
    const int nwarps_total = gridDim.x * WARPS;
    bool first = true;
    for (;;) {
        int k;
        if (first) {
            k = blockIdx.x + gridDim.x * wid;
            first = false;
        } else {
            if (lane == 0) k = nwarps_total + atomicAdd(counter, 1);
            k = __shfl_sync(0xffffffffu, k, 0);
        }
        if (k >= ntl) break;
        const int task = tlist[k];
        const int s = task * 32 + lane;
        const bool valid = s < p.nitems && p.order[s] >= 0;
        const int item = valid ? p.order[s] : 0;
        const int rows = valid ? p.rows[item] : 0;
        const int cols = valid ? p.cols[item] : 0;
        const int wmax = p.task_wmax[task];
        const int npass = p.task_npass[task];
        const int ti = p.nt ? item % p.nt : item;
        const uint8_t *tseq = p.targets + (valid ? p.toff[ti] : 0);
        /* query source */
        const uint8_t *qseq = nullptr;
        const int8_t *prof8 = nullptr;
        int lp = 0;
        if (p.mat8) {
            qseq = p.qall + (valid ? p.qoff[item] : 0);
        } else {
            /* an invalid lane (a task's padding) takes the task's query:
             * in the shared variant every lane writes part of the slice
             * from its own profile pointer */
            const int qitem = valid ? item : p.order[task * 32];
            const ProfDesc pd = p.profs[p.nt ? qitem / p.nt : 0];
            prof8 = pd.prof8;
            lp = pd.lp;
        }
        int rmax = rows;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) rmax = max(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
        const uint8_t *qseq0 = SHARED && p.mat8 ? p.qall + p.qoff[p.order[task * 32]] : nullptr;
        const P16Bounds bd = p16_bounds(ALG, rows, cols, open, gap, p.mmax, p.mmin);
        const int negv = bd.lb - open - 1;
        const uint32_t NEG = p16_splat(negv);
        uint4 *tbits = BITS ? p.bits + p.task_bits[task] : nullptr;
        int status = 0;

        /* end tracking */
        P16Best best = {0, 0, 0};
        bool have = false;
        int lc_h = INT_MIN, lc_i = -1;       /* SG: last column over rows < rows - 1 */
        int lr_h = INT_MIN, lr_j = -1;       /* SG: last row */
        int corner = 0;
        const int ilast = rows - 1;
        const int p_last = ilast >> 5, half_last = (ilast >> 4) & 1, r_last = ilast & 15;

        for (int pass = 0; pass < npass; ++pass) {
            const int r0 = pass * P16_PASS;
            /* scores of this pass's 32 rows against every letter: once per
             * warp (shared query) or once per lane; rows past the query
             * (past the task's longest in shared pairs mode) score 0 */
            if (SHARED) {
                __syncwarp();
                if (p.mat8) {
                    const int i = r0 + lane;
                    uint32_t c = i < rmax ? qseq0[i] : 255u;
                    if (c != 255u && c >= (uint32_t)L) { c = 0; status |= PB_ST_BADCODE; }
                    for (int a = 0; a < L; ++a)
                        wslice[a * P16_PASS + lane] = c == 255u ? (int8_t)0 : s_mat[a * L + c];
                } else {
                    for (int x = lane; x < 2 * L; x += 32) {
                        const int a = x >> 1, h = x & 1;
                        const int4 v = *reinterpret_cast<const int4 *>(prof8 + (size_t)a * lp + r0 + 16 * h);
                        *reinterpret_cast<int4 *>(wslice + a * P16_PASS + 16 * h) = v;
                    }
                }
            } else if (p.mat8) {
                uint32_t qc[8];
#pragma unroll
                for (int w = 0; w < 8; ++w) {
                    uint32_t word = 0;
#pragma unroll
                    for (int b = 0; b < 4; ++b) {
                        const int i = r0 + 4 * w + b;
                        uint32_t c = i < rows ? qseq[i] : 255u;
                        if (c != 255u && c >= (uint32_t)L) { c = 0; status |= PB_ST_BADCODE; }
                        word |= c << (8 * b);
                    }
                    qc[w] = word;
                }
                for (int a = 0; a < L; ++a) {
#pragma unroll
                    for (int w = 0; w < 8; ++w) {
                        uint32_t word = 0;
#pragma unroll
                        for (int b = 0; b < 4; ++b) {
                            const uint32_t c = (qc[w] >> (8 * b)) & 0xffu;
                            const uint32_t v = c == 255u ? 0u : (uint32_t)(uint8_t)s_mat[a * L + c];
                            word |= v << (8 * b);
                        }
                        *reinterpret_cast<uint32_t *>(myslice + a * P16_PASS + 4 * w) = word;
                    }
                }
            } else {
                /* db mode, lanes of different queries: each copies its own
                 * (a pass past this lane's profile rows, lp >= qlen + 32, is
                 * beyond its query: zeros) */
                const bool in = r0 + P16_PASS <= lp;
                for (int a = 0; a < L; ++a) {
                    const int4 z = make_int4(0, 0, 0, 0);
                    const int4 *src = reinterpret_cast<const int4 *>(prof8 + (size_t)a * lp + (in ? r0 : 0));
                    *reinterpret_cast<int4 *>(myslice + a * P16_PASS) = in ? src[0] : z;
                    *reinterpret_cast<int4 *>(myslice + a * P16_PASS + 16) = in ? src[1] : z;
                }
            }
            __syncwarp();
            const int8_t *sl = SHARED ? wslice : myslice;

            /* initial state: column -1 */
            uint32_t H[P16_R], E[P16_R];
#pragma unroll
            for (int r = 0; r < P16_R; ++r) {
                const int la = p16_left(ALG, sgf, r0 + r, open, gap);
                const int lb2 = p16_left(ALG, sgf, r0 + P16_R + r, open, gap);
                H[r] = (uint32_t)(uint16_t)la | ((uint32_t)(uint16_t)lb2 << 16);
                E[r] = NEG;
            }
            uint32_t dg = (uint32_t)(uint16_t)p16_left(ALG, sgf, r0 - 1, open, gap);
            uint32_t prev_h = (uint32_t)(uint16_t)p16_left(ALG, sgf, r0 + P16_R - 1, open, gap);
            uint32_t prev_f = NEG & 0xffffu;
            int top = p16_top(ALG, sgf, 0, open, gap);
            const int top_step = (ALG == PB_SW || (ALG == PB_SG && (sgf & PB_S2_BEG))) ? 0 : gap;
            P16Best sa = {0, -1, -1}, sb = {0, -1, -1};
            int cb = 0;
            const bool more = pass + 1 < npass;
            const bool lastpass = ENDS && ALG != PB_SW && pass == p_last;
            const uint32_t vnone = p16_prmt(0u, NEG, 0x5410u);
            auto code_at = [&](int j) -> int {
                int c = j < cols ? tseq[j] : 0;
                if (c >= L) { c = 0; status |= PB_ST_BADCODE; }
                return c;
            };
            int c_n1 = code_at(0);
            int c_n2 = code_at(1);
            uint32_t v_n1 = vnone, v_n2 = vnone;
            if (pass != 0) {
                if (0 <= wmax) v_n1 = __ldcg(&buf[lane]);
                if (1 <= wmax) v_n2 = __ldcg(&buf[32 + lane]);
            }
            /* unrolled by two: the prefetch registers then rotate by renaming
             * instead of by moves, which would wait for the loads */
#pragma unroll 2
            for (int j = 0; j <= wmax; ++j) {
                const int ca = c_n1;
                c_n1 = c_n2;
                c_n2 = code_at(j + 2);
                uint32_t hu, fu;
                if (pass == 0) {
                    hu = p16_prmt((uint32_t)(uint16_t)top, prev_h, 0x5410u);
                    fu = p16_prmt(NEG, prev_f, 0x5410u);
                    top -= top_step;
                } else {
                    const uint32_t v = v_n1;
                    v_n1 = v_n2;
                    v_n2 = j + 2 <= wmax ? __ldcg(&buf[(size_t)(j + 2) * 32 + lane]) : vnone;
                    hu = p16_prmt(v, prev_h, 0x5410u);       /* lo <- previous pass's strip B bottom */
                    fu = p16_prmt(v, prev_f, 0x5432u);
                }
                const uint4 pa4 = *reinterpret_cast<const uint4 *>(sl + ca * P16_PASS);
                const uint4 pb4 = *reinterpret_cast<const uint4 *>(sl + cb * P16_PASS + P16_R);
                uint32_t hd = dg;
                dg = hu;
                uint32_t cmax = 0u;
                uint32_t aD = 0u, aF = 0u, aE = 0u, aV = 0u;
                uint32_t lastv = 0u;
#pragma unroll
                for (int r = 0; r < P16_R; ++r) {
                    const uint32_t wa = r < 4 ? pa4.x : r < 8 ? pa4.y : r < 12 ? pa4.z : pa4.w;
                    const uint32_t wb = r < 4 ? pb4.x : r < 8 ? pb4.y : r < 12 ? pb4.z : pb4.w;
                    uint32_t sc;
                    switch (r & 3) {
                        case 0: sc = p16_pair<0>(wa, wb); break;
                        case 1: sc = p16_pair<1>(wa, wb); break;
                        case 2: sc = p16_pair<2>(wa, wb); break;
                        default: sc = p16_pair<3>(wa, wb); break;
                    }
                    uint32_t e, f, h;
                    if (BITS) {
                        const uint32_t ho = __vadd2(H[r], gO), ee = __vadd2(E[r], gE);
                        e = __vmaxs2(ho, ee);
                        const uint32_t fo = __vadd2(hu, gO), fe = __vadd2(fu, gE);
                        f = __vmaxs2(fo, fe);
                        const uint32_t hdg = __vadd2(hd, sc);
                        h = ALG == PB_SW ? __vimax3_s16x2_relu(hdg, e, f) : __vimax3_s16x2(hdg, e, f);
                        /* decision bits: sign of the difference of each half */
                        aD = (aD >> 1) | (__vsub2(hdg, h) & 0x80008000u);
                        aF = (aF >> 1) | (__vsub2(f, h) & 0x80008000u);
                        aE = (aE >> 1) | (__vsub2(ee, ho) & 0x80008000u);
                        aV = (aV >> 1) | (__vsub2(fe, fo) & 0x80008000u);
                    } else {
                        e = __viaddmax_s16x2(E[r], gE, __vadd2(H[r], gO));
                        f = __viaddmax_s16x2(hu, gO, __vadd2(fu, gE));
                        if (ALG == PB_SW) h = __vmaxs2(__viaddmax_s16x2_relu(hd, sc, e), f);
                        else h = __vmaxs2(__viaddmax_s16x2(hd, sc, e), f);
                    }
                    E[r] = e;
                    hd = H[r];
                    H[r] = h;
                    hu = h;
                    fu = f;
                    if (ENDS && ALG == PB_SW && (r & 1)) cmax = __vimax3_s16x2(cmax, H[r - 1], h);
                    if (lastpass && (sgf & PB_S2_END) && r == r_last) lastv = h;
                }
                if (BITS) tbits[((size_t)pass * (wmax + 1) + j) * 32 + lane] = make_uint4(aD, aF, aE, aV);
                if (j >= 1 && more) buf[(size_t)(j - 1) * 32 + lane] = p16_prmt(hu, fu, 0x7632u);
                prev_h = hu;
                prev_f = fu;
                cb = ca;
                if (j == 0) {
                    /* the high half computed column -1: restore strip B's
                     * left boundary (H(i,-1), E = -inf) */
#pragma unroll
                    for (int r = 0; r < P16_R; ++r) {
                        const int lb2 = p16_left(ALG, sgf, r0 + P16_R + r, open, gap);
                        H[r] = (H[r] & 0xffffu) | ((uint32_t)(uint16_t)lb2 << 16);
                        E[r] = (E[r] & 0xffffu) | (NEG & 0xffff0000u);
                    }
                }
                if (ENDS && ALG == PB_SW) {
                    /* a strictly higher column maximum than the strip's best
                     * so far: the first column reaching it, kept whole (the
                     * warp takes this branch whenever any lane improves; the
                     * smallest row is looked up once per pass) */
                    const int c_lo = p16_lo(cmax), c_hi = p16_hi(cmax);
                    if (c_lo > sa.score && j < cols) {
#pragma unroll
                        for (int k = 0; k < P16_R / 4; ++k)
                            save[k] = make_uint4(H[4 * k], H[4 * k + 1], H[4 * k + 2], H[4 * k + 3]);
                        sa.score = c_lo; sa.j = j;
                    }
                    if (c_hi > sb.score && j >= 1 && j <= cols) {
#pragma unroll
                        for (int k = 0; k < P16_R / 4; ++k)
                            save[P16_R / 4 + k] = make_uint4(H[4 * k], H[4 * k + 1], H[4 * k + 2], H[4 * k + 3]);
                        sb.score = c_hi; sb.j = j - 1;
                    }
                }
                if (ENDS && ALG != PB_SW) {
                    /* last column (strip A at j = cols - 1, strip B one
                     * iteration later): SG's last-column maximum over rows
                     * below rows - 1 (smallest row on ties), and the corner */
                    if (j == cols - 1 || j == cols) {
                        const int hsel = j == cols - 1 ? 0 : 1;
                        const int ib = r0 + hsel * P16_R;
#pragma unroll
                        for (int r = 0; r < P16_R; ++r) {
                            const int v = hsel ? p16_hi(H[r]) : p16_lo(H[r]);
                            const int i = ib + r;
                            if (ALG == PB_SG && (sgf & PB_S1_END) && i < ilast && v > lc_h) { lc_h = v; lc_i = i; }
                            if (i == ilast) corner = v;
                        }
                    }
                    if (lastpass && (sgf & PB_S2_END)) {
                        const int jj = j - half_last;
                        const int v = half_last ? p16_hi(lastv) : p16_lo(lastv);
                        if (jj >= 0 && jj < cols && v > lr_h) { lr_h = v; lr_j = jj; }
                    }
                }
            }
            if (ENDS && ALG == PB_SW) {
                if (sa.j >= 0) {
                    int rr = P16_R - 1;
#pragma unroll
                    for (int k = P16_R / 4 - 1; k >= 0; --k) {
                        const uint4 w = save[k];
                        const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
                        for (int x = 3; x >= 0; --x) if (p16_lo(ws[x]) == sa.score) rr = 4 * k + x;
                    }
                    sa.i = r0 + rr;
                }
                if (sb.j >= 0) {
                    int rr = P16_R - 1;
#pragma unroll
                    for (int k = P16_R / 4 - 1; k >= 0; --k) {
                        const uint4 w = save[P16_R / 4 + k];
                        const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
                        for (int x = 3; x >= 0; --x) if (p16_hi(ws[x]) == sb.score) rr = 4 * k + x;
                    }
                    sb.i = r0 + P16_R + rr;
                }
                const P16Best cand[2] = {sa, sb};
#pragma unroll
                for (int x = 0; x < 2; ++x) {
                    const P16Best c = cand[x];
                    if (c.j >= 0 && (!have || c.score > best.score || (c.score == best.score && c.j < best.j))) {
                        best = c;
                        have = true;
                    }
                }
            }
        }
        if (valid) {
            pb_pair_out o;
            if (ENDS) {
                int sc, eq, er;
                if (ALG == PB_SW) {
                    sc = have ? best.score : 0; eq = have ? best.i : 0; er = have ? best.j : 0;
                } else if (ALG == PB_NW) {
                    sc = corner; eq = ilast; er = cols - 1;
                } else {
                    /* src/sg.c:160-242 */
                    const bool s1e = sgf & PB_S1_END, s2e = sgf & PB_S2_END;
                    sc = INT_MIN; eq = rows; er = cols;
                    if (s1e && lc_i >= 0) { sc = lc_h; eq = lc_i; er = cols - 1; }
                    if (s1e && s2e) {
                        if (lr_h > sc || (lr_h == sc && lr_j < er)) { sc = lr_h; eq = ilast; er = lr_j; }
                    } else if (s2e) {
                        if (lr_h > sc) { sc = lr_h; eq = ilast; er = lr_j; }
                    }
                    if ((s1e && corner > sc) || (!s1e && !s2e)) { sc = corner; eq = ilast; er = cols - 1; }
                }
                o.score = sc; o.end_query = eq; o.end_ref = er;
                o.max_h = ALG == PB_SW ? sc : bd.ub;
            } else {
                o.score = 0; o.end_query = 0; o.end_ref = 0;
                o.max_h = bd.ub;
            }
            o.matches = o.similar = o.length = 0;
            /* the width verdicts read sound bounds (see p16_check) */
            o.min_h_real = bd.lb;
            o.min_f_real = bd.lb - open;
            o.max_stat_real = ((rows + 31) & ~31) + cols;
#pragma unroll
            for (int x = 0; x < 3; ++x) {
                o.min_h_pad[x] = bd.lb;
                o.max_stat_pad[x] = o.max_stat_real;
                o.min_f_pad[x] = bd.lb - open;
            }
            o.status = status | PB_ST_BOUNDED;
            p.out[item] = o;
        }
    }
}

/*
 * The statistics walk of one item: from its end cell back along the path
 * the reference's tie rules select, reading the direction bits of the
 * item's task (lane = its position in the task). Writes matches, similar
 * and length into out[item].
 */
template <int ALG>
__global__ void k_p16_walk(P16Params p, const int *__restrict__ tlist, int ntl, const pb_pair_out *__restrict__ ends,
                           int open, int gap)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ntl * 32) return;
    const int task = tlist[g >> 5], lane = g & 31;
    const int s = task * 32 + lane;
    if (s >= p.nitems) return;
    const int item = p.order[s];
    if (item < 0) return;
    const int wmax = p.task_wmax[task];
    const uint4 *tb = p.bits + p.task_bits[task];
    const pb_pair_out e = ends[item];
    const int ti = p.nt ? item % p.nt : item;
    const uint8_t *tseq = p.targets + p.toff[ti];
    const uint8_t *qseq;
    const int32_t *prof32 = nullptr;
    int lp = 0;
    if (p.mat8) {
        qseq = p.qall + p.qoff[item];
    } else {
        const ProfDesc pd = p.profs[p.nt ? item / p.nt : 0];
        qseq = pd.qcodes;
        prof32 = pd.prof;
        lp = pd.lp;
    }
    const int L = p.nletters;
    int i = e.end_query, j = e.end_ref;
    int v = e.score;
    pb_pair_out *o = p.out + item;
    if (i >= p.rows[item] || j >= p.cols[item]) {
        /* the end lies outside the computed region (a FASTSTATS item
         * whose prefix pass was not needed): nothing to walk */
        o->matches = o->similar = o->length = 0;
        return;
    }
    int M = 0, S = 0, Ln = 0;
    int state = 0;                                  /* 0 H, 1 F, 2 E */
    const int limit = p.rows[item] + p.cols[item] + 2;
    for (int step = 0; step <= 2 * limit; ++step) {
        if (i < 0 || j < 0) break;
        if (ALG == PB_SW && state == 0 && v <= 0) break;
        const int half = (i >> 4) & 1, bit = half * 16 + (i & 15);
        const uint4 w = tb[((size_t)(i >> 5) * (wmax + 1) + j + half) * 32 + lane];
        if (state == 0) {
            if (!((w.x >> bit) & 1u)) {
                int qc = qseq[i], tc = tseq[j];
                if (qc >= L) qc = 0;
                if (tc >= L) tc = 0;
                const int sc = p.mat32 ? p.mat32[tc * L + qc] : prof32[(size_t)tc * lp + i];
                M += qc == tc;
                S += sc > 0;
                Ln += 1;
                v -= sc;
                --i;
                --j;
            } else {
                state = ((w.y >> bit) & 1u) ? 2 : 1;
            }
        } else if (state == 1) {
            Ln += 1;
            if ((w.w >> bit) & 1u) { v += open; state = 0; } else { v += gap; }
            --i;
        } else {
            Ln += 1;
            if ((w.z >> bit) & 1u) { v += open; state = 0; } else { v += gap; }
            --j;
        }
    }
    o->matches = M;
    o->similar = S;
    o->length = Ln;
}

/*
 * The traceback path of one item: the walk of k_p16_walk, recording its
 * steps instead of counting them -- 0 a diagonal step (query and target
 * residue aligned), 1 a step up a vertical gap (a query residue against a
 * gap), 2 a step left along a horizontal gap (a target residue against a
 * gap) -- written backwards from the end of the item's op buffer, with
 * the cell where the walk stopped. These are the decisions the reference's
 * trace tables hold (src/sw_trace.c:138-147: DIAG when H == H_diag, else
 * DEL when H == F, else INS; DIAG_F / DIAG_E when the gap opened by strict
 * >), followed as its CIGAR builder does (src/cigar_template.c:143-243).
 */
template <int ALG>
__global__ void k_p16_path(P16Params p, const int *__restrict__ tlist, int ntl, const pb_pair_out *__restrict__ ends,
                           int open, int gap)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ntl * 32) return;
    const int task = tlist[g >> 5], lane = g & 31;
    const int s = task * 32 + lane;
    if (s >= p.nitems) return;
    const int item = p.order[s];
    if (item < 0) return;
    const int wmax = p.task_wmax[task];
    const uint4 *tb = p.bits + p.task_bits[task];
    const pb_pair_out e = ends[item];
    const int rows = p.rows[item], cols = p.cols[item];
    const int cap = rows + cols;
    uint8_t *ops = p.ops + p.ops_off[item];
    int *info = p.path_info + 3 * (size_t)item;
    int i = e.end_query, j = e.end_ref;
    int v = e.score;
    if (i >= rows || j >= cols || i < 0 || j < 0) {
        info[0] = -1; info[1] = i; info[2] = j;
        return;
    }
    const int ti = p.nt ? item % p.nt : item;
    const uint8_t *tseq = p.targets + p.toff[ti];
    const uint8_t *qseq;
    const int32_t *prof32 = nullptr;
    int lp = 0;
    if (p.mat8) {
        qseq = p.qall + p.qoff[item];
    } else {
        const ProfDesc pd = p.profs[p.nt ? item / p.nt : 0];
        qseq = pd.qcodes;
        prof32 = pd.prof;
        lp = pd.lp;
    }
    const int L = p.nletters;
    int n = 0, state = 0;                       /* 0 H, 1 F, 2 E */
    for (int step = 0; step <= 2 * cap + 2 && n < cap; ++step) {
        if (i < 0 || j < 0) break;
        if (ALG == PB_SW && state == 0 && v <= 0) break;
        const int half = (i >> 4) & 1, bit = half * 16 + (i & 15);
        const uint4 w = tb[((size_t)(i >> 5) * (wmax + 1) + j + half) * 32 + lane];
        if (state == 0) {
            if (!((w.x >> bit) & 1u)) {
                int qc = qseq[i], tc = tseq[j];
                if (qc >= L) qc = 0;
                if (tc >= L) tc = 0;
                v -= p.mat32 ? p.mat32[tc * L + qc] : prof32[(size_t)tc * lp + i];
                ops[cap - 1 - n++] = 0;
                --i;
                --j;
            } else {
                state = ((w.y >> bit) & 1u) ? 2 : 1;
            }
        } else if (state == 1) {
            ops[cap - 1 - n++] = 1;
            if ((w.w >> bit) & 1u) { v += open; state = 0; } else { v += gap; }
            --i;
        } else {
            ops[cap - 1 - n++] = 2;
            if ((w.z >> bit) & 1u) { v += open; state = 0; } else { v += gap; }
            --j;
        }
    }
    info[0] = n; info[1] = i; info[2] = j;
}

/* per item: rows, columns, eligibility and the sort key (eligible first,
 * then by query group, passes and columns, all descending) */
__global__ void k_p16_setup(P16Setup q, int *__restrict__ rows, int *__restrict__ cols,
                            unsigned long long *__restrict__ keys, int *__restrict__ idx,
                            int *__restrict__ counts)
{
    const int item = blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= q.nitems) return;
    const int ti = q.nt ? item % q.nt : item;
    int r = q.qlim ? q.qlim[item] : (q.qlen ? q.qlen[item] : q.prof_qlen[item / q.nt]);
    const int c = q.tlim ? q.tlim[item] : q.tlen[ti];
    rows[item] = r;
    cols[item] = c;
    idx[item] = item;
    bool ok = r >= 1 && c >= 1 && c <= q.max_cols && r <= 65535 && !((q.intra_mask >> p16_bucket(r, c)) & 1u);
    if (ok) {
        const P16Bounds b = p16_bounds(q.alg, r, c, q.open, q.gap, q.mmax, q.mmin);
        ok = p16_fits(b, q.open, q.gap);
    }
    if (ok) {
        const unsigned long long grp = q.group ? (unsigned long long)(q.group[item] & 0xfffff)
                                               : (q.nt ? (unsigned long long)(item / q.nt) & 0xfffff : 0ull);
        const unsigned long long np = (unsigned long long)((r + 31) / 32) & 0x7ff;
        keys[item] = (1ull << 63) | (grp << 43) | (np << 32) | ((unsigned long long)c & 0xffffffffull);
        atomicAdd(&counts[0], 1);
    } else {
        keys[item] = 0ull;
    }
}

/* per task (a warp each): widest target, passes, shared query, bits size */
__global__ void k_p16_tasks(P16Params p, int ntasks, const int *__restrict__ group, int *__restrict__ twmax,
                            int *__restrict__ tnpass, int *__restrict__ tshared, long long *__restrict__ tbits,
                            int bits)
{
    const int task = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (task >= ntasks) return;
    const int s = task * 32 + lane;
    const bool valid = s < p.nitems && p.order[s] >= 0;
    const int item = valid ? p.order[s] : -1;
    int c = valid ? p.cols[item] : 0, r = valid ? p.rows[item] : 0;
    long long src = -1;
    if (valid) {
        if (p.mat8) src = group ? (long long)group[item] : -2 - (long long)item;   /* pairs: one query per item */
        else src = p.nt ? item / p.nt : 0;
    }
    long long src0 = __shfl_sync(0xffffffffu, src, 0);
    const bool same = __all_sync(0xffffffffu, !valid || src == src0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        c = max(c, __shfl_xor_sync(0xffffffffu, c, o));
        r = max(r, __shfl_xor_sync(0xffffffffu, r, o));
    }
    if (lane == 0) {
        const int np = (r + P16_PASS - 1) / P16_PASS;
        twmax[task] = c;
        tnpass[task] = np;
        tshared[task] = p.mat8 ? (same && group != nullptr) : 1;
        tbits[task] = bits ? (long long)np * (c + 1) * 32 : 0;
    }
}

}  // namespace pb

namespace pb {

/* Is the record pb_chain_resolve builds from an item's bounded extremes
 * (pb_pair_out with PB_ST_BOUNDED: max_h an upper bound except in SW, where
 * it is the score; minima lower bounds; statistics maxima upper bounds) the
 * one it would build from exact extremes? Each width the chain visits must
 * either be CLEAN by the bounds (sound: the bounds contain the exact
 * values), be SAT by a value the item is known to reach (the score is a
 * visited H: above POS_LIMIT, or in a scan kernel below NEG_LIMIT), or be
 * decided by the lane-exact kernel, which does not read the extremes. */
__device__ bool p16_definite(const pb_job &job, const pb_pair_out &o, int qlen, int tlen)
{
    const pb_mode *m = &job.mode;
    if (job.bits < 0) return true;                         /* serial forms: exact values only */
    if (pb_job_is_faststats(&job)) return true;            /* score pass exact; prefix pass CLEAN or lane-exact */
    if (m->alg == PB_SW && !m->stats) return true;         /* SW score-only reads max_h = score only */
    const int w3[3] = {8, 16, 32};
    int f, l;
    pb_job_widths(&job, &f, &l);
    for (int t = f; t <= l; ++t) {
        const int w = w3[t];
        const int v = pb_resolve_tier(m, w, &o, qlen, tlen);
        if (pb_lane_applies(m, w) && (v != PB_CLEAN || pb_lane_forced(m, w))) continue;
        if (v == PB_CLEAN) return true;
        if (v != PB_SAT) return false;
        const int64_t imin = int_min_w(w), imax = int_max_w(w);
        const int64_t neg = ((-(int64_t)m->open < m->mmin) ? imin + m->open : imin - m->mmin) + 1;
        const int64_t pos = imax - m->mmax - 1;
        const int L = lanes_of(w);
        const int64_t padlen = ((int64_t)qlen + L - 1) / L * L;
        bool proven = (int64_t)o.score > pos;
        if (!m->striped && (int64_t)o.score < neg) proven = true;
        if (m->alg != PB_SW && m->striped && !m->stats && boundary_h(m, (int)padlen - 1, 0) - m->open < neg)
            proven = true;
        if (!proven) return false;
    }
    return true;
}

__global__ void k_p16_check(pb_job job, P16Params p, int *__restrict__ rest, int *__restrict__ nrest)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= p.nitems) return;
    const int item = p.order[s];
    if (item < 0) return;
    if (!p16_definite(job, p.out[item], p.rows[item], p.cols[item])) rest[atomicAdd(nrest, 1)] = item;
}

/* Task alignment to query groups: the eligible items sorted by (group,
 * passes, columns) are laid out so that every group starts a task (each
 * group padded with -1 entries to a multiple of 32). No task then mixes two
 * queries, and every task of a grouped batch takes the shared-query
 * variant. */
__global__ void k_pad_heads(const unsigned long long *__restrict__ keys, int n, int *__restrict__ head)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) head[s] = s == 0 || ((keys[s] >> 43) & 0xfffffull) != ((keys[s - 1] >> 43) & 0xfffffull);
}

__global__ void k_pad_counts(const int *__restrict__ gstart, int ng, int n, int *__restrict__ pcount)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < ng) pcount[g] = ((g + 1 < ng ? gstart[g + 1] : n) - gstart[g] + 31) & ~31;
}

__global__ void k_pad_scatter(const int *__restrict__ order, int n, const int *__restrict__ gid,
                              const int *__restrict__ gstart, const int *__restrict__ pstart, int *__restrict__ out)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) {
        const int g = gid[s] - 1;
        out[pstart[g] + (s - gstart[g])] = order[s];
    }
}

__global__ void k_mat_to_int8(const int32_t *__restrict__ m, int n, int8_t *__restrict__ m8)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) m8[k] = (int8_t)m[k];
}

__global__ void k_iota_int(int *__restrict__ v, int n)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) v[k] = k;
}

__global__ void k_copy_int(const int *__restrict__ src, int n, int *__restrict__ dst)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) dst[k] = src[k];
}

struct P16Frees {
    cudaStream_t st;
    std::vector<void *> v;
    explicit P16Frees(cudaStream_t s) : st(s) {}
    template <typename T> T *add(T *q) { if (q) v.push_back((void *)q); return q; }
    ~P16Frees() { for (void *q : v) cudaFreeAsync(q, st); }
};

namespace {

#define P16_CK(call)                                           \
    do {                                                       \
        if ((call) != cudaSuccess) {                           \
            fprintf(stderr, "pb_pair16: %s failed\n", #call);  \
            return -1;                                         \
        }                                                      \
    } while (0)

int p16_warps(bool shared, int L) { return shared || L <= 8 ? 8 : 4; }

size_t p16_smem(bool shared, int L, bool mat)
{
    const size_t mat_bytes = mat ? ((size_t)(L * L + 15) & ~(size_t)15) : 0;
    const size_t warp_bytes = shared ? (size_t)L * P16_PASS : 32 * ((size_t)L * P16_PASS + 16);
    return mat_bytes + warp_bytes * p16_warps(shared, L);
}

typedef void (*p16_kernel_t)(P16Params, const int *, int, int *);

template <int ALG, bool BITS, bool ENDS>
p16_kernel_t pick3(bool shared, int warps)
{
    if (shared) return k_p16<ALG, BITS, ENDS, true, 8>;
    return warps == 8 ? k_p16<ALG, BITS, ENDS, false, 8> : k_p16<ALG, BITS, ENDS, false, 4>;
}

p16_kernel_t pick(int alg, bool bits, bool ends, bool shared, int warps)
{
    if (alg == PB_SW) {
        if (!ends) return pick3<PB_SW, true, false>(shared, warps);
        return bits ? pick3<PB_SW, true, true>(shared, warps) : pick3<PB_SW, false, true>(shared, warps);
    }
    if (alg == PB_NW) return bits ? pick3<PB_NW, true, true>(shared, warps) : pick3<PB_NW, false, true>(shared, warps);
    return bits ? pick3<PB_SG, true, true>(shared, warps) : pick3<PB_SG, false, true>(shared, warps);
}

}  // namespace

int p16_pass(const pb_job &job, const pb_batch *b, int prefix, const pb_pair_out *ends, pb_pair_out *out,
             const int *group, int *d_rest, int *n_rest, cudaStream_t st,
             uint8_t *d_ops, const int64_t *d_ops_off, int *d_path_info, unsigned intra_mask)
{
    const pb_mode *m = &job.mode;
    const bool dbmode = b->nprofs > 0;
    const int N = dbmode ? b->npairs * b->nprofs : b->npairs;
    *n_rest = 0;
    if (N <= 0) return 0;
    if ((long long)(dbmode ? (long long)b->npairs * b->nprofs : b->npairs) > INT32_MAX) return -1;
    const bool paths = d_ops != nullptr;
    const bool bits = prefix || (m->stats && !pb_job_is_faststats(&job)) || paths;
    const bool walk = prefix || (m->stats && !pb_job_is_faststats(&job));
    const bool ends_on = !prefix;
    P16Frees frees(st);
    /* alphabet and score source; anything the kernels cannot take goes to the exact kernel */
    int L = 0, mmax = 0, mmin = 0;
    bool usable = true;
    int8_t *d_mat8 = nullptr;
    ProfDesc *d_profs = nullptr;
    int *d_pql = nullptr;
    if (dbmode) {
        L = b->profs[0]->size;
        mmax = b->profs[0]->mmax; mmin = b->profs[0]->mmin;
        std::vector<ProfDesc> h(b->nprofs);
        std::vector<int> ql(b->nprofs);
        for (int q = 0; q < b->nprofs; ++q) {
            const pb_device_profile *dp = b->profs[q];
            usable = usable && dp->fits8 && dp->size == L && dp->d_prof8;
            h[q].prof = dp->d_prof32; h[q].prof8 = dp->d_prof8; h[q].qcodes = dp->d_qcodes;
            h[q].qlen = dp->qlen; h[q].lp = dp->lp; h[q].size = dp->size; h[q].pad_ = 0;
            ql[q] = dp->qlen;
            mmax = dp->mmax > mmax ? dp->mmax : mmax;
            mmin = dp->mmin < mmin ? dp->mmin : mmin;
        }
        if (usable) {
            P16_CK(cudaMallocAsync((void **)&d_profs, sizeof(ProfDesc) * b->nprofs, st));
            frees.add(d_profs);
            P16_CK(cudaMallocAsync((void **)&d_pql, sizeof(int) * b->nprofs, st));
            frees.add(d_pql);
            P16_CK(cudaMemcpyAsync(d_profs, h.data(), sizeof(ProfDesc) * b->nprofs, cudaMemcpyHostToDevice, st));
            P16_CK(cudaMemcpyAsync(d_pql, ql.data(), sizeof(int) * b->nprofs, cudaMemcpyHostToDevice, st));
            P16_CK(cudaStreamSynchronize(st));      /* the host vectors die at return */
        }
    } else {
        L = b->msize; mmax = b->mmax; mmin = b->mmin;
        usable = b->d_mat && b->mmin >= -128 && b->mmax <= 127;
        if (usable) {
            P16_CK(cudaMallocAsync((void **)&d_mat8, (size_t)L * L, st));
            frees.add(d_mat8);
            k_mat_to_int8<<<(L * L + 255) / 256, 256, 0, st>>>(b->d_mat, L * L, d_mat8);
            pb_diag_count_launch(1);
        }
    }
    usable = usable && L >= 1 && L <= 32;
    if (!usable) {
        /* nothing for the pair kernels: every item to the exact kernel */
        k_iota_int<<<(N + 255) / 256, 256, 0, st>>>(d_rest, N);
        pb_diag_count_launch(1);
        *n_rest = N;
        P16_CK(cudaStreamSynchronize(st));
        return 0;
    }
    /* per item: rows, columns, eligibility, sort */
    int *rows = nullptr, *cols = nullptr, *idx = nullptr, *order = nullptr, *counts = nullptr;
    unsigned long long *keys = nullptr, *keys_sorted = nullptr;
    P16_CK(cudaMallocAsync((void **)&rows, sizeof(int) * N, st)); frees.add(rows);
    P16_CK(cudaMallocAsync((void **)&cols, sizeof(int) * N, st)); frees.add(cols);
    P16_CK(cudaMallocAsync((void **)&idx, sizeof(int) * N, st)); frees.add(idx);
    P16_CK(cudaMallocAsync((void **)&order, sizeof(int) * N, st)); frees.add(order);
    P16_CK(cudaMallocAsync((void **)&counts, sizeof(int) * 4, st)); frees.add(counts);
    P16_CK(cudaMallocAsync((void **)&keys, sizeof(unsigned long long) * N, st)); frees.add(keys);
    P16_CK(cudaMallocAsync((void **)&keys_sorted, sizeof(unsigned long long) * N, st)); frees.add(keys_sorted);
    P16_CK(cudaMemsetAsync(counts, 0, sizeof(int) * 4, st));
    P16Setup q;
    memset(&q, 0, sizeof q);
    q.alg = m->alg; q.open = m->open; q.gap = m->gap; q.mmax = mmax; q.mmin = mmin; q.nitems = N;
    q.nt = dbmode ? b->npairs : 0;
    q.max_cols = 65535;
    q.qlen = dbmode ? nullptr : b->d_qlen;
    q.prof_qlen = d_pql;
    q.tlen = b->d_tlen;
    q.qlim = b->d_qlim; q.tlim = b->d_tlim;
    q.group = dbmode ? nullptr : group;
    q.intra_mask = intra_mask;
    k_p16_setup<<<(N + 255) / 256, 256, 0, st>>>(q, rows, cols, keys, idx, counts);
    pb_diag_count_launch(1);
    size_t sort_bytes = 0;
    void *sort_tmp = nullptr;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, sort_bytes, keys, keys_sorted, idx, order, N, 0, 64, st);
    P16_CK(cudaMallocAsync(&sort_tmp, sort_bytes, st));
    frees.add(sort_tmp);
    cub::DeviceRadixSort::SortPairsDescending(sort_tmp, sort_bytes, keys, keys_sorted, idx, order, N, 0, 64, st);
    int nelig = 0;
    P16_CK(cudaMemcpyAsync(&nelig, counts, sizeof(int), cudaMemcpyDeviceToHost, st));
    P16_CK(cudaStreamSynchronize(st));
    /* the ineligible items (sorted last) start the rest list */
    if (N - nelig > 0) {
        k_copy_int<<<(N - nelig + 255) / 256, 256, 0, st>>>(order + nelig, N - nelig, d_rest);
        pb_diag_count_launch(1);
    }
    int nrest = N - nelig;
    /* grouped batches: every group starts a task */
    int nslots = nelig;
    int *porder = order;
    if (nelig > 0 && (dbmode || group)) {
        int *head = nullptr, *gid = nullptr, *gstart = nullptr, *pcount = nullptr, *pstart = nullptr, *iota = nullptr;
        int ng = 0, last_start = 0, last_count = 0;
        P16_CK(cudaMallocAsync((void **)&head, sizeof(int) * nelig, st)); frees.add(head);
        P16_CK(cudaMallocAsync((void **)&gid, sizeof(int) * nelig, st)); frees.add(gid);
        P16_CK(cudaMallocAsync((void **)&gstart, sizeof(int) * nelig, st)); frees.add(gstart);
        P16_CK(cudaMallocAsync((void **)&pcount, sizeof(int) * nelig, st)); frees.add(pcount);
        P16_CK(cudaMallocAsync((void **)&pstart, sizeof(int) * nelig, st)); frees.add(pstart);
        P16_CK(cudaMallocAsync((void **)&iota, sizeof(int) * nelig, st)); frees.add(iota);
        k_pad_heads<<<(nelig + 255) / 256, 256, 0, st>>>(keys_sorted, nelig, head);
        k_iota_int<<<(nelig + 255) / 256, 256, 0, st>>>(iota, nelig);
        pb_diag_count_launch(2);
        size_t b1 = 0, b2 = 0, b3 = 0;
        void *tmp = nullptr;
        P16_CK(cub::DeviceScan::InclusiveSum(nullptr, b1, head, gid, nelig, st));
        P16_CK(cub::DeviceSelect::Flagged(nullptr, b2, iota, head, gstart, counts + 2, nelig, st));
        P16_CK(cub::DeviceScan::ExclusiveSum(nullptr, b3, pcount, pstart, nelig, st));
        const size_t tb = std::max(b1, std::max(b2, b3));
        P16_CK(cudaMallocAsync(&tmp, tb, st)); frees.add(tmp);
        size_t b = tb;
        P16_CK(cub::DeviceScan::InclusiveSum(tmp, b, head, gid, nelig, st));
        b = tb;
        P16_CK(cub::DeviceSelect::Flagged(tmp, b, iota, head, gstart, counts + 2, nelig, st));
        P16_CK(cudaMemcpyAsync(&ng, counts + 2, sizeof(int), cudaMemcpyDeviceToHost, st));
        P16_CK(cudaStreamSynchronize(st));
        k_pad_counts<<<(ng + 255) / 256, 256, 0, st>>>(gstart, ng, nelig, pcount);
        pb_diag_count_launch(1);
        b = tb;
        P16_CK(cub::DeviceScan::ExclusiveSum(tmp, b, pcount, pstart, ng, st));
        P16_CK(cudaMemcpyAsync(&last_start, pstart + ng - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        P16_CK(cudaMemcpyAsync(&last_count, pcount + ng - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        P16_CK(cudaStreamSynchronize(st));
        nslots = last_start + last_count;
        P16_CK(cudaMallocAsync((void **)&porder, sizeof(int) * (size_t)nslots, st)); frees.add(porder);
        P16_CK(cudaMemsetAsync(porder, 0xff, sizeof(int) * (size_t)nslots, st));
        k_pad_scatter<<<(nelig + 255) / 256, 256, 0, st>>>(order, nelig, gid, gstart, pstart, porder);
        pb_diag_count_launch(1);
    }
    if (nelig > 0) {
        const int ntasks = (nslots + 31) / 32;
        P16Params p;
        memset(&p, 0, sizeof p);
        p.alg = m->alg; p.sgflags = m->sgflags; p.open = m->open; p.gap = m->gap; p.mmax = mmax; p.mmin = mmin;
        p.nletters = L; p.nitems = nslots; p.order = porder; p.rows = rows; p.cols = cols;
        p.mat8 = d_mat8; p.mat32 = dbmode ? nullptr : b->d_mat;
        p.qall = b->d_qall; p.qoff = b->d_qoff; p.profs = d_profs; p.nt = dbmode ? b->npairs : 0;
        p.targets = b->d_targets; p.toff = b->d_toff;
        p.out = out;
        p.ops = d_ops; p.ops_off = d_ops_off; p.path_info = d_path_info;
        int *twmax = nullptr, *tnpass = nullptr, *tshared = nullptr;
        long long *tbits = nullptr;
        P16_CK(cudaMallocAsync((void **)&twmax, sizeof(int) * ntasks, st)); frees.add(twmax);
        P16_CK(cudaMallocAsync((void **)&tnpass, sizeof(int) * ntasks, st)); frees.add(tnpass);
        P16_CK(cudaMallocAsync((void **)&tshared, sizeof(int) * ntasks, st)); frees.add(tshared);
        P16_CK(cudaMallocAsync((void **)&tbits, sizeof(long long) * ntasks, st)); frees.add(tbits);
        k_p16_tasks<<<(ntasks * 32 + 255) / 256, 256, 0, st>>>(p, ntasks, dbmode ? nullptr : group, twmax, tnpass,
                                                               tshared, tbits, bits ? 1 : 0);
        pb_diag_count_launch(1);
        std::vector<int> hw(ntasks), hn(ntasks), hs(ntasks);
        std::vector<long long> hb(ntasks);
        P16_CK(cudaMemcpyAsync(hw.data(), twmax, sizeof(int) * ntasks, cudaMemcpyDeviceToHost, st));
        P16_CK(cudaMemcpyAsync(hn.data(), tnpass, sizeof(int) * ntasks, cudaMemcpyDeviceToHost, st));
        P16_CK(cudaMemcpyAsync(hs.data(), tshared, sizeof(int) * ntasks, cudaMemcpyDeviceToHost, st));
        P16_CK(cudaMemcpyAsync(hb.data(), tbits, sizeof(long long) * ntasks, cudaMemcpyDeviceToHost, st));
        P16_CK(cudaStreamSynchronize(st));
        int maxlen = 0;
        for (int t = 0; t < ntasks; ++t) maxlen = hw[t] > maxlen ? hw[t] : maxlen;
        /* task order: most work first */
        std::vector<int> torder(ntasks);
        for (int t = 0; t < ntasks; ++t) torder[t] = t;
        std::stable_sort(torder.begin(), torder.end(), [&](int x, int y) {
            return (long long)hn[x] * (hw[x] + 1) > (long long)hn[y] * (hw[y] + 1);
        });
        /* chunks of tasks whose direction bits fit the budget: half of the
         * free device memory (at most 96 GiB), so that a chunk of the largest
         * tasks (about 36 MB of bits each at 1500 x 1500) still fills the
         * SMs; a budget of a few GiB left chunks of ~200 warps */
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        size_t budget = (size_t)96 << 30;
        if (free_b / 2 < budget) budget = free_b / 2;
        const size_t budget_u4 = budget / sizeof(uint4);
        /* launch shapes and the pass-boundary buffers, sized for the larger grid */
        int dev = 0, nsm = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        int grid[2] = {0, 0}, warps[2] = {0, 0};
        size_t smem[2] = {0, 0};
        p16_kernel_t kern[2];
        for (int sh = 0; sh < 2; ++sh) {
            warps[sh] = p16_warps(sh == 1, L);
            smem[sh] = p16_smem(sh == 1, L, d_mat8 != nullptr);
            kern[sh] = pick(m->alg, bits, ends_on, sh == 1, warps[sh]);
            int per_sm = 0;
            pb_raise_smem((const void *)kern[sh], (int)smem[sh]);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern[sh], warps[sh] * 32, smem[sh]);
            grid[sh] = (per_sm < 1 ? 1 : per_sm) * nsm;
        }
        const size_t rwarps = (size_t)std::max(grid[0] * warps[0], grid[1] * warps[1]);
        uint32_t *scratch = nullptr;
        P16_CK(cudaMallocAsync((void **)&scratch, sizeof(uint32_t) * (size_t)(maxlen + 1) * 32 * rwarps, st));
        frees.add(scratch);
        p.scratch = scratch;
        p.colsave = nullptr;
        if (ends_on && m->alg == PB_SW) {
            P16_CK(cudaMallocAsync((void **)&p.colsave, sizeof(uint4) * (P16_R / 2) * 32 * rwarps, st));
            frees.add(p.colsave);
        }
        p.maxlen = maxlen;
        p.task_wmax = twmax; p.task_npass = tnpass; p.task_bits = tbits;
        int *d_tlist = nullptr, *d_counter = nullptr;
        P16_CK(cudaMallocAsync((void **)&d_tlist, sizeof(int) * ntasks, st)); frees.add(d_tlist);
        P16_CK(cudaMallocAsync((void **)&d_counter, sizeof(int) * 2, st)); frees.add(d_counter);
        uint4 *bitsbuf = nullptr;
        size_t bits_cap = 0;
        std::vector<long long> hoff(ntasks, 0);
        int t0 = 0;
        while (t0 < ntasks) {
            /* the chunk [t0, t1) of torder, its tasks listed shared-first */
            int t1 = t0;
            size_t used = 0;
            while (t1 < ntasks && (t1 == t0 || used + (size_t)hb[torder[t1]] <= budget_u4)) used += (size_t)hb[torder[t1++]];
            std::vector<int> lst[2];
            for (int k = t0; k < t1; ++k) lst[hs[torder[k]] ? 1 : 0].push_back(torder[k]);
            size_t off = 0;
            for (int k = t0; k < t1; ++k) { hoff[torder[k]] = (long long)off; off += (size_t)hb[torder[k]]; }
            if (bits && off > bits_cap) {
                if (bitsbuf) cudaFreeAsync(bitsbuf, st);
                bitsbuf = nullptr;
                P16_CK(cudaMallocAsync((void **)&bitsbuf, sizeof(uint4) * (off + 1), st));
                bits_cap = off;
            }
            p.bits = bitsbuf;
            P16_CK(cudaMemcpyAsync(tbits, hoff.data(), sizeof(long long) * ntasks, cudaMemcpyHostToDevice, st));
            const int n1 = (int)lst[1].size(), n0 = (int)lst[0].size();
            std::vector<int> all(lst[1]);
            all.insert(all.end(), lst[0].begin(), lst[0].end());
            P16_CK(cudaMemcpyAsync(d_tlist, all.data(), sizeof(int) * all.size(), cudaMemcpyHostToDevice, st));
            for (int sh = 1; sh >= 0; --sh) {
                const int nl = sh ? n1 : n0;
                if (!nl) continue;
                const int *tl = d_tlist + (sh ? 0 : n1);
                int g = grid[sh];
                const int need = (nl + warps[sh] - 1) / warps[sh];
                if (g > need) g = need;
                P16_CK(cudaMemsetAsync(d_counter, 0, sizeof(int), st));
                kern[sh]<<<g, warps[sh] * 32, smem[sh], st>>>(p, tl, nl, d_counter);
                pb_diag_count_launch(1);
                P16_CK(cudaGetLastError());
            }
            if (paths) {
                const int nw = (int)all.size() * 32;
                if (m->alg == PB_SW) k_p16_path<PB_SW><<<(nw + 127) / 128, 128, 0, st>>>(p, d_tlist, (int)all.size(), out, m->open, m->gap);
                else if (m->alg == PB_NW) k_p16_path<PB_NW><<<(nw + 127) / 128, 128, 0, st>>>(p, d_tlist, (int)all.size(), out, m->open, m->gap);
                else k_p16_path<PB_SG><<<(nw + 127) / 128, 128, 0, st>>>(p, d_tlist, (int)all.size(), out, m->open, m->gap);
                pb_diag_count_launch(1);
                P16_CK(cudaGetLastError());
            }
            if (walk) {
                const int nw = (int)all.size() * 32;
                const pb_pair_out *e = prefix ? ends : out;
                if (m->alg == PB_SW) k_p16_walk<PB_SW><<<(nw + 127) / 128, 128, 0, st>>>(p, d_tlist, (int)all.size(), e, m->open, m->gap);
                else if (m->alg == PB_NW) k_p16_walk<PB_NW><<<(nw + 127) / 128, 128, 0, st>>>(p, d_tlist, (int)all.size(), e, m->open, m->gap);
                else k_p16_walk<PB_SG><<<(nw + 127) / 128, 128, 0, st>>>(p, d_tlist, (int)all.size(), e, m->open, m->gap);
                pb_diag_count_launch(1);
                P16_CK(cudaGetLastError());
            }
            /* the host vectors handed to the copies above change next chunk */
            P16_CK(cudaStreamSynchronize(st));
            t0 = t1;
        }
        if (bitsbuf) cudaFreeAsync(bitsbuf, st);
        /* items whose width verdicts need exact extremes */
        if (!prefix) {
            P16_CK(cudaMemsetAsync(counts + 1, 0, sizeof(int), st));
            k_p16_check<<<(nslots + 255) / 256, 256, 0, st>>>(job, p, d_rest + nrest, counts + 1);
            pb_diag_count_launch(1);
            int nx = 0;
            P16_CK(cudaMemcpyAsync(&nx, counts + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
            P16_CK(cudaStreamSynchronize(st));
            nrest += nx;
        }
    }
    *n_rest = nrest;
    P16_CK(cudaStreamSynchronize(st));
    return 0;
}

/* --- the intra-task wavefront kernel on a subset (global score-only) -------- */

namespace {

__global__ void k_wave_fill(pb_job job, const int *__restrict__ list, int n, const int *__restrict__ score,
                            const int *__restrict__ qlen, const int *__restrict__ tlen, pb_pair_out *__restrict__ out,
                            int *__restrict__ rest, int *__restrict__ nrest)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int item = list[k];
    const int rows = qlen[k], cols = tlen[k];
    const P16Bounds bd = p16_bounds(PB_NW, rows, cols, job.mode.open, job.mode.gap, job.mode.mmax, job.mode.mmin);
    pb_pair_out o;
    o.score = score[k]; o.end_query = rows - 1; o.end_ref = cols - 1;
    o.matches = o.similar = o.length = 0;
    o.max_h = bd.ub;
    o.min_h_real = bd.lb; o.min_f_real = bd.lb - job.mode.open; o.max_stat_real = ((rows + 31) & ~31) + cols;
    for (int x = 0; x < 3; ++x) { o.min_h_pad[x] = bd.lb; o.max_stat_pad[x] = o.max_stat_real; o.min_f_pad[x] = bd.lb - job.mode.open; }
    o.status = PB_ST_BOUNDED;
    out[item] = o;
    if (!p16_definite(job, o, rows, cols)) rest[atomicAdd(nrest, 1)] = item;
}

__global__ void k_gather_pairs(const int *__restrict__ list, int n, const int64_t *__restrict__ qoff,
                               const int *__restrict__ qlen, const int64_t *__restrict__ toff,
                               const int *__restrict__ tlen, int64_t *__restrict__ gqoff, int *__restrict__ gqlen,
                               int64_t *__restrict__ gtoff, int *__restrict__ gtlen)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int item = list[k];
    gqoff[k] = qoff[item]; gqlen[k] = qlen[item];
    gtoff[k] = toff[item]; gtlen[k] = tlen[item];
}

}  // namespace

bool wave_ok(const pb_job &job, const pb_batch *b)
{
    return job.mode.alg == PB_NW && !job.mode.stats && b->nprofs == 0 && b->d_mat && !b->d_qlim && !b->d_tlim &&
           b->msize <= 32 && b->mmax <= 127 && b->mmin >= -127;
}

int wave_subset(const pb_job &job, const pb_batch *b, const int *d_list, int n, pb_pair_out *out, int *d_rest2,
                int *n_rest2, cudaStream_t st)
{
    *n_rest2 = 0;
    if (n <= 0) return 0;
    P16Frees frees(st);
    int64_t *gq = nullptr, *gt = nullptr;
    int *gql = nullptr, *gtl = nullptr, *sc = nullptr, *cnt = nullptr;
    P16_CK(cudaMallocAsync((void **)&gq, sizeof(int64_t) * n, st)); frees.add(gq);
    P16_CK(cudaMallocAsync((void **)&gt, sizeof(int64_t) * n, st)); frees.add(gt);
    P16_CK(cudaMallocAsync((void **)&gql, sizeof(int) * n, st)); frees.add(gql);
    P16_CK(cudaMallocAsync((void **)&gtl, sizeof(int) * n, st)); frees.add(gtl);
    P16_CK(cudaMallocAsync((void **)&sc, sizeof(int) * n, st)); frees.add(sc);
    P16_CK(cudaMallocAsync((void **)&cnt, sizeof(int), st)); frees.add(cnt);
    k_gather_pairs<<<(n + 255) / 256, 256, 0, st>>>(d_list, n, b->d_qoff, b->d_qlen, b->d_toff, b->d_tlen, gq, gql,
                                                    gt, gtl);
    pb_diag_count_launch(1);
    std::vector<int> hl(n), hm((size_t)b->msize * b->msize);
    P16_CK(cudaMemcpyAsync(hl.data(), gtl, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
    P16_CK(cudaMemcpyAsync(hm.data(), b->d_mat, sizeof(int) * hm.size(), cudaMemcpyDeviceToHost, st));
    P16_CK(cudaMemsetAsync(cnt, 0, sizeof(int), st));
    P16_CK(cudaStreamSynchronize(st));
    int maxlen = 0;
    for (int x : hl) maxlen = x > maxlen ? x : maxlen;
    if (pb_cuda_nw_long(n, job.mode.open, job.mode.gap, hm.data(), b->msize, b->d_qall, gq, gql, b->d_targets, gt,
                        gtl, nullptr, nullptr, maxlen, sc) != 0)
        return -1;
    P16_CK(cudaDeviceSynchronize());
    k_wave_fill<<<(n + 255) / 256, 256, 0, st>>>(job, d_list, n, sc, gql, gtl, out, d_rest2, cnt);
    pb_diag_count_launch(1);
    P16_CK(cudaMemcpyAsync(n_rest2, cnt, sizeof(int), cudaMemcpyDeviceToHost, st));
    P16_CK(cudaStreamSynchronize(st));
    return 0;
}

/* --- the exact kernel on a subset of a batch's items ------------------------ */

namespace {

__global__ void k_gather_items(const int *__restrict__ list, int n, int nt, const int64_t *__restrict__ toff,
                               const int *__restrict__ tlen, const int64_t *__restrict__ qoff,
                               const int *__restrict__ qlen, const int *__restrict__ qlim,
                               const int *__restrict__ tlim, int64_t *__restrict__ g_toff, int *__restrict__ g_tlen,
                               int64_t *__restrict__ g_qoff, int *__restrict__ g_qlen, int *__restrict__ g_pidx,
                               int *__restrict__ g_qlim, int *__restrict__ g_tlim)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int item = list[k];
    const int ti = nt ? item % nt : item;
    g_toff[k] = toff[ti];
    g_tlen[k] = tlen[ti];
    if (nt) g_pidx[k] = item / nt;
    else { g_qoff[k] = qoff[item]; g_qlen[k] = qlen[item]; }
    if (qlim) g_qlim[k] = qlim[item];
    if (tlim) g_tlim[k] = tlim[item];
}

__global__ void k_scatter_items(const pb_pair_out *__restrict__ src, const int *__restrict__ list, int n,
                                pb_pair_out *__restrict__ dst)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) dst[list[k]] = src[k];
}

}  // namespace

int exact_subset(const pb_batch *b, const int *d_list, int n, int stats, int pad_rows, pb_pair_out *out,
                 cudaStream_t st)
{
    if (n <= 0) return 0;
    const bool dbmode = b->nprofs > 0;
    P16Frees frees(st);
    int64_t *g_toff = nullptr, *g_qoff = nullptr;
    int *g_tlen = nullptr, *g_qlen = nullptr, *g_pidx = nullptr, *g_qlim = nullptr, *g_tlim = nullptr;
    pb_pair_out *tmp = nullptr;
    P16_CK(cudaMallocAsync((void **)&g_toff, sizeof(int64_t) * n, st)); frees.add(g_toff);
    P16_CK(cudaMallocAsync((void **)&g_tlen, sizeof(int) * n, st)); frees.add(g_tlen);
    P16_CK(cudaMallocAsync((void **)&tmp, sizeof(pb_pair_out) * n, st)); frees.add(tmp);
    if (dbmode) {
        P16_CK(cudaMallocAsync((void **)&g_pidx, sizeof(int) * n, st)); frees.add(g_pidx);
    } else {
        P16_CK(cudaMallocAsync((void **)&g_qoff, sizeof(int64_t) * n, st)); frees.add(g_qoff);
        P16_CK(cudaMallocAsync((void **)&g_qlen, sizeof(int) * n, st)); frees.add(g_qlen);
    }
    if (b->d_qlim) { P16_CK(cudaMallocAsync((void **)&g_qlim, sizeof(int) * n, st)); frees.add(g_qlim); }
    if (b->d_tlim) { P16_CK(cudaMallocAsync((void **)&g_tlim, sizeof(int) * n, st)); frees.add(g_tlim); }
    k_gather_items<<<(n + 255) / 256, 256, 0, st>>>(d_list, n, dbmode ? b->npairs : 0, b->d_toff, b->d_tlen,
                                                    b->d_qoff, b->d_qlen, b->d_qlim, b->d_tlim, g_toff, g_tlen,
                                                    g_qoff, g_qlen, g_pidx, g_qlim, g_tlim);
    pb_diag_count_launch(1);
    P16_CK(cudaStreamSynchronize(st));
    pb_batch s = *b;
    s.npairs = n;
    s.stats = stats;
    s.pad_rows = pad_rows;
    s.d_toff = g_toff; s.d_tlen = g_tlen;
    s.d_qlim = g_qlim; s.d_tlim = g_tlim;
    s.d_out = tmp;
    if (dbmode) s.d_prof_index = g_pidx;
    else { s.d_qoff = g_qoff; s.d_qlen = g_qlen; }
    if (pb_cuda_align_exact(&s) != 0) return -1;
    k_scatter_items<<<(n + 255) / 256, 256, 0, st>>>(tmp, d_list, n, out);
    pb_diag_count_launch(1);
    P16_CK(cudaStreamSynchronize(st));
    return 0;
}

}  // namespace pb

namespace {

__global__ void k_p16_map(uint8_t *__restrict__ buf, int64_t n, const uint8_t *__restrict__ map)
{
    __shared__ uint8_t smap[256];
    for (int k = threadIdx.x; k < 256; k += blockDim.x) smap[k] = map[k];
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        buf[i] = smap[buf[i]];
}

__global__ void k_p16_ends(const pb_pair_out *__restrict__ o, int n, int *__restrict__ se)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    se[3 * k] = o[k].score;
    se[3 * k + 1] = o[k].end_query;
    se[3 * k + 2] = o[k].end_ref;
}

}  // namespace

/* Traceback paths of n pairs from host memory (pairs mode: tmpl carries the
 * matrix table on the device): characters copied and mapped on the device,
 * the pair kernels with direction bits and the path walk, then per pair
 * h_ends[3k..] = score, end_query, end_ref, the steps in
 * h_ops[h_ops_off[k] ..] (written backwards from the end of the pair's
 * qlen + tlen bytes) and h_info[3k..] = steps (-1: the pair is outside the
 * 16-bit bounds of the pair kernels and has no path), stop row, stop
 * column. */
extern "C" int pb_cuda_trace_pairs_host(const pb_job *job, const pb_batch *tmpl, const uint8_t *mapper256,
                                        const char *h_q, const int64_t *h_qoff, const int *h_qlen,
                                        const char *h_t, const int64_t *h_toff, const int *h_tlen, int n,
                                        int *h_ends, uint8_t *h_ops, const int64_t *h_ops_off, int *h_info)
{
    if (pb_cuda_init() != 0) return -1;
    if (n <= 0) return 0;
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return -1;
    int rc = 0;
    {
        pb::P16Frees frees(st);
        int64_t qb = 0, tb = 0, ob = 0;
        for (int i = 0; i < n; ++i) {
            qb = std::max(qb, h_qoff[i] + h_qlen[i]);
            tb = std::max(tb, h_toff[i] + h_tlen[i]);
            ob = std::max(ob, h_ops_off[i] + h_qlen[i] + h_tlen[i]);
        }
        uint8_t *d_q = nullptr, *d_t = nullptr, *d_map = nullptr, *d_ops = nullptr;
        int64_t *d_qoff = nullptr, *d_toff = nullptr, *d_ooff = nullptr;
        int *d_qlen = nullptr, *d_tlen = nullptr, *d_info = nullptr, *d_rest = nullptr, *d_se = nullptr;
        pb_pair_out *d_o = nullptr;
        if (cudaMallocAsync((void **)&d_q, qb + 16, st) || cudaMallocAsync((void **)&d_t, tb + 16, st) ||
            cudaMallocAsync((void **)&d_map, 256, st) || cudaMallocAsync((void **)&d_ops, ob + 16, st) ||
            cudaMallocAsync((void **)&d_qoff, sizeof(int64_t) * n, st) ||
            cudaMallocAsync((void **)&d_toff, sizeof(int64_t) * n, st) ||
            cudaMallocAsync((void **)&d_ooff, sizeof(int64_t) * n, st) ||
            cudaMallocAsync((void **)&d_qlen, sizeof(int) * n, st) || cudaMallocAsync((void **)&d_tlen, sizeof(int) * n, st) ||
            cudaMallocAsync((void **)&d_info, sizeof(int) * 3 * (size_t)n, st) ||
            cudaMallocAsync((void **)&d_se, sizeof(int) * 3 * (size_t)n, st) ||
            cudaMallocAsync((void **)&d_rest, sizeof(int) * n, st) ||
            cudaMallocAsync((void **)&d_o, sizeof(pb_pair_out) * n, st))
            rc = -1;
        void *ptrs[] = {d_q, d_t, d_map, d_ops, d_qoff, d_toff, d_ooff, d_qlen, d_tlen, d_info, d_se, d_rest, d_o};
        for (void *x : ptrs) frees.add(x);
        if (rc == 0) {
            cudaMemcpyAsync(d_q, h_q, qb, cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(d_t, h_t, tb, cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(d_map, mapper256, 256, cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(d_qoff, h_qoff, sizeof(int64_t) * n, cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(d_toff, h_toff, sizeof(int64_t) * n, cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(d_ooff, h_ops_off, sizeof(int64_t) * n, cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(d_qlen, h_qlen, sizeof(int) * n, cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(d_tlen, h_tlen, sizeof(int) * n, cudaMemcpyHostToDevice, st);
            cudaMemsetAsync(d_info, 0xff, sizeof(int) * 3 * (size_t)n, st);
            cudaMemsetAsync(d_o, 0, sizeof(pb_pair_out) * n, st);
            k_p16_map<<<148, 256, 0, st>>>(d_q, qb, d_map);
            k_p16_map<<<148, 256, 0, st>>>(d_t, tb, d_map);
            pb_diag_count_launch(2);
            if (cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
        }
        if (rc == 0) {
            pb_batch b = *tmpl;
            b.nprofs = 0;
            b.npairs = n;
            b.stats = 0;
            b.d_qall = d_q; b.d_qoff = d_qoff; b.d_qlen = d_qlen;
            b.d_targets = d_t; b.d_toff = d_toff; b.d_tlen = d_tlen;
            b.d_qlim = nullptr; b.d_tlim = nullptr;
            b.d_out = d_o;
            int nrest = 0;
            rc = pb::p16_pass(*job, &b, 0, nullptr, d_o, nullptr, d_rest, &nrest, st, d_ops, d_ooff, d_info);
        }
        if (rc == 0) {
            k_p16_ends<<<(n + 255) / 256, 256, 0, st>>>(d_o, n, d_se);
            pb_diag_count_launch(1);
            if (cudaMemcpyAsync(h_ends, d_se, sizeof(int) * 3 * (size_t)n, cudaMemcpyDeviceToHost, st) ||
                cudaMemcpyAsync(h_info, d_info, sizeof(int) * 3 * (size_t)n, cudaMemcpyDeviceToHost, st) ||
                cudaMemcpyAsync(h_ops, d_ops, ob, cudaMemcpyDeviceToHost, st))
                rc = -1;
        }
        if (cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
    }
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    return rc;
}

/* ---- the schedule table -------------------------------------------------------
 * Which length buckets of global score-only pairs run on the intra-task
 * wavefront kernel (one team of warps per pair) rather than the inter-task
 * pair kernel (one thread per pair). Written by the tuner
 * (parasail_b200/tune.py) as lines "mode bucket max_len inter_gcups
 * intra_gcups winner"; read from $PARASAIL_B200_SCHEDULE, else from
 * schedule.txt beside the library, on first use. */

namespace {

std::once_flag g_sched_once;
std::mutex g_sched_mu;
unsigned g_sched_nw = 0;

int sched_load_file(const char *path, unsigned *mask)
{
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    char line[256], mode[32], win[32];
    unsigned m = 0;
    int bucket, maxlen;
    double a, b;
    while (fgets(line, sizeof line, f)) {
        if (line[0] == '#') continue;
        if (sscanf(line, "%31s %d %d %lf %lf %31s", mode, &bucket, &maxlen, &a, &b, win) == 6 &&
            !strcmp(mode, "nw") && bucket >= 0 && bucket < 32 && !strcmp(win, "intra"))
            m |= 1u << bucket;
    }
    fclose(f);
    *mask = m;
    return 0;
}

void sched_init()
{
    unsigned m = 0;
    const char *env = getenv("PARASAIL_B200_SCHEDULE");
    if (env && *env) {
        if (sched_load_file(env, &m) == 0) g_sched_nw = m;
        return;
    }
    Dl_info info;
    if (dladdr((void *)&sched_init, &info) && info.dli_fname) {
        std::string dir(info.dli_fname);
        const size_t slash = dir.rfind('/');
        dir = slash == std::string::npos ? std::string(".") : dir.substr(0, slash);
        if (sched_load_file((dir + "/schedule.txt").c_str(), &m) == 0) g_sched_nw = m;
    }
}

}  // namespace

namespace pb {

unsigned pb_schedule_nw_mask()
{
    std::call_once(g_sched_once, sched_init);
    std::lock_guard<std::mutex> lk(g_sched_mu);
    return g_sched_nw;
}

}  // namespace pb

extern "C" unsigned parasail_b200_schedule_get(void)
{
    return pb::pb_schedule_nw_mask();
}

extern "C" void parasail_b200_schedule_set(unsigned intra_mask)
{
    std::call_once(g_sched_once, sched_init);
    std::lock_guard<std::mutex> lk(g_sched_mu);
    g_sched_nw = intra_mask;
}
