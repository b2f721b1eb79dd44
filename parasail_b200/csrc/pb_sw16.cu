/*
 * pb_sw16.cu -- Smith-Waterman score-only kernel in packed int16x2 lanes.
 *
 * Inter-task schedule: every thread aligns one query/target pair; a warp
 * takes 32 targets of similar length (targets are sorted by length) against
 * one query, and a persistent grid pulls such tasks for all queries of the
 * batch, longest first. The query is processed in passes of 2 x 16 rows:
 * the low 16-bit half of every register holds strip A (rows r0..r0+15) at
 * target column j, the high half strip B (rows r0+16..r0+31) at column j-1,
 * so strip B reads strip A's bottom row from the previous iteration and both
 * halves of one DPX instruction always do useful, independent work. A pass
 * hands its bottom row (H and the vertical-gap value F, 16 bits each) to the
 * next pass through a per-warp buffer laid out [column][lane]: one
 * contiguous 128-byte transaction per warp access. The int8 query profiles
 * of all the batch's queries live in shared memory; a column's 16 + 16
 * scores are two 16-byte loads expanded to int16x2 words by sign-extending
 * byte permutes. The recurrence is written so that two DPX operations per
 * row sit on the column's dependency chain (F = viaddmax(H_up, -open,
 * F_up - gap) and H = max(A, F), with A = max(H_diag + s, E, 0) computed off
 * the chain), and one in the biased form (k_sw16<true>, open >= gap): the
 * registers hold H - open and the profile s + open, and
 * F(i+1) = max(F(i) - gap, A(i) - open) since F(i) - open <= F(i) - gap.
 *
 * Semantics: the Smith-Waterman recurrence of the reference's striped/scan
 * kernels and of src/sw.c:131-158, with its end-position rule (first column
 * reaching the maximum, then the smallest query row; src/sw.c:150-158,
 * src/sw_striped_avx2_256_16.c:350-409). The 16-bit lanes hold exact values
 * while every H stays below 32767 - max(matrix) - 1; a pair that reaches
 * that bound is reported with PB_ST_OVERFLOW16 and must be rerun by the
 * exact 32-bit kernel. E and F start at -open, which is equivalent to -inf in
 * Smith-Waterman (H is clamped at 0) and keeps E - gap, F - gap in range.
 */
#include <cstdio>
#include <cstdint>
#include <climits>
#include <cuda_runtime.h>

#include "pb_cuda.h"
#include "pb_kernels.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <vector>
#include <mutex>

namespace pb {

static constexpr int SW16_R = 16;          /* query rows per strip (two strips per pass) */
static constexpr int SW16_WARPS = 8;       /* warps per block */

/* Packs two signed bytes (byte k of a and of b) into one int16x2 word:
 * low half from a, high half from b, each sign-extended (prmt sign mode). */
template <int K>
__device__ __forceinline__ uint32_t pack_pair(uint32_t a, uint32_t b)
{
    constexpr uint32_t sel = (K) | ((K | 8) << 4) | ((4 + K) << 8) | (((4 + K) | 8) << 12);
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
    return d;
}

__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel)
{
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
    return d;
}

__device__ __forceinline__ int s16lo(uint32_t x) { return (int)(int16_t)(x & 0xffffu); }
__device__ __forceinline__ int s16hi(uint32_t x) { return (int)(int16_t)(x >> 16); }
__device__ __forceinline__ uint32_t splat16(int v) { return ((uint32_t)(uint16_t)v) | ((uint32_t)(uint16_t)v << 16); }

struct Sw16Best {
    int score, i, j;
};

__device__ __forceinline__ void fold_best(Sw16Best &best, bool &have, const Sw16Best &s)
{
    /* higher score, then smaller column; an equal column keeps the earlier
     * (smaller) row, which was folded first */
    if (s.j >= 0 && (!have || s.score > best.score || (s.score == best.score && s.j < best.j))) {
        best = s;
        have = true;
    }
}

template <bool BIAS>
__global__ void __launch_bounds__(SW16_WARPS * 32, 2)
k_sw16(Sw16Params p, int *task_counter)
{
    extern __shared__ __align__(16) int8_t s_prof[];
    {
        const int4 *src = reinterpret_cast<const int4 *>(p.prof_all);
        int4 *dst = reinterpret_cast<int4 *>(s_prof);
        const int n16 = p.prof_bytes / 16;
        /* BIAS: every score + open (the host checked that it stays in int8) */
        const uint32_t b4 = BIAS ? 0x01010101u * (uint32_t)(uint8_t)p.open : 0u;
        for (int k = threadIdx.x; k < n16; k += blockDim.x) {
            int4 v = src[k];
            if (BIAS) {
                v.x = (int)__vadd4((uint32_t)v.x, b4); v.y = (int)__vadd4((uint32_t)v.y, b4);
                v.z = (int)__vadd4((uint32_t)v.z, b4); v.w = (int)__vadd4((uint32_t)v.w, b4);
            }
            dst[k] = v;
        }
    }
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    /* the block's SW16_WARPS buffers: warp w's is team_buf + w * maxlen * 32;
     * an entry is strip B's bottom row at one column, H in the low and F in
     * the high 16 bits */
    uint32_t *team_buf = p.scratch + (size_t)blockIdx.x * SW16_WARPS * p.maxlen * 32;
    const uint32_t gapO = splat16(-p.open);
    const uint32_t gapE = splat16(-p.gap);
    /* BIAS: the H registers, the pass buffer, the column maxima and the
     * best-so-far hold H - open, so "H = 0" reads as -open */
    const uint32_t zeroH = BIAS ? gapO : 0u;
    const int bias = BIAS ? p.open : 0;
    /* team tasks: the tasks at the front of the list (the most expensive,
     * each more than a fair share of the work per warp) are run by all
     * warps of a block together, pass k of the task on warp k % SW16_WARPS;
     * a pass reads the previous one's bottom row from that warp's buffer,
     * published every 32 columns through s_prog (generation-tagged, so that
     * it only grows) */
    __shared__ volatile long long s_prog[SW16_WARPS];
    __shared__ int s_task;
    __shared__ Sw16Best s_best[SW16_WARPS][32];
    __shared__ int s_have[SW16_WARPS][32];
    __shared__ int s_status[SW16_WARPS][32];
    volatile int *verr = task_counter + 2;
    /* this thread's copies of its strips' best columns: A's 16 words, then B's */
    uint4 *save = p.colsave + ((size_t)blockIdx.x * blockDim.x + threadIdx.x) * (SW16_R / 2);
    bool team = p.nteam > 0;

    /* warp tasks: the first of each warp block-strided, so that the largest
     * ones (the list is sorted by cost) are spread one per block instead of
     * landing on the first blocks' SMs; then from the shared counter */
    const int nwarps_total = gridDim.x * SW16_WARPS;
    bool first = true;
    for (;;) {
        int task = 0, trank = 0, tsize = 1;
        if (team) {
            __syncthreads();
            if (threadIdx.x == 0) s_task = atomicAdd(task_counter + 1, 1);
            if (threadIdx.x < SW16_WARPS) s_prog[threadIdx.x] = 0;
            __syncthreads();
            task = s_task;
            if (task >= p.nteam) { team = false; continue; }
            trank = wid;
            tsize = SW16_WARPS;
        } else {
            if (first) {
                task = p.nteam + blockIdx.x + gridDim.x * wid;
                first = false;
            } else {
                if (lane == 0) task = p.nteam + nwarps_total + atomicAdd(task_counter, 1);
                task = __shfl_sync(0xffffffffu, task, 0);
            }
            if (task >= p.ntasks) break;
        }
        uint32_t *out_buf = team_buf + (size_t)(team ? trank : wid) * p.maxlen * 32;
        const uint32_t *in_buf = team ? team_buf + (size_t)((trank + tsize - 1) % tsize) * p.maxlen * 32 : out_buf;
        const Sw16Task T = p.tasks[task];
        const Sw16Query Q = p.queries[T.q];
        const int s = T.first + lane;
        const bool valid = s < p.npairs;
        const int pid = valid ? p.order[s] : 0;
        const int len = valid ? p.tlen[pid] : 0;
        const uint8_t *tseq = p.targets + (valid ? p.toff[pid] : 0);
        int wmax = len;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) wmax = max(wmax, __shfl_xor_sync(0xffffffffu, wmax, o));
        const int8_t *prof = s_prof + Q.prof_off;
        const int lp = Q.lp, ql = Q.qlen;

        Sw16Best best = {0, 0, 0};
        bool have = false;
        int status = 0;

        const long long stride = (long long)wmax + 1;
        for (int r0 = 2 * SW16_R * trank; r0 < ql; r0 += 2 * SW16_R * tsize) {
            const int sp = r0 / (2 * SW16_R);            /* pass index */
            /* team: the previous pass (warp trank-1) must have published
             * column c before it is read */
            const long long in_base = (long long)((sp - 1) / tsize) * stride + 1;
            const long long out_base = (long long)(sp / tsize) * stride + 1;
            auto wait_for = [&](int c) -> bool {
                if (!team || sp == 0) return true;
                const int need = min(c, wmax - 1);
                bool ok = true;
                if (lane == 0 && need >= 0) {
                    const long long t0 = clock64();
                    while (s_prog[(trank + tsize - 1) % tsize] < in_base + need) {
                        if (*verr) { ok = false; break; }
                        if (clock64() - t0 > (1ll << 32)) { atomicExch(task_counter + 2, 1); ok = false; break; }
                    }
                    __threadfence_block();
                }
                ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
                __syncwarp();
                return ok;
            };
            if (!wait_for(33)) break;
            uint32_t H[SW16_R], E[SW16_R];
#pragma unroll
            for (int r = 0; r < SW16_R; ++r) { H[r] = zeroH; E[r] = gapO; }
            uint32_t dg = zeroH;            /* lo: H(r0-1, j-1); hi: H(r0+15, j-2) */
            uint32_t prev_h = zeroH, prev_f = gapO;   /* lo halves: strip A bottom at j-1 */
            Sw16Best sa = {0, -1, -1}, sb = {0, -1, -1};
            uint32_t sbest = zeroH;
            int cb = 0;                     /* residue of column j-1 (strip B) */
            const int8_t *pa_base = prof + r0;
            const int8_t *pb_base = prof + r0 + SW16_R;
            const bool more = r0 + 2 * SW16_R < ql;
            /* the residue and the previous pass's boundary of a column are
             * loaded two and three columns ahead: both come from L2 or DRAM,
             * and the chain of one column is too short to cover that latency
             * (this pass overwrites buf[j-1] at column j, never buf[j+3]) */
            const uint32_t vnone = prmt(zeroH, gapO, 0x5410u);
            int c_n1 = 0 < len ? tseq[0] : 0;
            int c_n2 = 1 < len ? tseq[1] : 0;
            uint32_t v_n1 = vnone, v_n2 = vnone, v_n3 = vnone;
            if (r0 != 0) {
                if (0 < wmax) v_n1 = __ldcg(&in_buf[lane]);
                if (1 < wmax) v_n2 = __ldcg(&in_buf[32 + lane]);
                if (2 < wmax) v_n3 = __ldcg(&in_buf[64 + lane]);
            }
            bool aborted = false;
            /* unrolled by two: the prefetch registers then rotate by renaming
             * instead of by moves, which would wait for the loads */
#pragma unroll 2
            for (int j = 0; j <= wmax; ++j) {
                if (team && j > 0 && (j & 31) == 0 && !wait_for(j + 33)) { aborted = true; break; }
                const int ca = c_n1;
                c_n1 = c_n2;
                c_n2 = j + 2 < len ? tseq[j + 2] : 0;
                uint32_t hu, fu;
                if (r0 == 0) {
                    hu = prmt(zeroH, prev_h, 0x5410u);      /* top row H = 0 */
                    fu = prmt(gapO, prev_f, 0x5410u);       /* top row F = -inf */
                } else {
                    const uint32_t v = v_n1;
                    v_n1 = v_n2;
                    v_n2 = v_n3;
                    v_n3 = j + 3 < wmax ? __ldcg(&in_buf[(size_t)(j + 3) * 32 + lane]) : vnone;
                    hu = prmt(v, prev_h, 0x5410u);          /* lo <- previous pass's strip B bottom */
                    fu = prmt(v, prev_f, 0x5432u);
                }
                const uint4 pa4 = *reinterpret_cast<const uint4 *>(pa_base + (size_t)ca * lp);
                const uint4 pb4 = *reinterpret_cast<const uint4 *>(pb_base + (size_t)cb * lp);
                uint32_t hd = dg;
                dg = hu;
                uint32_t cmax = zeroH;
                uint32_t aop = 0u;          /* BIAS: the previous row's max(H_diag + s, E, 0) - open */
#pragma unroll
                for (int r = 0; r < SW16_R; ++r) {
                    const uint32_t wa = r < 4 ? pa4.x : r < 8 ? pa4.y : r < 12 ? pa4.z : pa4.w;
                    const uint32_t wb = r < 4 ? pb4.x : r < 8 ? pb4.y : r < 12 ? pb4.z : pb4.w;
                    uint32_t sc;
                    switch (r & 3) {
                        case 0: sc = pack_pair<0>(wa, wb); break;
                        case 1: sc = pack_pair<1>(wa, wb); break;
                        case 2: sc = pack_pair<2>(wa, wb); break;
                        default: sc = pack_pair<3>(wa, wb); break;
                    }
                    if (BIAS) {
                        /* registers hold HO = H - open and the profile s + open:
                         *   E(i,j) = max(E(i,j-1) - gap, HO(i,j-1))
                         *   a      = max(HO(i-1,j-1) + (s + open), E, 0)
                         *   F(i,j) = max(F(i-1,j) - gap, HO(i-1,j))
                         *          = max(F(i-1,j) - gap, a(i-1) - open)  (open >= gap)
                         *   HO     = max(a - open, F - open)
                         * so one DPX operation per row sits on the chain */
                        const uint32_t e = __viaddmax_s16x2(E[r], gapE, H[r]);
                        const uint32_t a = __viaddmax_s16x2_relu(hd, sc, e);
                        const uint32_t ao = __vadd2(a, gapO);
                        const uint32_t f = __viaddmax_s16x2(fu, gapE, r == 0 ? hu : aop);
                        const uint32_t ho = __viaddmax_s16x2(f, gapO, ao);
                        E[r] = e;
                        hd = H[r];
                        H[r] = ho;
                        hu = ho;
                        fu = f;
                        aop = ao;
                        if (r & 1) cmax = __vimax3_s16x2(cmax, H[r - 1], ho);
                    } else {
                        /* E(i,j) = max(E(i,j-1) - gap, H(i,j-1) - open): off the chain */
                        const uint32_t e = __viaddmax_s16x2(E[r], gapE, __vadd2(H[r], gapO));
                        const uint32_t a = __viaddmax_s16x2_relu(hd, sc, e);
                        /* F(i,j) = max(H(i-1,j) - open, F(i-1,j) - gap): on the chain */
                        const uint32_t f = __viaddmax_s16x2(hu, gapO, __vadd2(fu, gapE));
                        const uint32_t h = __vmaxs2(a, f);
                        E[r] = e;
                        hd = H[r];
                        H[r] = h;
                        hu = h;
                        fu = f;
                        if (r & 1) cmax = __vimax3_s16x2(cmax, H[r - 1], h);
                    }
                }
                if (j >= 1 && more) {
                    out_buf[(size_t)(j - 1) * 32 + lane] = prmt(hu, fu, 0x7632u);
                    /* team: publish every 32 columns and the last one */
                    if (team && (((j - 1) & 31) == 31 || j - 1 == wmax - 1)) {
                        __threadfence_block();
                        __syncwarp();
                        if (lane == 0) s_prog[trank] = out_base + (j - 1);
                    }
                }
                prev_h = hu;
                prev_f = fu;
                cb = ca;
                if (j == 0) {
                    /* the high half computed column -1: restore strip B's
                     * left boundary (H = 0, E = -inf) */
#pragma unroll
                    for (int r = 0; r < SW16_R; ++r) {
                        H[r] = (H[r] & 0xffffu) | (zeroH & 0xffff0000u);
                        E[r] = (E[r] & 0xffffu) | (gapO & 0xffff0000u);
                    }
                }
                bool ge_lo, ge_hi;
                (void)__vibmax_s16x2(sbest, cmax, &ge_hi, &ge_lo);
                const bool up_a = !ge_lo && j < len;
                const bool up_b = !ge_hi && j >= 1 && j <= len;
                if (up_a || up_b) {
                    /* a new strip maximum: keep the column (the warp takes
                     * this branch whenever any lane improves, so the row is
                     * looked up once per pass, from the saved column) */
                    if (up_a) {
                        const int c = s16lo(cmax);
#pragma unroll
                        for (int k = 0; k < SW16_R / 4; ++k)
                            save[k] = make_uint4(H[4 * k], H[4 * k + 1], H[4 * k + 2], H[4 * k + 3]);
                        sa.score = c + bias; sa.j = j;
                        if (c + bias >= Q.posmax) status |= PB_ST_OVERFLOW16;
                    }
                    if (up_b) {
                        const int c = s16hi(cmax);
#pragma unroll
                        for (int k = 0; k < SW16_R / 4; ++k)
                            save[SW16_R / 4 + k] = make_uint4(H[4 * k], H[4 * k + 1], H[4 * k + 2], H[4 * k + 3]);
                        sb.score = c + bias; sb.j = j - 1;
                        if (c + bias >= Q.posmax) status |= PB_ST_OVERFLOW16;
                    }
                    sbest = (uint32_t)(uint16_t)(sa.score - bias) | ((uint32_t)(uint16_t)(sb.score - bias) << 16);
                }
            }
            if (aborted) break;
            /* the first row of each strip's best column reaching its maximum */
            if (sa.j >= 0) {
                int rr = SW16_R - 1;
#pragma unroll
                for (int k = SW16_R / 4 - 1; k >= 0; --k) {
                    const uint4 w = save[k];
                    const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
                    for (int x = 3; x >= 0; --x) if (s16lo(ws[x]) == sa.score - bias) rr = 4 * k + x;
                }
                sa.i = r0 + rr;
            }
            if (sb.j >= 0) {
                int rr = SW16_R - 1;
#pragma unroll
                for (int k = SW16_R / 4 - 1; k >= 0; --k) {
                    const uint4 w = save[SW16_R / 4 + k];
                    const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
                    for (int x = 3; x >= 0; --x) if (s16hi(ws[x]) == sb.score - bias) rr = 4 * k + x;
                }
                sb.i = r0 + SW16_R + rr;
            }
            fold_best(best, have, sa);
            fold_best(best, have, sb);
        }
        if (team) {
            /* merge the warps' per-lane bests: highest score, then smallest
             * column, then smallest row (the reference's first maximum) */
            s_best[wid][lane] = best;
            s_have[wid][lane] = have ? 1 : 0;
            s_status[wid][lane] = status;
            __syncthreads();
            if (wid != 0) continue;
            have = false;
            status = 0;
            for (int w = 0; w < SW16_WARPS; ++w) {
                status |= s_status[w][lane];
                if (!s_have[w][lane]) continue;
                const Sw16Best c = s_best[w][lane];
                if (!have || c.score > best.score || (c.score == best.score && (c.j < best.j ||
                                                        (c.j == best.j && c.i < best.i)))) {
                    best = c;
                    have = true;
                }
            }
        }
        /* no positive cell: score 0 at (0, 0), the first cell (src/sw.c:150-158) */
        if (valid) {
            pb_pair_out o = {};
            o.score = have ? best.score : 0;
            o.end_query = have ? best.i : 0;
            o.end_ref = have ? best.j : 0;
            o.max_h = o.score;
            o.status = status;
            p.out[(size_t)T.q * p.npairs + pid] = o;
        }
    }
}

/*
 * Small searches (few warp tasks, e.g. one query against 1,000 targets):
 * the intra-task wavefront. One warp aligns one (query, target) pair in
 * exact int32: a pass covers 256 query rows, 8 per lane, and lane k
 * computes column t - k at iteration t, so the warp's 32 lanes work on 32
 * columns of one pair at once and the row-to-row dependency chain is 8
 * rows long instead of the inter-task kernel's per-target 16-row strips on
 * a handful of SMs. Row above a lane's first row: the previous lane's last
 * row by __shfl_up_sync, or, for lane 0, the previous pass's bottom row
 * from the warp's buffer (passes of one pair run one after the other on
 * the warp). The recurrence and end rule are src/sw.c:102-158's: H =
 * max(0, H_diag + s, E, F), the first maximum in column-major order, score
 * 0 at (0, 0) when no cell is positive; with open >= gap, F of the next
 * row is max(F - gap, max(a, 0) - open) with a = max(H_diag + s, E), one
 * dependent operation per row.
 */
/* RL query rows per lane (4, 8, 12 or 16; a pass covers 32 * RL rows),
 * chosen per launch from the query lengths (wave_rows) */
template <bool GE, int RL>
__global__ void __launch_bounds__(SW16_WARPS * 32, 2)
k_sw_wave(Sw16Params p, int *counter)
{
    extern __shared__ __align__(16) int8_t s_prof[];
    {
        const int4 *src = reinterpret_cast<const int4 *>(p.prof_all);
        int4 *dst = reinterpret_cast<int4 *>(s_prof);
        const int n16 = p.prof_bytes / 16;
        for (int k = threadIdx.x; k < n16; k += blockDim.x) dst[k] = src[k];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    int2 *buf = reinterpret_cast<int2 *>(p.scratch) + (size_t)(blockIdx.x * SW16_WARPS + wid) * p.maxlen;
    const int open = p.open, gap = p.gap;
    const int NEG = INT_MIN / 4;
    const long long nitems = (long long)p.nq * p.npairs;
    for (;;) {
        long long w = 0;
        if (lane == 0) w = atomicAdd(counter, 1);
        w = __shfl_sync(0xffffffffu, w, 0);
        if (w >= nitems) break;
        const int q = (int)(w / p.npairs);
        const int pid = p.order[w % p.npairs];
        const Sw16Query Q = p.queries[q];
        const int n = Q.qlen, m = p.tlen[pid];
        const uint8_t *ts = p.targets + p.toff[pid];
        const int8_t *prof = s_prof + Q.prof_off;
        const int npass = (n + 32 * RL - 1) / (32 * RL);
        Sw16Best best = {0, -1, -1};
        int status = 0;
        for (int pass = 0; pass < npass; ++pass) {
            const int R0 = pass * 32 * RL + lane * RL;
            /* a lane whose rows reach past lp (a multiple of 64, at least
             * qlen + 32) holds only dummy rows: they score 0 */
            const bool rows_in = R0 + RL <= Q.lp;
            int Hl[RL], E[RL];
#pragma unroll
            for (int r = 0; r < RL; ++r) { Hl[r] = 0; E[r] = NEG; }
            int dg = 0;                               /* H(R0 - 1, j - 1); H(i, -1) = 0 */
            int sh_h = 0, sh_f = NEG;
            int2 cur = make_int2(0, NEG);
            const int nreal = min(RL, max(0, n - R0));
            auto res_at = [&](int c) -> int { return (c >= 0 && c < m) ? (int)ts[c] : 0; };
            int tc_n1 = res_at(-lane), tc_n2 = res_at(1 - lane);
            for (int it = 0; it <= m - 1 + 31; ++it) {
                const int j = it - lane;
                if (((it & 31) == 0) && pass > 0) {
                    const int c = it + lane;
                    cur = c < m ? __ldcg(&buf[c]) : make_int2(0, NEG);
                }
                const int vh = __shfl_sync(0xffffffffu, cur.x, it & 31);
                const int vf = __shfl_sync(0xffffffffu, cur.y, it & 31);
                int up_h = __shfl_up_sync(0xffffffffu, sh_h, 1);
                int up_f = __shfl_up_sync(0xffffffffu, sh_f, 1);
                const int tc_raw = tc_n1;
                tc_n1 = tc_n2;
                tc_n2 = res_at(j + 2);
                if (lane == 0) {
                    /* row above the pass: row -1 (H = 0, F = -inf) or the
                     * previous pass's bottom row */
                    up_h = pass > 0 ? vh : 0;
                    up_f = pass > 0 ? vf : NEG;
                }
                if (j >= 0 && j < m) {
                    int tc = tc_raw;
                    if (tc >= p.nletters) { status |= PB_ST_BADCODE; tc = 0; }
                    /* R0 and lp are multiples of 4: word loads */
                    uint32_t sw[RL / 4];
#pragma unroll
                    for (int k = 0; k < RL / 4; ++k)
                        sw[k] = rows_in ? reinterpret_cast<const uint32_t *>(prof + (size_t)tc * Q.lp + R0)[k] : 0u;
                    int hd = dg;
                    int f = max(up_f - gap, up_h - open);
                    int cmax = 0, last_h = 0, last_f = 0;
#pragma unroll
                    for (int r = 0; r < RL; ++r) {
                        const int sc = (int)(int8_t)((sw[r >> 2] >> (8 * (r & 3))) & 0xffu);
                        const int e = max(E[r] - gap, Hl[r] - open);
                        const int a = __viaddmax_s32(hd, sc, e);
                        const int h = __vimax_s32_relu(a, f);
                        if (r < nreal) cmax = max(cmax, h);
                        last_h = h;
                        last_f = f;
                        if (GE) f = __viaddmax_s32(f, -gap, max(a, 0) - open);
                        else f = __viaddmax_s32(f, -gap, h - open);
                        E[r] = e;
                        hd = Hl[r];
                        Hl[r] = h;
                    }
                    /* a higher maximum than the lane's best, or the same one
                     * in an earlier column (a later pass revisits the
                     * columns): the first row reaching it in this column */
                    if (cmax > best.score || (cmax == best.score && j < best.j)) {
                        int rr = 0;
#pragma unroll
                        for (int r = RL - 1; r >= 0; --r) if (r < nreal && Hl[r] == cmax) rr = r;
                        best.score = cmax; best.j = j; best.i = R0 + rr;
                    }
                    dg = up_h;
                    sh_h = last_h;
                    sh_f = last_f;
                    if (lane == 31 && pass + 1 < npass) buf[j] = make_int2(last_h, last_f);
                }
            }
            __syncwarp();
        }
        /* the lanes' bests in the reference's order: higher score, then
         * smaller column, then smaller row */
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const int os = __shfl_xor_sync(0xffffffffu, best.score, o);
            const int oj = __shfl_xor_sync(0xffffffffu, best.j, o);
            const int oi = __shfl_xor_sync(0xffffffffu, best.i, o);
            const bool take = oj >= 0 && (best.j < 0 || os > best.score ||
                                          (os == best.score && (oj < best.j || (oj == best.j && oi < best.i))));
            if (take) { best.score = os; best.j = oj; best.i = oi; }
        }
        status = __reduce_or_sync(0xffffffffu, status);
        if (lane == 0) {
            pb_pair_out o = {};
            o.score = best.j >= 0 ? best.score : 0;
            o.end_query = best.j >= 0 ? best.i : 0;
            o.end_ref = best.j >= 0 ? best.j : 0;
            o.max_h = o.score;
            o.status = status;
            p.out[(size_t)q * p.npairs + pid] = o;
        }
    }
}

}  // namespace pb

namespace {

__global__ void k_iota(int *v, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

__global__ void k_collect_overflow(const pb_pair_out *out, int n, int *list, int *count,
                                   const int64_t *toff, const int *tlen,
                                   int64_t *otoff, int *otlen)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && (out[i].status & PB_ST_OVERFLOW16)) {
        const int k = atomicAdd(count, 1);
        list[k] = i;
        otoff[k] = toff[i];
        otlen[k] = tlen[i];
    }
}

__global__ void k_scatter(const pb_pair_out *src, const int *list, int n, pb_pair_out *dst)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) dst[list[k]] = src[k];
}

}  // namespace

/* Everything the score kernel needs for a batch that depends only on the
 * profiles and the target lengths: the length order of the targets, the
 * task list (most cells first, team tasks at the front), the concatenated
 * int8 profiles and the per-warp pass buffers. Buffers come from st's pool
 * and are released by sw16_release. */
struct Sw16Prep {
    pb::Sw16Params p;
    int blocks;
    bool wave;                    /* few tasks: the intra-task wavefront k_sw_wave */
    int wave_rl;                  /* its rows per lane */
    size_t prof_bytes;
    int *counter;                 /* [warp tasks, team tasks, error, spare] */
    void *bufs[10];
};

static void sw16_release(Sw16Prep *pr, cudaStream_t st)
{
    for (void *x : pr->bufs) if (x) cudaFreeAsync(x, st);
    memset(pr->bufs, 0, sizeof pr->bufs);
}

typedef void (*WaveKernel)(pb::Sw16Params, int *);

/* k_sw_wave for (open >= gap, rows per lane) */
static WaveKernel wave_kernel(bool ge, int rl)
{
    if (ge) {
        switch (rl) {
            case 4: return pb::k_sw_wave<true, 4>;
            case 12: return pb::k_sw_wave<true, 12>;
            case 16: return pb::k_sw_wave<true, 16>;
            default: return pb::k_sw_wave<true, 8>;
        }
    }
    switch (rl) {
        case 4: return pb::k_sw_wave<false, 4>;
        case 12: return pb::k_sw_wave<false, 12>;
        case 16: return pb::k_sw_wave<false, 16>;
        default: return pb::k_sw_wave<false, 8>;
    }
}

static void wave_set_smem(int bytes)
{
    for (int ge = 0; ge < 2; ++ge)
        for (int rl = 4; rl <= 16; rl += 4)
            pb_raise_smem((const void *)wave_kernel(ge != 0, rl), bytes);
}

static int sw16_prepare(const pb_batch *b, pb_pair_out *d_out_all, size_t prof_bytes, cudaStream_t st,
                        Sw16Prep *pr)
{
    const int n = b->npairs, nq = b->nprofs;
    memset(pr, 0, sizeof *pr);
    pr->prof_bytes = prof_bytes;
    /* targets sorted by length, descending */
    int *keys_sorted = nullptr, *idx = nullptr, *order = nullptr, *counter = nullptr;
    void *tmp = nullptr;
    int8_t *prof_all = nullptr;
    pb::Sw16Task *d_tasks = nullptr;
    pb::Sw16Query *d_q = nullptr;
    size_t tmp_sort = 0;
    /* an allocation that fails ends the call before anything writes
     * through it, releasing what was allocated */
    auto give_up = [&]() {
        void *owned[10] = {keys_sorted, idx, order, counter, tmp, prof_all, d_tasks, d_q, nullptr, nullptr};
        memcpy(pr->bufs, owned, sizeof owned);
        sw16_release(pr, st);
        cudaGetLastError();
        return -1;
    };
    if (cudaMallocAsync((void **)&keys_sorted, sizeof(int) * n, st) != cudaSuccess ||
        cudaMallocAsync((void **)&idx, sizeof(int) * n, st) != cudaSuccess ||
        cudaMallocAsync((void **)&order, sizeof(int) * n, st) != cudaSuccess ||
        cudaMallocAsync((void **)&counter, sizeof(int) * 4, st) != cudaSuccess)
        return give_up();
    k_iota<<<(n + 255) / 256, 256, 0, st>>>(idx, n);
    cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp_sort, b->d_tlen, keys_sorted, idx, order, n, 0, 32, st);
    if (cudaMallocAsync(&tmp, tmp_sort, st) != cudaSuccess) return give_up();
    cub::DeviceRadixSort::SortPairsDescending(tmp, tmp_sort, b->d_tlen, keys_sorted, idx, order, n, 0, 32, st);
    std::vector<int> hlen(n);
    cudaMemcpyAsync(hlen.data(), keys_sorted, sizeof(int) * n, cudaMemcpyDeviceToHost, st);
    cudaMemsetAsync(counter, 0, sizeof(int) * 4, st);   /* warp tasks, team tasks, error */
    /* concatenated int8 profiles */
    std::vector<pb::Sw16Query> hq(nq);
    if (cudaMallocAsync((void **)&prof_all, prof_bytes, st) != cudaSuccess) return give_up();
    {
        size_t off = 0;
        for (int q = 0; q < nq; ++q) {
            const pb_device_profile *dp = b->profs[q];
            const size_t bytes = (size_t)dp->size * dp->lp;
            cudaMemcpyAsync(prof_all + off, dp->d_prof8, bytes, cudaMemcpyDeviceToDevice, st);
            hq[q].prof_off = (int)off;
            hq[q].qlen = dp->qlen;
            hq[q].lp = dp->lp;
            hq[q].posmax = 32767 - dp->mmax - 1;
            off += bytes;
        }
    }
    cudaStreamSynchronize(st);
    /* tasks: (query, block of 32 sorted targets), most cells first */
    const int nblk = (n + 31) / 32;
    std::vector<pb::Sw16Task> tasks((size_t)nq * nblk);
    std::vector<int64_t> cost((size_t)nq * nblk);
    for (int q = 0; q < nq; ++q)
        for (int k = 0; k < nblk; ++k) {
            tasks[(size_t)q * nblk + k].q = q;
            tasks[(size_t)q * nblk + k].first = 32 * k;
        }
    std::vector<int> perm(tasks.size());
    for (size_t k = 0; k < perm.size(); ++k) perm[k] = (int)k;
    std::sort(perm.begin(), perm.end(), [&](int x, int y) {
        const int64_t cx = (int64_t)hq[tasks[x].q].qlen * hlen[tasks[x].first];
        const int64_t cy = (int64_t)hq[tasks[y].q].qlen * hlen[tasks[y].first];
        return cx > cy;
    });
    std::vector<pb::Sw16Task> sorted_tasks(tasks.size());
    for (size_t k = 0; k < perm.size(); ++k) sorted_tasks[k] = tasks[perm[k]];
    if (cudaMallocAsync((void **)&d_tasks, sizeof(pb::Sw16Task) * sorted_tasks.size(), st) != cudaSuccess ||
        cudaMallocAsync((void **)&d_q, sizeof(pb::Sw16Query) * nq, st) != cudaSuccess)
        return give_up();
    cudaMemcpyAsync(d_tasks, sorted_tasks.data(), sizeof(pb::Sw16Task) * sorted_tasks.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(d_q, hq.data(), sizeof(pb::Sw16Query) * nq, cudaMemcpyHostToDevice, st);

    int per_sm = 0, nsm = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    /* the biased kernel (one DPX operation per row on the dependency
     * chain) needs open >= gap and every score + open inside int8 */
    bool bias = b->open >= b->gap;
    for (int q = 0; q < nq; ++q)
        if (b->profs[q]->mmax + b->open > 127 || b->profs[q]->mmin + b->open < -128) bias = false;
    pb_raise_smem((const void *)pb::k_sw16<true>, (int)prof_bytes);
    pb_raise_smem((const void *)pb::k_sw16<false>, (int)prof_bytes);
    if (bias)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pb::k_sw16<true>, pb::SW16_WARPS * 32, prof_bytes);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pb::k_sw16<false>, pb::SW16_WARPS * 32, prof_bytes);
    if (per_sm < 1) per_sm = 1;
    int blocks = per_sm * nsm;
    const int need = (int)((sorted_tasks.size() + pb::SW16_WARPS - 1) / pb::SW16_WARPS);
    /* few tasks (a small database, e.g. one query against 1,000 targets):
     * every task gets a block of its own and is run as a team task, its
     * passes spread over the block's warps, instead of leaving most SMs
     * idle with one warp per task */
    const bool few = (int)sorted_tasks.size() <= blocks;
    if (few) blocks = (int)sorted_tasks.size();
    else if (blocks > need) blocks = need;
    const int maxlen = hlen[0] + 1;
    /* few tasks: the intra-task wavefront, a warp per pair, as many warps
     * as pairs (up to the resident warps) */
    pr->wave = few;
    if (few) {
        /* rows per lane: the fewest row-steps over the batch's queries,
         * npass * (RL + 4) per column, the 4 standing for the per-column
         * shuffles and loads (one query of 300 rows: one pass of 12 rows
         * per lane instead of two of 8) */
        int best_rl = 8;
        double best_cost = -1.0;
        for (int rl = 4; rl <= 16; rl += 4) {
            double cost = 0.0;
            for (int q = 0; q < nq; ++q) cost += (double)((hq[q].qlen + 32 * rl - 1) / (32 * rl)) * (rl + 4);
            if (best_cost < 0.0 || cost < best_cost) { best_cost = cost; best_rl = rl; }
        }
        pr->wave_rl = best_rl;
        int wper = 0;
        wave_set_smem((int)prof_bytes);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&wper, wave_kernel(b->open >= b->gap, best_rl),
                                                      pb::SW16_WARPS * 32, prof_bytes);
        if (wper < 1) wper = 1;
        const long long items = (long long)n * nq;
        const long long want = (items + pb::SW16_WARPS - 1) / pb::SW16_WARPS;
        blocks = (int)std::min<long long>(want, (long long)wper * nsm);
    }
    uint32_t *scratch = nullptr;
    const size_t scratch_bytes = few ? sizeof(int2) * (size_t)maxlen * blocks * pb::SW16_WARPS
                                     : sizeof(uint32_t) * (size_t)maxlen * 32 * blocks * pb::SW16_WARPS;
    if (cudaMallocAsync((void **)&scratch, scratch_bytes, st) != cudaSuccess)
        scratch = nullptr;
    /* k_sw16: per thread, the two strips' best columns (2 x 16 words) */
    uint4 *colsave = nullptr;
    if (!few && cudaMallocAsync((void **)&colsave, sizeof(uint4) * (pb::SW16_R / 2) * (size_t)blocks * pb::SW16_WARPS * 32,
                                st) != cudaSuccess)
        colsave = nullptr;
    /* team tasks: those above a fair share of the work per warp, which one
     * warp alone would finish last */
    int nteam = few ? (int)sorted_tasks.size() : 0;
    if (!few) {
        double total = 0.0;
        for (const auto &t : sorted_tasks) total += (double)hq[t.q].qlen * hlen[t.first];
        const double fair = total / ((double)blocks * pb::SW16_WARPS);
        while (nteam < (int)sorted_tasks.size() &&
               (double)hq[sorted_tasks[nteam].q].qlen * hlen[sorted_tasks[nteam].first] > fair)
            ++nteam;
    }
    pb::Sw16Params &p = pr->p;
    p.open = b->open; p.gap = b->gap; p.npairs = n; p.nq = nq; p.nletters = b->profs[0]->size;
    p.bias = bias ? 1 : 0;
    p.ntasks = (int)sorted_tasks.size(); p.maxlen = maxlen; p.nteam = nteam;
    p.queries = d_q; p.prof_all = prof_all; p.prof_bytes = (int)prof_bytes;
    p.order = order; p.tasks = d_tasks;
    p.targets = b->d_targets; p.toff = b->d_toff; p.tlen = b->d_tlen;
    p.scratch = scratch; p.out = d_out_all; p.colsave = colsave;
    pr->blocks = blocks;
    pr->counter = counter;
    void *owned[10] = {keys_sorted, idx, order, counter, tmp, prof_all, d_tasks, d_q, scratch, colsave};
    memcpy(pr->bufs, owned, sizeof owned);
    if (!keys_sorted || !idx || !order || !counter || !tmp || !prof_all || !d_tasks || !d_q || !scratch ||
        (!few && !colsave) ||
        cudaGetLastError() != cudaSuccess) {
        sw16_release(pr, st);
        return -1;
    }
    return 0;
}

/* the kernel on a prepared batch (its counters zeroed first) */
static void sw16_launch(const Sw16Prep &pr, cudaStream_t st)
{
    cudaMemsetAsync(pr.counter, 0, sizeof(int) * 4, st);
    if (pr.wave) {
        wave_kernel(pr.p.open >= pr.p.gap, pr.wave_rl)<<<pr.blocks, pb::SW16_WARPS * 32, pr.prof_bytes, st>>>(
            pr.p, pr.counter);
    } else {
        if (pr.p.bias)
            pb::k_sw16<true><<<pr.blocks, pb::SW16_WARPS * 32, pr.prof_bytes, st>>>(pr.p, pr.counter);
        else
            pb::k_sw16<false><<<pr.blocks, pb::SW16_WARPS * 32, pr.prof_bytes, st>>>(pr.p, pr.counter);
    }
}

/* nq profiles against the same targets; out[q * npairs + i]. */
extern "C" int pb_cuda_align_sw16_multi(const pb_batch *b, pb_pair_out *d_out_all)
{
    if (pb_cuda_init() != 0) return -1;
    const int n = b->npairs, nq = b->nprofs;
    if (n <= 0 || nq <= 0) return 0;
    bool ok = b->alg == PB_SW && !b->stats && !b->d_qlim && !b->d_tlim && b->open + b->gap <= 30000;
    size_t prof_bytes = 0;
    for (int q = 0; q < nq && ok; ++q) {
        const pb_device_profile *dp = b->profs[q];
        ok = dp->fits8 && dp->size == b->profs[0]->size;
        prof_bytes += (size_t)dp->size * dp->lp;
    }
    if (!ok || prof_bytes > 200 * 1024) {
        /* outside this kernel's domain: the exact kernel, one profile at a time */
        for (int q = 0; q < nq; ++q) {
            pb_batch one = *b;
            one.profs = &b->profs[q];
            one.nprofs = 1;
            one.d_out = d_out_all + (size_t)q * n;
            if (pb_cuda_align_exact(&one) != 0) return -1;
        }
        return 0;
    }
    cudaStream_t st = 0;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    int rc = 0;
    Sw16Prep prep;
    if (sw16_prepare(b, d_out_all, prof_bytes, st, &prep) != 0) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
        return -1;
    }
    int *counter = prep.counter;
    cudaEvent_t ev0, ev1;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    cudaEventRecord(ev0, st);
    sw16_launch(prep, st);
    cudaEventRecord(ev1, st);
    if (cudaGetLastError() != cudaSuccess) rc = -1;
    pb_diag_count_launch(2);   /* k_iota, k_sw16 */
    {
        int herr = 0;
        cudaMemcpyAsync(&herr, counter + 2, sizeof(int), cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        if (herr) {
            fprintf(stderr, "pb_cuda_align_sw16_multi: a pass wait exceeded its bound\n");
            rc = -1;
        }
    }
    {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev0, ev1);
        pb_diag_sw16_time(ms);
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
    }
    /* pairs that left the 16-bit range: the exact kernel, per query */
    int *list = nullptr, *otlen = nullptr;
    int64_t *otoff = nullptr;
    if (cudaMallocAsync((void **)&list, sizeof(int) * n, st) != cudaSuccess ||
        cudaMallocAsync((void **)&otlen, sizeof(int) * n, st) != cudaSuccess ||
        cudaMallocAsync((void **)&otoff, sizeof(int64_t) * n, st) != cudaSuccess) {
        cudaGetLastError();
        rc = -1;   /* nothing below runs; the buffers that exist are freed */
    }
    for (int q = 0; q < nq && rc == 0; ++q) {
        int nover = 0;
        pb_pair_out *oq = d_out_all + (size_t)q * n;
        cudaMemsetAsync(counter + 1, 0, sizeof(int), st);
        k_collect_overflow<<<(n + 255) / 256, 256, 0, st>>>(oq, n, list, counter + 1, b->d_toff,
                                                            b->d_tlen, otoff, otlen);
        pb_diag_count_launch(1);
        cudaMemcpyAsync(&nover, counter + 1, sizeof(int), cudaMemcpyDeviceToHost, st);
        cudaStreamSynchronize(st);
        if (nover > 0) {
            pb_pair_out *tmpo = nullptr;
            if (cudaMallocAsync((void **)&tmpo, sizeof(pb_pair_out) * nover, st) != cudaSuccess) {
                cudaGetLastError();
                rc = -1;
                break;
            }
            cudaStreamSynchronize(st);
            pb_batch sub = *b;
            sub.profs = &b->profs[q];
            sub.nprofs = 1;
            sub.npairs = nover;
            sub.d_toff = otoff;
            sub.d_tlen = otlen;
            sub.d_out = tmpo;
            sub.d_prof_index = nullptr;
            rc = pb_cuda_align_exact(&sub);
            k_scatter<<<(nover + 255) / 256, 256, 0, st>>>(tmpo, list, nover, oq);
            pb_diag_count_launch(1);
            cudaFreeAsync(tmpo, st);
        }
    }
    if (list) cudaFreeAsync(list, st);
    if (otlen) cudaFreeAsync(otlen, st);
    if (otoff) cudaFreeAsync(otoff, st);
    sw16_release(&prep, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
    cudaStreamDestroy(st);
    return rc;
}

/* One SW score pair from host target codes: the wavefront kernel on one
 * warp (exact int32, no overflow rerun), its descriptors and the codes in
 * one upload to the thread's arena, the output in one download. */
extern "C" int pb_cuda_sw_single(const pb_device_profile *dp, int open, int gap, const uint8_t *h_codes, int tlen,
                                 pb_pair_out *h_out)
{
    if (pb_cuda_init() != 0) return -1;
    if (!dp->fits8 || !dp->d_prof8 || tlen <= 0 || open + gap > 30000) return -2;
    cudaGetLastError();   /* a launch error below is this call's own */
    const size_t prof_bytes = (size_t)dp->size * dp->lp;
    /* the kernels' shared-memory limit raised to this profile (never lowered) */
    {
        int dev = 0, optin = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        if ((long long)prof_bytes > optin) return -2;
        wave_set_smem((int)prof_bytes);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            pb_cuda_set_error("single-pair SW shared memory", cudaGetErrorString(e));
            return -1;
        }
    }
    /* [Sw16Query][toff int64][order, tlen, counter x4: int][out][codes] then the scratch of 8 warps */
    const size_t o_q = 0, o_toff = 16, o_ints = 24, o_out = 48;
    const size_t o_codes = (o_out + sizeof(pb_pair_out) + 15) & ~(size_t)15;
    const size_t up = (o_codes + (size_t)tlen + 16 + 15) & ~(size_t)15;
    const size_t total = up + sizeof(int2) * (size_t)(tlen + 1) * pb::SW16_WARPS;
    char *h = nullptr;
    char *d = pb_single_arena(total, up, &h);
    if (!d) { pb_cuda_set_error("single-pair arena", "allocation failed"); return -1; }
    pb::Sw16Query q;
    q.prof_off = 0; q.qlen = dp->qlen; q.lp = dp->lp; q.posmax = 32767 - dp->mmax - 1;
    memcpy(h + o_q, &q, sizeof q);
    const int ints[6] = {0, tlen, 0, 0, 0, 0};
    memcpy(h + o_ints, ints, sizeof ints);
    memcpy(h + o_codes, h_codes, (size_t)tlen);
    cudaStream_t st = (cudaStream_t)pb_cuda_stream();
    if (cudaMemcpyAsync(d, h, up, cudaMemcpyHostToDevice, st) != cudaSuccess) {
        pb_cuda_set_error("single-pair upload", cudaGetErrorString(cudaGetLastError()));
        return -1;
    }
    pb::Sw16Params p;
    memset(&p, 0, sizeof p);
    p.open = open; p.gap = gap; p.npairs = 1; p.nq = 1; p.ntasks = 1; p.maxlen = tlen + 1;
    p.nletters = dp->size;
    p.queries = reinterpret_cast<const pb::Sw16Query *>(d + o_q);
    p.prof_all = dp->d_prof8; p.prof_bytes = (int)prof_bytes;
    p.order = reinterpret_cast<const int *>(d + o_ints);
    p.targets = reinterpret_cast<const uint8_t *>(d + o_codes);
    p.toff = reinterpret_cast<const int64_t *>(d + o_toff);
    p.tlen = reinterpret_cast<const int *>(d + o_ints) + 1;
    p.scratch = reinterpret_cast<uint32_t *>(d + up);
    p.out = reinterpret_cast<pb_pair_out *>(d + o_out);
    int rl = 8;
    double best = -1.0;
    for (int r = 4; r <= 16; r += 4) {
        const double c = (double)((dp->qlen + 32 * r - 1) / (32 * r)) * (r + 4);
        if (best < 0.0 || c < best) { best = c; rl = r; }
    }
    int *counter = reinterpret_cast<int *>(d + o_ints) + 2;
    wave_kernel(open >= gap, rl)<<<1, pb::SW16_WARPS * 32, prof_bytes, st>>>(p, counter);
    pb_diag_count_launch(1);
    {
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            pb_cuda_set_error("single-pair SW launch", cudaGetErrorString(e));
            return -1;
        }
    }
    if (cudaMemcpyAsync(h_out, d + o_out, sizeof(pb_pair_out), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
        pb_cuda_set_error("single-pair SW", cudaGetErrorString(cudaGetLastError()));
        return -1;
    }
    return 0;
}

extern "C" int pb_cuda_align_sw16(const pb_batch *b)
{
    if (b->nprofs != 1 || b->d_prof_index) return pb_cuda_align_exact(b);
    return pb_cuda_align_sw16_multi(b, b->d_out);
}

/* ---- database-search plans: the search as one CUDA graph ------------------ */

namespace {

__global__ void k_count_overflow(const pb_pair_out *__restrict__ out, int n, int *__restrict__ count)
{
    int c = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        c += (out[i].status & PB_ST_OVERFLOW16) != 0;
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

struct DbPlan {
    cudaStream_t st = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    Sw16Prep prep;
    bool prepared = false;
    pb_pair_out *o1 = nullptr;
    int *need = nullptr, *counts = nullptr;   /* counts[0..2] lane lists (unused), [4] overflow */
    pb_job job;
    pb_batch b;
    std::vector<const pb_device_profile *> profs;
    pb_record *rec = nullptr;
    uint8_t *map = nullptr;                   /* device mapper of plan runs from host memory */
};

void plan_destroy(DbPlan *pl)
{
    if (pl->exec) cudaGraphExecDestroy(pl->exec);
    if (pl->graph) cudaGraphDestroy(pl->graph);
    if (pl->st) {
        if (pl->prepared) sw16_release(&pl->prep, pl->st);
        if (pl->o1) cudaFreeAsync(pl->o1, pl->st);
        if (pl->need) cudaFreeAsync(pl->need, pl->st);
        if (pl->counts) cudaFreeAsync(pl->counts, pl->st);
        if (pl->map) cudaFreeAsync(pl->map, pl->st);
        cudaStreamSynchronize(pl->st);
        cudaStreamDestroy(pl->st);
    }
    delete pl;
}

}  // namespace

/* A Smith-Waterman score-only database search (every profile of b against
 * every target) whose host-side preparation -- the length order of the
 * targets, the task list, the concatenated profiles, every buffer -- is done
 * once, and whose device work -- the int16x2 score kernel, the count of
 * pairs past the 16-bit range and the width resolution writing d_rec -- is
 * recorded once as a CUDA graph. Running the plan replays the graph on the
 * current contents of b's target buffers (same lengths). Returns -1 when
 * the job is outside what the graph holds (statistics, lane-exact widths,
 * the score kernel's domain). */
extern "C" int pb_cuda_db_plan_create(const pb_job *job, const pb_batch *b, pb_record *d_rec, void **out)
{
    *out = nullptr;
    if (pb_cuda_init() != 0) return -1;
    const int n = b->npairs, nq = b->nprofs;
    const pb_mode *m = &job->mode;
    if (n <= 0 || nq <= 0 || m->alg != PB_SW || m->stats || job->bits < 0) return -1;
    for (int w = 8; w <= 32; w *= 2) if (pb_lane_forced(m, w)) return -1;
    if (b->open + b->gap > 30000 || (long long)n * nq > INT32_MAX) return -1;
    size_t prof_bytes = 0;
    for (int q = 0; q < nq; ++q) {
        const pb_device_profile *dp = b->profs[q];
        if (!dp->fits8 || dp->size != b->profs[0]->size) return -1;
        prof_bytes += (size_t)dp->size * dp->lp;
    }
    if (prof_bytes > 200 * 1024) return -1;
    DbPlan *pl = new DbPlan();
    pl->job = *job;
    pl->profs.assign(b->profs, b->profs + nq);
    pl->b = *b;
    pl->b.profs = pl->profs.data();
    pl->rec = d_rec;
    int rc = 0;
    if (cudaStreamCreateWithFlags(&pl->st, cudaStreamNonBlocking) != cudaSuccess) { pl->st = nullptr; rc = -1; }
    const size_t N = (size_t)n * nq;
    if (rc == 0 && (cudaMallocAsync((void **)&pl->o1, sizeof(pb_pair_out) * N, pl->st) != cudaSuccess ||
                    cudaMallocAsync((void **)&pl->need, sizeof(int) * 3 * (size_t)n, pl->st) != cudaSuccess ||
                    cudaMallocAsync((void **)&pl->counts, sizeof(int) * 8, pl->st) != cudaSuccess))
        rc = -1;
    if (rc == 0) {
        pb_batch bb = pl->b;
        bb.stats = 0; bb.pad_rows = 0; bb.d_qlim = nullptr; bb.d_tlim = nullptr;
        rc = sw16_prepare(&bb, pl->o1, prof_bytes, pl->st, &pl->prep);
        pl->prepared = rc == 0;
    }
    if (rc == 0 && cudaStreamSynchronize(pl->st) != cudaSuccess) rc = -1;
    if (rc == 0 && cudaStreamBeginCapture(pl->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) rc = -1;
    if (rc == 0) {
        sw16_launch(pl->prep, pl->st);
        cudaMemsetAsync(pl->counts, 0, sizeof(int) * 8, pl->st);
        k_count_overflow<<<148, 256, 0, pl->st>>>(pl->o1, (int)N, pl->counts + 4);
        for (int q = 0; q < nq; ++q)
            pb::launch_resolve_plain(pl->job, pl->o1 + (size_t)q * n, pl->profs[q]->qlen, b->d_tlen, n,
                                     d_rec + (size_t)q * n, pl->need, pl->counts, pl->st);
        if (cudaStreamEndCapture(pl->st, &pl->graph) != cudaSuccess) rc = -1;
    }
    if (rc == 0 && cudaGraphInstantiate(&pl->exec, pl->graph, 0) != cudaSuccess) rc = -1;
    if (rc != 0) {
        cudaGetLastError();
        plan_destroy(pl);
        return -1;
    }
    *out = pl;
    return 0;
}

/* Replays the plan's graph; pairs past the 16-bit range (rare: a score
 * above 32767 - max(matrix) - 1) send the whole search once through the
 * batch pipeline, which reruns them in 32 bits. */
extern "C" int pb_cuda_db_plan_run(void *plan)
{
    DbPlan *pl = (DbPlan *)plan;
    if (!pl) return -1;
    int h[8] = {0};
    if (cudaGraphLaunch(pl->exec, pl->st) != cudaSuccess) return -1;
    pb_diag_count_launch(2 + (long)pl->profs.size());   /* k_sw16, overflow count, resolution */
    if (cudaMemcpyAsync(h, pl->counts, sizeof h, cudaMemcpyDeviceToHost, pl->st) != cudaSuccess) return -1;
    int herr = 0;
    if (cudaMemcpyAsync(&herr, pl->prep.counter + 2, sizeof(int), cudaMemcpyDeviceToHost, pl->st) != cudaSuccess)
        return -1;
    if (cudaStreamSynchronize(pl->st) != cudaSuccess) return -1;
    if (herr) {
        fprintf(stderr, "pb_cuda_db_plan_run: a pass wait exceeded its bound\n");
        return -1;
    }
    if (h[4] > 0) return pb_cuda_batch_run(&pl->job, &pl->b, pl->rec);
    return 0;
}

namespace {

__global__ void k_map_inplace(uint8_t *__restrict__ buf, int64_t n, const uint8_t *__restrict__ map)
{
    __shared__ uint8_t smap[256];
    for (int k = threadIdx.x; k < 256; k += blockDim.x) smap[k] = map[k];
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        buf[i] = smap[buf[i]];
}

}  // namespace

/* A plan run from host memory: the targets' characters (the layout the
 * plan was created with) are copied into d_codes and mapped there, the
 * graph replays, and the records come back into h_rec, all on the plan's
 * stream. */
extern "C" int pb_cuda_db_plan_run_host(void *plan, const char *h_chars, size_t nbytes, uint8_t *d_codes,
                                        const uint8_t *mapper256, pb_record *h_rec)
{
    DbPlan *pl = (DbPlan *)plan;
    if (!pl) return -1;
    if (!pl->map) {
        if (cudaMallocAsync((void **)&pl->map, 256, pl->st) != cudaSuccess) return -1;
        if (cudaMemcpyAsync(pl->map, mapper256, 256, cudaMemcpyHostToDevice, pl->st) != cudaSuccess) return -1;
    }
    if (nbytes && cudaMemcpyAsync(d_codes, h_chars, nbytes, cudaMemcpyHostToDevice, pl->st) != cudaSuccess)
        return -1;
    if (nbytes) {
        int dev = 0, nsm = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        const int64_t want = ((int64_t)nbytes + 255) / 256;
        k_map_inplace<<<(int)(want < 2 * nsm ? want : 2 * nsm), 256, 0, pl->st>>>(d_codes, (int64_t)nbytes, pl->map);
        pb_diag_count_launch(1);
    }
    if (pb_cuda_db_plan_run(plan) != 0) return -1;
    const size_t nrec = (size_t)pl->b.npairs * pl->profs.size();
    if (cudaMemcpyAsync(h_rec, pl->rec, sizeof(pb_record) * nrec, cudaMemcpyDeviceToHost, pl->st) != cudaSuccess)
        return -1;
    return cudaStreamSynchronize(pl->st) == cudaSuccess ? 0 : -1;
}

extern "C" void pb_cuda_db_plan_free(void *plan)
{
    if (plan) plan_destroy((DbPlan *)plan);
}
