/*
 * pb_sw16.cu -- Smith-Waterman score-only kernel in packed int16x2 lanes.
 *
 * Inter-task schedule: every thread aligns TWO targets against the same query
 * at once, one per 16-bit half of each register (targets are sorted by
 * length so the two halves, and the 32 threads of a warp, run similar
 * lengths). The query is processed in strips of R rows held in registers;
 * each strip sweeps the targets' columns and hands its bottom row (H and the
 * vertical-gap value F) to the next strip through a per-warp buffer laid out
 * [column][lane] so that every access of a warp is one contiguous 256-byte
 * transaction. The int8 query profile lives in shared memory; a column's R
 * scores for both targets are two 16-byte loads expanded to R int16x2 words
 * by sign-extending byte permutes. The recurrence uses the Hopper/Blackwell
 * DPX instructions (viaddmax, vimax3, vibmax).
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

namespace pb {

static constexpr int SW16_R = 16;          /* query rows per strip */
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

__device__ __forceinline__ uint32_t lo16(uint32_t x) { return x & 0xffffu; }
__device__ __forceinline__ int s16lo(uint32_t x) { return (int)(int16_t)(x & 0xffffu); }
__device__ __forceinline__ int s16hi(uint32_t x) { return (int)(int16_t)(x >> 16); }
__device__ __forceinline__ uint32_t splat16(int v) { return ((uint32_t)(uint16_t)v) | ((uint32_t)(uint16_t)v << 16); }

struct Sw16Best {
    int score, i, j;
};

/*
 * One warp task = 64 consecutive pairs of the length-sorted order; lane l
 * takes sorted positions 2l (low half) and 2l+1 (high half).
 */
__global__ void __launch_bounds__(SW16_WARPS * 32)
k_sw16(Sw16Params p, int ntasks, int *task_counter)
{
    extern __shared__ __align__(16) int8_t s_prof[];
    const ProfDesc pd = p.profs[0];
    const int lp = pd.lp;
    const int size = pd.size;
    const int ql = pd.qlen;
    /* whole int8 profile into shared memory, 16 bytes per thread-step */
    {
        const int4 *src = reinterpret_cast<const int4 *>(pd.prof8);
        int4 *dst = reinterpret_cast<int4 *>(s_prof);
        const int n16 = size * lp / 16;
        for (int k = threadIdx.x; k < n16; k += blockDim.x) dst[k] = src[k];
    }
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const uint32_t gapO = splat16(-p.open);
    const uint32_t gapE = splat16(-p.gap);
    const int posmax = p.posmax;       /* H + max(matrix) must stay <= 32767 */

    for (;;) {
        int task = 0;
        if (lane == 0) task = atomicAdd(task_counter, 1);
        task = __shfl_sync(0xffffffffu, task, 0);
        if (task >= ntasks) break;

        const int s0 = task * 64 + 2 * lane, s1 = s0 + 1;
        const bool v0 = s0 < p.npairs, v1 = s1 < p.npairs;
        const int pa = v0 ? p.order[s0] : -1, pbid = v1 ? p.order[s1] : -1;
        const int la = v0 ? p.tlen[pa] : 0, lb = v1 ? p.tlen[pbid] : 0;
        const uint8_t *ta = v0 ? p.targets + p.toff[pa] : nullptr;
        const uint8_t *tb = v1 ? p.targets + p.toff[pbid] : nullptr;
        int wmax = max(la, lb);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) wmax = max(wmax, __shfl_xor_sync(0xffffffffu, wmax, o));
        uint2 *buf = reinterpret_cast<uint2 *>(p.scratch + p.woff[task]);

        Sw16Best ba = {0, ql, la}, bb = {0, ql, lb};
        bool have_a = false, have_b = false;
        int status_a = 0, status_b = 0;

        for (int r0 = 0; r0 < ql; r0 += SW16_R) {
            uint32_t H[SW16_R], E[SW16_R];
#pragma unroll
            for (int r = 0; r < SW16_R; ++r) { H[r] = 0u; E[r] = gapO; }
            uint32_t dg = 0u;                 /* H(r0-1, j-1) */
            Sw16Best sa = {0, -1, -1}, sb = {0, -1, -1};   /* strip-local first max */
            uint32_t sbest = 0u;
            const int8_t *prow_base = s_prof + r0;
            for (int j = 0; j < wmax; ++j) {
                const int ca = j < la ? ta[j] : 0;
                const int cb = j < lb ? tb[j] : 0;
                uint32_t hu, fu;
                if (r0 == 0) { hu = 0u; fu = gapO; }
                else { const uint2 v = buf[(size_t)j * 32 + lane]; hu = v.x; fu = v.y; }
                const uint4 pa4 = *reinterpret_cast<const uint4 *>(prow_base + (size_t)ca * lp);
                const uint4 pb4 = *reinterpret_cast<const uint4 *>(prow_base + (size_t)cb * lp);
                uint32_t hd = dg;
                dg = hu;
                uint32_t cmax = 0u;
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
                    /* F: vertical gap from the row above, E: horizontal gap */
                    const uint32_t ho_up = __vadd2(hu, gapO);
                    const uint32_t f = __viaddmax_s16x2(fu, gapE, ho_up);
                    const uint32_t ho_left = __vadd2(H[r], gapO);
                    const uint32_t e = __viaddmax_s16x2(E[r], gapE, ho_left);
                    const uint32_t h = __viaddmax_s16x2_relu(hd, sc, __vmaxs2(e, f));
                    E[r] = e;
                    hd = H[r];
                    H[r] = h;
                    hu = h;
                    fu = f;
                    cmax = __vmaxs2(cmax, h);
                }
                if (r0 + SW16_R < ql) buf[(size_t)j * 32 + lane] = make_uint2(hu, fu);
                /* strip-local first column reaching a new maximum */
                bool ge_lo, ge_hi;
                (void)__vibmax_s16x2(sbest, cmax, &ge_hi, &ge_lo);
                const bool up_a = !ge_lo && j < la, up_b = !ge_hi && j < lb;
                if (up_a || up_b) {
                    if (up_a) {
                        const int c = s16lo(cmax);
                        int rr = -1;
#pragma unroll
                        for (int r = SW16_R - 1; r >= 0; --r) if (s16lo(H[r]) == c) rr = r;
                        sa.score = c; sa.j = j; sa.i = r0 + rr;
                        if (c >= posmax) status_a |= PB_ST_OVERFLOW16;
                    }
                    if (up_b) {
                        const int c = s16hi(cmax);
                        int rr = -1;
#pragma unroll
                        for (int r = SW16_R - 1; r >= 0; --r) if (s16hi(H[r]) == c) rr = r;
                        sb.score = c; sb.j = j; sb.i = r0 + rr;
                        if (c >= posmax) status_b |= PB_ST_OVERFLOW16;
                    }
                    sbest = (uint32_t)(uint16_t)sa.score | ((uint32_t)(uint16_t)sb.score << 16);
                }
            }
            /* fold the strip into the pair's best: higher score, then smaller
             * column; an equal column keeps the earlier strip (smaller row) */
            if (sa.j >= 0 && (!have_a || sa.score > ba.score || (sa.score == ba.score && sa.j < ba.j))) {
                ba = sa; have_a = true;
            }
            if (sb.j >= 0 && (!have_b || sb.score > bb.score || (sb.score == bb.score && sb.j < bb.j))) {
                bb = sb; have_b = true;
            }
        }
        /* no positive cell: score 0 at (0, 0), the first cell (src/sw.c:150-158) */
        if (v0) {
            pb_pair_out o = {};
            o.score = have_a ? ba.score : 0;
            o.end_query = have_a ? ba.i : 0;
            o.end_ref = have_a ? ba.j : 0;
            o.max_h = o.score;
            o.status = status_a;
            p.out[pa] = o;
        }
        if (v1) {
            pb_pair_out o = {};
            o.score = have_b ? bb.score : 0;
            o.end_query = have_b ? bb.i : 0;
            o.end_ref = have_b ? bb.j : 0;
            o.max_h = o.score;
            o.status = status_b;
            p.out[pbid] = o;
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

/* words of per-warp strip buffer: longest target of the task x 32 lanes x 2 */
__global__ void k_task_sizes(const int *sorted_len, int npairs, int ntasks, int64_t *sz)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < ntasks) sz[t] = (int64_t)sorted_len[t * 64] * 64;
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

extern "C" int pb_cuda_align_sw16(const pb_batch *b)
{
    static thread_local char err[160];
    (void)err;
    if (pb_cuda_init() != 0) return -1;
    if (b->npairs <= 0) return 0;
    const pb_device_profile *dp = b->profs[0];
    if (b->alg != PB_SW || b->stats || b->nprofs != 1 || !dp->fits8 || b->d_qlim || b->d_tlim ||
        b->open + b->gap > 30000) {
        return pb_cuda_align_exact(b);   /* outside this kernel's domain: the exact kernel */
    }
    const size_t smem = (size_t)dp->size * dp->lp;
    if (smem > 200 * 1024) return pb_cuda_align_exact(b);
    cudaStream_t st = 0;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    const int n = b->npairs;
    const int ntasks = (n + 63) / 64;
    int *keys_sorted = nullptr, *idx = nullptr, *order = nullptr, *counter = nullptr;
    int64_t *tsz = nullptr, *woff = nullptr;
    void *tmp = nullptr;
    size_t tmp_sort = 0, tmp_scan = 0;
    cudaMallocAsync((void **)&keys_sorted, sizeof(int) * n, st);
    cudaMallocAsync((void **)&idx, sizeof(int) * n, st);
    cudaMallocAsync((void **)&order, sizeof(int) * n, st);
    cudaMallocAsync((void **)&tsz, sizeof(int64_t) * ntasks, st);
    cudaMallocAsync((void **)&woff, sizeof(int64_t) * ntasks, st);
    cudaMallocAsync((void **)&counter, sizeof(int) * 2, st);
    k_iota<<<(n + 255) / 256, 256, 0, st>>>(idx, n);
    cub::DeviceRadixSort::SortPairsDescending(nullptr, tmp_sort, b->d_tlen, keys_sorted, idx, order, n, 0, 32, st);
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_scan, tsz, woff, ntasks, st);
    cudaMallocAsync(&tmp, tmp_sort > tmp_scan ? tmp_sort : tmp_scan, st);
    cub::DeviceRadixSort::SortPairsDescending(tmp, tmp_sort, b->d_tlen, keys_sorted, idx, order, n, 0, 32, st);
    k_task_sizes<<<(ntasks + 255) / 256, 256, 0, st>>>(keys_sorted, n, ntasks, tsz);
    cub::DeviceScan::ExclusiveSum(tmp, tmp_scan, tsz, woff, ntasks, st);
    int64_t last_off = 0, last_sz = 0;
    cudaMemcpyAsync(&last_off, woff + ntasks - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&last_sz, tsz + ntasks - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st);
    cudaMemsetAsync(counter, 0, sizeof(int) * 2, st);
    cudaStreamSynchronize(st);
    uint32_t *scratch = nullptr;
    if (cudaMallocAsync((void **)&scratch, sizeof(uint32_t) * (size_t)(last_off + last_sz + 64), st) != cudaSuccess) {
        cudaStreamDestroy(st);
        return -1;
    }
    pb::ProfDesc hd;
    hd.prof = dp->d_prof32; hd.prof8 = dp->d_prof8; hd.qcodes = dp->d_qcodes;
    hd.qlen = dp->qlen; hd.lp = dp->lp; hd.size = dp->size; hd.pad_ = 0;
    pb::ProfDesc *d_pd = nullptr;
    cudaMallocAsync((void **)&d_pd, sizeof hd, st);
    cudaMemcpyAsync(d_pd, &hd, sizeof hd, cudaMemcpyHostToDevice, st);

    pb::Sw16Params p;
    p.open = b->open; p.gap = b->gap; p.npairs = n;
    p.posmax = 32767 - dp->mmax - 1;
    p.profs = d_pd; p.order = order;
    p.targets = b->d_targets; p.toff = b->d_toff; p.tlen = b->d_tlen;
    p.scratch = scratch; p.woff = woff; p.out = b->d_out;
    cudaFuncSetAttribute(pb::k_sw16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0, nsm = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pb::k_sw16, pb::SW16_WARPS * 32, smem);
    if (per_sm < 1) per_sm = 1;
    int blocks = per_sm * nsm;
    const int need = (ntasks + pb::SW16_WARPS - 1) / pb::SW16_WARPS;
    if (blocks > need) blocks = need;
    cudaEvent_t ev0, ev1;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    cudaEventRecord(ev0, st);
    pb::k_sw16<<<blocks, pb::SW16_WARPS * 32, smem, st>>>(p, ntasks, counter);
    cudaEventRecord(ev1, st);
    cudaError_t e = cudaGetLastError();
    pb_diag_count_launch(4);   /* k_iota, k_task_sizes, k_sw16, k_collect_overflow */

    /* pairs that left the 16-bit range: the exact kernel */
    int *list = nullptr, *otlen = nullptr, nover = 0;
    int64_t *otoff = nullptr;
    cudaMallocAsync((void **)&list, sizeof(int) * n, st);
    cudaMallocAsync((void **)&otlen, sizeof(int) * n, st);
    cudaMallocAsync((void **)&otoff, sizeof(int64_t) * n, st);
    k_collect_overflow<<<(n + 255) / 256, 256, 0, st>>>(b->d_out, n, list, counter + 1, b->d_toff,
                                                        b->d_tlen, otoff, otlen);
    cudaMemcpyAsync(&nover, counter + 1, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, ev0, ev1);
        pb_diag_sw16_time(ms);
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
    }
    int rc = (e == cudaSuccess) ? 0 : -1;
    if (rc == 0 && nover > 0) {
        pb_pair_out *tmpo = nullptr;
        cudaMallocAsync((void **)&tmpo, sizeof(pb_pair_out) * nover, st);
        cudaStreamSynchronize(st);
        pb_batch sub = *b;
        sub.npairs = nover;
        sub.d_toff = otoff;
        sub.d_tlen = otlen;
        sub.d_out = tmpo;
        sub.d_prof_index = nullptr;
        rc = pb_cuda_align_exact(&sub);
        k_scatter<<<(nover + 255) / 256, 256, 0, st>>>(tmpo, list, nover, b->d_out);
        pb_diag_count_launch(1);
        cudaFreeAsync(tmpo, st);
    }
    cudaFreeAsync(list, st); cudaFreeAsync(otlen, st); cudaFreeAsync(otoff, st);
    cudaFreeAsync(scratch, st); cudaFreeAsync(d_pd, st); cudaFreeAsync(tmp, st);
    cudaFreeAsync(keys_sorted, st); cudaFreeAsync(idx, st); cudaFreeAsync(order, st);
    cudaFreeAsync(tsz, st); cudaFreeAsync(woff, st); cudaFreeAsync(counter, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
    cudaStreamDestroy(st);
    return rc;
}
