/*
 * pb_nwlong.cu -- global alignment of long pairs: one warp per pair,
 * anti-diagonal wavefront across the warp's lanes, exact 32-bit values,
 * optionally restricted to a band of diagonals.
 *
 * Intra-task schedule: a pass covers 32 x NWL_RL query rows; lane k owns
 * rows r0 + k*NWL_RL .. + NWL_RL - 1 and, at iteration t, computes target
 * column t - k. Lane k therefore receives the bottom row of lane k-1 (H and
 * the vertical-gap value F at the same column) through one warp shuffle of
 * the previous iteration's outputs, and lane 0 reads the previous pass's
 * bottom row from a per-warp buffer that lane 31 writes. Scores come from a
 * square substitution table in shared memory indexed by (target letter,
 * query letter); for alphabets of at most 8 letters one byte-permute selects
 * the score from the target letter's table row held in two registers.
 *
 * Semantics: the global recurrence of the reference (src/nw.c:102-156,
 * boundaries H(-1,j) = -open - j*gap, H(i,-1) = -open - i*gap, score at the
 * corner), which its nw_scan/nw_striped kernels reproduce. With a band
 * [lo, hi] every cell -- boundary cells included -- whose diagonal i - j
 * lies outside it is -infinity, i.e. the result is the best global
 * alignment among paths that stay inside the band.
 */
#include <cstdint>
#include <climits>
#include <vector>
#include <algorithm>
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>

#include "pb_cuda.h"

namespace pb {

static constexpr int NWL_RL = 8;          /* query rows per lane */
static constexpr int NWL_WARPS = 4;       /* warps per block */
static constexpr int NWL_NEG = INT32_MIN / 4;

struct NwWaveParams {
    int npairs, open, gap, msize, small_alpha;
    const int8_t *mat;            /* [msize][msize], row = target letter (vector orientation) */
    const uint8_t *q; const int64_t *qoff; const int *qlen;
    const uint8_t *t; const int64_t *toff; const int *tlen;
    const int *lo; const int *hi; /* per pair band (diagonal i - j), or nullptr */
    const int *order;             /* pairs, most cells first */
    int2 *scratch;                /* per resident warp: [maxlen] (H, F) */
    int maxlen;
    int *score;                   /* per pair */
};

__device__ __forceinline__ int sext_byte(uint32_t lo, uint32_t hi, int k)
{
    /* byte k of {hi:lo}, sign-extended to 32 bits */
    const uint32_t sel = (uint32_t)k | (((uint32_t)k | 8u) << 4) | (((uint32_t)k | 8u) << 8) | (((uint32_t)k | 8u) << 12);
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(lo), "r"(hi), "r"(sel));
    return (int)d;
}

template <bool BANDED>
__global__ void __launch_bounds__(NWL_WARPS * 32)
k_nw_wave(NwWaveParams p, int *counter)
{
    __shared__ __align__(16) int8_t s_mat[32 * 32];
    for (int k = threadIdx.x; k < p.msize * p.msize; k += blockDim.x) {
        const int r = k / p.msize, c = k % p.msize;
        s_mat[r * 32 + c] = p.mat[k];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int slot = blockIdx.x * NWL_WARPS + (threadIdx.x >> 5);
    int2 *buf = p.scratch + (size_t)slot * p.maxlen;
    const int open = p.open, gap = p.gap;

    for (;;) {
        int w = 0;
        if (lane == 0) w = atomicAdd(counter, 1);
        w = __shfl_sync(0xffffffffu, w, 0);
        if (w >= p.npairs) break;
        const int pid = p.order[w];
        const int n = p.qlen[pid], m = p.tlen[pid];
        const uint8_t *qs = p.q + p.qoff[pid];
        const uint8_t *ts = p.t + p.toff[pid];
        const int lo = BANDED ? p.lo[pid] : -(m + 1);
        const int hi = BANDED ? p.hi[pid] : n + 1;
        int result = NWL_NEG;
        int prev_jhi = -1;

        for (int r0 = 0; r0 < n; r0 += 32 * NWL_RL) {
            const int R0 = r0 + lane * NWL_RL;
            int qc[NWL_RL];
#pragma unroll
            for (int r = 0; r < NWL_RL; ++r) qc[r] = (R0 + r < n) ? qs[R0 + r] : 0;
            /* columns this pass touches */
            int jlo = 0, jhi = m - 1;
            if (BANDED) {
                jlo = max(0, r0 - hi);
                jhi = min(m - 1, r0 + 32 * NWL_RL - 1 - lo);
            }
            /* left state: column jlo - 1 */
            int Hl[NWL_RL], E[NWL_RL];
#pragma unroll
            for (int r = 0; r < NWL_RL; ++r) {
                const int i = R0 + r;
                int v = NWL_NEG;
                if (jlo == 0 && (!BANDED || (i + 1 >= lo && i + 1 <= hi))) v = -open - i * gap;
                Hl[r] = v;
                E[r] = NWL_NEG;
            }
            /* diagonal of each lane's first row at column jlo: H(R0 - 1, jlo - 1) */
            int dg;
            if (jlo == 0) {
                dg = (R0 == 0) ? 0 : ((!BANDED || (R0 >= lo && R0 <= hi)) ? -open - (R0 - 1) * gap : NWL_NEG);
            } else if (lane == 0 && jlo - 1 <= prev_jhi) {
                dg = buf[jlo - 1].x;    /* H(r0 - 1, jlo - 1), on the band's edge */
            } else {
                dg = NWL_NEG;           /* outside the band */
            }
            int sh_h = NWL_NEG, sh_f = NWL_NEG;   /* outputs of the previous iteration (this lane's bottom) */
            const int tend = jhi + 31;
            for (int it = jlo; it <= tend; ++it) {
                const int j = it - lane;
                /* bottom row of lane-1 at column j (computed last iteration) */
                int up_h = __shfl_up_sync(0xffffffffu, sh_h, 1);
                int up_f = __shfl_up_sync(0xffffffffu, sh_f, 1);
                const bool active = j >= jlo && j <= jhi;
                if (lane == 0 && active) {
                    if (r0 == 0) {
                        const bool inb = !BANDED || (-1 - j >= lo && -1 - j <= hi);
                        up_h = inb ? -open - j * gap : NWL_NEG;
                        up_f = NWL_NEG;
                    } else if (j <= prev_jhi) {
                        const int2 v = buf[j];
                        up_h = v.x;
                        up_f = v.y;
                    } else {
                        up_h = NWL_NEG;
                        up_f = NWL_NEG;
                    }
                }
                if (active) {
                    const int tc = ts[j];
                    int hd = dg;
                    int hu = up_h, fu = up_f;
                    uint32_t row_lo = 0, row_hi = 0;
                    if (p.small_alpha) {
                        row_lo = *reinterpret_cast<const uint32_t *>(s_mat + tc * 32);
                        row_hi = *reinterpret_cast<const uint32_t *>(s_mat + tc * 32 + 4);
                    }
#pragma unroll
                    for (int r = 0; r < NWL_RL; ++r) {
                        const int i = R0 + r;
                        const int sc = p.small_alpha ? sext_byte(row_lo, row_hi, qc[r]) : (int)s_mat[tc * 32 + qc[r]];
                        const int e = max(E[r] - gap, Hl[r] - open);
                        const int f = max(fu - gap, hu - open);
                        int h = max(max(hd + sc, e), f);
                        int ee = e, ff = f;
                        if (BANDED) {
                            const int d = i - j;
                            if (d < lo || d > hi) { h = NWL_NEG; ee = NWL_NEG; ff = NWL_NEG; }
                        }
                        if (i == n - 1 && j == m - 1) result = h;
                        E[r] = ee;
                        hd = Hl[r];
                        Hl[r] = h;
                        hu = h;
                        fu = ff;
                    }
                    dg = up_h;
                    sh_h = hu;
                    sh_f = fu;
                    if (lane == 31 && r0 + 32 * NWL_RL < n) buf[j] = make_int2(hu, fu);
                }
            }
            prev_jhi = jhi;
            __syncwarp();
        }
        /* the corner's owner holds the result */
        const int owner = ((n - 1) % (32 * NWL_RL)) / NWL_RL;
        result = __shfl_sync(0xffffffffu, result, owner);
        if (lane == 0) p.score[pid] = result;
    }
}

__global__ void k_iota_nw(int *v, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

__global__ void k_cells(const int *ql, const int *tl, int n, int64_t *cells)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) cells[i] = (int64_t)ql[i] * tl[i];
}

}  // namespace pb

/* Global alignment scores of npairs device-resident pairs (codes), query i =
 * q[qoff[i] ..+qlen[i]), target i likewise, scored through the square matrix
 * d_mat (msize x msize int32, row = target letter). d_lo/d_hi: optional
 * per-pair band. Scores to d_score. */
extern "C" int pb_cuda_nw_long(int npairs, int open, int gap, const int32_t *h_mat, int msize,
                               const uint8_t *d_q, const int64_t *d_qoff, const int *d_qlen,
                               const uint8_t *d_t, const int64_t *d_toff, const int *d_tlen,
                               const int *d_lo, const int *d_hi, int maxlen, int *d_score)
{
    if (pb_cuda_init() != 0) return -1;
    if (npairs <= 0) return 0;
    if (msize > 32) return -1;
    cudaStream_t st = nullptr;
    cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    std::vector<int8_t> hm((size_t)msize * msize);
    int small = msize <= 8;
    for (int k = 0; k < msize * msize; ++k) {
        if (h_mat[k] < -128 || h_mat[k] > 127) { cudaStreamDestroy(st); return -1; }
        hm[k] = (int8_t)h_mat[k];
    }
    int8_t *d_mat = nullptr;
    int *idx = nullptr, *order = nullptr, *counter = nullptr;
    int64_t *cells = nullptr, *cells_sorted = nullptr;
    void *tmp = nullptr;
    size_t tmpb = 0;
    cudaMallocAsync((void **)&d_mat, hm.size(), st);
    cudaMemcpyAsync(d_mat, hm.data(), hm.size(), cudaMemcpyHostToDevice, st);
    cudaMallocAsync((void **)&idx, sizeof(int) * npairs, st);
    cudaMallocAsync((void **)&order, sizeof(int) * npairs, st);
    cudaMallocAsync((void **)&cells, sizeof(int64_t) * npairs, st);
    cudaMallocAsync((void **)&cells_sorted, sizeof(int64_t) * npairs, st);
    cudaMallocAsync((void **)&counter, sizeof(int), st);
    cudaMemsetAsync(counter, 0, sizeof(int), st);
    pb::k_iota_nw<<<(npairs + 255) / 256, 256, 0, st>>>(idx, npairs);
    pb::k_cells<<<(npairs + 255) / 256, 256, 0, st>>>(d_qlen, d_tlen, npairs, cells);
    cub::DeviceRadixSort::SortPairsDescending(nullptr, tmpb, cells, cells_sorted, idx, order, npairs, 0, 64, st);
    cudaMallocAsync(&tmp, tmpb, st);
    cub::DeviceRadixSort::SortPairsDescending(tmp, tmpb, cells, cells_sorted, idx, order, npairs, 0, 64, st);
    int nsm = 0, dev = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (d_lo) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pb::k_nw_wave<true>, pb::NWL_WARPS * 32, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pb::k_nw_wave<false>, pb::NWL_WARPS * 32, 0);
    if (per_sm < 1) per_sm = 1;
    int blocks = per_sm * nsm;
    const int need = (npairs + pb::NWL_WARPS - 1) / pb::NWL_WARPS;
    if (blocks > need) blocks = need;
    int2 *scratch = nullptr;
    int rc = 0;
    if (cudaMallocAsync((void **)&scratch, sizeof(int2) * (size_t)(maxlen + 1) * blocks * pb::NWL_WARPS, st) != cudaSuccess)
        rc = -1;
    if (rc == 0) {
        pb::NwWaveParams p;
        p.npairs = npairs; p.open = open; p.gap = gap; p.msize = msize; p.small_alpha = small;
        p.mat = d_mat; p.q = d_q; p.qoff = d_qoff; p.qlen = d_qlen;
        p.t = d_t; p.toff = d_toff; p.tlen = d_tlen; p.lo = d_lo; p.hi = d_hi;
        p.order = order; p.scratch = scratch; p.maxlen = maxlen + 1; p.score = d_score;
        if (d_lo) pb::k_nw_wave<true><<<blocks, pb::NWL_WARPS * 32, 0, st>>>(p, counter);
        else pb::k_nw_wave<false><<<blocks, pb::NWL_WARPS * 32, 0, st>>>(p, counter);
        if (cudaGetLastError() != cudaSuccess) rc = -1;
        pb_diag_count_launch(3);
    }
    cudaFreeAsync(d_mat, st); cudaFreeAsync(idx, st); cudaFreeAsync(order, st);
    cudaFreeAsync(cells, st); cudaFreeAsync(cells_sorted, st); cudaFreeAsync(counter, st);
    cudaFreeAsync(tmp, st);
    if (scratch) cudaFreeAsync(scratch, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
    cudaStreamDestroy(st);
    return rc;
}
