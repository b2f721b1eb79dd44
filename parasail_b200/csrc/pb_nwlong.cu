/*
 * pb_nwlong.cu -- global alignment of long pairs: one CTA per pair,
 * anti-diagonal wavefront across each warp's lanes, exact 32-bit values,
 * optionally restricted to a band of diagonals.
 *
 * Intra-task schedule: a pass covers 32 x NWL_RL query rows; lane k owns
 * rows r0 + k*NWL_RL .. + NWL_RL - 1 and, at iteration t, computes target
 * column t - k. Lane k therefore receives the bottom row of lane k-1 (H and
 * the vertical-gap value F at the same column) through one warp shuffle of
 * the previous iteration's outputs. The passes of one pair are spread over
 * the warps of a CTA and pipelined: lane 0 of pass p reads the bottom row
 * that lane 31 of pass p-1 (the previous warp) publishes. Scores come from a
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
#include <cstdio>

#include "pb_cuda.h"

namespace pb {

static constexpr int NWL_RL = 8;          /* query rows per lane */
static constexpr int NWL_WARPS = 8;       /* warps per CTA, one CTA per pair */
static constexpr int NWL_NEG = INT32_MIN / 4;

struct NwWaveParams {
    int npairs, open, gap, msize, small_alpha;
    const int8_t *mat;            /* [msize][msize], row = target letter (vector orientation) */
    const uint8_t *q; const int64_t *qoff; const int *qlen;
    const uint8_t *t; const int64_t *toff; const int *tlen;
    const int *lo; const int *hi; /* per pair band (diagonal i - j), or nullptr */
    const int *order;             /* pairs, most cells first */
    int2 *scratch;                /* per CTA: NWL_WARPS ring buffers of [maxlen] (H, F) */
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

/*
 * One CTA of NWL_WARPS warps per pair. Pass p (rows p*256 .. p*256+255) is
 * run by warp p % NWL_WARPS; its lane 0 reads pass p-1's bottom row from
 * ring buffer (p-1) % NWL_WARPS, which pass p-1's lane 31 fills column by
 * column and publishes through a progress counter in shared memory every 32
 * columns. Waits are bounded: a spin that exceeds NWL_SPIN polls sets the
 * error flag and abandons the pair (the host reports the failure).
 */
static constexpr long long NWL_SPIN = 1ll << 26;

template <bool BANDED, bool GE>
__global__ void __launch_bounds__(NWL_WARPS * 32, 3)
k_nw_wave(NwWaveParams p, int *counter, int *error)
{
    __shared__ __align__(16) int8_t s_mat[32 * 32];
    /* progress of ring buffer k: g * (m + 1) + j + 1 once generation g (the
     * pass g * NWL_WARPS + k) has published column j; monotone, so a reader
     * never mistakes an older pass's progress for its predecessor's */
    __shared__ volatile long long s_prog[NWL_WARPS];
    __shared__ int s_pair;
    __shared__ volatile int s_abort;
    for (int k = threadIdx.x; k < p.msize * p.msize; k += blockDim.x) {
        const int r = k / p.msize, c = k % p.msize;
        s_mat[r * 32 + c] = p.mat[k];
    }
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int open = p.open, gap = p.gap;
    int2 *ring = p.scratch + (size_t)blockIdx.x * NWL_WARPS * p.maxlen;

    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) { s_pair = atomicAdd(counter, 1); s_abort = 0; }
        if (threadIdx.x < NWL_WARPS) s_prog[threadIdx.x] = 0;
        __syncthreads();
        const int w = s_pair;
        if (w >= p.npairs) break;
        const int pid = p.order[w];
        const int n = p.qlen[pid], m = p.tlen[pid];
        const uint8_t *qs = p.q + p.qoff[pid];
        const uint8_t *ts = p.t + p.toff[pid];
        const int lo = BANDED ? p.lo[pid] : -(m + 1);
        const int hi = BANDED ? p.hi[pid] : n + 1;
        const int npass = (n + 32 * NWL_RL - 1) / (32 * NWL_RL);
        int result = NWL_NEG;
        bool have_result = false;

        for (int pass = warp; pass < npass; pass += NWL_WARPS) {
            const int r0 = pass * 32 * NWL_RL;
            const int R0 = r0 + lane * NWL_RL;
            int2 *in_buf = ring + (size_t)((pass + NWL_WARPS - 1) % NWL_WARPS) * p.maxlen;
            int2 *out_buf = ring + (size_t)(pass % NWL_WARPS) * p.maxlen;
            const long long stride = (long long)m + 1;
            volatile long long *in_prog = &s_prog[(pass + NWL_WARPS - 1) % NWL_WARPS];
            volatile long long *out_prog = &s_prog[pass % NWL_WARPS];
            const long long in_base = pass > 0 ? (long long)((pass - 1) / NWL_WARPS) * stride + 1 : 0;
            const long long out_base = (long long)(pass / NWL_WARPS) * stride + 1;
            int qc[NWL_RL];
#pragma unroll
            for (int r = 0; r < NWL_RL; ++r) qc[r] = (R0 + r < n) ? qs[R0 + r] : 0;
            int jlo = 0, jhi = m - 1, prev_jlo = 0, prev_jhi = m - 1;
            if (BANDED) {
                jlo = max(0, r0 - hi);
                jhi = min(m - 1, r0 + 32 * NWL_RL - 1 - lo);
                prev_jlo = max(0, r0 - 32 * NWL_RL - hi);
                prev_jhi = min(m - 1, r0 - 1 - lo);
            }
            if (pass == 0) prev_jhi = -1;
            /* the previous pass must have published column c before it is read */
            auto wait_for = [&](int c) -> bool {
                if (pass == 0) return true;
                const int need = min(c, prev_jhi);
                if (need < 0) return true;
                long long spins = 0;
                while (*in_prog < in_base + need) {
                    if (s_abort) return false;
                    if (++spins > NWL_SPIN) { s_abort = 1; atomicExch(error, 1); return false; }
                }
                __threadfence_block();
                return true;
            };
            int Hl[NWL_RL], E[NWL_RL];
#pragma unroll
            for (int r = 0; r < NWL_RL; ++r) {
                const int i = R0 + r;
                int v = NWL_NEG;
                if (jlo == 0 && (!BANDED || (i + 1 >= lo && i + 1 <= hi))) v = -open - i * gap;
                Hl[r] = v;
                E[r] = NWL_NEG;
            }
            int dg;
            if (jlo == 0) {
                dg = (R0 == 0) ? 0 : ((!BANDED || (R0 >= lo && R0 <= hi)) ? -open - (R0 - 1) * gap : NWL_NEG);
            } else {
                dg = NWL_NEG;
                bool ok = true;
                if (lane == 0) ok = wait_for(jlo - 1);
                ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0);
                if (!ok) break;
                if (lane == 0 && jlo - 1 <= prev_jhi && jlo - 1 >= prev_jlo) dg = __ldcg(&in_buf[jlo - 1]).x;
            }
            int sh_h = NWL_NEG, sh_f = NWL_NEG;
            const int tend = jhi + 31;
            /* this lane's target residues, loaded two columns ahead */
            auto res_at = [&](int c) -> int { return (c >= jlo && c <= jhi) ? (int)ts[c] : 0; };
            int tc_n1 = res_at(jlo - lane), tc_n2 = res_at(jlo - lane + 1);
            /* the previous pass's bottom row, one 32-column chunk per
             * register (lane l holds column chunk start + l; lane 0 takes its
             * column by shuffle), loaded one chunk ahead so that the L2
             * latency is off the column loop. A chunk is read only after the
             * previous pass has published the next one. */
            auto ring_at = [&](int c) -> int2 {
                return (pass > 0 && c >= prev_jlo && c <= prev_jhi) ? __ldcg(&in_buf[c])
                                                                      : make_int2(NWL_NEG, NWL_NEG);
            };
            int2 cur_v = make_int2(NWL_NEG, NWL_NEG), nxt_v = cur_v;
            bool aborted = false;
            for (int it = jlo; it <= tend; ++it) {
                const int j = it - lane;
                const int cpos = (it - jlo) & 31;
                if (cpos == 0) {
                    bool ok = true;
                    if (lane == 0) ok = wait_for(it + 63);
                    ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0);
                    if (!ok) { aborted = true; break; }
                    cur_v = it == jlo ? ring_at(it + lane) : nxt_v;
                    nxt_v = ring_at(it + 32 + lane);
                }
                const int vh = __shfl_sync(0xffffffffu, cur_v.x, cpos);
                const int vf = __shfl_sync(0xffffffffu, cur_v.y, cpos);
                int up_h = __shfl_up_sync(0xffffffffu, sh_h, 1);
                int up_f = __shfl_up_sync(0xffffffffu, sh_f, 1);
                const bool active = j >= jlo && j <= jhi;
                const int tc = tc_n1;
                tc_n1 = tc_n2;
                tc_n2 = res_at(j + 2);
                if (lane == 0 && active) {
                    if (r0 == 0) {
                        const bool inb = !BANDED || (-1 - j >= lo && -1 - j <= hi);
                        up_h = inb ? -open - j * gap : NWL_NEG;
                        up_f = NWL_NEG;
                    } else {
                        up_h = vh;
                        up_f = vf;
                    }
                }
                if (active) {
                    int hd = dg;
                    uint32_t row_lo = 0, row_hi = 0;
                    if (p.small_alpha) {
                        row_lo = *reinterpret_cast<const uint32_t *>(s_mat + tc * 32);
                        row_hi = *reinterpret_cast<const uint32_t *>(s_mat + tc * 32 + 4);
                    }
                    /* F of row R0 from the row above (previous lane or pass) */
                    int f = max(up_f - gap, up_h - open);
                    /* row R0 + r lies in the band iff 0 <= R0 + r - j - lo <= hi - lo */
                    const int dlo = R0 - j - lo;
                    const unsigned bw = (unsigned)(hi - lo);
                    int last_h = 0, last_f = 0;
#pragma unroll
                    for (int r = 0; r < NWL_RL; ++r) {
                        const int sc = p.small_alpha ? sext_byte(row_lo, row_hi, qc[r]) : (int)s_mat[tc * 32 + qc[r]];
                        /* E and the diagonal/E part a are off the row-to-row chain */
                        int e = max(E[r] - gap, Hl[r] - open);
                        int a = __viaddmax_s32(hd, sc, e);
                        if (BANDED) {
                            const bool in = (unsigned)(dlo + r) <= bw;
                            e = in ? e : NWL_NEG;
                            a = in ? a : NWL_NEG;
                            f = in ? f : NWL_NEG;
                        }
                        const int h = max(a, f);
                        last_h = h;
                        last_f = f;
                        /* F of the next row: max(F - gap, H - open). With
                         * open >= gap, H - open = max(a, F) - open and
                         * F - open <= F - gap, so only a - open is needed:
                         * one dependent operation per row */
                        if (GE) f = __viaddmax_s32(f, -gap, a - open);
                        else f = max(f - gap, h - open);
                        E[r] = e;
                        hd = Hl[r];
                        Hl[r] = h;
                    }
                    if (j == m - 1 && R0 <= n - 1 && n - 1 < R0 + NWL_RL) {
#pragma unroll
                        for (int r = 0; r < NWL_RL; ++r)
                            if (R0 + r == n - 1) { result = Hl[r]; have_result = true; }
                    }
                    dg = up_h;
                    sh_h = last_h;
                    sh_f = last_f;
                    if (lane == 31 && pass + 1 < npass) {
                        out_buf[j] = make_int2(last_h, last_f);
                        if (((j - jlo) & 31) == 31 || j == jhi) {
                            __threadfence_block();
                            *out_prog = out_base + j;
                        }
                    }
                }
            }
            if (aborted) break;
            __syncwarp();
        }
        /* the corner's owner publishes the result */
        __shared__ int s_result;
        if (have_result) s_result = result;
        __syncthreads();
        if (threadIdx.x == 0) p.score[pid] = s_abort ? NWL_NEG : s_result;
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
    /* the one-operation F chain needs open >= gap */
    const bool ge = open >= gap;
    void (*kern)(pb::NwWaveParams, int *, int *) =
        d_lo ? (ge ? pb::k_nw_wave<true, true> : pb::k_nw_wave<true, false>)
             : (ge ? pb::k_nw_wave<false, true> : pb::k_nw_wave<false, false>);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, pb::NWL_WARPS * 32, 0);
    if (per_sm < 1) per_sm = 1;
    int blocks = per_sm * nsm;
    if (blocks > npairs) blocks = npairs;
    int2 *scratch = nullptr;
    int *d_err = nullptr;
    int rc = 0, herr = 0;
    cudaMallocAsync((void **)&d_err, sizeof(int), st);
    cudaMemsetAsync(d_err, 0, sizeof(int), st);
    if (cudaMallocAsync((void **)&scratch, sizeof(int2) * (size_t)(maxlen + 1) * blocks * pb::NWL_WARPS, st) != cudaSuccess)
        rc = -1;
    if (rc == 0) {
        pb::NwWaveParams p;
        p.npairs = npairs; p.open = open; p.gap = gap; p.msize = msize; p.small_alpha = small;
        p.mat = d_mat; p.q = d_q; p.qoff = d_qoff; p.qlen = d_qlen;
        p.t = d_t; p.toff = d_toff; p.tlen = d_tlen; p.lo = d_lo; p.hi = d_hi;
        p.order = order; p.scratch = scratch; p.maxlen = maxlen + 1; p.score = d_score;
        kern<<<blocks, pb::NWL_WARPS * 32, 0, st>>>(p, counter, d_err);
        if (cudaGetLastError() != cudaSuccess) rc = -1;
        pb_diag_count_launch(3);
        cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
    }
    cudaFreeAsync(d_mat, st); cudaFreeAsync(idx, st); cudaFreeAsync(order, st);
    cudaFreeAsync(cells, st); cudaFreeAsync(cells_sorted, st); cudaFreeAsync(counter, st);
    cudaFreeAsync(tmp, st);
    if (scratch) cudaFreeAsync(scratch, st);
    cudaFreeAsync(d_err, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
    if (herr) {
        fprintf(stderr, "pb_cuda_nw_long: a pipeline wait exceeded its bound; pair abandoned\n");
        rc = -1;
    }
    cudaStreamDestroy(st);
    return rc;
}
