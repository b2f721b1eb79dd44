/*
 * pb_batch.cu -- the batch pipeline: score pass, optional prefix stats pass
 * (SW stats striped, the reference's FASTSTATS wrapper), and the width
 * resolution of every pair on the device, producing compact records.
 */
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <vector>
#include <cuda_runtime.h>

#include "pb_cuda.h"
#include "pb_kernels.cuh"
#include "pb_resolve.h"

namespace pb {

/* The lane results of pair i as the chain reads them: `e` holds the last
 * lane-exact result of the pair (valid = its width). The chain moves past a
 * width whose lane result it read only when that result saturated, so every
 * narrower width it read is given back as a saturated result. */
__device__ inline void lane_views(const pb_lane_res *e, int i, pb_lane_res x[3])
{
    const int w3[3] = {8, 16, 32};
    pb_lane_res s;
    memset(x, 0, 3 * sizeof(pb_lane_res));
    if (!e) return;
    s = e[i];
    for (int t = 0; t < 3; ++t) {
        if (s.valid == w3[t]) x[t] = s;
        else if (s.valid > w3[t]) { x[t].valid = w3[t]; x[t].saturated = 1; }
    }
}

/* Resolves pairs (all n, or the n listed) and lists by width the pairs that
 * still wait for a lane-exact kernel: need + w * n, counts[w]. */
__global__ void k_resolve(pb_job job, const pb_pair_out *__restrict__ o1,
                          const pb_pair_out *__restrict__ o2, const int *__restrict__ qlen,
                          int qlen_all, const int *__restrict__ tlen, int n_all, int n,
                          const int *__restrict__ list, const pb_lane_res *__restrict__ e,
                          pb_record *__restrict__ rec, int *__restrict__ need, int *__restrict__ counts)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int i = list ? list[k] : k;
    const pb_pair_out a = o1[i];
    pb_pair_out b;
    if (o2) b = o2[i];
    pb_lane_res x[3];
    lane_views(e, i, x);
    pb_record r = pb_chain_resolve(&job, &a, o2 ? &b : nullptr, qlen ? qlen[i] : qlen_all, tlen[i],
                                   &x[0], &x[1], &x[2]);
    const int t = r.ambig == 8 ? 0 : r.ambig == 16 ? 1 : r.ambig == 32 ? 2 : -1;
    /* a finished record goes out as the public record, whose last field
     * (here the fallback note) is reserved and 0 */
    if (t < 0) r.ambig = 0;
    rec[i] = r;
    if (t >= 0) need[(size_t)t * n_all + atomicAdd(&counts[t], 1)] = i;
}

__global__ void k_max_int(const int *__restrict__ v, int n, int *__restrict__ out)
{
    int m = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = max(m, v[i]);
    for (int o = 16; o; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

/* prefix limits of the FASTSTATS stats pass; pairs that need none get a
 * 1x1 problem */
__global__ void k_prefix_limits(pb_job job, const pb_pair_out *__restrict__ o1, int n,
                                int *__restrict__ qlim, int *__restrict__ tlim)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const pb_pair_out a = o1[i];
    const bool need = pb_needs_pass2(&job, &a);
    qlim[i] = need ? a.end_query + 1 : 1;
    tlim[i] = need ? a.end_ref + 1 : 1;
}

/*
 * Resolution of n pairs with the lane-exact rounds: resolve every pair; the
 * pairs that need the 8-, 16- or 32-bit lane kernel are listed by width,
 * emulated and resolved again, until none is left (at most one round per
 * width). `la` describes the query side (profile or matrix mode) and the
 * targets. Work memory: from `work` (work_bytes, 256-byte aligned) when
 * given, otherwise from the stream's pool. Synchronises the stream once per
 * round. Returns 0; -1 on a device error; -2 when `work` is smaller than
 * the lists and results; -3 when what `work` has left after them does not
 * hold one warp's lane-exact arrays.
 */
int resolve_rounds(const pb_job &job, const pb_lane_args &la, const pb_pair_out *o1, const pb_pair_out *o2,
                   const int *qlen, int qlen_all, const int *tlen, int n, pb_record *rec, cudaStream_t st,
                   void *work, size_t work_bytes)
{
    if (n <= 0) return 0;
    /* work layout: counts | lists A (3n) | lists B (3n) | results (n) | lane scratch */
    const size_t b_counts = 256;
    const size_t b_lists = ((sizeof(int) * 3 * (size_t)n) + 255) & ~(size_t)255;
    const size_t b_res = ((sizeof(pb_lane_res) * (size_t)n) + 255) & ~(size_t)255;
    const size_t fixed = b_counts + 2 * b_lists + b_res;
    unsigned char *base = (unsigned char *)work;
    bool own = false;
    if (!base) {
        if (cudaMallocAsync((void **)&base, fixed, st) != cudaSuccess) return -1;
        own = true;
    } else if (work_bytes < fixed) {
        return -2;
    }
    int *counts = (int *)base;
    int *lists[2] = {(int *)(base + b_counts), (int *)(base + b_counts + b_lists)};
    pb_lane_res *res = (pb_lane_res *)(base + b_counts + 2 * b_lists);
    unsigned char *lane_scratch = own ? nullptr : base + fixed;
    const size_t lane_bytes = own ? 0 : work_bytes - fixed;
    const int w3[3] = {8, 16, 32};
    int rc = 0;
    cudaMemsetAsync(counts, 0, 3 * sizeof(int), st);
    cudaMemsetAsync(res, 0, b_res, st);
    k_resolve<<<(n + 255) / 256, 256, 0, st>>>(job, o1, o2, qlen, qlen_all, tlen, n, n, nullptr, nullptr,
                                               rec, lists[0], counts);
    pb_diag_count_launch(1);
    int cur = 0;
    pb_lane_args a = la;
    bool have_max = a.max_qlen > 0;
    for (int round = 0; rc == 0; ++round) {
        int hc[3] = {0, 0, 0};
        if (cudaMemcpyAsync(hc, counts, sizeof hc, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) { rc = -1; break; }
        if (hc[0] + hc[1] + hc[2] == 0) break;
        if (round == 3) { rc = -1; break; }   /* a width cannot be asked for twice */
        if (!have_max) {
            /* matrix mode: the longest query sizes the lane scratch */
            int *dm = counts + 4;
            int hm = 0;
            cudaMemsetAsync(dm, 0, sizeof(int), st);
            k_max_int<<<64, 256, 0, st>>>(a.qlens, n, dm);
            pb_diag_count_launch(1);
            cudaMemcpyAsync(&hm, dm, sizeof(int), cudaMemcpyDeviceToHost, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) { rc = -1; break; }
            a.max_qlen = hm;
            have_max = true;
        }
        a.kind = pb_lane_kind(&job.mode);
        a.sgflags = job.mode.sgflags;
        a.open = job.mode.open; a.gap = job.mode.gap;
        for (int t = 0; t < 3 && rc == 0; ++t)
            if (hc[t]) {
                const int lr = pb_cuda_lane_run(w3[t], &a, lists[cur] + (size_t)t * n, hc[t], res, lane_scratch,
                                                lane_bytes, st);
                if (lr != 0) rc = lr == -3 ? -3 : -1;
            }
        if (rc) break;
        const int nxt = cur ^ 1;
        cudaMemsetAsync(counts, 0, 3 * sizeof(int), st);
        for (int t = 0; t < 3; ++t)
            if (hc[t]) {
                k_resolve<<<(hc[t] + 255) / 256, 256, 0, st>>>(job, o1, o2, qlen, qlen_all, tlen, n, hc[t],
                                                               lists[cur] + (size_t)t * n, res, rec, lists[nxt],
                                                               counts);
                pb_diag_count_launch(1);
            }
        if (cudaGetLastError() != cudaSuccess) { rc = -1; break; }
        cur = nxt;
    }
    if (own) cudaFreeAsync(base, st);
    return rc;
}

/* One resolution pass of n pairs of one query (no lane-exact rounds): the
 * width verdicts of jobs whose every width the exact values settle. */
void launch_resolve_plain(const pb_job &job, const pb_pair_out *o1, int qlen_all, const int *tlen, int n,
                          pb_record *rec, int *need, int *counts, cudaStream_t st)
{
    k_resolve<<<(n + 255) / 256, 256, 0, st>>>(job, o1, nullptr, nullptr, qlen_all, tlen, n, n, nullptr, nullptr,
                                               rec, need, counts);
}

/* the lane arguments of query q of a batch */
pb_lane_args lane_args_of(const pb_batch *b, int q, const pb_pair_out *o1)
{
    pb_lane_args a;
    memset(&a, 0, sizeof a);
    if (b->nprofs > 0) {
        const pb_device_profile *p = b->profs[q];
        a.prof = p->d_prof32; a.qcodes = p->d_qcodes; a.lp = p->lp; a.qlen = p->qlen; a.size = p->size;
        a.mmax = p->mmax; a.mmin = p->mmin; a.max_qlen = p->qlen;
    } else {
        a.mat = b->d_mat; a.msize = b->msize; a.qall = b->d_qall; a.qoff = b->d_qoff; a.qlens = b->d_qlen;
        a.mmax = b->mmax; a.mmin = b->mmin; a.max_qlen = 0;
    }
    a.targets = b->d_targets; a.toff = b->d_toff; a.tlen = b->d_tlen;
    a.o1 = o1;
    return a;
}

}  // namespace pb

extern "C" int pb_cuda_batch_run(const pb_job *job, const pb_batch *tmpl, pb_record *d_rec)
{
    if (pb_cuda_init() != 0) return -1;
    const int n = tmpl->npairs;
    if (n <= 0) return 0;
    const pb_mode *m = &job->mode;
    const int nq = tmpl->nprofs > 0 ? tmpl->nprofs : 1;   /* pairs mode: one "query set" */
    const size_t nitems = (size_t)n * nq;
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return -1;
    pb_pair_out *o1 = nullptr, *o2 = nullptr;
    int *qlim = nullptr, *tlim = nullptr;
    int rc = 0;
    /* every buffer is checked before any launch that would write through it */
    if (cudaMallocAsync((void **)&o1, sizeof(pb_pair_out) * nitems, st) != cudaSuccess) rc = -1;
    const bool faststats = pb_job_is_faststats(job);
    int *rest = nullptr;      /* items the 16-bit pair kernels leave to the exact kernel */
    if (rc == 0 && faststats &&
        (cudaMallocAsync((void **)&o2, sizeof(pb_pair_out) * nitems, st) != cudaSuccess ||
         cudaMallocAsync((void **)&qlim, sizeof(int) * nitems, st) != cudaSuccess ||
         cudaMallocAsync((void **)&tlim, sizeof(int) * nitems, st) != cudaSuccess))
        rc = -1;
    if (rc == 0 && cudaMallocAsync((void **)&rest, sizeof(int) * nitems, st) != cudaSuccess) rc = -1;
    if (rc == 0 && cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
    const bool sw_score = m->alg == PB_SW && (!m->stats || faststats) && job->bits >= 0;
    const int *group = tmpl->nprofs > 0 ? nullptr : tmpl->d_qgroup;
    if (rc == 0 && sw_score && tmpl->nprofs >= 1) {
        pb_batch b = *tmpl;
        b.stats = 0;
        b.pad_rows = 0;
        b.d_qlim = nullptr;
        b.d_tlim = nullptr;
        rc = pb_cuda_align_sw16_multi(&b, o1);
    } else if (rc == 0) {
        /* every item on the int16x2 pair kernels where the 16-bit bounds
         * hold, the rest (and items whose width verdicts need exact
         * extremes) on the exact kernel */
        pb_batch b = *tmpl;
        b.d_out = o1;
        b.d_qlim = nullptr;
        b.d_tlim = nullptr;
        b.stats = sw_score ? 0 : m->stats;
        b.pad_rows = (job->bits < 0 || (m->alg == PB_SW && !m->stats)) ? 0
                   : (job->bits == 0 || job->bits == 8) ? 32 : job->bits == 16 ? 16 : 8;
        int nrest = 0;
        /* global score-only pairs: the length buckets the schedule table
         * gives the intra-task wavefront kernel go there, with every pair
         * the pair kernels cannot take */
        const bool wave = pb::wave_ok(*job, &b);
        rc = pb::p16_pass(*job, &b, 0, nullptr, o1, group, rest, &nrest, st, nullptr, nullptr, nullptr,
                          wave ? pb::pb_schedule_nw_mask() : 0u);
        if (rc == 0 && wave && nrest > 0) {
            int *rest2 = nullptr, nrest2 = 0;
            if (cudaMallocAsync((void **)&rest2, sizeof(int) * (size_t)nrest, st) != cudaSuccess) rc = -1;
            if (rc == 0) rc = pb::wave_subset(*job, &b, rest, nrest, o1, rest2, &nrest2, st);
            if (rc == 0 && nrest2 > 0) rc = pb::exact_subset(&b, rest2, nrest2, b.stats, b.pad_rows, o1, st);
            if (rest2) cudaFreeAsync(rest2, st);
            nrest = 0;
        }
        if (rc == 0 && nrest > 0) rc = pb::exact_subset(&b, rest, nrest, b.stats, b.pad_rows, o1, st);
    }
    if (rc == 0 && faststats) {
        /* the prefix statistics pass of every item: limits per (query,
         * target) item, query-major like o1; statistics by the direction-bit
         * walk from the score pass's ends */
        pb::k_prefix_limits<<<(int)((nitems + 255) / 256), 256, 0, st>>>(*job, o1, (int)nitems, qlim, tlim);
        pb_diag_count_launch(1);
        if (cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
        pb_batch b2 = *tmpl;
        b2.stats = 1;
        b2.pad_rows = 32;
        b2.d_qlim = qlim;
        b2.d_tlim = tlim;
        b2.d_out = o2;
        int nrest = 0;
        if (rc == 0) rc = pb::p16_pass(*job, &b2, 1, o1, o2, group, rest, &nrest, st);
        if (rc == 0 && nrest > 0) rc = pb::exact_subset(&b2, rest, nrest, 1, 32, o2, st);
    }
    for (int q = 0; q < nq && rc == 0; ++q) {
        const int qall = tmpl->nprofs > 0 ? tmpl->profs[q]->qlen : 0;
        const pb_lane_args la = pb::lane_args_of(tmpl, q, o1 + (size_t)q * n);
        rc = pb::resolve_rounds(*job, la, o1 + (size_t)q * n, o2 ? o2 + (size_t)q * n : nullptr,
                                tmpl->nprofs > 0 ? nullptr : tmpl->d_qlen, qall, tmpl->d_tlen, n,
                                d_rec + (size_t)q * n, st, nullptr, 0);
    }
    if (o1) cudaFreeAsync(o1, st);
    if (o2) cudaFreeAsync(o2, st);
    if (rest) cudaFreeAsync(rest, st);
    if (qlim) cudaFreeAsync(qlim, st);
    if (tlim) cudaFreeAsync(tlim, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
    cudaStreamDestroy(st);
    return rc;
}

namespace {

__global__ void k_map_codes(uint8_t *__restrict__ buf, int64_t n, const uint8_t *__restrict__ map)
{
    __shared__ uint8_t smap[256];
    for (int k = threadIdx.x; k < 256; k += blockDim.x) smap[k] = map[k];
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        buf[i] = smap[buf[i]];
}

}  // namespace

namespace {

/* characters [lo, hi) of raw to codes at the same offsets */
__global__ void k_map_into(const uint8_t *__restrict__ raw, uint8_t *__restrict__ codes, int64_t lo, int64_t hi,
                           const uint8_t *__restrict__ map)
{
    __shared__ uint8_t smap[256];
    for (int k = threadIdx.x; k < 256; k += blockDim.x) smap[k] = map[k];
    __syncthreads();
    for (int64_t i = lo + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < hi; i += (int64_t)gridDim.x * blockDim.x)
        codes[i] = smap[raw[i]];
}

}  // namespace

/* Host-memory batch: copies the characters of targets (and, in pairs mode,
 * queries) to the device, maps them to codes there, runs the pipeline and
 * copies the records back. With one query set (pairs mode or a single
 * profile) and enough pairs, the items run in chunks whose copies overlap
 * the previous chunk's alignment: chunk k + 1's characters go up and chunk
 * k - 1's records come back on a copy stream while chunk k runs. Every
 * chunk's characters land at their own offsets in one device buffer (a
 * separate raw buffer is mapped into it, so chunks whose byte ranges
 * overlap map the same bytes to the same codes). */
extern "C" int pb_cuda_batch_host(const pb_job *job, const pb_batch *tmpl, const uint8_t *mapper256,
                                  const char *h_targets, const int64_t *h_toff, const int *h_tlen,
                                  const char *h_queries, const int64_t *h_qoff, const int *h_qlen,
                                  int n, pb_record *h_rec)
{
    if (pb_cuda_init() != 0) return -1;
    if (n <= 0) return 0;
    const int nq = tmpl->nprofs > 0 ? tmpl->nprofs : 1;
    /* chunks: at least 65,536 items each, at most 4 */
    constexpr int CH_MIN = 1 << 16;
    const int nch = nq == 1 ? std::max(1, std::min(4, n / CH_MIN)) : 1;
    std::vector<int> cut(nch + 1);
    for (int k = 0; k <= nch; ++k) cut[k] = (int)((int64_t)n * k / nch);
    /* each chunk's byte ranges [lo, hi) of targets and queries */
    std::vector<int64_t> tlo(nch, INT64_MAX), thi(nch, 0), qlo(nch, INT64_MAX), qhi(nch, 0);
    int64_t tbytes = 0, qbytes = 0;
    for (int k = 0; k < nch; ++k)
        for (int i = cut[k]; i < cut[k + 1]; ++i) {
            tlo[k] = std::min(tlo[k], h_toff[i]);
            thi[k] = std::max(thi[k], h_toff[i] + h_tlen[i]);
            if (h_queries) {
                qlo[k] = std::min(qlo[k], h_qoff[i]);
                qhi[k] = std::max(qhi[k], h_qoff[i] + h_qlen[i]);
            }
        }
    for (int k = 0; k < nch; ++k) { tbytes = std::max(tbytes, thi[k]); if (h_queries) qbytes = std::max(qbytes, qhi[k]); }
    cudaStream_t cs = nullptr;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) return -1;
    std::vector<cudaEvent_t> ready(nch, nullptr);
    uint8_t *d_t = nullptr, *d_traw = nullptr, *d_q = nullptr, *d_qraw = nullptr, *d_map = nullptr;
    int64_t *d_toff = nullptr, *d_qoff = nullptr;
    int *d_tlen = nullptr, *d_qlen = nullptr;
    pb_record *d_rec = nullptr;
    int rc = 0;
    for (int k = 0; k < nch && rc == 0; ++k)
        if (cudaEventCreateWithFlags(&ready[k], cudaEventDisableTiming) != cudaSuccess) rc = -1;
    if (rc == 0 &&
        (cudaMallocAsync((void **)&d_t, tbytes + 16, cs) != cudaSuccess ||
         cudaMallocAsync((void **)&d_traw, tbytes + 16, cs) != cudaSuccess ||
         cudaMallocAsync((void **)&d_toff, sizeof(int64_t) * n, cs) != cudaSuccess ||
         cudaMallocAsync((void **)&d_tlen, sizeof(int) * n, cs) != cudaSuccess ||
         cudaMallocAsync((void **)&d_map, 256, cs) != cudaSuccess ||
         cudaMallocAsync((void **)&d_rec, sizeof(pb_record) * n * (size_t)nq, cs) != cudaSuccess))
        rc = -1;
    if (rc == 0 && h_queries &&
        (cudaMallocAsync((void **)&d_q, qbytes + 16, cs) != cudaSuccess ||
         cudaMallocAsync((void **)&d_qraw, qbytes + 16, cs) != cudaSuccess ||
         cudaMallocAsync((void **)&d_qoff, sizeof(int64_t) * n, cs) != cudaSuccess ||
         cudaMallocAsync((void **)&d_qlen, sizeof(int) * n, cs) != cudaSuccess))
        rc = -1;
    auto stage = [&](int k) {
        /* chunk k's offsets, lengths and characters, mapped to codes */
        const size_t i0 = (size_t)cut[k], ni = (size_t)(cut[k + 1] - cut[k]);
        cudaMemcpyAsync(d_toff + i0, h_toff + i0, sizeof(int64_t) * ni, cudaMemcpyHostToDevice, cs);
        cudaMemcpyAsync(d_tlen + i0, h_tlen + i0, sizeof(int) * ni, cudaMemcpyHostToDevice, cs);
        cudaMemcpyAsync(d_traw + tlo[k], h_targets + tlo[k], thi[k] - tlo[k], cudaMemcpyHostToDevice, cs);
        k_map_into<<<296, 256, 0, cs>>>(d_traw, d_t, tlo[k], thi[k], d_map);
        pb_diag_count_launch(1);
        if (h_queries) {
            cudaMemcpyAsync(d_qoff + i0, h_qoff + i0, sizeof(int64_t) * ni, cudaMemcpyHostToDevice, cs);
            cudaMemcpyAsync(d_qlen + i0, h_qlen + i0, sizeof(int) * ni, cudaMemcpyHostToDevice, cs);
            cudaMemcpyAsync(d_qraw + qlo[k], h_queries + qlo[k], qhi[k] - qlo[k], cudaMemcpyHostToDevice, cs);
            k_map_into<<<296, 256, 0, cs>>>(d_qraw, d_q, qlo[k], qhi[k], d_map);
            pb_diag_count_launch(1);
        }
        cudaEventRecord(ready[k], cs);
    };
    if (rc == 0) {
        cudaMemcpyAsync(d_map, mapper256, 256, cudaMemcpyHostToDevice, cs);
        stage(0);
    }
    for (int k = 0; k < nch && rc == 0; ++k) {
        if (k + 1 < nch) stage(k + 1);
        if (cudaEventSynchronize(ready[k]) != cudaSuccess) { rc = -1; break; }
        const int i0 = cut[k];
        pb_batch b = *tmpl;
        b.npairs = cut[k + 1] - i0;
        b.d_targets = d_t; b.d_toff = d_toff + i0; b.d_tlen = d_tlen + i0;
        if (h_queries) { b.d_qall = d_q; b.d_qoff = d_qoff + i0; b.d_qlen = d_qlen + i0; }
        rc = pb_cuda_batch_run(job, &b, d_rec + (size_t)i0 * nq);
        if (rc == 0 && cudaMemcpyAsync(h_rec + (size_t)i0 * nq, d_rec + (size_t)i0 * nq,
                                       sizeof(pb_record) * (size_t)b.npairs * nq, cudaMemcpyDeviceToHost,
                                       cs) != cudaSuccess)
            rc = -1;
    }
    if (d_t) cudaFreeAsync(d_t, cs);
    if (d_traw) cudaFreeAsync(d_traw, cs);
    if (d_toff) cudaFreeAsync(d_toff, cs);
    if (d_tlen) cudaFreeAsync(d_tlen, cs);
    if (d_map) cudaFreeAsync(d_map, cs);
    if (d_rec) cudaFreeAsync(d_rec, cs);
    if (d_q) cudaFreeAsync(d_q, cs);
    if (d_qraw) cudaFreeAsync(d_qraw, cs);
    if (d_qoff) cudaFreeAsync(d_qoff, cs);
    if (d_qlen) cudaFreeAsync(d_qlen, cs);
    if (cudaStreamSynchronize(cs) != cudaSuccess) rc = -1;
    for (int k = 0; k < nch; ++k) if (ready[k]) cudaEventDestroy(ready[k]);
    cudaStreamDestroy(cs);
    return rc;
}

namespace {

/* pair p of the upper triangle of n sequences -> (i, j), i < j, row-major:
 * row i starts at i*n - i*(i+1)/2 */
__global__ void k_all_pairs(const int64_t *__restrict__ off, const int *__restrict__ len, int n, int npairs,
                            int64_t *__restrict__ qoff, int *__restrict__ qlen, int64_t *__restrict__ toff,
                            int *__restrict__ tlen, int *__restrict__ grp)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    const int64_t N = n;
    int lo = 0, hi = n - 2;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((int64_t)mid * N - (int64_t)mid * (mid + 1) / 2 <= p) lo = mid; else hi = mid - 1;
    }
    const int i = lo;
    const int j = i + 1 + (int)(p - ((int64_t)i * N - (int64_t)i * (i + 1) / 2));
    qoff[p] = off[i]; qlen[p] = len[i];
    toff[p] = off[j]; tlen[p] = len[j];
    grp[p] = i;
}

}  // namespace

extern "C" int pb_cuda_batch_all(const pb_job *job, const pb_batch *tmpl, const uint8_t *d_codes,
                                 const int64_t *d_off, const int *d_len, int n, pb_record *d_rec)
{
    if (pb_cuda_init() != 0) return -1;
    if (n < 2) return 0;
    const int npairs = (int)((int64_t)n * (n - 1) / 2);
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return -1;
    int64_t *qoff = nullptr, *toff = nullptr;
    int *qlen = nullptr, *tlen = nullptr, *grp = nullptr;
    int rc = 0;
    if (cudaMallocAsync((void **)&qoff, sizeof(int64_t) * npairs, st) != cudaSuccess ||
        cudaMallocAsync((void **)&toff, sizeof(int64_t) * npairs, st) != cudaSuccess ||
        cudaMallocAsync((void **)&qlen, sizeof(int) * npairs, st) != cudaSuccess ||
        cudaMallocAsync((void **)&tlen, sizeof(int) * npairs, st) != cudaSuccess ||
        cudaMallocAsync((void **)&grp, sizeof(int) * npairs, st) != cudaSuccess)
        rc = -1;
    if (rc == 0) {
        k_all_pairs<<<(npairs + 255) / 256, 256, 0, st>>>(d_off, d_len, n, npairs, qoff, qlen, toff, tlen, grp);
        pb_diag_count_launch(1);
        if (cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
    }
    if (rc == 0) {
        pb_batch b = *tmpl;
        b.nprofs = 0;
        b.npairs = npairs;
        b.d_qall = d_codes; b.d_qoff = qoff; b.d_qlen = qlen;
        b.d_targets = d_codes; b.d_toff = toff; b.d_tlen = tlen;
        b.d_qgroup = grp;
        rc = pb_cuda_batch_run(job, &b, d_rec);
    }
    if (grp) cudaFreeAsync(grp, st);
    if (qoff) cudaFreeAsync(qoff, st);
    if (toff) cudaFreeAsync(toff, st);
    if (qlen) cudaFreeAsync(qlen, st);
    if (tlen) cudaFreeAsync(tlen, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
    cudaStreamDestroy(st);
    return rc;
}

extern "C" int pb_cuda_batch_all_host(const pb_job *job, const pb_batch *tmpl, const uint8_t *mapper256,
                                      const char *h_seqs, const int64_t *h_off, const int *h_len, int n,
                                      pb_record *h_rec)
{
    if (pb_cuda_init() != 0) return -1;
    if (n < 2) return 0;
    const size_t npairs = (size_t)n * (n - 1) / 2;
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return -1;
    int64_t bytes = 0;
    for (int i = 0; i < n; ++i) bytes = h_off[i] + h_len[i] > bytes ? h_off[i] + h_len[i] : bytes;
    uint8_t *d_s = nullptr, *d_map = nullptr;
    int64_t *d_off = nullptr;
    int *d_len = nullptr;
    pb_record *d_rec = nullptr;
    int rc = 0;
    if (cudaMallocAsync((void **)&d_s, bytes + 16, st) != cudaSuccess ||
        cudaMallocAsync((void **)&d_off, sizeof(int64_t) * n, st) != cudaSuccess ||
        cudaMallocAsync((void **)&d_len, sizeof(int) * n, st) != cudaSuccess ||
        cudaMallocAsync((void **)&d_map, 256, st) != cudaSuccess ||
        cudaMallocAsync((void **)&d_rec, sizeof(pb_record) * npairs, st) != cudaSuccess)
        rc = -1;
    if (rc == 0) {
        cudaMemcpyAsync(d_s, h_seqs, bytes, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_off, h_off, sizeof(int64_t) * n, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_len, h_len, sizeof(int) * n, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_map, mapper256, 256, cudaMemcpyHostToDevice, st);
        k_map_codes<<<296, 256, 0, st>>>(d_s, bytes, d_map);
        pb_diag_count_launch(1);
        if (cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
    }
    if (rc == 0) rc = pb_cuda_batch_all(job, tmpl, d_s, d_off, d_len, n, d_rec);
    if (rc == 0 && cudaMemcpyAsync(h_rec, d_rec, sizeof(pb_record) * npairs, cudaMemcpyDeviceToHost, st) != cudaSuccess)
        rc = -1;
    if (d_s) cudaFreeAsync(d_s, st);
    if (d_off) cudaFreeAsync(d_off, st);
    if (d_len) cudaFreeAsync(d_len, st);
    if (d_map) cudaFreeAsync(d_map, st);
    if (d_rec) cudaFreeAsync(d_rec, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
    cudaStreamDestroy(st);
    return rc;
}
