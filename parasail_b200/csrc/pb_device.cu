/*
 * pb_device.cu -- device management, profile construction, memory helpers
 * and the launch entry points of the C ABI in pb_cuda.h.
 *
 * Every host thread gets its own non-blocking stream; device memory comes
 * from the stream-ordered pool allocator, whose release threshold is raised
 * so that repeated calls reuse memory instead of returning it to the driver.
 */
#include <cstdio>
#include <cstring>
#include <cstdint>
#include <vector>
#include <mutex>

#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_radix_sort.cuh>

#include "pb_cuda.h"
#include "pb_kernels.cuh"

namespace {

thread_local char g_err[256] = "";
thread_local cudaStream_t g_stream = nullptr;
std::once_flag g_init_once;
int g_init_rc = -1;

void set_err(const char *what, cudaError_t e)
{
    snprintf(g_err, sizeof g_err, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call)                                   \
    do {                                           \
        cudaError_t e_ = (call);                   \
        if (e_ != cudaSuccess) {                   \
            set_err(#call, e_);                    \
            return -1;                             \
        }                                          \
    } while (0)

cudaStream_t stream()
{
    if (!g_stream) cudaStreamCreateWithFlags(&g_stream, cudaStreamNonBlocking);
    return g_stream;
}

/* A second stream and an event per host thread, for work that runs beside
 * the thread's main stream; created once and kept. */
thread_local cudaStream_t g_stream2 = nullptr;
thread_local cudaEvent_t g_event2 = nullptr;

int side_stream(cudaStream_t *st2, cudaEvent_t *ev)
{
    if (!g_stream2 && cudaStreamCreateWithFlags(&g_stream2, cudaStreamNonBlocking) != cudaSuccess) {
        g_stream2 = nullptr;
        return -1;
    }
    if (!g_event2 && cudaEventCreateWithFlags(&g_event2, cudaEventDisableTiming) != cudaSuccess) {
        g_event2 = nullptr;
        return -1;
    }
    *st2 = g_stream2;
    *ev = g_event2;
    return 0;
}

/* Stream-ordered frees of a call's pool allocations, on every return path
 * (an early error return included). */
struct PoolFrees {
    cudaStream_t st;
    void *p[16];
    int n = 0;
    explicit PoolFrees(cudaStream_t s) : st(s) {}
    template <typename T> T *add(T *q) { if (q && n < 16) p[n++] = (void *)q; return q; }
    ~PoolFrees() { for (int k = 0; k < n; ++k) cudaFreeAsync(p[k], st); }
};

void do_init()
{
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n <= 0) {
        snprintf(g_err, sizeof g_err, "no CUDA device available (%s)",
                 e != cudaSuccess ? cudaGetErrorString(e) : "count 0");
        g_init_rc = -1;
        return;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    g_init_rc = 0;
}

__global__ void k_build_profile(const int *__restrict__ table, int is_pssm, int size,
                                const uint8_t *__restrict__ qcodes, int qlen, int lp,
                                int32_t *__restrict__ prof32, int8_t *__restrict__ prof8)
{
    const int64_t n = (int64_t)size * lp;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < n;
         idx += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(idx / lp), i = (int)(idx % lp);
        int v = 0;
        if (i < qlen) v = is_pssm ? table[(int64_t)i * size + k] : table[(int64_t)k * size + qcodes[i]];
        prof32[idx] = v;
        if (prof8) prof8[idx] = (int8_t)v;
    }
}

/* bytes -> codes through a 256-entry table, in place */
__global__ void k_map_bytes(uint8_t *__restrict__ buf, int64_t n, const uint8_t *__restrict__ map)
{
    __shared__ uint8_t smap[256];
    for (int k = threadIdx.x; k < 256; k += blockDim.x) smap[k] = map[k];
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        buf[i] = smap[buf[i]];
}

__global__ void k_scratch_sizes(const int *__restrict__ tlen, const int *__restrict__ tlim,
                                int n, int nv, int64_t *__restrict__ sizes)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n) sizes[p] = (int64_t)(tlim ? tlim[p] : tlen[p]) * nv;
}

/* one query per pair (its own codes, qlen[k], or a profile per pair,
 * profs[prof_index[k]], or one profile for all, profs[0]): each pair's work
 * (query length x target length),
 * with the warp-per-pair items (the rule of k_exact_db_items) flagged in
 * bit 62 */
__global__ void k_exact_pair_items(const int *__restrict__ qlen, const pb::ProfDesc *__restrict__ profs,
                                   const int *__restrict__ prof_index, const int *__restrict__ tlen,
                                   const int *__restrict__ qlim, const int *__restrict__ tlim, int n,
                                   unsigned long long *__restrict__ keys, int *__restrict__ idx, int *nwarp)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int q = qlen ? qlen[k] : profs[prof_index ? prof_index[k] : 0].qlen;
    const int ql = qlim ? qlim[k] : q, tl = tlim ? tlim[k] : tlen[k];
    const long long cells = (long long)ql * tl;
    const bool w = ql >= 32 || (ql >= 8 && cells >= (1LL << 14));
    keys[k] = (unsigned long long)cells | (w ? 1ull << 62 : 0ull);
    idx[k] = k;
    if (w) atomicAdd(nwarp, 1);
}

/* every query against every target: scratch per (query, target) item,
 * query-major, and the item's work (query length x target length) */
__global__ void k_exact_db_items(const int *__restrict__ tlen, const int *__restrict__ qlens,
                                 const int *__restrict__ qlim, const int *__restrict__ tlim, int n, int nq, int nv,
                                 int warp_min_qlen, int64_t *__restrict__ sizes,
                                 unsigned long long *__restrict__ keys, int *__restrict__ idx, int *nwarp)
{
    const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (k >= (long long)n * nq) return;
    const int t = (int)(k % n), q = (int)(k / n);
    /* per-item limits (a prefix of the pair) when given */
    const int ql = qlim ? qlim[k] : qlens[q], tl = tlim ? tlim[k] : tlen[t];
    sizes[k] = (int64_t)tl * nv;
    /* items for the warp-per-pair kernel sort first (bit 62): every query of
     * 32 rows or more, and shorter ones (8 or more) whose pair has 2^14
     * cells or more. On 5 queries (100-2000) x 20,000 targets this beat
     * one thread per pair at every size: NW 455 GCUPS against 288 with the
     * warp kernel only for pairs of 2^18 cells and queries that fill a
     * pass, and NW statistics 227 against 74 */
    const long long cells = (long long)ql * tl;
    const bool w = warp_min_qlen > 0 && (ql >= 32 || (ql >= 8 && cells >= (1LL << 14)));
    keys[k] = (unsigned long long)cells | (w ? 1ull << 62 : 0ull);
    idx[k] = (int)k;
    if (w) atomicAdd(nwarp, 1);
}

/* Copies the host descriptors of the batch's profiles to the device. */
pb::ProfDesc *upload_profs(const pb_batch *b, cudaStream_t st)
{
    std::vector<pb::ProfDesc> h(b->nprofs);
    for (int k = 0; k < b->nprofs; ++k) {
        const pb_device_profile *p = b->profs[k];
        h[k].prof = p->d_prof32;
        h[k].prof8 = p->d_prof8;
        h[k].qcodes = p->d_qcodes;
        h[k].qlen = p->qlen;
        h[k].lp = p->lp;
        h[k].size = p->size;
        h[k].pad_ = 0;
    }
    pb::ProfDesc *d = nullptr;
    if (cudaMallocAsync((void **)&d, sizeof(pb::ProfDesc) * h.size(), st) != cudaSuccess) return nullptr;
    cudaMemcpyAsync(d, h.data(), sizeof(pb::ProfDesc) * h.size(), cudaMemcpyHostToDevice, st);
    /* the host vector dies at return: make the copy complete first */
    cudaStreamSynchronize(st);
    return d;
}

}  // namespace

extern "C" {

int pb_cuda_init(void)
{
    std::call_once(g_init_once, do_init);
    return g_init_rc;
}

const char *pb_cuda_last_error(void) { return g_err; }
void pb_cuda_set_error(const char *what, const char *detail)
{
    snprintf(g_err, sizeof g_err, "%s: %s", what, detail ? detail : "");
}

int pb_cuda_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

void *pb_cuda_malloc(size_t bytes)
{
    void *p = nullptr;
    if (pb_cuda_init() != 0) return nullptr;
    if (cudaMallocAsync(&p, bytes ? bytes : 1, stream()) != cudaSuccess) {
        snprintf(g_err, sizeof g_err, "device allocation of %zu bytes failed", bytes);
        return nullptr;
    }
    return p;
}

void pb_cuda_free(void *p)
{
    if (p) cudaFreeAsync(p, stream());
}

int pb_cuda_h2d(void *dst, const void *src, size_t bytes)
{
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream()));
    return 0;
}

int pb_cuda_d2h(void *dst, const void *src, size_t bytes)
{
    CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream()));
    CK(cudaStreamSynchronize(stream()));
    return 0;
}

int pb_cuda_sync(void)
{
    CK(cudaStreamSynchronize(stream()));
    return 0;
}

/* copies n host characters to d_buf and maps them to codes there */
int pb_cuda_h2d_mapped(uint8_t *d_buf, const char *h_chars, int64_t n, const uint8_t *mapper256)
{
    if (n <= 0) return 0;
    cudaStream_t st = stream();
    uint8_t *d_map = nullptr;
    CK(cudaMallocAsync((void **)&d_map, 256, st));
    CK(cudaMemcpyAsync(d_map, mapper256, 256, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_buf, h_chars, (size_t)n, cudaMemcpyHostToDevice, st));
    k_map_bytes<<<296, 256, 0, st>>>(d_buf, n, d_map);
    pb_diag_count_launch(1);
    CK(cudaGetLastError());
    CK(cudaFreeAsync(d_map, st));
    /* the host mapper copy dies at return */
    CK(cudaStreamSynchronize(st));
    return 0;
}

/* waits for all work on the device, the legacy default stream included */
int pb_cuda_device_sync(void)
{
    CK(cudaDeviceSynchronize());
    return 0;
}

int pb_cuda_memset(void *p, int v, size_t bytes)
{
    CK(cudaMemsetAsync(p, v, bytes, stream()));
    CK(cudaStreamSynchronize(stream()));
    return 0;
}

int pb_cuda_profile_create(const int *table, int is_pssm, int size,
                           const uint8_t *qcodes, int qlen, int mmax, int mmin,
                           pb_device_profile *out)
{
    if (pb_cuda_init() != 0) return -1;
    memset(out, 0, sizeof *out);
    const int lp = ((qlen + 32 + 63) / 64) * 64;
    const size_t tsz = (size_t)(is_pssm ? qlen : size) * size;
    cudaStream_t st = stream();
    int vmin = 0, vmax = 0;
    for (size_t k = 0; k < tsz; ++k) {
        vmin = table[k] < vmin ? table[k] : vmin;
        vmax = table[k] > vmax ? table[k] : vmax;
    }
    const int fits8 = vmin >= -128 && vmax <= 127;
    int *d_table = nullptr;
    std::vector<uint8_t> hq(lp, 255);
    memcpy(hq.data(), qcodes, qlen);
    CK(cudaMallocAsync((void **)&d_table, tsz * sizeof(int), st));
    CK(cudaMallocAsync((void **)&out->d_qcodes, lp, st));
    CK(cudaMallocAsync((void **)&out->d_prof32, (size_t)size * lp * sizeof(int32_t), st));
    if (fits8) CK(cudaMallocAsync((void **)&out->d_prof8, (size_t)size * lp, st));
    CK(cudaMemcpyAsync(d_table, table, tsz * sizeof(int), cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(out->d_qcodes, hq.data(), lp, cudaMemcpyHostToDevice, st));
    k_build_profile<<<148, 256, 0, st>>>(d_table, is_pssm, size, out->d_qcodes, qlen, lp,
                                         out->d_prof32, fits8 ? out->d_prof8 : nullptr);
    CK(cudaGetLastError());
    CK(cudaFreeAsync(d_table, st));
    CK(cudaStreamSynchronize(st));
    out->qlen = qlen;
    out->lp = lp;
    out->size = size;
    out->fits8 = fits8;
    out->mmax = mmax;
    out->mmin = mmin;
    cudaGetDevice(&out->device);
    return 0;
}

void pb_cuda_profile_destroy(pb_device_profile *p)
{
    if (!p) return;
    cudaStream_t st = stream();
    if (p->d_prof32) cudaFreeAsync(p->d_prof32, st);
    if (p->d_prof8) cudaFreeAsync(p->d_prof8, st);
    if (p->d_qcodes) cudaFreeAsync(p->d_qcodes, st);
    cudaStreamSynchronize(st);
    memset(p, 0, sizeof *p);
}

int pb_cuda_align_exact(const pb_batch *b)
{
    if (pb_cuda_init() != 0) return -1;
    if (b->npairs <= 0) return 0;
    cudaStream_t st = stream();
    PoolFrees frees(st);
    const int nv = b->stats ? 8 : 2;
    int64_t *sizes = nullptr, *soff = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    CK(cudaMallocAsync((void **)&sizes, sizeof(int64_t) * b->npairs, st));
    frees.add(sizes);
    CK(cudaMallocAsync((void **)&soff, sizeof(int64_t) * b->npairs, st));
    frees.add(soff);
    k_scratch_sizes<<<(b->npairs + 255) / 256, 256, 0, st>>>(b->d_tlen, b->d_tlim, b->npairs, nv, sizes);
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, sizes, soff, b->npairs, st);
    CK(cudaMallocAsync(&tmp, tmp_bytes, st));
    frees.add(tmp);
    cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, sizes, soff, b->npairs, st);
    int64_t last_off = 0, last_size = 0;
    CK(cudaMemcpyAsync(&last_off, soff + b->npairs - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&last_size, sizes + b->npairs - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    int *scratch = nullptr;
    CK(cudaMallocAsync((void **)&scratch, sizeof(int) * (size_t)(last_off + last_size + 1), st));
    frees.add(scratch);
    pb::ProfDesc *d_profs = nullptr;
    if (b->nprofs > 0) {
        d_profs = frees.add(upload_profs(b, st));
        if (!d_profs) { snprintf(g_err, sizeof g_err, "profile descriptor upload failed"); return -1; }
    }

    pb::ExactParams p;
    p.alg = b->alg; p.sgflags = b->sgflags; p.open = b->open; p.gap = b->gap;
    p.pad_rows = b->pad_rows; p.npairs = b->npairs;
    p.profs = d_profs; p.prof_index = b->d_prof_index;
    p.targets = b->d_targets; p.toff = b->d_toff; p.tlen = b->d_tlen;
    p.qlim = b->d_qlim; p.tlim = b->d_tlim;
    p.scratch = scratch; p.soff = soff; p.out = b->d_out;
    p.mat = b->d_mat; p.msize = b->msize; p.qall = b->d_qall; p.qoff = b->d_qoff; p.qlen = b->d_qlen;
    /* the exact kernels score through the matrix whenever one is given;
     * profile mode without an index is one profile against every target
     * (the single calls of parasail.h among them) */
    const bool per_pair = (b->d_mat && b->d_qlen) || (!b->d_mat && b->nprofs > 0);
    if (per_pair) {
        /* one query per pair (its own codes, or a profile per pair): long
         * pairs one per warp on a side stream (most cells first), the rest
         * one per thread beside them */
        const int n = b->npairs;
        unsigned long long *keys = nullptr, *keys_sorted = nullptr;
        int *idx = nullptr, *order = nullptr, *d_nwarp = nullptr;
        void *stmp = nullptr;
        size_t stmp_bytes = 0;
        CK(cudaMallocAsync((void **)&keys, sizeof(unsigned long long) * n, st));
        frees.add(keys);
        CK(cudaMallocAsync((void **)&keys_sorted, sizeof(unsigned long long) * n, st));
        frees.add(keys_sorted);
        CK(cudaMallocAsync((void **)&idx, sizeof(int) * n, st));
        frees.add(idx);
        CK(cudaMallocAsync((void **)&order, sizeof(int) * n, st));
        frees.add(order);
        CK(cudaMallocAsync((void **)&d_nwarp, sizeof(int), st));
        frees.add(d_nwarp);
        CK(cudaMemsetAsync(d_nwarp, 0, sizeof(int), st));
        const bool matmode = b->d_mat != nullptr;
        k_exact_pair_items<<<(n + 255) / 256, 256, 0, st>>>(matmode ? b->d_qlen : nullptr, d_profs,
                                                           matmode ? nullptr : b->d_prof_index, b->d_tlen,
                                                           b->d_qlim, b->d_tlim, n, keys, idx, d_nwarp);
        if (n > 1) {
            cub::DeviceRadixSort::SortPairsDescending(nullptr, stmp_bytes, keys, keys_sorted, idx, order, n, 0, 64,
                                                      st);
            CK(cudaMallocAsync(&stmp, stmp_bytes, st));
            frees.add(stmp);
            cub::DeviceRadixSort::SortPairsDescending(stmp, stmp_bytes, keys, keys_sorted, idx, order, n, 0, 64, st);
        } else {
            order = idx;     /* one pair: nothing to order */
        }
        int nwarp = 0;
        CK(cudaMemcpyAsync(&nwarp, d_nwarp, sizeof(int), cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        p.order = order;
        cudaStream_t st2 = nullptr;
        cudaEvent_t ev = nullptr;
        if (nwarp > 0) {
            if (side_stream(&st2, &ev) != 0) { snprintf(g_err, sizeof g_err, "side stream creation failed"); return -1; }
            CK(cudaEventRecord(ev, st));
            CK(cudaStreamWaitEvent(st2, ev, 0));
            pb::launch_exact_warp(p, b->alg, b->stats != 0, nwarp, st2);
            pb_diag_count_launch(1);
        }
        if (n - nwarp > 0) {
            pb::ExactParams pt = p;
            pt.order = order + nwarp;
            pt.npairs = n - nwarp;
            pb::launch_exact(pt, b->alg, b->stats != 0, st);
            pb_diag_count_launch(1);
        }
        if (st2) {
            CK(cudaEventRecord(ev, st2));
            CK(cudaStreamWaitEvent(st, ev, 0));
        }
        pb_diag_count_launch(2);   /* k_scratch_sizes, k_exact_pair_items (plus the library sort) */
    } else {
        pb::launch_exact(p, b->alg, b->stats != 0, st);
        pb_diag_count_launch(2);   /* k_scratch_sizes, k_exact */
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    return 0;
}

/*
 * Every profile of the batch against every target in one exact-kernel
 * launch (outputs query-major: d_out[q * npairs + t]). One thread aligns
 * one pair, so a warp runs as long as its longest pair: the items go to
 * the threads in order of work, largest first, which gives each warp pairs
 * of like size and starts the longest ones first.
 */
int pb_cuda_align_exact_db(const pb_batch *b)
{
    if (pb_cuda_init() != 0) return -1;
    const int n = b->npairs, nq = b->nprofs;
    if (n <= 0 || nq <= 0) return 0;
    if ((long long)n * nq > INT32_MAX) { snprintf(g_err, sizeof g_err, "batch too large"); return -1; }
    const int N = n * nq;
    cudaStream_t st = stream();
    const int nv = b->stats ? 8 : 2;
    int64_t *sizes = nullptr, *soff = nullptr;
    unsigned long long *keys = nullptr, *keys_sorted = nullptr;
    int *idx = nullptr, *order = nullptr, *d_qlens = nullptr, *d_nwarp = nullptr;
    void *tmp = nullptr, *stmp = nullptr;
    size_t tmp_bytes = 0, stmp_bytes = 0;
    std::vector<int> hq(nq);
    for (int q = 0; q < nq; ++q) hq[q] = b->profs[q]->qlen;
    PoolFrees frees(st);
    CK(cudaMallocAsync((void **)&sizes, sizeof(int64_t) * N, st));
    frees.add(sizes);
    CK(cudaMallocAsync((void **)&soff, sizeof(int64_t) * N, st));
    frees.add(soff);
    CK(cudaMallocAsync((void **)&keys, sizeof(unsigned long long) * N, st));
    frees.add(keys);
    CK(cudaMallocAsync((void **)&keys_sorted, sizeof(unsigned long long) * N, st));
    frees.add(keys_sorted);
    CK(cudaMallocAsync((void **)&idx, sizeof(int) * N, st));
    frees.add(idx);
    CK(cudaMallocAsync((void **)&order, sizeof(int) * N, st));
    frees.add(order);
    CK(cudaMallocAsync((void **)&d_qlens, sizeof(int) * nq, st));
    frees.add(d_qlens);
    CK(cudaMallocAsync((void **)&d_nwarp, sizeof(int), st));
    frees.add(d_nwarp);
    CK(cudaMemcpyAsync(d_qlens, hq.data(), sizeof(int) * nq, cudaMemcpyHostToDevice, st));
    CK(cudaMemsetAsync(d_nwarp, 0, sizeof(int), st));
    /* pairs go one per warp (k_exact_db_items) */
    const int warp_min_qlen = pb::exact_warp_pass_rows(b->stats != 0);
    k_exact_db_items<<<(N + 255) / 256, 256, 0, st>>>(b->d_tlen, d_qlens, b->d_qlim, b->d_tlim, n, nq, nv,
                                                      warp_min_qlen, sizes, keys, idx, d_nwarp);
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, sizes, soff, N, st);
    cub::DeviceRadixSort::SortPairsDescending(nullptr, stmp_bytes, keys, keys_sorted, idx, order, N, 0, 64, st);
    CK(cudaMallocAsync(&tmp, tmp_bytes, st));
    frees.add(tmp);
    CK(cudaMallocAsync(&stmp, stmp_bytes, st));
    frees.add(stmp);
    cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, sizes, soff, N, st);
    cub::DeviceRadixSort::SortPairsDescending(stmp, stmp_bytes, keys, keys_sorted, idx, order, N, 0, 64, st);
    int64_t last_off = 0, last_size = 0;
    int nwarp = 0;
    CK(cudaMemcpyAsync(&last_off, soff + N - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&last_size, sizes + N - 1, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(&nwarp, d_nwarp, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    int *scratch = nullptr;
    CK(cudaMallocAsync((void **)&scratch, sizeof(int) * (size_t)(last_off + last_size + 1), st));
    frees.add(scratch);
    pb::ProfDesc *d_profs = frees.add(upload_profs(b, st));
    if (!d_profs) { snprintf(g_err, sizeof g_err, "profile descriptor upload failed"); return -1; }

    pb::ExactParams p;
    p.alg = b->alg; p.sgflags = b->sgflags; p.open = b->open; p.gap = b->gap;
    p.pad_rows = b->pad_rows; p.npairs = N;
    p.profs = d_profs; p.prof_index = nullptr;
    p.targets = b->d_targets; p.toff = b->d_toff; p.tlen = b->d_tlen;
    p.qlim = b->d_qlim; p.tlim = b->d_tlim;      /* per item (query-major), or none */
    p.scratch = scratch; p.soff = soff; p.out = b->d_out;
    p.mat = nullptr; p.msize = 0; p.qall = nullptr; p.qoff = nullptr; p.qlen = nullptr;
    p.order = order; p.nt = n;
    /* the warp-per-pair items (sorted first) on the thread's side stream,
     * the rest one per thread beside them */
    cudaStream_t st2 = nullptr;
    cudaEvent_t ev = nullptr;
    if (nwarp > 0) {
        if (side_stream(&st2, &ev) != 0) { snprintf(g_err, sizeof g_err, "side stream creation failed"); return -1; }
        CK(cudaEventRecord(ev, st));
        CK(cudaStreamWaitEvent(st2, ev, 0));
        pb::launch_exact_warp(p, b->alg, b->stats != 0, nwarp, st2);
        pb_diag_count_launch(1);
    }
    if (N - nwarp > 0) {
        pb::ExactParams pt = p;
        pt.order = order + nwarp;
        pt.npairs = N - nwarp;
        pb::launch_exact(pt, b->alg, b->stats != 0, st);
        pb_diag_count_launch(1);
    }
    if (st2) {
        CK(cudaEventRecord(ev, st2));
        CK(cudaStreamWaitEvent(st, ev, 0));
    }
    pb_diag_count_launch(1);   /* k_exact_db_items (plus the library scan and sort) */
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
    return 0;
}

/* ---- single pairs (the one-pair calls of parasail.h) ----------------------
 * A per-thread device arena holds one pair's descriptors, target codes,
 * scratch and output: one upload, one launch, one download and one
 * synchronisation per call, instead of the batch pipeline's set-up. */

namespace {

struct SingleArena {
    char *d = nullptr;
    size_t cap = 0;
    std::vector<char> h;     /* host staging of the upload */
};
thread_local SingleArena g_single;

size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

}  // namespace

/* the calling thread's stream of the library */
void *pb_cuda_stream(void) { return (void *)stream(); }

/* Raises a kernel's dynamic shared-memory limit to at least `bytes`, never
 * lowering it: a limit set for a small launch must not fail a larger one of
 * another call, another host thread or a recorded graph. */
int pb_raise_smem(const void *func, int bytes)
{
    static std::mutex mu;
    static std::vector<std::pair<const void *, int>> seen;
    std::lock_guard<std::mutex> lock(mu);
    for (auto &x : seen)
        if (x.first == func) {
            if (bytes <= x.second) return 0;
            if (cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess)
                return -1;
            x.second = bytes;
            return 0;
        }
    const int want = bytes > 48 * 1024 ? bytes : 48 * 1024;
    if (cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, want) != cudaSuccess) return -1;
    seen.emplace_back(func, want);
    return 0;
}

/* the calling thread's arena of at least `bytes` device bytes, and (host)
 * a zeroed host staging buffer of host_bytes */
char *pb_single_arena(size_t bytes, size_t host_bytes, char **host)
{
    if (bytes > g_single.cap) {
        if (g_single.d) cudaFree(g_single.d);
        size_t cap = bytes < ((size_t)1 << 20) ? ((size_t)1 << 20) : bytes;
        cap = (cap + 4095) & ~(size_t)4095;
        if (cudaMalloc((void **)&g_single.d, cap) != cudaSuccess) {
            g_single.d = nullptr;
            g_single.cap = 0;
            return nullptr;
        }
        g_single.cap = cap;
    }
    g_single.h.assign(host_bytes, 0);
    if (host) *host = g_single.h.data();
    return g_single.d;
}

/* One pair on the exact kernel from host target codes: the warp kernel for a
 * pair of 32 rows or more (or of 8 rows and 2^14 cells), else one thread.
 * qlim/tlim > 0 limit the pair to a prefix (the FASTSTATS pass). */
int pb_cuda_exact_single(const pb_batch *tmpl, const uint8_t *h_codes, int tlen, int qlim, int tlim,
                         pb_pair_out *h_out)
{
    if (pb_cuda_init() != 0) return -1;
    if (tmpl->nprofs != 1 || tlen <= 0) return -1;
    cudaGetLastError();   /* a launch error below is this call's own */
    const pb_device_profile *dp = tmpl->profs[0];
    const int nv = tmpl->stats ? 8 : 2;
    const int ql = qlim > 0 ? qlim : dp->qlen, tl = tlim > 0 ? tlim : tlen;
    /* [ProfDesc][soff, toff: int64][order, tlen, qlim, tlim: int][out][codes] then scratch */
    const size_t o_pd = 0, o_soff = align16(sizeof(pb::ProfDesc)), o_toff = o_soff + 8, o_ints = o_toff + 8;
    const size_t o_out = align16(o_ints + 16), o_codes = align16(o_out + sizeof(pb_pair_out));
    const size_t up = align16(o_codes + (size_t)tlen + 16);
    const size_t total = up + sizeof(int) * ((size_t)tl * nv + 16);
    char *h = nullptr;
    char *d = pb_single_arena(total, up, &h);
    if (!d) { snprintf(g_err, sizeof g_err, "single-pair arena allocation failed"); return -1; }
    pb::ProfDesc pd;
    pd.prof = dp->d_prof32; pd.prof8 = dp->d_prof8; pd.qcodes = dp->d_qcodes;
    pd.qlen = dp->qlen; pd.lp = dp->lp; pd.size = dp->size; pd.pad_ = 0;
    memcpy(h + o_pd, &pd, sizeof pd);
    const int ints[4] = {0, tlen, qlim, tlim};
    memcpy(h + o_ints, ints, sizeof ints);
    memcpy(h + o_codes, h_codes, (size_t)tlen);
    cudaStream_t st = stream();
    CK(cudaMemcpyAsync(d, h, up, cudaMemcpyHostToDevice, st));
    pb::ExactParams p;
    p.alg = tmpl->alg; p.sgflags = tmpl->sgflags; p.open = tmpl->open; p.gap = tmpl->gap;
    p.pad_rows = tmpl->pad_rows; p.npairs = 1;
    p.profs = reinterpret_cast<const pb::ProfDesc *>(d + o_pd); p.prof_index = nullptr;
    p.targets = reinterpret_cast<const uint8_t *>(d + o_codes);
    p.toff = reinterpret_cast<const int64_t *>(d + o_toff);
    p.tlen = reinterpret_cast<const int *>(d + o_ints) + 1;
    p.qlim = qlim > 0 ? reinterpret_cast<const int *>(d + o_ints) + 2 : nullptr;
    p.tlim = tlim > 0 ? reinterpret_cast<const int *>(d + o_ints) + 3 : nullptr;
    p.scratch = reinterpret_cast<int *>(d + up);
    p.soff = reinterpret_cast<const int64_t *>(d + o_soff);
    p.out = reinterpret_cast<pb_pair_out *>(d + o_out);
    p.mat = nullptr; p.msize = 0; p.qall = nullptr; p.qoff = nullptr; p.qlen = nullptr;
    p.order = reinterpret_cast<const int *>(d + o_ints);
    p.nt = 0;
    p.scan_vgap = tmpl->scan_vgap;
    const long long cells = (long long)ql * tl;
    if (ql >= 32 || (ql >= 8 && cells >= (1LL << 14))) pb::launch_exact_warp(p, tmpl->alg, tmpl->stats != 0, 1, st);
    else pb::launch_exact(p, tmpl->alg, tmpl->stats != 0, st);
    pb_diag_count_launch(1);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(h_out, d + o_out, sizeof(pb_pair_out), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return 0;
}

int pb_cuda_align_host(int kernel, const pb_batch *tmpl,
                       const uint8_t *h_targets, const int64_t *h_toff,
                       const int *h_tlen, const int *h_qlim, const int *h_tlim,
                       const int *h_prof_index, int npairs, pb_pair_out *h_out)
{
    if (pb_cuda_init() != 0) return -1;
    if (npairs <= 0) return 0;
    cudaStream_t st = stream();
    int64_t total = 0;
    for (int p = 0; p < npairs; ++p) {
        const int64_t e = h_toff[p] + h_tlen[p];
        total = e > total ? e : total;
    }
    pb_batch b = *tmpl;
    uint8_t *d_t = nullptr;
    int64_t *d_off = nullptr;
    int *d_len = nullptr, *d_ql = nullptr, *d_tl = nullptr, *d_pi = nullptr;
    pb_pair_out *d_out = nullptr;
    CK(cudaMallocAsync((void **)&d_t, total + 16, st));
    CK(cudaMallocAsync((void **)&d_off, sizeof(int64_t) * npairs, st));
    CK(cudaMallocAsync((void **)&d_len, sizeof(int) * npairs, st));
    CK(cudaMallocAsync((void **)&d_out, sizeof(pb_pair_out) * npairs, st));
    CK(cudaMemcpyAsync(d_t, h_targets, total, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_off, h_toff, sizeof(int64_t) * npairs, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(d_len, h_tlen, sizeof(int) * npairs, cudaMemcpyHostToDevice, st));
    if (h_qlim) {
        CK(cudaMallocAsync((void **)&d_ql, sizeof(int) * npairs, st));
        CK(cudaMemcpyAsync(d_ql, h_qlim, sizeof(int) * npairs, cudaMemcpyHostToDevice, st));
    }
    if (h_tlim) {
        CK(cudaMallocAsync((void **)&d_tl, sizeof(int) * npairs, st));
        CK(cudaMemcpyAsync(d_tl, h_tlim, sizeof(int) * npairs, cudaMemcpyHostToDevice, st));
    }
    if (h_prof_index) {
        CK(cudaMallocAsync((void **)&d_pi, sizeof(int) * npairs, st));
        CK(cudaMemcpyAsync(d_pi, h_prof_index, sizeof(int) * npairs, cudaMemcpyHostToDevice, st));
    }
    b.npairs = npairs;
    b.d_targets = d_t; b.d_toff = d_off; b.d_tlen = d_len;
    b.d_qlim = d_ql; b.d_tlim = d_tl; b.d_prof_index = d_pi;
    b.d_out = d_out;
    int rc = kernel == 1 ? pb_cuda_align_sw16(&b) : pb_cuda_align_exact(&b);
    if (rc == 0) {
        CK(cudaMemcpyAsync(h_out, d_out, sizeof(pb_pair_out) * npairs, cudaMemcpyDeviceToHost, st));
    }
    cudaFreeAsync(d_t, st);
    cudaFreeAsync(d_off, st);
    cudaFreeAsync(d_len, st);
    cudaFreeAsync(d_out, st);
    if (d_ql) cudaFreeAsync(d_ql, st);
    if (d_tl) cudaFreeAsync(d_tl, st);
    if (d_pi) cudaFreeAsync(d_pi, st);
    CK(cudaStreamSynchronize(st));
    return rc;
}

}  // extern "C"
