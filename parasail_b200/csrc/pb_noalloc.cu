/*
 * pb_noalloc.cu -- one profile against device-resident targets without any
 * device allocation: the exact kernel (pb_exact.cu) and the width resolution
 * (pb_batch.cu) run with their scratch carved out of one file-scope device
 * array of fixed size, PB_NOALLOC_SCRATCH_BYTES.
 *
 * Layout of the array for a call of n pairs (each region 256-byte aligned):
 *   [profile descriptor | n per-pair kernel outputs | n + 1 strip offsets |
 *    strip buffers: (target length) x (2 ints score-only, 8 with statistics)]
 * Once the exact kernel is done, the strip region is reused for the
 * resolution's work area (lists and results of the lane-exact rounds, and
 * the lane kernel's per-warp arrays).
 * Every region is written by the call before it is read (descriptor copy,
 * offset scan, the exact kernel's per-pair outputs; a strip buffer's first
 * strip reads the top boundary, not the buffer), so nothing has to start at
 * zero and the contents left by an earlier call are never observed.
 *
 * The array is shared by every call on a device: calls that overlap in time
 * on one device (two host threads, or two streams) race on it and must be
 * serialised by the caller.
 */
#include <cstdio>
#include <cstdint>
#include <mutex>
#include <cuda_runtime.h>
#include <cub/block/block_scan.cuh>

#include "pb_cuda.h"
#include "pb_kernels.cuh"
#include "pb_resolve.h"

namespace {

constexpr size_t PB_NOALLOC_SCRATCH_BYTES = (size_t)32 << 20;
constexpr int PB_NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[PB_NOALLOC_SCRATCH_BYTES];

std::mutex g_noalloc_mu;
unsigned char *g_noalloc_addr[PB_NOALLOC_MAX_DEVICES];
thread_local cudaStream_t g_noalloc_stream[PB_NOALLOC_MAX_DEVICES];
thread_local char g_noalloc_err[256] = "";

constexpr size_t round256(size_t x) { return (x + 255) & ~(size_t)255; }

/* exclusive scan of the strip-buffer sizes (ints) in one CTA; soff[n] is
 * the total */
constexpr int SCAN_THREADS = 1024;

__global__ void __launch_bounds__(SCAN_THREADS)
k_noalloc_offsets(const int *__restrict__ tlen, int n, int nv, int64_t *__restrict__ soff)
{
    typedef cub::BlockScan<int64_t, SCAN_THREADS> Scan;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ int64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += SCAN_THREADS) {
        const int i = base + threadIdx.x;
        const int64_t v = i < n ? (int64_t)max(tlen[i], 0) * nv : 0;
        int64_t ex, total;
        Scan(tmp).ExclusiveSum(v, ex, total);
        if (i < n) soff[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) soff[n] = carry;
}

/* the array's device address on the current device; the first call on a
 * device looks it up (cudaGetSymbolAddress) */
unsigned char *scratch_base(int dev)
{
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void *ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) {
            snprintf(g_noalloc_err, sizeof g_noalloc_err, "cudaGetSymbolAddress of the static scratch failed: %s",
                     cudaGetErrorString(e));
            return nullptr;
        }
        g_noalloc_addr[dev] = (unsigned char *)ptr;
    }
    return g_noalloc_addr[dev];
}

}  // namespace

extern "C" {

size_t pb_cuda_noalloc_capacity(void) { return PB_NOALLOC_SCRATCH_BYTES; }

int pb_cuda_noalloc_max_pairs(void)
{
    /* descriptor + outputs + offsets must leave room for at least one strip */
    return (int)((PB_NOALLOC_SCRATCH_BYTES / 2) / (sizeof(pb_pair_out) + sizeof(int64_t)));
}

const char *pb_cuda_noalloc_last_error(void) { return g_noalloc_err; }

int pb_cuda_noalloc_run(const pb_job *job, const pb_batch *b, pb_record *d_rec)
{
    g_noalloc_err[0] = 0;
    if (pb_cuda_init() != 0) {
        snprintf(g_noalloc_err, sizeof g_noalloc_err, "%s", pb_cuda_last_error());
        return -1;
    }
    const int n = b->npairs;
    if (n <= 0) return 0;
    if (b->nprofs != 1 || !b->profs || !b->profs[0]) {
        snprintf(g_noalloc_err, sizeof g_noalloc_err, "exactly one profile is required");
        return -1;
    }
    if (n > pb_cuda_noalloc_max_pairs()) {
        snprintf(g_noalloc_err, sizeof g_noalloc_err, "%d pairs exceed the static scratch's limit of %d pairs", n,
                 pb_cuda_noalloc_max_pairs());
        return -1;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= PB_NOALLOC_MAX_DEVICES) {
        snprintf(g_noalloc_err, sizeof g_noalloc_err, "no usable current device");
        return -1;
    }
    const pb_device_profile *prof = b->profs[0];
    if (prof->device != dev) {
        snprintf(g_noalloc_err, sizeof g_noalloc_err, "the profile lives on device %d, the current device is %d",
                 prof->device, dev);
        return -1;
    }
    unsigned char *base = scratch_base(dev);
    if (!base) return -1;
    if (!g_noalloc_stream[dev] && cudaStreamCreateWithFlags(&g_noalloc_stream[dev], cudaStreamNonBlocking) != cudaSuccess) {
        snprintf(g_noalloc_err, sizeof g_noalloc_err, "stream creation failed");
        return -1;
    }
    cudaStream_t st = g_noalloc_stream[dev];

    const int nv = b->stats ? 8 : 2;
    const size_t off_out = round256(sizeof(pb::ProfDesc));
    const size_t off_soff = off_out + round256(sizeof(pb_pair_out) * (size_t)n);
    const size_t off_strip = off_soff + round256(sizeof(int64_t) * ((size_t)n + 1));
    pb::ProfDesc *d_desc = (pb::ProfDesc *)base;
    pb_pair_out *d_out = (pb_pair_out *)(base + off_out);
    int64_t *d_soff = (int64_t *)(base + off_soff);
    int *d_strip = (int *)(base + off_strip);

    pb::ProfDesc h;
    h.prof = prof->d_prof32; h.prof8 = prof->d_prof8; h.qcodes = prof->d_qcodes;
    h.qlen = prof->qlen; h.lp = prof->lp; h.size = prof->size; h.pad_ = 0;
    int64_t total = 0;
    if (cudaMemcpyAsync(d_desc, &h, sizeof h, cudaMemcpyHostToDevice, st) != cudaSuccess) goto fail;
    k_noalloc_offsets<<<1, SCAN_THREADS, 0, st>>>(b->d_tlen, n, nv, d_soff);
    pb_diag_count_launch(1);
    if (cudaMemcpyAsync(&total, d_soff + n, sizeof total, cudaMemcpyDeviceToHost, st) != cudaSuccess) goto fail;
    if (cudaStreamSynchronize(st) != cudaSuccess) goto fail;
    if (off_strip + sizeof(int) * (size_t)total > PB_NOALLOC_SCRATCH_BYTES) {
        snprintf(g_noalloc_err, sizeof g_noalloc_err,
                 "the batch needs %zu bytes of scratch (%d pairs, %lld target residues x %d ints); "
                 "the static scratch holds %zu",
                 off_strip + sizeof(int) * (size_t)total, n, (long long)(total / nv), nv, PB_NOALLOC_SCRATCH_BYTES);
        return -1;
    }
    {
        pb::ExactParams p;
        p.alg = b->alg; p.sgflags = b->sgflags; p.open = b->open; p.gap = b->gap;
        p.pad_rows = b->pad_rows; p.npairs = n;
        p.profs = d_desc; p.prof_index = nullptr;
        p.targets = b->d_targets; p.toff = b->d_toff; p.tlen = b->d_tlen;
        p.qlim = nullptr; p.tlim = nullptr;
        p.scratch = d_strip; p.soff = d_soff; p.out = d_out;
        p.mat = nullptr; p.msize = 0; p.qall = nullptr; p.qoff = nullptr; p.qlen = nullptr;
        pb::launch_exact(p, b->alg, b->stats != 0, st);
        pb_diag_count_launch(1);
        if (cudaGetLastError() != cudaSuccess) goto fail;
        /* the resolution's work area (lane-exact rounds) reuses the strip
         * region: the exact kernel is done with it, in stream order */
        const pb_lane_args la = pb::lane_args_of(b, 0, d_out);
        const int rr = pb::resolve_rounds(*job, la, d_out, nullptr, nullptr, prof->qlen, b->d_tlen, n, d_rec, st,
                                          base + off_strip, PB_NOALLOC_SCRATCH_BYTES - off_strip);
        if (rr == -2) {
            snprintf(g_noalloc_err, sizeof g_noalloc_err,
                     "%d pairs need more resolution work space than the static scratch has left", n);
            return -1;
        }
        if (rr == -3) {
            size_t need = 0;
            for (int w = 8; w <= 32; w *= 2) {
                const size_t x = pb_cuda_lane_scratch_per_warp(w, pb_lane_kind(&job->mode), prof->qlen);
                need = x > need ? x : need;
            }
            snprintf(g_noalloc_err, sizeof g_noalloc_err,
                     "the lane-exact kernel needs up to %zu bytes per warp for this query (%d rows), more than the "
                     "%zu bytes of static scratch left after the batch's other regions",
                     need, prof->qlen, (size_t)PB_NOALLOC_SCRATCH_BYTES - off_strip);
            return -1;
        }
        if (rr != 0) goto fail;
    }
    if (cudaGetLastError() != cudaSuccess) goto fail;
    if (cudaStreamSynchronize(st) != cudaSuccess) goto fail;
    return 0;
fail:
    snprintf(g_noalloc_err, sizeof g_noalloc_err, "CUDA error: %s", cudaGetErrorString(cudaGetLastError()));
    return -1;
}

}  // extern "C"
