/*
 * pb_filter.cu -- candidate pairs of the aligner's exact-match filter on the
 * GPU.
 *
 * The reference aligner (apps/parasail_aligner.cpp:1316-1420, :1816-1904)
 * builds an enhanced suffix array of the '$'-separated text and walks its
 * lcp-interval tree: every pair of sequences with a left-maximal common
 * substring of at least `cutoff` characters (not crossing a sentinel) is a
 * candidate, kept in a std::set. That set is exactly the pairs of sequences
 * sharing a substring of `cutoff` characters: a shared substring extends
 * left to a left-maximal one of at least the same length, and the interval
 * of its two suffixes pairs them. So the filter needs no suffix tree:
 *
 *   1. every start position whose next `cutoff` characters hold no sentinel
 *      (its sequence id from a prefix count of sentinels);
 *   2. the positions sorted by those characters: stable LSD radix sorts
 *      over 8-byte big-endian chunks, last chunk first (exact, no hashing);
 *   3. groups of equal prefixes (adjacent compare), then the distinct
 *      sequence ids of each group (sort of group << 32 | id, unique);
 *   4. every pair of distinct ids of a group -- (smaller, larger), or with a
 *      query file (query, database) across the crossover -- emitted by one
 *      thread per pair (a binary search over the groups' pair counts and a
 *      closed-form row decode), in chunks of a fixed device budget;
 *   5. sort + unique of the 64-bit pair keys: the set in its ascending
 *      order.
 * All of it is integer/byte work bound by HBM and the radix sorts.
 */
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <vector>

#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>

#include "pb_cuda.h"

namespace {

#define FL_CK(call)                                              \
    do {                                                         \
        if ((call) != cudaSuccess) {                             \
            fprintf(stderr, "pb_filter: %s failed\n", #call);    \
            rc = -1;                                             \
            goto done;                                           \
        }                                                        \
    } while (0)

__global__ void k_sep_flags(const uint8_t *__restrict__ T, int n, uint8_t sep, int *__restrict__ f)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) f[i] = T[i] == sep;
}

/* incl[i] = sentinels in [0, i]: position p starts a window of c residues
 * when p + c <= n and no sentinel lies in [p, p + c) */
__global__ void k_windows(const int *__restrict__ incl, const uint8_t *__restrict__ T, uint8_t sep, int n, int c,
                          int *__restrict__ pos, int *__restrict__ count)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int before = incl[p] - (T[p] == sep);
    if (p + c > n || incl[p + c - 1] != before) return;
    pos[atomicAdd(count, 1)] = p;
}

/* the sequence id of each window: the sentinels before its first residue
 * (incl[p], the residue itself being none) */
__global__ void k_window_sid(const int *__restrict__ incl, const int *__restrict__ pos, int m, int *__restrict__ sid)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) sid[i] = incl[pos[i]];
}

/* big-endian 8-byte chunk k of the window at pos[i] (bytes past the window
 * are 0; every window has the same length) */
__global__ void k_chunk_keys(const uint8_t *__restrict__ T, const int *__restrict__ pos, int m, int c, int k,
                             unsigned long long *__restrict__ key)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    const int b0 = 8 * k, nb = min(8, c - b0);
    const uint8_t *s = T + pos[i] + b0;
    unsigned long long v = 0;
    for (int b = 0; b < 8; ++b) v = (v << 8) | (b < nb ? (unsigned long long)s[b] : 0ull);
    key[i] = v;
}

/* 1 where the window differs from its predecessor in sorted order */
__global__ void k_group_heads(const uint8_t *__restrict__ T, const int *__restrict__ pos, int m, int c,
                              int *__restrict__ head)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    int h = i == 0;
    if (!h) {
        const uint8_t *a = T + pos[i - 1], *b = T + pos[i];
        for (int x = 0; x < c; ++x)
            if (a[x] != b[x]) { h = 1; break; }
    }
    head[i] = h;
}

__global__ void k_group_sid_keys(const int *__restrict__ gincl, const int *__restrict__ sid_sorted, int m,
                                 unsigned long long *__restrict__ key)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m) key[i] = ((unsigned long long)(unsigned)(gincl[i] - 1) << 32) | (unsigned)sid_sorted[i];
}

__global__ void k_seg_heads(const unsigned long long *__restrict__ u, int nu, int *__restrict__ head)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nu) head[i] = i == 0 || (u[i] >> 32) != (u[i - 1] >> 32);
}

__global__ void k_iota(int *__restrict__ v, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

/* pairs of each segment [start[s], start[s+1]) of distinct sorted ids;
 * with a crossover, only database x query (ids < cross are database) */
__global__ void k_seg_pairs(const unsigned long long *__restrict__ u, const int *__restrict__ start, int nseg,
                            int nu, int cross, long long *__restrict__ npairs, int *__restrict__ ndb)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    const int b = start[s], e = s + 1 < nseg ? start[s + 1] : nu;
    const long long m = e - b;
    if (cross < 0) {
        npairs[s] = m * (m - 1) / 2;
        ndb[s] = 0;
    } else {
        int lo = b, hi = e;                  /* first id >= cross */
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if ((int)(unsigned)u[mid] < cross) lo = mid + 1;
            else hi = mid;
        }
        const long long d = lo - b;
        npairs[s] = d * (m - d);
        ndb[s] = (int)d;
    }
}

/* pair e0 + t of the concatenated segment pair lists: its segment by binary
 * search over the exclusive prefix `off`, then the pair inside it */
__global__ void k_emit(const unsigned long long *__restrict__ u, const int *__restrict__ start, int nseg, int nu,
                       const long long *__restrict__ off, const int *__restrict__ ndb, int cross, long long e0,
                       long long ne, unsigned long long *__restrict__ out)
{
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= ne) return;
    const long long e = e0 + t;
    int lo = 0, hi = nseg - 1;                /* last segment with off <= e */
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (off[mid] <= e) lo = mid;
        else hi = mid - 1;
    }
    const int s = lo;
    const int b = start[s], en = s + 1 < nseg ? start[s + 1] : nu;
    const long long m = en - b, r = e - off[s];
    unsigned first, second;
    if (cross < 0) {
        /* row x holds pairs (x, x+1 .. m-1): rows before x hold x(2m-1-x)/2 */
        const double mm = 2.0 * (double)m - 1.0;
        long long x = (long long)floor((mm - sqrt(mm * mm - 8.0 * (double)r)) / 2.0);
        if (x > m - 2) x = m - 2;
        if (x < 0) x = 0;
        while (x > 0 && x * (2 * m - 1 - x) / 2 > r) --x;
        while ((x + 1) * (2 * m - 2 - x) / 2 <= r) ++x;
        const long long y = x + 1 + (r - x * (2 * m - 1 - x) / 2);
        first = (unsigned)u[b + x];
        second = (unsigned)u[b + y];
    } else {
        const long long d = ndb[s];
        first = (unsigned)u[b + d + r / d];   /* query */
        second = (unsigned)u[b + r % d];      /* database */
    }
    out[t] = ((unsigned long long)first << 32) | second;
}

template <typename K, typename V>
int radix_pairs(const K *kin, K *kout, const V *vin, V *vout, int n, int end_bit, cudaStream_t st)
{
    size_t bytes = 0;
    void *tmp = nullptr;
    if (cub::DeviceRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, n, 0, end_bit, st) != cudaSuccess)
        return -1;
    if (cudaMallocAsync(&tmp, bytes, st) != cudaSuccess) return -1;
    const cudaError_t e = cub::DeviceRadixSort::SortPairs(tmp, bytes, kin, kout, vin, vout, n, 0, end_bit, st);
    cudaFreeAsync(tmp, st);
    return e == cudaSuccess ? 0 : -1;
}

/* sort + unique of n keys in place (scratch of n keys); returns the count */
long long sort_unique(unsigned long long *keys, unsigned long long *scratch, long long n, int *d_num,
                      cudaStream_t st)
{
    if (n <= 0) return 0;
    size_t bytes = 0;
    void *tmp = nullptr;
    long long out = -1;
    int h = 0;
    if (cub::DeviceRadixSort::SortKeys(nullptr, bytes, keys, scratch, (int)n, 0, 64, st) != cudaSuccess) return -1;
    size_t b2 = 0;
    if (cub::DeviceSelect::Unique(nullptr, b2, scratch, keys, d_num, (int)n, st) != cudaSuccess) return -1;
    if (b2 > bytes) bytes = b2;
    if (cudaMallocAsync(&tmp, bytes, st) != cudaSuccess) return -1;
    size_t b = bytes;
    if (cub::DeviceRadixSort::SortKeys(tmp, b, keys, scratch, (int)n, 0, 64, st) == cudaSuccess) {
        b = bytes;
        if (cub::DeviceSelect::Unique(tmp, b, scratch, keys, d_num, (int)n, st) == cudaSuccess &&
            cudaMemcpyAsync(&h, d_num, sizeof(int), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
            cudaStreamSynchronize(st) == cudaSuccess)
            out = h;
    }
    cudaFreeAsync(tmp, st);
    return out;
}

inline int nblk(long long n) { return (int)((n + 255) / 256); }

}  // namespace

/*
 * Candidate pairs of `text` (n bytes, every sequence followed by `sep`):
 * the pairs of sequences sharing a substring of `cutoff` characters, as
 * 64-bit keys first << 32 | second in ascending order (malloc'd, *count of
 * them). cross < 0: all against all, first < second; otherwise ids below
 * cross are database sequences and only (query, database) pairs are kept.
 * `budget` bounds the pair keys held on the device at once. Returns 0, or
 * -1 on a CUDA error.
 */
extern "C" int pb_cuda_candidate_pairs(const uint8_t *h_text, long long n_in, uint8_t sep, int cutoff, int cross,
                                       long long budget, unsigned long long **h_pairs, long long *count)
{
    *h_pairs = nullptr;
    *count = 0;
    if (pb_cuda_init() != 0) return -1;
    if (n_in <= 0 || cutoff < 1) return 0;
    if (n_in > 0x7fffffffLL) return -1;
    const int n = (int)n_in;
    int rc = 0, m = 0, nu = 0, nseg = 0;
    cudaStream_t st = nullptr;
    uint8_t *T = nullptr;
    int *flags = nullptr, *incl = nullptr, *pos = nullptr, *pos2 = nullptr, *sid = nullptr;
    int *head = nullptr, *cnt = nullptr, *seg = nullptr, *ndb = nullptr, *idx = nullptr;
    unsigned long long *key = nullptr, *key2 = nullptr, *acc = nullptr, *accs = nullptr;
    long long *np = nullptr, *off = nullptr;
    long long nacc = 0, acc_cap = 0, total = 0;
    FL_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    FL_CK(cudaMallocAsync((void **)&T, (size_t)n, st));
    FL_CK(cudaMallocAsync((void **)&flags, sizeof(int) * (size_t)n, st));
    FL_CK(cudaMallocAsync((void **)&incl, sizeof(int) * (size_t)n, st));
    FL_CK(cudaMallocAsync((void **)&cnt, sizeof(int) * 2, st));
    FL_CK(cudaMemcpyAsync(T, h_text, (size_t)n, cudaMemcpyHostToDevice, st));
    FL_CK(cudaMemsetAsync(cnt, 0, sizeof(int) * 2, st));
    k_sep_flags<<<nblk(n), 256, 0, st>>>(T, n, sep, flags);
    pb_diag_count_launch(1);
    {
        size_t bytes = 0;
        void *tmp = nullptr;
        FL_CK(cub::DeviceScan::InclusiveSum(nullptr, bytes, flags, incl, n, st));
        FL_CK(cudaMallocAsync(&tmp, bytes, st));
        FL_CK(cub::DeviceScan::InclusiveSum(tmp, bytes, flags, incl, n, st));
        cudaFreeAsync(tmp, st);
    }
    FL_CK(cudaMallocAsync((void **)&pos, sizeof(int) * (size_t)n, st));
    k_windows<<<nblk(n), 256, 0, st>>>(incl, T, sep, n, cutoff, pos, cnt);
    pb_diag_count_launch(1);
    FL_CK(cudaMemcpyAsync(&m, cnt, sizeof(int), cudaMemcpyDeviceToHost, st));
    FL_CK(cudaStreamSynchronize(st));
    cudaFreeAsync(flags, st);
    flags = nullptr;
    if (m < 2) goto done;
    /* window order: stable LSD radix sorts over 8-byte chunks, last first,
     * positions carried along (each chunk's used bytes are its high ones) */
    FL_CK(cudaMallocAsync((void **)&key, sizeof(unsigned long long) * (size_t)m, st));
    FL_CK(cudaMallocAsync((void **)&key2, sizeof(unsigned long long) * (size_t)m, st));
    FL_CK(cudaMallocAsync((void **)&pos2, sizeof(int) * (size_t)m, st));
    FL_CK(cudaMallocAsync((void **)&idx, sizeof(int) * (size_t)m, st));
    FL_CK(cudaMallocAsync((void **)&sid, sizeof(int) * (size_t)m, st));
    for (int k = (cutoff - 1) / 8; k >= 0; --k) {
        const int nb = cutoff - 8 * k < 8 ? cutoff - 8 * k : 8;
        k_chunk_keys<<<nblk(m), 256, 0, st>>>(T, pos, m, cutoff, k, key);
        pb_diag_count_launch(1);
        size_t bytes = 0;
        void *tmp = nullptr;
        FL_CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, key, key2, pos, pos2, m, 64 - 8 * nb, 64, st));
        FL_CK(cudaMallocAsync(&tmp, bytes, st));
        FL_CK(cub::DeviceRadixSort::SortPairs(tmp, bytes, key, key2, pos, pos2, m, 64 - 8 * nb, 64, st));
        cudaFreeAsync(tmp, st);
        int *t = pos;
        pos = pos2;
        pos2 = t;
    }
    k_window_sid<<<nblk(m), 256, 0, st>>>(incl, pos, m, sid);
    pb_diag_count_launch(1);
    /* groups of equal windows: head flags, group index = inclusive count */
    FL_CK(cudaMallocAsync((void **)&head, sizeof(int) * (size_t)m, st));
    k_group_heads<<<nblk(m), 256, 0, st>>>(T, pos, m, cutoff, head);
    pb_diag_count_launch(1);
    {
        size_t bytes = 0;
        void *tmp = nullptr;
        FL_CK(cub::DeviceScan::InclusiveSum(nullptr, bytes, head, pos2, m, st));
        FL_CK(cudaMallocAsync(&tmp, bytes, st));
        FL_CK(cub::DeviceScan::InclusiveSum(tmp, bytes, head, pos2, m, st));
        cudaFreeAsync(tmp, st);
    }
    k_group_sid_keys<<<nblk(m), 256, 0, st>>>(pos2, sid, m, key);
    pb_diag_count_launch(1);
    {
        size_t bytes = 0, b2 = 0;
        void *tmp = nullptr;
        FL_CK(cub::DeviceRadixSort::SortKeys(nullptr, bytes, key, key2, m, 0, 64, st));
        FL_CK(cub::DeviceSelect::Unique(nullptr, b2, key2, key, cnt + 1, m, st));
        if (b2 > bytes) bytes = b2;
        FL_CK(cudaMallocAsync(&tmp, bytes, st));
        size_t b = bytes;
        FL_CK(cub::DeviceRadixSort::SortKeys(tmp, b, key, key2, m, 0, 64, st));
        b = bytes;
        FL_CK(cub::DeviceSelect::Unique(tmp, b, key2, key, cnt + 1, m, st));
        cudaFreeAsync(tmp, st);
        FL_CK(cudaMemcpyAsync(&nu, cnt + 1, sizeof(int), cudaMemcpyDeviceToHost, st));
        FL_CK(cudaStreamSynchronize(st));
    }
    /* segments of equal group among the unique (group, id) keys */
    k_seg_heads<<<nblk(nu), 256, 0, st>>>(key, nu, head);
    pb_diag_count_launch(1);
    FL_CK(cudaMallocAsync((void **)&seg, sizeof(int) * (size_t)nu, st));
    k_iota<<<nblk(nu), 256, 0, st>>>(idx, nu);
    pb_diag_count_launch(1);
    {
        size_t bytes = 0;
        void *tmp = nullptr;
        FL_CK(cub::DeviceSelect::Flagged(nullptr, bytes, idx, head, seg, cnt, nu, st));
        FL_CK(cudaMallocAsync(&tmp, bytes, st));
        FL_CK(cub::DeviceSelect::Flagged(tmp, bytes, idx, head, seg, cnt, nu, st));
        cudaFreeAsync(tmp, st);
        FL_CK(cudaMemcpyAsync(&nseg, cnt, sizeof(int), cudaMemcpyDeviceToHost, st));
        FL_CK(cudaStreamSynchronize(st));
    }
    FL_CK(cudaMallocAsync((void **)&np, sizeof(long long) * (size_t)nseg, st));
    FL_CK(cudaMallocAsync((void **)&off, sizeof(long long) * (size_t)nseg, st));
    FL_CK(cudaMallocAsync((void **)&ndb, sizeof(int) * (size_t)nseg, st));
    k_seg_pairs<<<nblk(nseg), 256, 0, st>>>(key, seg, nseg, nu, cross, np, ndb);
    pb_diag_count_launch(1);
    {
        size_t bytes = 0;
        void *tmp = nullptr;
        FL_CK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, np, off, nseg, st));
        FL_CK(cudaMallocAsync(&tmp, bytes, st));
        FL_CK(cub::DeviceScan::ExclusiveSum(tmp, bytes, np, off, nseg, st));
        cudaFreeAsync(tmp, st);
    }
    {
        long long last_off = 0, last_np = 0;
        FL_CK(cudaMemcpyAsync(&last_off, off + nseg - 1, sizeof(long long), cudaMemcpyDeviceToHost, st));
        FL_CK(cudaMemcpyAsync(&last_np, np + nseg - 1, sizeof(long long), cudaMemcpyDeviceToHost, st));
        FL_CK(cudaStreamSynchronize(st));
        total = last_off + last_np;
    }
    if (total == 0) goto done;
    /* emit in chunks of at most `budget` keys, merging unique keys */
    if (budget < 1024) budget = 1024;
    for (long long e0 = 0; e0 < total; e0 += budget) {
        const long long ne = total - e0 < budget ? total - e0 : budget;
        if (nacc + ne > acc_cap) {
            const long long cap = (nacc + ne) * 2;
            unsigned long long *a = nullptr, *s = nullptr;
            FL_CK(cudaMallocAsync((void **)&a, sizeof(unsigned long long) * (size_t)cap, st));
            FL_CK(cudaMallocAsync((void **)&s, sizeof(unsigned long long) * (size_t)cap, st));
            if (nacc) FL_CK(cudaMemcpyAsync(a, acc, sizeof(unsigned long long) * (size_t)nacc,
                                            cudaMemcpyDeviceToDevice, st));
            if (acc) cudaFreeAsync(acc, st);
            if (accs) cudaFreeAsync(accs, st);
            acc = a;
            accs = s;
            acc_cap = cap;
        }
        k_emit<<<nblk(ne), 256, 0, st>>>(key, seg, nseg, nu, off, ndb, cross, e0, ne, acc + nacc);
        pb_diag_count_launch(1);
        if (nacc + ne > 0x7fffffffLL) { rc = -1; goto done; }
        const long long u = sort_unique(acc, accs, nacc + ne, cnt, st);
        if (u < 0) { rc = -1; goto done; }
        nacc = u;
    }
    *h_pairs = (unsigned long long *)malloc(sizeof(unsigned long long) * (size_t)(nacc ? nacc : 1));
    if (!*h_pairs) { rc = -1; goto done; }
    FL_CK(cudaMemcpyAsync(*h_pairs, acc, sizeof(unsigned long long) * (size_t)nacc, cudaMemcpyDeviceToHost, st));
    FL_CK(cudaStreamSynchronize(st));
    *count = nacc;
done:
    if (rc != 0 && *h_pairs) { free(*h_pairs); *h_pairs = nullptr; *count = 0; }
    void *bufs[] = {T, flags, incl, pos, pos2, sid, head, cnt, seg, ndb, idx, key, key2, acc, accs, np, off};
    for (void *b : bufs)
        if (b) cudaFreeAsync(b, st);
    if (st) {
        if (cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
        cudaStreamDestroy(st);
    }
    return rc;
}
