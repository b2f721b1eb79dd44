/*
 * pb_lane.cu -- the lane-exact striped kernels (pb_lane.cuh) on the GPU: one
 * warp per pair, AVX2 lane l = warp lane l. The vector shift of the
 * reference's striped loop (_mm256_slli_si256 by one lane) is a warp shuffle,
 * _mm256_movemask_epi8 of a comparison is a warp vote, and each of the
 * kernel's per-segment vector arrays (pvHStore, pvE, ...) is a [segLen][32]
 * int16 array in this warp's slice of a scratch buffer, so every thread only
 * touches its own lane's elements.
 *
 * Runs only on the pairs whose narrow-width result the exact values cannot
 * settle (pb_resolve.h), so it is built for exactness, not speed.
 */
#include <cstdio>
#include <cstdint>
#include <climits>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>

#include "pb_cuda.h"
#include "pb_lane.cuh"
#include "pb_resolve.h"

namespace pb {
namespace lane {

/* storage of one lane value: 16 bits hold the 8- and 16-bit kernels' lanes */
template <int W> struct LaneElem { typedef int16_t T; };
template <> struct LaneElem<32> { typedef int32_t T; };

template <int W> struct WarpVec {
    static constexpr int L = Lim<W>::LANES;
    typedef int V;
    typedef typename LaneElem<W>::T E;
    struct Arr { E *p; };
    int lane;
    E *scratch;

    __device__ __forceinline__ Arr arr(int a, int segLen) { return Arr{scratch + (size_t)a * segLen * 32}; }
    __device__ __forceinline__ V load(Arr a, int i) { return a.p[i * 32 + lane]; }
    __device__ __forceinline__ void store(Arr a, int i, V x) { a.p[i * 32 + lane] = (E)x; }
    __device__ __forceinline__ V set1(int x) { return x; }
    template <int W2> __device__ __forceinline__ V adds(V a, V b) { return lane_arith<W2>((long long)a + b); }
    template <int W2> __device__ __forceinline__ V subs(V a, V b) { return lane_arith<W2>((long long)a - b); }
    __device__ __forceinline__ V max(V a, V b) { return a > b ? a : b; }
    __device__ __forceinline__ V min(V a, V b) { return a < b ? a : b; }
    __device__ __forceinline__ V cmpgt(V a, V b) { return a > b ? -1 : 0; }
    __device__ __forceinline__ V cmpeq(V a, V b) { return a == b ? -1 : 0; }
    __device__ __forceinline__ V blend(V a, V b, V m) { return m ? b : a; }
    __device__ __forceinline__ V and_(V a, V b) { return a & b; }
    __device__ __forceinline__ V or_(V a, V b) { return a | b; }
    __device__ __forceinline__ V andnot(V a, V b) { return ~a & b; }
    __device__ __forceinline__ V shift1(V a)
    {
        const int y = __shfl_up_sync(0xffffffffu, a, 1);
        return lane == 0 ? 0 : y;
    }
    __device__ __forceinline__ V insert0(V a, int x) { return lane == 0 ? x : a; }
    __device__ __forceinline__ bool any(V m) { return __any_sync(0xffffffffu, lane < L && m != 0) != 0; }
    __device__ __forceinline__ int extract(V a, int l) { return __shfl_sync(0xffffffffu, a, l); }
    __device__ __forceinline__ int hmax(V a)
    {
        int m = lane < L ? a : INT_MIN;
        for (int o = 16; o; o >>= 1) {
            const int y = __shfl_xor_sync(0xffffffffu, m, o);
            m = y > m ? y : m;
        }
        return m;
    }
    __device__ __forceinline__ V lane_eq(int k) { return lane == k ? -1 : 0; }
    template <int W2> __device__ __forceinline__ void init_he(V &h, V &e, int i, int segLen, int s1_beg, int open, int gap)
    {
        long long tmp = s1_beg ? 0 : (-(long long)open - (long long)gap * (lane * segLen + i));
        h = tmp < Lim<W2>::MIN ? Lim<W2>::MIN : (int)tmp;
        tmp = tmp - open;
        e = tmp < Lim<W2>::MIN ? Lim<W2>::MIN : (int)tmp;
    }
    template <int W2> __device__ __forceinline__ int boundary(const Problem &pr, int j)
    {
        if (j == 0) return 0;
        const long long tmp = pr.s2_beg ? 0 : (-(long long)pr.open - (long long)pr.gap * (j - 1));
        return tmp < Lim<W2>::MIN ? Lim<W2>::MIN : (int)tmp;
    }
    template <int W2> __device__ __forceinline__ V prof(const Problem &pr, int k, int i, int segLen)
    {
        const int row = lane * segLen + i;
        return (lane < L && row < pr.qlen) ? wrap<W2>(prof_value(pr, k, row)) : 0;
    }
    template <int W2> __device__ __forceinline__ V match(const Problem &pr, int k, int i, int segLen)
    {
        const int row = lane * segLen + i;
        return (lane < L && row < pr.qlen) ? (k == pr.qcodes[row] ? 1 : 0) : 0;
    }
    template <int W2> __device__ __forceinline__ V similar(const Problem &pr, int k, int i, int segLen)
    {
        return prof<W2>(pr, k, i, segLen) > 0 ? 1 : 0;
    }
};

struct LaneJob {
    int kind;                                  /* 0 nw/sg, 1 nw/sg stats, 2 sw stats prefix, 3 sw,
                                                  4 nw/sg striped trace, 5 nw/sg scan trace,
                                                  6 nw/sg scan, 7 sw scan, 8 nw/sg scan stats */
    int open, gap, mmax, mmin;
    int s1_beg, s1_end, s2_beg, s2_end;
    /* profile mode */
    const int32_t *prof; const uint8_t *qcodes; int lp; int qlen; int size;
    /* matrix (pairs) mode */
    const int32_t *mat; int msize; const uint8_t *qall; const int64_t *qoff; const int *qlens;
    const uint8_t *targets; const int64_t *toff; const int *tlen;
    const pb_pair_out *o1;                     /* kind 2: prefix = o1 ends */
    const int *list; int nlist;
    pb_lane_res *res;                          /* indexed by pair id */
    void *scratch; int seg_max; int narr;
};

PB_LHD int lane_narr(int kind)
{
    return kind == 0 || (kind >= 4 && kind <= 6) ? 3 : kind == 1 ? 12 : kind == 2 ? 16 : kind == 8 ? 8 : 4;
}

constexpr int LANE_THREADS = 256;

template <int W>
__global__ void __launch_bounds__(LANE_THREADS) k_lane(LaneJob J)
{
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    WarpVec<W> v;
    v.lane = lane;
    v.scratch = reinterpret_cast<typename WarpVec<W>::E *>(J.scratch) + (size_t)warp * J.narr * J.seg_max * 32;
    for (int k = warp; k < J.nlist; k += nwarps) {
        const int pid = J.list[k];
        Problem pr;
        pr.open = J.open; pr.gap = J.gap; pr.mmax = J.mmax; pr.mmin = J.mmin;
        pr.s1_beg = J.s1_beg; pr.s1_end = J.s1_end; pr.s2_beg = J.s2_beg; pr.s2_end = J.s2_end;
        if (J.mat) {
            pr.prof = nullptr; pr.lp = 0; pr.mat = J.mat; pr.msize = J.msize; pr.size = J.msize;
            pr.qcodes = J.qall + J.qoff[pid]; pr.qlen = J.qlens[pid];
        } else {
            pr.prof = J.prof; pr.lp = J.lp; pr.mat = nullptr; pr.msize = 0; pr.size = J.size;
            pr.qcodes = J.qcodes; pr.qlen = J.qlen;
        }
        pr.t = J.targets + J.toff[pid];
        pr.tlen = J.tlen[pid];
        if (J.kind == 2) {
            pr.qlen = J.o1[pid].end_query + 1;
            pr.tlen = J.o1[pid].end_ref + 1;
        }
        Out o;
        if (J.kind == 0) striped_nwsg<WarpVec<W>, W>(v, pr, o);
        else if (J.kind == 1) striped_nwsg_stats<WarpVec<W>, W>(v, pr, o);
        else if (J.kind == 3) striped_sw<WarpVec<W>, W>(v, pr, o);
        else if (J.kind == 4) striped_nwsg<WarpVec<W>, W, true>(v, pr, o);
        else if (J.kind == 5) { if (W != 32) scan_nwsg_trace<WarpVec<W>, W>(v, pr, o); }
        else if (J.kind == 6) scan_nwsg<WarpVec<W>, W>(v, pr, o);
        else if (J.kind == 7) scan_sw<WarpVec<W>, W>(v, pr, o);
        else if (J.kind == 8) scan_stats<WarpVec<W>, W, false>(v, pr, o);
        else if (W != 32) striped_sw_stats_bias<WarpVec<W>, W>(v, pr, o);
        if (lane == 0) {
            pb_lane_res r;
            r.score = o.score; r.end_query = o.end_query; r.end_ref = o.end_ref;
            r.matches = o.matches; r.similar = o.similar; r.length = o.length;
            r.saturated = o.saturated; r.valid = W;
            J.res[pid] = r;
        }
        __syncwarp();
    }
}

/* characters to matrix codes in place */
__global__ void k_lane_map(uint8_t *__restrict__ buf, int64_t n, const uint8_t *__restrict__ map)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        buf[i] = map[buf[i]];
}

}  // namespace lane
}  // namespace pb

extern "C" {

size_t pb_cuda_lane_scratch_per_warp(int bits, int kind, int max_qlen)
{
    const int L = 256 / bits;
    const int seg = (max_qlen + L - 1) / L;
    return (bits == 32 ? 4 : 2) * (size_t)pb::lane::lane_narr(kind) * seg * 32;
}

int pb_cuda_lane_run(int bits, const pb_lane_args *a, const int *d_list, int nlist, pb_lane_res *d_res,
                     void *scratch, size_t scratch_bytes, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    using namespace pb::lane;
    if (nlist <= 0) return 0;
    if ((bits != 8 && bits != 16 && bits != 32) || (bits == 32 && (a->kind == 2 || a->kind == 5))) return -1;
    LaneJob J;
    J.kind = a->kind; J.open = a->open; J.gap = a->gap; J.mmax = a->mmax; J.mmin = a->mmin;
    J.s1_beg = (a->sgflags & PB_S1_BEG) != 0; J.s1_end = (a->sgflags & PB_S1_END) != 0;
    J.s2_beg = (a->sgflags & PB_S2_BEG) != 0; J.s2_end = (a->sgflags & PB_S2_END) != 0;
    J.prof = a->prof; J.qcodes = a->qcodes; J.lp = a->lp; J.qlen = a->qlen; J.size = a->size;
    J.mat = a->mat; J.msize = a->msize; J.qall = a->qall; J.qoff = a->qoff; J.qlens = a->qlens;
    J.targets = a->targets; J.toff = a->toff; J.tlen = a->tlen; J.o1 = a->o1;
    J.list = d_list; J.nlist = nlist; J.res = d_res;
    const int L = 256 / bits;
    J.seg_max = (a->max_qlen + L - 1) / L;
    if (J.seg_max < 1) J.seg_max = 1;
    J.narr = lane_narr(a->kind);
    const size_t per_warp = (bits == 32 ? 4 : 2) * (size_t)J.narr * J.seg_max * 32;
    int nsm = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int wpb = LANE_THREADS / 32;
    /* warps launched: one per listed pair up to 8 per SM; every launched warp
     * owns one per_warp slice of the scratch */
    long long warps = nlist < nsm * 8 ? nlist : (long long)nsm * 8;
    int threads = LANE_THREADS;
    bool own = false;
    if (scratch) {
        const long long fit = (long long)(scratch_bytes / per_warp);
        if (fit < 1) return -3;   /* the given scratch does not hold one warp's arrays */
        if (warps > fit) warps = fit;
    }
    if (warps >= wpb) {
        warps = (warps / wpb) * wpb;
    } else {
        threads = 32;
    }
    if (!scratch) {
        if (cudaMallocAsync(&scratch, per_warp * warps, st) != cudaSuccess) return -1;
        own = true;
    }
    J.scratch = scratch;
    const int blocks = (int)(warps * 32 / threads);
    if (bits == 8) k_lane<8><<<blocks, threads, 0, st>>>(J);
    else if (bits == 16) k_lane<16><<<blocks, threads, 0, st>>>(J);
    else k_lane<32><<<blocks, threads, 0, st>>>(J);
    pb_diag_count_launch(1);
    const cudaError_t e = cudaGetLastError();
    if (own) cudaFreeAsync(scratch, st);
    return e == cudaSuccess ? 0 : -1;
}

int pb_cuda_lane_pair(int bits, const pb_device_profile *dp, const struct pb_mode *m, const uint8_t *h_codes,
                      int tlen, const pb_pair_out *h_o1, pb_lane_res *h_res)
{
    if (pb_cuda_init() != 0) return -1;
    cudaGetLastError();   /* a launch error below is this call's own */
    /* the thread's single-pair arena: [toff int64][tlen, list: int][o1][res][codes] then one warp's scratch */
    const int kind = pb_lane_kind(m);
    const size_t o_toff = 0, o_ints = 8, o_o1 = 16;
    const size_t o_res = (o_o1 + sizeof(pb_pair_out) + 15) & ~(size_t)15;
    const size_t o_codes = (o_res + sizeof(pb_lane_res) + 15) & ~(size_t)15;
    const size_t up = (o_codes + (size_t)tlen + 16 + 255) & ~(size_t)255;
    const size_t per_warp = pb_cuda_lane_scratch_per_warp(bits, kind, dp->qlen);
    char *h = nullptr;
    char *d = pb_single_arena(up + per_warp, up, &h);
    if (!d) { pb_cuda_set_error("single-pair arena", "allocation failed"); return -1; }
    const int ints[2] = {tlen, 0};
    memcpy(h + o_ints, ints, sizeof ints);
    memcpy(h + o_o1, h_o1, sizeof(pb_pair_out));
    memcpy(h + o_codes, h_codes, (size_t)tlen);
    cudaStream_t st = (cudaStream_t)pb_cuda_stream();
    if (cudaMemcpyAsync(d, h, up, cudaMemcpyHostToDevice, st) != cudaSuccess) return -1;
    pb_lane_args a;
    memset(&a, 0, sizeof a);
    a.kind = kind; a.sgflags = m->sgflags; a.open = m->open; a.gap = m->gap;
    a.mmax = dp->mmax; a.mmin = dp->mmin; a.max_qlen = dp->qlen;
    a.prof = dp->d_prof32; a.qcodes = dp->d_qcodes; a.lp = dp->lp; a.qlen = dp->qlen; a.size = dp->size;
    a.targets = reinterpret_cast<const uint8_t *>(d + o_codes);
    a.toff = reinterpret_cast<const int64_t *>(d + o_toff);
    a.tlen = reinterpret_cast<const int *>(d + o_ints);
    a.o1 = reinterpret_cast<const pb_pair_out *>(d + o_o1);
    pb_lane_res *d_res = reinterpret_cast<pb_lane_res *>(d + o_res);
    int rc = pb_cuda_lane_run(bits, &a, reinterpret_cast<const int *>(d + o_ints) + 1, 1, d_res, d + up, per_warp, st);
    if (rc == 0 && cudaMemcpyAsync(h_res, d_res, sizeof(pb_lane_res), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        rc = -1;
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
    if (rc != 0) pb_cuda_set_error("single-pair lane-exact kernel", cudaGetErrorString(cudaGetLastError()));
    return rc;
}

int pb_cuda_trace_sat_host(int bits, int kind, int sgflags, int open, int gap, int mmax, int mmin,
                           const int32_t *h_mat, int msize, const uint8_t *map, const char *q, const int64_t *qoff,
                           const int *qlen, const char *t, const int64_t *toff, const int *tlen, const int *list,
                           int nlist, int *sat)
{
    using namespace pb::lane;
    if (nlist <= 0) return 0;
    if ((bits != 8 && bits != 16) || (kind != 4 && kind != 5) || msize <= 0) return -1;
    if (pb_cuda_init() != 0) return -1;
    /* the listed pairs, packed: queries then targets, in list order */
    std::vector<int64_t> hqo(nlist), hto(nlist);
    std::vector<int> hql(nlist), htl(nlist), hid(nlist);
    int64_t nq = 0, nt = 0;
    int maxq = 1;
    for (int k = 0; k < nlist; ++k) {
        const int p = list[k];
        hqo[k] = nq; hql[k] = qlen[p]; nq += qlen[p];
        hto[k] = nt; htl[k] = tlen[p]; nt += tlen[p];
        hid[k] = k;
        if (qlen[p] > maxq) maxq = qlen[p];
    }
    std::vector<uint8_t> chars((size_t)(nq + nt));
    for (int k = 0; k < nlist; ++k) {
        const int p = list[k];
        memcpy(chars.data() + hqo[k], q + qoff[p], (size_t)qlen[p]);
        memcpy(chars.data() + nq + hto[k], t + toff[p], (size_t)tlen[p]);
    }
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return -1;
    uint8_t *d_chars = nullptr, *d_map = nullptr;
    int32_t *d_mat = nullptr;
    int64_t *d_qo = nullptr, *d_to = nullptr;
    int *d_ql = nullptr, *d_tl = nullptr, *d_list = nullptr;
    pb_lane_res *d_res = nullptr;
    int rc = 0;
    if (cudaMallocAsync((void **)&d_chars, (size_t)(nq + nt) + 16, st) != cudaSuccess ||
        cudaMallocAsync((void **)&d_map, 256, st) != cudaSuccess ||
        cudaMallocAsync((void **)&d_mat, sizeof(int32_t) * (size_t)msize * msize, st) != cudaSuccess ||
        cudaMallocAsync((void **)&d_qo, sizeof(int64_t) * nlist, st) != cudaSuccess ||
        cudaMallocAsync((void **)&d_to, sizeof(int64_t) * nlist, st) != cudaSuccess ||
        cudaMallocAsync((void **)&d_ql, sizeof(int) * nlist, st) != cudaSuccess ||
        cudaMallocAsync((void **)&d_tl, sizeof(int) * nlist, st) != cudaSuccess ||
        cudaMallocAsync((void **)&d_list, sizeof(int) * nlist, st) != cudaSuccess ||
        cudaMallocAsync((void **)&d_res, sizeof(pb_lane_res) * nlist, st) != cudaSuccess)
        rc = -1;
    std::vector<pb_lane_res> hres;
    if (rc == 0) {
        cudaMemcpyAsync(d_chars, chars.data(), (size_t)(nq + nt), cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_map, map, 256, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_mat, h_mat, sizeof(int32_t) * (size_t)msize * msize, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_qo, hqo.data(), sizeof(int64_t) * nlist, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_to, hto.data(), sizeof(int64_t) * nlist, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_ql, hql.data(), sizeof(int) * nlist, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_tl, htl.data(), sizeof(int) * nlist, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_list, hid.data(), sizeof(int) * nlist, cudaMemcpyHostToDevice, st);
        const int64_t n = nq + nt;
        const int blocks = (int)((n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024);
        k_lane_map<<<blocks, 256, 0, st>>>(d_chars, n, d_map);
        pb_diag_count_launch(1);
        pb_lane_args a;
        memset(&a, 0, sizeof a);
        a.kind = kind; a.sgflags = sgflags; a.open = open; a.gap = gap; a.mmax = mmax; a.mmin = mmin;
        a.max_qlen = maxq;
        a.mat = d_mat; a.msize = msize; a.qall = d_chars; a.qoff = d_qo; a.qlens = d_ql;
        a.targets = d_chars + nq; a.toff = d_to; a.tlen = d_tl;
        rc = pb_cuda_lane_run(bits, &a, d_list, nlist, d_res, nullptr, 0, st);
        if (rc == 0) {
            hres.resize(nlist);
            cudaMemcpyAsync(hres.data(), d_res, sizeof(pb_lane_res) * nlist, cudaMemcpyDeviceToHost, st);
        }
    }
    cudaFreeAsync(d_chars, st); cudaFreeAsync(d_map, st); cudaFreeAsync(d_mat, st);
    cudaFreeAsync(d_qo, st); cudaFreeAsync(d_to, st); cudaFreeAsync(d_ql, st); cudaFreeAsync(d_tl, st);
    cudaFreeAsync(d_list, st); cudaFreeAsync(d_res, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
    cudaStreamDestroy(st);
    for (int k = 0; rc == 0 && k < nlist; ++k) {
        if (hres[k].valid != bits) { rc = -1; break; }
        sat[k] = hres[k].saturated;
    }
    return rc;
}

}  // extern "C"
