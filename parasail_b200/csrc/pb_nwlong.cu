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
#include <cooperative_groups.h>
#include <cuda/atomic>
#include <cstdio>
#include <type_traits>

#include "pb_cuda.h"
#include "pb_cert.cuh"

namespace pb {

static constexpr int NWL_RL = 8;          /* query rows per lane */
static constexpr int NWL_WARPS = 8;       /* warps per CTA */
/* team classes: class c runs each pair on a cluster of c + 1 CTAs (class 0:
 * one CTA); one launch per class */
static constexpr int NWL_CLASSES = 8;
static constexpr int NWL_NEG = INT32_MIN / 4;

/* How large a team a pair gets (k_team_class). `share`: a pair gets the
 * smallest team whose warps hold its share of the work (its cells over the
 * launch's cells per warp, divided by share); `max_class` caps it; `jump`:
 * every pair above one CTA's share gets the largest team instead. */
struct TeamPolicy { int max_class; float share; int jump; };

struct NwWaveParams {
    int npairs, open, gap, msize, small_alpha;
    const int8_t *mat;            /* [msize][msize], row = target letter (vector orientation) */
    const uint8_t *q; const int64_t *qoff; const int *qlen;
    const uint8_t *t; const int64_t *toff; const int *tlen;
    const int *lo; const int *hi; /* per pair band (diagonal i - j), or nullptr */
    int cert;                     /* banded: certify each pair, widen and rerun on failure */
    CostModel cm;
    int *lo_out, *hi_out;         /* cert: the band of pairs that ran twice */
    int *rounds;                  /* cert: 2 for pairs that ran twice */
    const int *order;             /* pairs, cooperative ones first, then most cells first */
    const unsigned long long *keys; /* sorted keys; bit 62 set: run by a whole cluster */
    int2 *scratch;                /* per warp slot: a ring buffer of [maxlen] (H, F) */
    long long *prog;              /* per warp slot: publication progress of its ring */
    int maxlen;
    int *score;                   /* per pair */
};

static constexpr unsigned long long NWL_COOP_BIT = 1ull << 62;

__device__ __forceinline__ int sext_byte(uint32_t lo, uint32_t hi, int k)
{
    /* byte k of {hi:lo}, sign-extended to 32 bits */
    const uint32_t sel = (uint32_t)k | (((uint32_t)k | 8u) << 4) | (((uint32_t)k | 8u) << 8) | (((uint32_t)k | 8u) << 12);
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(lo), "r"(hi), "r"(sel));
    return (int)d;
}

/*
 * A team of warps per pair: the NWL_WARPS warps of one CTA, or, for pairs
 * flagged cooperative, the warps of all CTAs of a thread-block cluster
 * (which the hardware schedules together). Pass p (rows p*256 .. p*256+255)
 * runs on team warp p % T; its lane 0 reads pass p-1's bottom row from that
 * warp slot's ring buffer, which pass p-1's lane 31 fills column by column
 * and publishes every 32 columns through the slot's progress counter
 * (device-scope release / acquire, so it works across the cluster's CTAs).
 * Waits are bounded: a wait that exceeds NWL_SPIN_CYCLES, or sees the
 * launch's error flag set, gives up; the host reports the failure.
 */
static constexpr long long NWL_SPIN_CYCLES = 1ll << 32;

/* BIAS (with GE): the H registers, the pass ring and the lane hand-off hold
 * H - open, and the score table s + open (the host checked that it stays in
 * int8); E = max(E - gap, HO), A = max(HO_diag + s', E), F = max(F - gap,
 * A - open), HO = max(A - open, F - open) */
template <bool BANDED, bool GE, bool BIAS>
__global__ void __launch_bounds__(NWL_WARPS * 32, 3)
k_nw_wave(NwWaveParams p, int *counter, int *error)
{
    namespace cg = cooperative_groups;
    __shared__ __align__(16) int8_t s_mat[32 * 32];
    __shared__ int s_pair;
    for (int k = threadIdx.x; k < p.msize * p.msize; k += blockDim.x) {
        const int r = k / p.msize, c = k % p.msize;
        s_mat[r * 32 + c] = p.mat[k];
    }
    cg::cluster_group cluster = cg::this_cluster();
    const int C = (int)cluster.num_blocks();
    const int crank = (int)cluster.block_rank();
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int open = p.open, gap = p.gap;
    volatile int *verr = error;
    bool coop = C > 1;

    for (;;) {
        int w;
        if (coop) {
            cluster.sync();
            if (crank == 0 && threadIdx.x == 0) s_pair = atomicAdd(counter, 1);
            cluster.sync();
            w = *cluster.map_shared_rank(&s_pair, 0);
            /* every CTA has read rank 0's pair before it is overwritten */
            cluster.sync();
            if (w < p.npairs && !(p.keys[w] & NWL_COOP_BIT)) {
                /* the cooperative pairs are done: from here on each CTA
                 * takes pairs of its own (rank 0 keeps this one) */
                coop = false;
                if (crank != 0) {
                    if (threadIdx.x == 0) s_pair = atomicAdd(counter, 1);
                    __syncthreads();
                    w = s_pair;
                }
            }
        } else {
            __syncthreads();
            if (threadIdx.x == 0) s_pair = atomicAdd(counter, 1);
            __syncthreads();
            w = s_pair;
        }
        if (w >= p.npairs) break;
        const int T = coop ? C * NWL_WARPS : NWL_WARPS;           /* warps of the team */
        const int tw = coop ? crank * NWL_WARPS + warp : warp;    /* this warp in the team */
        const long long slot0 = coop ? (long long)(blockIdx.x / C) * C * NWL_WARPS
                                     : (long long)blockIdx.x * NWL_WARPS;
        const int pid = p.order[w];
        const int n = p.qlen[pid], m = p.tlen[pid];
        const uint8_t *qs = p.q + p.qoff[pid];
        const uint8_t *ts = p.t + p.toff[pid];
        int lo = BANDED ? p.lo[pid] : -(m + 1);
        int hi = BANDED ? p.hi[pid] : n + 1;
        const int npass = (n + 32 * NWL_RL - 1) / (32 * NWL_RL);
        /* with p.cert, a band whose score fails the certificate is widened
         * to (its band) U (the label band of its own cost) and the pair runs
         * once more: that band always passes (its optimum costs at most the
         * first one's, and the label band of that cost covers it) */
        for (int round = 0; round < (BANDED && p.cert ? 2 : 1); ++round) {
        /* this CTA's slots start the pair unpublished */
        if (threadIdx.x < NWL_WARPS)
            cuda::atomic_ref<long long, cuda::thread_scope_device>(p.prog[(long long)blockIdx.x * NWL_WARPS + threadIdx.x])
                .store(0, cuda::memory_order_relaxed);
        if (coop) cluster.sync(); else __syncthreads();
        int result = NWL_NEG;
        bool have_result = false;

        for (int pass = tw; pass < npass; pass += T) {
            const int r0 = pass * 32 * NWL_RL;
            const int R0 = r0 + lane * NWL_RL;
            const long long in_slot = slot0 + (pass + T - 1) % T, out_slot = slot0 + pass % T;
            int2 *in_buf = p.scratch + in_slot * p.maxlen;
            int2 *out_buf = p.scratch + out_slot * p.maxlen;
            const long long stride = (long long)m + 1;
            cuda::atomic_ref<long long, cuda::thread_scope_device> in_prog(p.prog[in_slot]);
            cuda::atomic_ref<long long, cuda::thread_scope_device> out_prog(p.prog[out_slot]);
            const long long in_base = pass > 0 ? (long long)((pass - 1) / T) * stride + 1 : 0;
            const long long out_base = (long long)(pass / T) * stride + 1;
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
                const long long t0 = clock64();
                unsigned ns = 32;
                while (in_prog.load(cuda::memory_order_acquire) < in_base + need) {
                    if (*verr) return false;
                    if (clock64() - t0 > NWL_SPIN_CYCLES) { atomicExch(error, 1); return false; }
                    /* back off, so that waiting warps leave the memory
                     * system and the issue slots to the producers */
                    __nanosleep(ns);
                    if (ns < 1024) ns <<= 1;
                }
                return true;
            };
            int Hl[NWL_RL], E[NWL_RL];
#pragma unroll
            for (int r = 0; r < NWL_RL; ++r) {
                const int i = R0 + r;
                int v = NWL_NEG;
                if (jlo == 0 && (!BANDED || (i + 1 >= lo && i + 1 <= hi))) v = -open - i * gap - (BIAS ? open : 0);
                Hl[r] = v;
                E[r] = NWL_NEG;
            }
            int dg;
            if (jlo == 0) {
                dg = (R0 == 0) ? 0 : ((!BANDED || (R0 >= lo && R0 <= hi)) ? -open - (R0 - 1) * gap : NWL_NEG);
                if (BIAS && dg != NWL_NEG) dg -= open;
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
             * column by shuffle), loaded when the chunk starts, as soon as the
             * previous pass has published it. Loading a chunk ahead would hide
             * one L2 latency per 32 columns, but it makes each pass wait for
             * its predecessor to be 32 columns further along; a banded pair's
             * passes then start about 350 instead of 318 columns apart, and
             * the largest pairs, which keep only (band + 287) / lag warps
             * busy, take longer: 0.089 vs 0.080 s for the 300-pair
             * learned-band call. */
            auto ring_at = [&](int c) -> int2 {
                return (pass > 0 && c >= prev_jlo && c <= prev_jhi) ? __ldcg(&in_buf[c])
                                                                      : make_int2(NWL_NEG, NWL_NEG);
            };
            int2 cur_v = make_int2(NWL_NEG, NWL_NEG);
            bool aborted = false;
            for (int it = jlo; it <= tend; ++it) {
                const int j = it - lane;
                const int cpos = (it - jlo) & 31;
                if (cpos == 0) {
                    bool ok = true;
                    if (lane == 0) ok = wait_for(it + 31);
                    ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0);
                    if (!ok) { aborted = true; break; }
                    cur_v = ring_at(it + lane);
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
                        up_h = inb ? -open - j * gap - (BIAS ? open : 0) : NWL_NEG;
                        up_f = NWL_NEG;
                    } else {
                        up_h = vh;
                        up_f = vf;
                    }
                }
                /* banded: do all active lanes of the warp hold all their
                 * rows inside the band at this column? */
                bool full_in = true;
                if (BANDED) {
                    const unsigned bwl = (unsigned)(hi - lo);
                    const bool mine = !active || (bwl >= NWL_RL - 1 && (unsigned)(R0 - j - lo) <= bwl - (NWL_RL - 1));
                    full_in = __all_sync(0xffffffffu, mine);
                }
                if (active) {
                    int hd = dg;
                    uint32_t row_lo = 0, row_hi = 0;
                    if (p.small_alpha) {
                        row_lo = *reinterpret_cast<const uint32_t *>(s_mat + tc * 32);
                        row_hi = *reinterpret_cast<const uint32_t *>(s_mat + tc * 32 + 4);
                    }
                    /* F of row R0 from the row above (previous lane or pass) */
                    int f = BIAS ? __viaddmax_s32(up_f, -gap, up_h) : max(up_f - gap, up_h - open);
                    /* row R0 + r lies in the band iff 0 <= R0 + r - j - lo <= hi - lo */
                    const int dlo = R0 - j - lo;
                    const unsigned bw = (unsigned)(hi - lo);
                    int last_h = 0, last_f = 0;
                    /* one column of this lane's rows; MASK: rows outside the
                     * band are -infinity */
                    auto rows = [&](auto mask_tag) {
                        constexpr bool MASK = decltype(mask_tag)::value;
#pragma unroll
                        for (int r = 0; r < NWL_RL; ++r) {
                            const int sc = p.small_alpha ? sext_byte(row_lo, row_hi, qc[r]) : (int)s_mat[tc * 32 + qc[r]];
                            /* E and the diagonal/E part a are off the row-to-row chain */
                            int e = BIAS ? __viaddmax_s32(E[r], -gap, Hl[r]) : max(E[r] - gap, Hl[r] - open);
                            int a = __viaddmax_s32(hd, sc, e);
                            if (MASK) {
                                const bool in = (unsigned)(dlo + r) <= bw;
                                e = in ? e : NWL_NEG;
                                a = in ? a : NWL_NEG;
                                f = in ? f : NWL_NEG;
                            }
                            int h;
                            if (BIAS) {
                                const int ao = a - open;
                                h = __viaddmax_s32(f, -open, ao);     /* H - open */
                                last_h = h;
                                last_f = f;
                                f = __viaddmax_s32(f, -gap, ao);
                            } else {
                                h = max(a, f);
                                last_h = h;
                                last_f = f;
                                /* F of the next row: max(F - gap, H - open). With
                                 * open >= gap, H - open = max(a, F) - open and
                                 * F - open <= F - gap, so only a - open is needed:
                                 * one dependent operation per row */
                                if (GE) f = __viaddmax_s32(f, -gap, a - open);
                                else f = max(f - gap, h - open);
                            }
                            E[r] = e;
                            hd = Hl[r];
                            Hl[r] = h;
                        }
                    };
                    if (BANDED && !full_in) {
                        rows(std::integral_constant<bool, true>());
                    } else {
                        /* unbanded, or a column where every active lane of a
                         * wide band holds all its rows: no masks */
                        rows(std::integral_constant<bool, false>());
                    }
                    if (j == m - 1 && R0 <= n - 1 && n - 1 < R0 + NWL_RL) {
#pragma unroll
                        for (int r = 0; r < NWL_RL; ++r)
                            if (R0 + r == n - 1) { result = Hl[r] + (BIAS ? open : 0); have_result = true; }
                    }
                    dg = up_h;
                    sh_h = last_h;
                    sh_f = last_f;
                    if (lane == 31 && pass + 1 < npass) {
                        out_buf[j] = make_int2(last_h, last_f);
                        if (((j - jlo) & 31) == 31 || j == jhi)
                            out_prog.store(out_base + j, cuda::memory_order_release);
                    }
                }
            }
            if (aborted) break;
            __syncwarp();
        }
        /* the corner's owner publishes the result */
        if (have_result) p.score[pid] = result;
        if (!(BANDED && p.cert)) break;
        /* every thread of the team reads the one published score, so all
         * take the same branch (and the same barriers) below */
        if (coop) cluster.sync(); else __syncthreads();
        const int sc = *(volatile int *)&p.score[pid];
        const bool whole = lo <= -(m + 1) && hi >= n + 1;
        bool ok = whole;
        if (!whole && cert_valid(p.cm) && sc > NWL_NEG / 2)
            ok = cost2_of(p.cm, n, m, sc) <= exit_cost2(p.cm, n, m, lo, hi);
        if (ok || round == 1) break;
        if (cert_valid(p.cm) && sc > NWL_NEG / 2) {
            int l2, h2;
            label_band(p.cm, n, m, cost2_of(p.cm, n, m, sc), &l2, &h2);
            lo = min(lo, l2);
            hi = max(hi, h2);
        } else {
            lo = -(m + 1);
            hi = n + 1;
        }
        if (threadIdx.x == 0 && (!coop || crank == 0)) {
            p.lo_out[pid] = lo;
            p.hi_out[pid] = hi;
            p.rounds[pid] = 2;
        }
        }   /* rounds */
    }
    /* no CTA leaves while another of its cluster may still read its pair */
    if (coop) cluster.sync();
}

__global__ void k_iota_nw(int *v, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

/* sort key: the pair's work (cells, or for a band its rows x the columns
 * its passes sweep); the total goes to *total for k_team_class */
__global__ void k_cells(const int *ql, const int *tl, const int *lo, const int *hi, int n,
                        unsigned long long *keys, unsigned long long *total)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long k = 0;
    if (i < n) {
        const unsigned long long cols = lo ? (unsigned long long)min((long long)tl[i],
                                                  (long long)hi[i] - lo[i] + 32 * NWL_RL)
                                           : (unsigned long long)tl[i];
        k = (unsigned long long)ql[i] * cols;
        keys[i] = k;
    }
    for (int o = 16; o; o >>= 1) k += __shfl_xor_sync(0xffffffffu, k, o);
    if ((threadIdx.x & 31) == 0 && k) atomicAdd(total, k);
}

/*
 * The team class of every pair, in the key's bits 59-61 (and NWL_COOP_BIT
 * for classes >= 1), counted per class. A team of T warps is busy only
 * while T passes are in flight: a pass takes (its columns + 31) iterations
 * and the next one starts at most (256 + 94) columns later when banded (the
 * band moves 256 columns per pass; 31 of lane skew and up to 63 of the
 * 32-column hand-off), 94 otherwise, so a pair keeps at least
 * kappa = (columns + 31) / lag warps busy. The team is the smallest number
 * of CTAs that holds the pair's share of the warps, or kappa if that is
 * smaller, and every warp of the team gets a pass.
 */
__global__ void k_team_class(const int *ql, const int *tl, const int *lo, const int *hi, int n, int nwarps,
                             TeamPolicy pol, const unsigned long long *total, unsigned long long *keys,
                             int *count)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned long long k = keys[i];
    const int npass = (ql[i] + 32 * NWL_RL - 1) / (32 * NWL_RL);
    const long long m = tl[i];
    const bool narrow = lo && (long long)hi[i] - lo[i] + 32 * NWL_RL < m;
    const double cols = narrow ? (double)((long long)hi[i] - lo[i] + 32 * NWL_RL) : (double)m;
    const double kappa = (cols + 31.0) / (narrow ? 32.0 * NWL_RL + 94.0 : 94.0);
    const double share = (double)k * nwarps / ((double)*total * pol.share);
    int c = 0;
    if (pol.jump) {
        if (share > NWL_WARPS && npass >= NWL_WARPS * (pol.max_class + 1)) c = pol.max_class;
    } else {
        const double want = share < kappa ? share : kappa;
        while (c < pol.max_class && NWL_WARPS * (c + 1) < want && npass >= NWL_WARPS * (c + 2)) ++c;
    }
    keys[i] = k | (c ? NWL_COOP_BIT | ((unsigned long long)c << 59) : 0ull);
    atomicAdd(&count[c], 1);
}

}  // namespace pb

/* Global alignment scores of npairs device-resident pairs (codes), query i =
 * q[qoff[i] ..+qlen[i]), target i likewise, scored through the square matrix
 * d_mat (msize x msize int32, row = target letter). d_lo/d_hi: optional
 * per-pair band. Scores to d_score. */
static int nw_long_impl(int npairs, int open, int gap, const int32_t *h_mat, int msize,
                        const uint8_t *d_q, const int64_t *d_qoff, const int *d_qlen,
                        const uint8_t *d_t, const int64_t *d_toff, const int *d_tlen,
                        const int *d_lo, const int *d_hi, int maxlen, int *d_score,
                        int cert_a, int *d_lo_out, int *d_hi_out, int *d_rounds)
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
    unsigned long long *keys = nullptr, *keys_sorted = nullptr;
    void *tmp = nullptr;
    size_t tmpb = 0;
    int nsm = 0, dev = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    /* the one-operation F chain needs open >= gap; the biased form also every
     * score + open inside int8 */
    const bool ge = open >= gap;
    bool bias = ge;
    for (int k = 0; k < msize * msize; ++k)
        if (h_mat[k] + open > 127 || h_mat[k] + open < -128) bias = false;
    if (bias)
        for (int k = 0; k < msize * msize; ++k) hm[k] = (int8_t)(h_mat[k] + open);
    void (*kern)(pb::NwWaveParams, int *, int *) =
        d_lo ? (bias ? pb::k_nw_wave<true, true, true> : ge ? pb::k_nw_wave<true, true, false>
                                                            : pb::k_nw_wave<true, false, false>)
             : (bias ? pb::k_nw_wave<false, true, true> : ge ? pb::k_nw_wave<false, true, false>
                                                             : pb::k_nw_wave<false, false, false>);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, pb::NWL_WARPS * 32, 0);
    if (per_sm < 1) per_sm = 1;
    const int plain_max = per_sm * nsm;
    /* the largest cluster class the device runs, and how many clusters of
     * each class fit at once */
    /* full DP: kappa is in the hundreds, the largest pairs take 8-CTA teams;
     * banded: teams as large as the pair's share, bounded by what its band
     * keeps busy, and by 4 CTAs (larger teams leave fewer slots to the other
     * pairs than they gain: 0.064 vs 0.073 s for 300 long pairs on their
     * certified bands) */
    pb::TeamPolicy pol = d_lo ? pb::TeamPolicy{3, 1.0f, 0} : pb::TeamPolicy{7, 1.0f, 1};
    int maxclusters[pb::NWL_CLASSES] = {plain_max, 0, 0, 0, 0, 0, 0, 0};
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(pb::NWL_WARPS * 32);
    cfg.dynamicSmemBytes = 0;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    for (int c = 1; c <= pol.max_class; ++c) {
        attr[0].val.clusterDim.x = c + 1;
        cfg.gridDim = dim3((c + 1) * nsm);
        if (cudaOccupancyMaxActiveClusters(&maxclusters[c], (const void *)kern, &cfg) != cudaSuccess ||
            maxclusters[c] < 1) {
            cudaGetLastError();
            pol.max_class = c - 1;
            break;
        }
    }
    /* the work-queue buffers, each checked before any launch writes
     * through it; a failure frees what was allocated and ends the call */
    auto give_up = [&]() {
        if (d_mat) cudaFreeAsync(d_mat, st);
        if (idx) cudaFreeAsync(idx, st);
        if (order) cudaFreeAsync(order, st);
        if (keys) cudaFreeAsync(keys, st);
        if (keys_sorted) cudaFreeAsync(keys_sorted, st);
        if (counter) cudaFreeAsync(counter, st);
        if (tmp) cudaFreeAsync(tmp, st);
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
        cudaGetLastError();
        return -1;
    };
    if (cudaMallocAsync((void **)&d_mat, hm.size(), st) != cudaSuccess ||
        cudaMallocAsync((void **)&idx, sizeof(int) * npairs, st) != cudaSuccess ||
        cudaMallocAsync((void **)&order, sizeof(int) * npairs, st) != cudaSuccess ||
        cudaMallocAsync((void **)&keys, sizeof(unsigned long long) * npairs, st) != cudaSuccess ||
        cudaMallocAsync((void **)&keys_sorted, sizeof(unsigned long long) * npairs, st) != cudaSuccess ||
        cudaMallocAsync((void **)&counter, sizeof(int) * 32, st) != cudaSuccess)
        return give_up();
    cudaMemcpyAsync(d_mat, hm.data(), hm.size(), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(counter, 0, sizeof(int) * 32, st);
    /* counter[0..7]: pair counters of the class launches; [8..9]: total
     * work; [16..23]: pairs per class */
    unsigned long long *total = reinterpret_cast<unsigned long long *>(counter + 8);
    pb::k_iota_nw<<<(npairs + 255) / 256, 256, 0, st>>>(idx, npairs);
    pb::k_cells<<<(npairs + 255) / 256, 256, 0, st>>>(d_qlen, d_tlen, d_lo, d_hi, npairs, keys, total);
    pb::k_team_class<<<(npairs + 255) / 256, 256, 0, st>>>(d_qlen, d_tlen, d_lo, d_hi, npairs,
                                                           plain_max * pb::NWL_WARPS, pol, total, keys,
                                                           counter + 16);
    pb_diag_count_launch(3);
    cub::DeviceRadixSort::SortPairsDescending(nullptr, tmpb, keys, keys_sorted, idx, order, npairs, 0, 64, st);
    if (cudaMallocAsync(&tmp, tmpb, st) != cudaSuccess) return give_up();
    cub::DeviceRadixSort::SortPairsDescending(tmp, tmpb, keys, keys_sorted, idx, order, npairs, 0, 64, st);
    /* pairs sorted by class, largest first; one launch per class, each on
     * its own stream, the largest teams first; they never wait on each other */
    int ncls[pb::NWL_CLASSES] = {0, 0, 0, 0, 0, 0, 0, 0};
    cudaMemcpyAsync(ncls, counter + 16, sizeof ncls, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    /* Each launch gets as many teams as fit at once (or as it has pairs);
     * CTAs beyond what is resident only wait for a slot. If the launches
     * together exceed four times the resident CTAs, all are scaled down by
     * the same factor (each keeps at least one team), which bounds the ring
     * buffers without leaving any launch a handful of teams for many pairs
     * (a budget taken largest team first did that: one launch of many
     * pairs then ran on a single cluster). */
    int cblocks[pb::NWL_CLASSES], first[pb::NWL_CLASSES], blocks = 0, before = 0;
    long long want = 0;
    for (int c = pb::NWL_CLASSES - 1; c >= 0; --c) {
        const int nc = ncls[c] < maxclusters[c] ? ncls[c] : maxclusters[c];
        cblocks[c] = nc * (c + 1);
        want += cblocks[c];
    }
    const long long cap = 4LL * plain_max;
    for (int c = pb::NWL_CLASSES - 1; c >= 0; --c) {
        const int C = c + 1;
        int nc = cblocks[c] / C;
        if (want > cap && nc > 0) {
            nc = (int)((long long)nc * cap / want);
            if (nc < 1) nc = 1;
        }
        cblocks[c] = ncls[c] > 0 ? nc * C : 0;
        first[c] = before;
        before += ncls[c];
        blocks += cblocks[c];
    }
    int2 *scratch = nullptr;
    long long *prog = nullptr;
    int *d_err = nullptr;
    int rc = 0, herr = 0;
    cudaStream_t sc[pb::NWL_CLASSES] = {};
    cudaEvent_t ev = nullptr, evc[pb::NWL_CLASSES] = {};
    if (cudaMallocAsync((void **)&d_err, sizeof(int), st) != cudaSuccess) rc = -1;
    else cudaMemsetAsync(d_err, 0, sizeof(int), st);
    if (rc != 0 || cudaMallocAsync((void **)&scratch, sizeof(int2) * (size_t)(maxlen + 1) * blocks * pb::NWL_WARPS, st) != cudaSuccess ||
        cudaMallocAsync((void **)&prog, sizeof(long long) * (size_t)blocks * pb::NWL_WARPS, st) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
        rc = -1;
    for (int c = 0; c < pb::NWL_CLASSES && rc == 0; ++c)
        if (cblocks[c] > 0 &&
            (cudaStreamCreateWithFlags(&sc[c], cudaStreamNonBlocking) != cudaSuccess ||
             cudaEventCreateWithFlags(&evc[c], cudaEventDisableTiming) != cudaSuccess))
            rc = -1;
    if (rc == 0) {
        cudaMemsetAsync(prog, 0, sizeof(long long) * (size_t)blocks * pb::NWL_WARPS, st);
        cudaEventRecord(ev, st);
        pb::NwWaveParams p;
        p.open = open; p.gap = gap; p.msize = msize; p.small_alpha = small;
        p.mat = d_mat; p.q = d_q; p.qoff = d_qoff; p.qlen = d_qlen;
        p.t = d_t; p.toff = d_toff; p.tlen = d_tlen; p.lo = d_lo; p.hi = d_hi;
        p.maxlen = maxlen + 1; p.score = d_score;
        p.cert = d_lo && d_rounds ? 1 : 0;
        p.cm.a = cert_a; p.cm.open = open; p.cm.ext = gap;
        p.lo_out = d_lo_out; p.hi_out = d_hi_out; p.rounds = d_rounds;
        size_t slot = 0;
        int nlaunch = 0;
        for (int c = pb::NWL_CLASSES - 1; c >= 0; --c) {
            if (cblocks[c] <= 0) continue;
            cudaStreamWaitEvent(sc[c], ev, 0);
            pb::NwWaveParams pc = p;
            pc.npairs = ncls[c]; pc.order = order + first[c]; pc.keys = keys_sorted + first[c];
            pc.scratch = scratch + slot * p.maxlen;
            pc.prog = prog + slot;
            slot += (size_t)cblocks[c] * pb::NWL_WARPS;
            if (c > 0) {
                attr[0].val.clusterDim.x = c + 1;
                cfg.gridDim = dim3(cblocks[c]);
                cfg.stream = sc[c];
                if (cudaLaunchKernelEx(&cfg, kern, pc, counter + c, d_err) != cudaSuccess) rc = -1;
            } else {
                kern<<<cblocks[c], pb::NWL_WARPS * 32, 0, sc[c]>>>(pc, counter + c, d_err);
            }
            ++nlaunch;
            cudaEventRecord(evc[c], sc[c]);
            cudaStreamWaitEvent(st, evc[c], 0);
        }
        pb_diag_count_launch(nlaunch);
        if (cudaGetLastError() != cudaSuccess) rc = -1;
        cudaMemcpyAsync(&herr, d_err, sizeof(int), cudaMemcpyDeviceToHost, st);
    }
    cudaFreeAsync(d_mat, st); cudaFreeAsync(idx, st); cudaFreeAsync(order, st);
    cudaFreeAsync(keys, st); cudaFreeAsync(keys_sorted, st); cudaFreeAsync(counter, st);
    cudaFreeAsync(tmp, st);
    if (scratch) cudaFreeAsync(scratch, st);
    if (prog) cudaFreeAsync(prog, st);
    if (d_err) cudaFreeAsync(d_err, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) rc = -1;
    for (int c = 0; c < pb::NWL_CLASSES; ++c) {
        if (sc[c]) cudaStreamDestroy(sc[c]);
        if (evc[c]) cudaEventDestroy(evc[c]);
    }
    if (ev) cudaEventDestroy(ev);
    if (herr) {
        fprintf(stderr, "pb_cuda_nw_long: a pipeline wait exceeded its bound; pair abandoned\n");
        rc = -1;
    }
    cudaStreamDestroy(st);
    return rc;
}

extern "C" int pb_cuda_nw_long(int npairs, int open, int gap, const int32_t *h_mat, int msize,
                               const uint8_t *d_q, const int64_t *d_qoff, const int *d_qlen,
                               const uint8_t *d_t, const int64_t *d_toff, const int *d_tlen,
                               const int *d_lo, const int *d_hi, int maxlen, int *d_score)
{
    return nw_long_impl(npairs, open, gap, h_mat, msize, d_q, d_qoff, d_qlen, d_t, d_toff, d_tlen, d_lo, d_hi,
                        maxlen, d_score, 0, nullptr, nullptr, nullptr);
}

extern "C" int pb_cuda_nw_long_cert(int npairs, int open, int gap, const int32_t *h_mat, int msize, int a,
                                    const uint8_t *d_q, const int64_t *d_qoff, const int *d_qlen,
                                    const uint8_t *d_t, const int64_t *d_toff, const int *d_tlen,
                                    int *d_lo, int *d_hi, int maxlen, int *d_score, int *d_rounds)
{
    return nw_long_impl(npairs, open, gap, h_mat, msize, d_q, d_qoff, d_qlen, d_t, d_toff, d_tlen, d_lo, d_hi,
                        maxlen, d_score, a, d_lo, d_hi, d_rounds);
}
