/*
 * pb_band.cu -- learned band for long global alignments.
 *
 * Pipeline per batch of pairs:
 *   1. k_kmer_hist   k = 8 diagonal-offset histogram of every pair (256 bins
 *                    around the mid diagonal, normalised) + both lengths
 *   2. k_mlp_fwd     258 -> 128 -> 128 -> 2 MLP (ReLU, BF16 weights, FP32
 *                    accumulation): band centre and half-width, in units
 *                    of the longer sequence's length
 *   3. k_band_from_pred  band of diagonals [lo, hi] centred on (n - m) / 2
 *                    (where the certificate centres every label band), of
 *                    the predicted half-width; it always contains the start
 *                    and end diagonals
 *   4. banded global DP (pb_nwlong.cu) with the exactness certificate
 *                    checked in the launch: a pair that fails it reruns at
 *                    once on its band joined with the label band of its own
 *                    banded cost, which always passes
 *   5. k_certify     the certificate on its own, for caller-given bands
 *                    (parasail_b200_nw_banded_certified)
 *
 * Certificate. With a = the matrix's largest score, any global alignment
 * of lengths n (query) and m (target) has cost C = a(n+m)/2 - score, a sum
 * of non-negative terms: a - s per aligned pair, a/2 + ext per gap column
 * and open - ext per gap (open >= ext and a + 2 ext > 0 required). A path
 * that reaches diagonal hi+1 (i - j, above the band) needs at least
 * 2(hi+1) - d_end gap columns in at least two gaps, d_end = n - m, so its
 * cost is at least C_up = (2(hi+1) - d_end)(a/2 + ext) + 2(open - ext);
 * below the band, C_dn = (d_end - 2(lo-1))(a/2 + ext) + 2(open - ext). If the
 * banded optimum's cost is <= min(C_up, C_dn), no path leaving the band
 * scores more, so the banded score is the full optimum. The smallest band
 * that passes this test for the optimal cost C* is the training label.
 */
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <vector>
#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include "pb_cuda.h"
#include "pb_cert.cuh"

namespace pb {

static constexpr int KMER_K = 8;
static constexpr int HIST_BINS = 256;
static constexpr int MLP_IN = HIST_BINS + 2;
static constexpr int MLP_H = 128;
static constexpr int MLP_OUT = 2;

/* ---- 1. k-mer diagonal-offset histograms ------------------------------- */

/* table: per CTA slot, 4^8 entries holding the first query position of each
 * 8-mer (0xffffffff = absent); restored to absent before the CTA moves on. */
__global__ void __launch_bounds__(256)
k_kmer_hist(int npairs, const uint8_t *q, const int64_t *qoff, const int *qlen,
            const uint8_t *t, const int64_t *toff, const int *tlen,
            uint32_t *tables, float *features, int *counter)
{
    __shared__ unsigned int s_hist[HIST_BINS];
    __shared__ int s_pair;
    uint32_t *table = tables + (size_t)blockIdx.x * (1u << (2 * KMER_K));
    for (;;) {
        if (threadIdx.x == 0) s_pair = atomicAdd(counter, 1);
        for (int b = threadIdx.x; b < HIST_BINS; b += blockDim.x) s_hist[b] = 0;
        __syncthreads();
        const int p = s_pair;
        if (p >= npairs) break;
        const uint8_t *a = q + qoff[p];
        const uint8_t *bseq = t + toff[p];
        const int n = qlen[p], m = tlen[p];
        /* first occurrence of every query 8-mer (letters 0..3 only) */
        for (int i = threadIdx.x; i + KMER_K <= n; i += blockDim.x) {
            uint32_t code = 0;
            bool ok = true;
#pragma unroll
            for (int k = 0; k < KMER_K; ++k) {
                const uint32_t c = a[i + k];
                ok &= c < 4;
                code = (code << 2) | (c & 3u);
            }
            if (ok) atomicMin(&table[code], (uint32_t)i);
        }
        __syncthreads();
        const float L = (float)max(n, m);
        const float mid = 0.5f * (float)(n - m);
        const float scale = (float)HIST_BINS / (0.5f * L);   /* bins cover mid +- L/4 */
        unsigned int nk = 0;
        for (int j = threadIdx.x; j + KMER_K <= m; j += blockDim.x) {
            uint32_t code = 0;
            bool ok = true;
#pragma unroll
            for (int k = 0; k < KMER_K; ++k) {
                const uint32_t c = bseq[j + k];
                ok &= c < 4;
                code = (code << 2) | (c & 3u);
            }
            if (!ok) continue;
            ++nk;
            const uint32_t i = table[code];
            if (i == 0xffffffffu) continue;
            const float d = (float)((int)i - j) - mid;
            int bin = (int)floorf(d * scale) + HIST_BINS / 2;
            bin = min(max(bin, 0), HIST_BINS - 1);
            atomicAdd(&s_hist[bin], 1u);
        }
        /* number of target k-mers, for normalisation */
        __shared__ unsigned int s_nk;
        if (threadIdx.x == 0) s_nk = 0;
        __syncthreads();
        atomicAdd(&s_nk, nk);
        __syncthreads();
        float *f = features + (size_t)p * MLP_IN;
        const float inv = 1.0f / (float)max(1u, s_nk);
        for (int b = threadIdx.x; b < HIST_BINS; b += blockDim.x) f[b] = (float)s_hist[b] * inv * 16.0f;
        if (threadIdx.x == 0) {
            f[HIST_BINS] = logf((float)n) / 11.0f;
            f[HIST_BINS + 1] = logf((float)m) / 11.0f;
        }
        /* restore the table */
        for (int i = threadIdx.x; i + KMER_K <= n; i += blockDim.x) {
            uint32_t code = 0;
            bool ok = true;
#pragma unroll
            for (int k = 0; k < KMER_K; ++k) {
                const uint32_t c = a[i + k];
                ok &= c < 4;
                code = (code << 2) | (c & 3u);
            }
            if (ok) table[code] = 0xffffffffu;
        }
        __syncthreads();
    }
}

/* ---- 2. the MLP -------------------------------------------------------- */

struct MlpWeights {   /* BF16 copies used by the forward pass */
    const __nv_bfloat16 *w1, *w2, *w3;   /* [H][IN], [H][H], [OUT][H] */
    const float *b1, *b2, *b3;
};

/* one block of MLP_H threads per sample; activations saved for backward */
__global__ void __launch_bounds__(MLP_H)
k_mlp_fwd(int nsamp, const float *x, MlpWeights w, float *h1, float *h2, float *y)
{
    __shared__ float s_x[MLP_IN];
    __shared__ float s_h1[MLP_H];
    __shared__ float s_h2[MLP_H];
    const int s = blockIdx.x;
    if (s >= nsamp) return;
    const int u = threadIdx.x;
    for (int k = u; k < MLP_IN; k += MLP_H) s_x[k] = x[(size_t)s * MLP_IN + k];
    __syncthreads();
    float acc = w.b1[u];
    for (int k = 0; k < MLP_IN; ++k) acc = fmaf(__bfloat162float(w.w1[u * MLP_IN + k]), s_x[k], acc);
    acc = fmaxf(acc, 0.0f);
    s_h1[u] = acc;
    if (h1) h1[(size_t)s * MLP_H + u] = acc;
    __syncthreads();
    acc = w.b2[u];
    for (int k = 0; k < MLP_H; ++k) acc = fmaf(__bfloat162float(w.w2[u * MLP_H + k]), s_h1[k], acc);
    acc = fmaxf(acc, 0.0f);
    s_h2[u] = acc;
    if (h2) h2[(size_t)s * MLP_H + u] = acc;
    __syncthreads();
    if (u < MLP_OUT) {
        float o = w.b3[u];
        for (int k = 0; k < MLP_H; ++k) o = fmaf(__bfloat162float(w.w3[u * MLP_H + k]), s_h2[k], o);
        y[(size_t)s * MLP_OUT + u] = o;
    }
}

/* Loss per sample: squared error on the centre, pinball (quantile tau) on
 * the half-width so that predictions err on the wide side. dY = dLoss/dY
 * (mean over the batch). Per-sample deltas of both hidden layers follow. */
__global__ void __launch_bounds__(MLP_H)
k_mlp_delta(int nsamp, const float *y, const float *target, float tau, MlpWeights w,
            const float *h1, const float *h2, float *dy, float *d2, float *d1, float *loss)
{
    __shared__ float s_dy[MLP_OUT];
    __shared__ float s_d2[MLP_H];
    const int s = blockIdx.x;
    if (s >= nsamp) return;
    const int u = threadIdx.x;
    const float invb = 1.0f / (float)nsamp;
    if (u == 0) {
        const float ec = y[s * 2 + 0] - target[s * 2 + 0];
        const float ew = target[s * 2 + 1] - y[s * 2 + 1];
        s_dy[0] = 2.0f * ec * invb;
        s_dy[1] = (ew > 0.0f ? -tau : (1.0f - tau)) * invb;
        dy[s * 2 + 0] = s_dy[0];
        dy[s * 2 + 1] = s_dy[1];
        loss[s] = ec * ec + (ew > 0.0f ? tau * ew : (tau - 1.0f) * ew);
    }
    __syncthreads();
    float g = 0.0f;
    for (int o = 0; o < MLP_OUT; ++o) g = fmaf(__bfloat162float(w.w3[o * MLP_H + u]), s_dy[o], g);
    g = h2[(size_t)s * MLP_H + u] > 0.0f ? g : 0.0f;
    s_d2[u] = g;
    d2[(size_t)s * MLP_H + u] = g;
    __syncthreads();
    float g1 = 0.0f;
    for (int k = 0; k < MLP_H; ++k) g1 = fmaf(__bfloat162float(w.w2[k * MLP_H + u]), s_d2[k], g1);
    g1 = h1[(size_t)s * MLP_H + u] > 0.0f ? g1 : 0.0f;
    d1[(size_t)s * MLP_H + u] = g1;
}

/* Weight gradients, one thread per weight, summing over the batch in a fixed
 * order (deterministic): G[r][c] = sum_s D[s][r] * A[s][c]; bias gradient
 * GB[r] = sum_s D[s][r] (thread c == ncols). */
__global__ void k_mlp_wgrad(int nsamp, int nrows, int ncols, const float *D, const float *A,
                            float *G, float *GB)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    const int total = nrows * (ncols + 1);
    if (idx >= total) return;
    const int r = idx / (ncols + 1), c = idx % (ncols + 1);
    float acc = 0.0f;
    if (c < ncols) {
        for (int s = 0; s < nsamp; ++s) acc = fmaf(D[(size_t)s * nrows + r], A[(size_t)s * ncols + c], acc);
        G[r * ncols + c] = acc;
    } else {
        for (int s = 0; s < nsamp; ++s) acc += D[(size_t)s * nrows + r];
        GB[r] = acc;
    }
}

/* Adam on FP32 master weights; refreshes the BF16 copy. */
__global__ void k_adam(int n, float *w, const float *g, float *m1, float *m2, __nv_bfloat16 *wb,
                       float lr, float b1, float b2, float eps, float bc1, float bc2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi;
    const float v = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = v;
    const float upd = lr * (a / bc1) / (sqrtf(v / bc2) + eps);
    w[i] -= upd;
    if (wb) wb[i] = __float2bfloat16(w[i]);
}

/* ---- 3. bands and labels ---------------------------------------------- */

__global__ void k_labels(int npairs, CostModel c, const int *qlen, const int *tlen, const int *score,
                         float *target, int *lo_out, int *hi_out)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    const int n = qlen[p], m = tlen[p];
    const long long c2 = (long long)c.a * (n + m) - 2LL * score[p];
    int lo, hi;
    label_band(c, n, m, c2, &lo, &hi);
    const float L = (float)max(n, m);
    target[p * 2 + 0] = 0.5f * (float)(lo + hi) / L;
    target[p * 2 + 1] = 0.5f * (float)(hi - lo) / L;
    if (lo_out) lo_out[p] = lo;
    if (hi_out) hi_out[p] = hi;
}

__global__ void k_band_from_pred(int npairs, const int *qlen, const int *tlen, const float *y,
                                 float widen, int slack, int *lo_out, int *hi_out)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    const int n = qlen[p], m = tlen[p];
    const float L = (float)max(n, m);
    /* The centre is the label band's own, (n - m) / 2: the certificate's two
     * exits cost the same per gap column, so the narrowest certified band of
     * any cost is symmetric about d_end / 2 (label_band). Only the width is
     * predicted; taking the model's centre output instead cost a wider band
     * for the same coverage (on 300 config-5 pairs: widen 1.15 and 22% of the
     * cells, against 1.05 and 20%, 0.079 vs 0.069 s). */
    const float c = 0.5f * (float)(n - m);
    const float w = fmaxf(y[p * 2 + 1], 0.0f) * L * widen + (float)slack;
    long long lo = (long long)floorf(c - w), hi = (long long)ceilf(c + w);
    const long long dend = (long long)n - m;
    if (lo > (dend < 0 ? dend : 0)) lo = dend < 0 ? dend : 0;
    if (hi < (dend > 0 ? dend : 0)) hi = dend > 0 ? dend : 0;
    if (lo < -(long long)m - 1) lo = -(long long)m - 1;
    if (hi > (long long)n + 1) hi = (long long)n + 1;
    lo_out[p] = (int)lo;
    hi_out[p] = (int)hi;
}

/* certified[p] = 1 when the banded score is provably the full optimum */
__global__ void k_certify(int npairs, CostModel c, const int *qlen, const int *tlen, const int *lo,
                          const int *hi, const int *band_score, int *certified, int *fail_count)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    const int n = qlen[p], m = tlen[p];
    int ok;
    if (lo[p] <= -m - 1 && hi[p] >= n + 1) {
        ok = 1;                                   /* the band is the whole matrix */
    } else if (band_score[p] <= INT32_MIN / 8 || c.open < c.ext || c.a + 2 * c.ext <= 0) {
        ok = 0;
    } else {
        const long long c2 = (long long)c.a * (n + m) - 2LL * band_score[p];
        ok = c2 <= exit_cost2(c, n, m, lo[p], hi[p]);
    }
    certified[p] = ok;
    if (!ok) atomicAdd(fail_count, 1);
}

__global__ void k_band_cells(int npairs, const int *qlen, const int *tlen, const int *lo, const int *hi,
                             unsigned long long *cells)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    const long long n = qlen[p], m = tlen[p];
    /* cells (i, j) of the matrix with lo <= i - j <= hi: sum over diagonals */
    long long tot = 0;
    const long long dlo = lo[p] > -(m - 1) ? lo[p] : -(m - 1);
    const long long dhi = hi[p] < n - 1 ? hi[p] : n - 1;
    for (long long d = dlo; d <= dhi; ++d) {
        /* i = j + d, 0 <= i < n, 0 <= j < m */
        const long long jmin = d < 0 ? -d : 0;
        const long long jmax = (n - 1 - d) < (m - 1) ? (n - 1 - d) : (m - 1);
        if (jmax >= jmin) tot += jmax - jmin + 1;
    }
    atomicAdd(cells, (unsigned long long)tot);
}

/* cells (i, j) of an n x m matrix with lo <= i - j <= hi */
__device__ inline long long band_cells_of(long long n, long long m, long long lo, long long hi)
{
    long long tot = 0;
    const long long dlo = lo > -(m - 1) ? lo : -(m - 1);
    const long long dhi = hi < n - 1 ? hi : n - 1;
    for (long long d = dlo; d <= dhi; ++d) {
        const long long jmin = d < 0 ? -d : 0;
        const long long jmax = (n - 1 - d) < (m - 1) ? (n - 1 - d) : (m - 1);
        if (jmax >= jmin) tot += jmax - jmin + 1;
    }
    return tot;
}

/* expected cost of a band choice, in cells: the band's cells, plus, for
 * every pair whose band does not contain its label band (so the certificate
 * fails), a rerun on (band) U (label band of the first run's cost). That
 * cost is at least the optimum's, so the rerun band is at least the union
 * with the label band. A rerun counts 6 times that union's cells: it starts
 * only when its pair's first band is done, so it lengthens that pair's
 * latency (often the batch's tail) rather than adding to throughput. */
static constexpr int BAND_RERUN_WEIGHT = 6;

__global__ void k_tune_cost(int npairs, const int *qlen, const int *tlen, const int *lo, const int *hi,
                            const int *lab_lo, const int *lab_hi, unsigned long long *cost)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    const long long n = qlen[p], m = tlen[p];
    long long tot = band_cells_of(n, m, lo[p], hi[p]);
    if (lo[p] > lab_lo[p] || hi[p] < lab_hi[p])
        tot += BAND_RERUN_WEIGHT * band_cells_of(n, m, min(lo[p], lab_lo[p]), max(hi[p], lab_hi[p]));
    atomicAdd(cost, (unsigned long long)tot);
}

}  // namespace pb

/* ======================================================================== */

struct pb_band_model {
    /* FP32 master weights, Adam moments, BF16 copies (device) */
    float *w;        /* concatenated w1 | w2 | w3 */
    float *b;        /* b1 | b2 | b3 */
    float *mw1, *mw2, *mb1, *mb2;
    __nv_bfloat16 *wb;
    int step;
    /* band scaling chosen on held-out pairs after training */
    float widen;
    int slack;
};

static const int NW1 = pb::MLP_H * pb::MLP_IN, NW2 = pb::MLP_H * pb::MLP_H, NW3 = pb::MLP_OUT * pb::MLP_H;
static const int NWT = NW1 + NW2 + NW3;
static const int NBT = pb::MLP_H + pb::MLP_H + pb::MLP_OUT;

static pb::MlpWeights weights_of(const pb_band_model *m)
{
    pb::MlpWeights w;
    w.w1 = m->wb;
    w.w2 = m->wb + NW1;
    w.w3 = m->wb + NW1 + NW2;
    w.b1 = m->b;
    w.b2 = m->b + pb::MLP_H;
    w.b3 = m->b + 2 * pb::MLP_H;
    return w;
}

extern "C" pb_band_model *pb_cuda_band_model_new(unsigned seed)
{
    if (pb_cuda_init() != 0) return nullptr;
    pb_band_model *m = new pb_band_model();
    m->widen = 1.1f;
    m->slack = 32;
    std::vector<float> hw(NWT), hb(NBT, 0.0f);
    /* He-uniform initialisation from a fixed LCG (reproducible) */
    uint64_t s = 0x9E3779B97F4A7C15ull ^ seed;
    auto uni = [&]() {
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        return (float)((s >> 40) & 0xffffff) / 16777216.0f * 2.0f - 1.0f;
    };
    const float a1 = sqrtf(6.0f / pb::MLP_IN), a2 = sqrtf(6.0f / pb::MLP_H), a3 = sqrtf(3.0f / pb::MLP_H);
    for (int k = 0; k < NW1; ++k) hw[k] = a1 * uni();
    for (int k = 0; k < NW2; ++k) hw[NW1 + k] = a2 * uni();
    for (int k = 0; k < NW3; ++k) hw[NW1 + NW2 + k] = 0.1f * a3 * uni();
    hb[2 * pb::MLP_H + 0] = 0.0f;
    hb[2 * pb::MLP_H + 1] = 0.05f;
    std::vector<__nv_bfloat16> hwb(NWT);
    for (int k = 0; k < NWT; ++k) hwb[k] = __float2bfloat16(hw[k]);
    cudaMalloc(&m->w, sizeof(float) * NWT);
    cudaMalloc(&m->b, sizeof(float) * NBT);
    cudaMalloc(&m->mw1, sizeof(float) * NWT);
    cudaMalloc(&m->mw2, sizeof(float) * NWT);
    cudaMalloc(&m->mb1, sizeof(float) * NBT);
    cudaMalloc(&m->mb2, sizeof(float) * NBT);
    cudaMalloc(&m->wb, sizeof(__nv_bfloat16) * NWT);
    cudaMemcpy(m->w, hw.data(), sizeof(float) * NWT, cudaMemcpyHostToDevice);
    cudaMemcpy(m->b, hb.data(), sizeof(float) * NBT, cudaMemcpyHostToDevice);
    cudaMemcpy(m->wb, hwb.data(), sizeof(__nv_bfloat16) * NWT, cudaMemcpyHostToDevice);
    cudaMemset(m->mw1, 0, sizeof(float) * NWT);
    cudaMemset(m->mw2, 0, sizeof(float) * NWT);
    cudaMemset(m->mb1, 0, sizeof(float) * NBT);
    cudaMemset(m->mb2, 0, sizeof(float) * NBT);
    m->step = 0;
    return m;
}

extern "C" void pb_cuda_band_model_free(pb_band_model *m)
{
    if (!m) return;
    cudaFree(m->w); cudaFree(m->b); cudaFree(m->mw1); cudaFree(m->mw2);
    cudaFree(m->mb1); cudaFree(m->mb2); cudaFree(m->wb);
    delete m;
}

/* weights as FP32 (w: NWT, b: NBT) to/from host; set also refreshes BF16 */
extern "C" int pb_cuda_band_model_get(const pb_band_model *m, float *w, float *b)
{
    if (w && cudaMemcpy(w, m->w, sizeof(float) * NWT, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    if (b && cudaMemcpy(b, m->b, sizeof(float) * NBT, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
    return 0;
}

extern "C" int pb_cuda_band_model_set(pb_band_model *m, const float *w, const float *b)
{
    std::vector<__nv_bfloat16> hwb(NWT);
    for (int k = 0; k < NWT; ++k) hwb[k] = __float2bfloat16(w[k]);
    if (cudaMemcpy(m->w, w, sizeof(float) * NWT, cudaMemcpyHostToDevice) != cudaSuccess) return -1;
    if (cudaMemcpy(m->b, b, sizeof(float) * NBT, cudaMemcpyHostToDevice) != cudaSuccess) return -1;
    if (cudaMemcpy(m->wb, hwb.data(), sizeof(__nv_bfloat16) * NWT, cudaMemcpyHostToDevice) != cudaSuccess) return -1;
    return 0;
}

extern "C" int pb_cuda_band_sizes(int *n_in, int *n_hidden, int *n_out, int *nw, int *nb)
{
    *n_in = pb::MLP_IN; *n_hidden = pb::MLP_H; *n_out = pb::MLP_OUT; *nw = NWT; *nb = NBT;
    return 0;
}

/* features [npairs][258] of device-resident pairs (DNA codes 0..3) */
extern "C" int pb_cuda_band_features(int npairs, const uint8_t *d_q, const int64_t *d_qoff, const int *d_qlen,
                                     const uint8_t *d_t, const int64_t *d_toff, const int *d_tlen, float *d_feat)
{
    if (npairs <= 0) return 0;
    int nsm = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = std::min(npairs, nsm * 4);
    uint32_t *tables = nullptr;
    int *counter = nullptr;
    /* stream-ordered pool memory: a plain cudaMalloc/cudaFree of these
     * tables (tens of MB per call) can stall while the pool holds most of
     * the device's memory */
    const size_t tbytes = sizeof(uint32_t) * ((size_t)1 << (2 * pb::KMER_K)) * blocks;
    if (cudaMallocAsync((void **)&tables, tbytes, 0) != cudaSuccess) return -1;
    if (cudaMallocAsync((void **)&counter, sizeof(int), 0) != cudaSuccess) { cudaFreeAsync(tables, 0); return -1; }
    cudaMemsetAsync(tables, 0xff, tbytes, 0);
    cudaMemsetAsync(counter, 0, sizeof(int), 0);
    pb::k_kmer_hist<<<blocks, 256>>>(npairs, d_q, d_qoff, d_qlen, d_t, d_toff, d_tlen, tables, d_feat, counter);
    pb_diag_count_launch(1);
    cudaFreeAsync(tables, 0);
    cudaFreeAsync(counter, 0);
    cudaError_t e = cudaDeviceSynchronize();
    return e == cudaSuccess ? 0 : -1;
}

/* forward pass; d_h1/d_h2 may be NULL (inference) */
extern "C" int pb_cuda_band_forward(const pb_band_model *m, int n, const float *d_x, float *d_h1, float *d_h2,
                                    float *d_y)
{
    if (n <= 0) return 0;
    pb::k_mlp_fwd<<<n, pb::MLP_H>>>(n, d_x, weights_of(m), d_h1, d_h2, d_y);
    pb_diag_count_launch(1);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

/* gradients of the batch loss w.r.t. all weights (FP32, host-visible layout
 * w1|w2|w3, b1|b2|b3) -- exposed so the tests can check them against a CPU
 * oracle; returns the mean loss */
extern "C" int pb_cuda_band_gradients(const pb_band_model *m, int n, const float *d_x, const float *d_target,
                                      float tau, float *d_gw, float *d_gb, float *loss_out)
{
    if (n <= 0) return -1;
    float *h1 = nullptr, *h2 = nullptr, *y = nullptr, *dy = nullptr, *d2 = nullptr, *d1 = nullptr, *loss = nullptr;
    float **const bufs[7] = {&h1, &h2, &d1, &d2, &y, &dy, &loss};
    const size_t per[7] = {pb::MLP_H, pb::MLP_H, pb::MLP_H, pb::MLP_H, pb::MLP_OUT, pb::MLP_OUT, 1};
    /* every buffer checked before any kernel writes through it */
    for (int b = 0; b < 7; ++b) {
        if (cudaMallocAsync((void **)bufs[b], sizeof(float) * n * per[b], 0) != cudaSuccess) {
            for (int c = 0; c < b; ++c) cudaFreeAsync(*bufs[c], 0);
            cudaGetLastError();
            return -1;
        }
    }
    const pb::MlpWeights w = weights_of(m);
    pb::k_mlp_fwd<<<n, pb::MLP_H>>>(n, d_x, w, h1, h2, y);
    pb::k_mlp_delta<<<n, pb::MLP_H>>>(n, y, d_target, tau, w, h1, h2, dy, d2, d1, loss);
    const int t1 = pb::MLP_H * (pb::MLP_IN + 1), t2 = pb::MLP_H * (pb::MLP_H + 1), t3 = pb::MLP_OUT * (pb::MLP_H + 1);
    pb::k_mlp_wgrad<<<(t1 + 255) / 256, 256>>>(n, pb::MLP_H, pb::MLP_IN, d1, d_x, d_gw, d_gb);
    pb::k_mlp_wgrad<<<(t2 + 255) / 256, 256>>>(n, pb::MLP_H, pb::MLP_H, d2, h1, d_gw + NW1, d_gb + pb::MLP_H);
    pb::k_mlp_wgrad<<<(t3 + 255) / 256, 256>>>(n, pb::MLP_OUT, pb::MLP_H, dy, h2, d_gw + NW1 + NW2, d_gb + 2 * pb::MLP_H);
    pb_diag_count_launch(5);
    std::vector<float> hl(n);
    cudaMemcpy(hl.data(), loss, sizeof(float) * n, cudaMemcpyDeviceToHost);
    double tot = 0;
    for (int k = 0; k < n; ++k) tot += hl[k];
    if (loss_out) *loss_out = (float)(tot / n);
    cudaFreeAsync(h1, 0); cudaFreeAsync(h2, 0); cudaFreeAsync(d1, 0); cudaFreeAsync(d2, 0); cudaFreeAsync(y, 0); cudaFreeAsync(dy, 0); cudaFreeAsync(loss, 0);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int pb_cuda_band_adam(pb_band_model *m, const float *d_gw, const float *d_gb, float lr)
{
    m->step += 1;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float bc1 = 1.0f - powf(b1, (float)m->step), bc2 = 1.0f - powf(b2, (float)m->step);
    pb::k_adam<<<(NWT + 255) / 256, 256>>>(NWT, m->w, d_gw, m->mw1, m->mw2, m->wb, lr, b1, b2, eps, bc1, bc2);
    pb::k_adam<<<(NBT + 255) / 256, 256>>>(NBT, m->b, d_gb, m->mb1, m->mb2, nullptr, lr, b1, b2, eps, bc1, bc2);
    pb_diag_count_launch(2);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int pb_cuda_band_labels(int npairs, int a, int open, int ext, const int *d_qlen, const int *d_tlen,
                                   const int *d_score, float *d_target, int *d_lo, int *d_hi)
{
    pb::CostModel c = {a, open, ext};
    pb::k_labels<<<(npairs + 255) / 256, 256>>>(npairs, c, d_qlen, d_tlen, d_score, d_target, d_lo, d_hi);
    pb_diag_count_launch(1);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int pb_cuda_band_from_pred(int npairs, const int *d_qlen, const int *d_tlen, const float *d_y,
                                      float widen, int slack, int *d_lo, int *d_hi)
{
    pb::k_band_from_pred<<<(npairs + 255) / 256, 256>>>(npairs, d_qlen, d_tlen, d_y, widen, slack, d_lo, d_hi);
    pb_diag_count_launch(1);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int pb_cuda_band_certify(int npairs, int a, int open, int ext, const int *d_qlen, const int *d_tlen,
                                    const int *d_lo, const int *d_hi, const int *d_score, int *d_cert,
                                    int *h_failures)
{
    pb::CostModel c = {a, open, ext};
    int *d_fail = nullptr;
    if (npairs <= 0) { if (h_failures) *h_failures = 0; return 0; }
    if (cudaMallocAsync((void **)&d_fail, sizeof(int), 0) != cudaSuccess) { cudaGetLastError(); return -1; }
    cudaMemset(d_fail, 0, sizeof(int));
    pb::k_certify<<<(npairs + 255) / 256, 256>>>(npairs, c, d_qlen, d_tlen, d_lo, d_hi, d_score, d_cert, d_fail);
    pb_diag_count_launch(1);
    cudaMemcpy(h_failures, d_fail, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFreeAsync(d_fail, 0);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int pb_cuda_band_cells(int npairs, const int *d_qlen, const int *d_tlen, const int *d_lo,
                                  const int *d_hi, unsigned long long *h_cells)
{
    unsigned long long *d = nullptr;
    if (cudaMallocAsync((void **)&d, sizeof(unsigned long long), 0) != cudaSuccess) return -1;
    cudaMemsetAsync(d, 0, sizeof(unsigned long long), 0);
    pb::k_band_cells<<<(npairs + 127) / 128, 128>>>(npairs, d_qlen, d_tlen, d_lo, d_hi, d);
    pb_diag_count_launch(1);
    cudaMemcpyAsync(h_cells, d, sizeof(unsigned long long), cudaMemcpyDeviceToHost, 0);
    cudaFreeAsync(d, 0);
    const cudaError_t e = cudaStreamSynchronize(0);
    return e == cudaSuccess && cudaGetLastError() == cudaSuccess ? 0 : -1;
}

/* Chooses the model's band scaling on n held-out pairs (features d_x,
 * label bands d_lab_lo/d_lab_hi): the widen factor of a fixed grid with the
 * least expected DP work (k_tune_cost). */
extern "C" int pb_cuda_band_tune(pb_band_model *m, int n, const float *d_x, const int *d_qlen, const int *d_tlen,
                                 const int *d_lab_lo, const int *d_lab_hi, float *chosen)
{
    static const float grid[] = {1.0f, 1.05f, 1.1f, 1.15f, 1.2f, 1.3f, 1.4f, 1.5f, 1.75f, 2.0f, 2.5f, 3.0f};
    if (n <= 0) return -1;
    float *y = nullptr;
    int *lo = nullptr, *hi = nullptr;
    unsigned long long *cost = nullptr;
    if (cudaMallocAsync((void **)&y, sizeof(float) * n * pb::MLP_OUT, 0) != cudaSuccess ||
        cudaMallocAsync((void **)&lo, sizeof(int) * n, 0) != cudaSuccess ||
        cudaMallocAsync((void **)&hi, sizeof(int) * n, 0) != cudaSuccess ||
        cudaMallocAsync((void **)&cost, sizeof(unsigned long long), 0) != cudaSuccess) {
        /* nothing has been launched: free what was allocated */
        if (y) cudaFreeAsync(y, 0);
        if (lo) cudaFreeAsync(lo, 0);
        if (hi) cudaFreeAsync(hi, 0);
        cudaGetLastError();
        return -1;
    }
    int rc = pb_cuda_band_forward(m, n, d_x, nullptr, nullptr, y);
    unsigned long long best = ~0ull;
    float bw = m->widen;
    for (unsigned g = 0; rc == 0 && g < sizeof grid / sizeof grid[0]; ++g) {
        unsigned long long c = 0;
        rc = pb_cuda_band_from_pred(n, d_qlen, d_tlen, y, grid[g], m->slack, lo, hi);
        cudaMemsetAsync(cost, 0, sizeof(unsigned long long), 0);
        pb::k_tune_cost<<<(n + 127) / 128, 128>>>(n, d_qlen, d_tlen, lo, hi, d_lab_lo, d_lab_hi, cost);
        pb_diag_count_launch(1);
        if (cudaMemcpy(&c, cost, sizeof c, cudaMemcpyDeviceToHost) != cudaSuccess) rc = -1;
        if (rc == 0 && c < best) { best = c; bw = grid[g]; }
    }
    if (rc == 0) m->widen = bw;
    if (chosen) *chosen = m->widen;
    cudaFreeAsync(y, 0); cudaFreeAsync(lo, 0); cudaFreeAsync(hi, 0); cudaFreeAsync(cost, 0);
    return rc;
}

extern "C" void pb_cuda_band_scaling(const pb_band_model *m, float *widen, int *slack)
{
    if (widen) *widen = m->widen;
    if (slack) *slack = m->slack;
}

/* bands of the pairs that ran twice (d_rounds == 2), empty bands (no
 * cells) for the others */
__global__ void k_band_select(int npairs, const int *rounds, const int *lo, const int *hi, int *slo, int *shi)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    const bool twice = rounds[p] == 2;
    slo[p] = twice ? lo[p] : 1;
    shi[p] = twice ? hi[p] : 0;
}

extern "C" int pb_cuda_band_select(int npairs, const int *d_rounds, const int *d_lo, const int *d_hi, int *sel_lo,
                                   int *sel_hi)
{
    k_band_select<<<(npairs + 255) / 256, 256>>>(npairs, d_rounds, d_lo, d_hi, sel_lo, sel_hi);
    pb_diag_count_launch(1);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

/* host mirror of the certificate arithmetic, for the C host code */
extern "C" void pb_band_label_host(int a, int open, int ext, int n, int m, long long c2, int *lo, int *hi)
{
    pb::CostModel c = {a, open, ext};
    pb::label_band(c, n, m, c2, lo, hi);
}
