/*
 * pb_banded.cu -- parasail_nw_banded on the GPU.
 *
 * k_nw_banded_one follows the reference's banded global recurrence
 * (src/nw_banded.c:29-189): the band of query positions
 * [j + low, j + k] (low = min(0, s1Len - s2Len) - k style bounds, :92-96) is
 * held as one column of colLen = k - low + 1 cells that slides down one row
 * per target column; cells outside the query are skipped, the column's
 * sentinels are NEG_INF, and the score is read at the band position of the
 * bottom-right corner (:179). The column lives in global scratch.
 */
#include <cstdint>
#include <climits>
#include <cuda_runtime.h>

#include "pb_cuda.h"

namespace {

constexpr int NEG_INF = INT32_MIN / 2;

__global__ void k_nw_banded_one(const int32_t *__restrict__ prof, int lp,
                                const uint8_t *__restrict__ s2, int s1Len, int s2Len,
                                int open, int gap, int k, int *__restrict__ HB,
                                int *__restrict__ EB, int *__restrict__ out)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int low = s1Len - s2Len - k;
    if (s1Len > s2Len) low = s2Len - s1Len - k;
    const int colLen = k - low + 1;
    int colOff = s1Len > s2Len ? -k : low;
    int *H = HB + 1, *E = EB + 1;
    for (int i = -1; i <= colLen; ++i) { H[i] = 0; E[i] = 0; }
    for (int i = -colOff + 1, j = 0; i < colLen; ++i, ++j) {
        H[i] = -open - j * gap;
        E[i] = NEG_INF;
    }
    H[-colOff - 1] = -open;
    E[-colOff - 1] = NEG_INF;
    H[-colOff] = 0;
    E[-colOff] = NEG_INF;
    H[-1] = NEG_INF;
    E[-1] = NEG_INF;
    H[colLen] = NEG_INF;
    E[colLen] = NEG_INF;
    for (int j = 0; j < s2Len; ++j) {
        int F = NEG_INF;
        const int32_t *prow = prof + (size_t)s2[j] * lp;
        if (colOff < 0) H[-colOff - 1] = -open - j * gap;
        for (int i = 0; i < colLen; ++i) {
            const int pos = colOff + i;
            if (pos < 0 || pos >= s1Len) continue;
            const int hdag = H[i] + prow[pos];
            const int e = max(H[i + 1] - open, E[i + 1] - gap);
            F = max(H[i - 1] - open, F - gap);
            E[i] = e;
            H[i] = max(max(e, F), hdag);
        }
        colOff += 1;
    }
    out[0] = s1Len > s2Len ? H[-low] : H[k];
}

}  // namespace

extern "C" int pb_cuda_nw_banded(const pb_device_profile *dp, const uint8_t *h_s2, int s2Len,
                                 int open, int gap, int k, int *score)
{
    const int s1Len = dp->qlen;
    int low = s1Len - s2Len - k;
    if (s1Len > s2Len) low = s2Len - s1Len - k;
    const long colLen = (long)k - low + 1;
    cudaStream_t st = nullptr;
    uint8_t *d_s2 = nullptr;
    int *d_h = nullptr, *d_e = nullptr, *d_out = nullptr;
    if (cudaMallocAsync((void **)&d_s2, s2Len, 0) != cudaSuccess) return -1;
    if (cudaMallocAsync((void **)&d_h, sizeof(int) * (colLen + 2), 0) != cudaSuccess) { cudaFreeAsync(d_s2, 0); return -1; }
    if (cudaMallocAsync((void **)&d_e, sizeof(int) * (colLen + 2), 0) != cudaSuccess) { cudaFreeAsync(d_s2, 0); cudaFreeAsync(d_h, 0); return -1; }
    if (cudaMallocAsync((void **)&d_out, sizeof(int), 0) != cudaSuccess) { cudaFreeAsync(d_s2, 0); cudaFreeAsync(d_h, 0); cudaFreeAsync(d_e, 0); return -1; }
    cudaMemcpyAsync(d_s2, h_s2, s2Len, cudaMemcpyHostToDevice, st);
    k_nw_banded_one<<<1, 1, 0, st>>>(dp->d_prof32, dp->lp, d_s2, s1Len, s2Len, open, gap, k, d_h, d_e, d_out);
    cudaError_t e = cudaMemcpyAsync(score, d_out, sizeof(int), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    cudaFreeAsync(d_s2, 0); cudaFreeAsync(d_h, 0); cudaFreeAsync(d_e, 0); cudaFreeAsync(d_out, 0);
    return (e == cudaSuccess && cudaGetLastError() == cudaSuccess) ? 0 : -1;
}
