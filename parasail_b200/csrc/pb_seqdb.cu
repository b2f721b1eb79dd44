/*
 * pb_seqdb.cu -- device-resident packed sequence sets.
 *
 * The '$'-separated text of parasail_sequences_pack (src/parser.c:235-258 of
 * the reference) is mapped through a matrix's mapper on the GPU and stored
 * in 32-bit words at the narrowest width its codes allow: 2 bits (16
 * residues a word) when every code is below 4, 5 bits (6 a word) below 32,
 * else 8 bits (4 a word). Residue i of the text sits in word i / per at bit
 * (i % per) * bits; sentinels store code 0 (they lie outside every
 * sequence). Unpacking to the one-byte codes the DP kernels read is an
 * HBM-bound pass: each thread loads one 16-byte group of 4 words and writes
 * its 64 / 24 / 16 codes with 16-, 8- and 16-byte stores.
 */
#include <cstdint>
#include <cstdio>
#include <cstring>

#include <cuda_runtime.h>

#include "pb_cuda.h"

namespace {

__global__ void k_max_code(const uint8_t *__restrict__ T, int64_t n, uint8_t sep, const int *__restrict__ map,
                           int *__restrict__ mx)
{
    __shared__ int smap[256];
    __shared__ int bmax;
    for (int k = threadIdx.x; k < 256; k += blockDim.x) smap[k] = map[k];
    if (threadIdx.x == 0) bmax = 0;
    __syncthreads();
    int v = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (T[i] != sep) v = max(v, smap[T[i]]);
    atomicMax(&bmax, v);
    __syncthreads();
    if (threadIdx.x == 0) atomicMax(mx, bmax);
}

__global__ void k_pack(const uint8_t *__restrict__ T, int64_t n, uint8_t sep, const int *__restrict__ map, int bits,
                       int per, int64_t nwords, uint32_t *__restrict__ words)
{
    __shared__ int smap[256];
    for (int k = threadIdx.x; k < 256; k += blockDim.x) smap[k] = map[k];
    __syncthreads();
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < nwords;
         w += (int64_t)gridDim.x * blockDim.x) {
        uint32_t v = 0;
        const int64_t i0 = w * per;
        for (int k = 0; k < per; ++k) {
            const int64_t i = i0 + k;
            const uint32_t c = i < n && T[i] != sep ? (uint32_t)smap[T[i]] : 0u;
            v |= c << (k * bits);
        }
        words[w] = v;
    }
}

template <int BITS>
__device__ __forceinline__ uint32_t code_of(uint32_t w, int k)
{
    return (w >> (k * BITS)) & ((1u << BITS) - 1u);
}

/* one thread per 16-byte group of 4 words */
template <int BITS, int PER>
__global__ void k_unpack(const uint4 *__restrict__ groups, int64_t ngroups, int64_t n, uint8_t *__restrict__ out)
{
    constexpr int G = 4 * PER;                  /* codes per group */
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ngroups;
         g += (int64_t)gridDim.x * blockDim.x) {
        const uint4 q = groups[g];
        const uint32_t w[4] = {q.x, q.y, q.z, q.w};
        uint8_t c[G];
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
            for (int k = 0; k < PER; ++k) c[x * PER + k] = (uint8_t)code_of<BITS>(w[x], k);
        const int64_t base = g * G;
        if (base + G <= n) {
            if (G % 16 == 0) {
#pragma unroll
                for (int s = 0; s < G / 16; ++s) {
                    uint4 v;
                    memcpy(&v, c + 16 * s, 16);
                    reinterpret_cast<uint4 *>(out + base)[s] = v;
                }
            } else {
#pragma unroll
                for (int s = 0; s < G / 8; ++s) {
                    uint2 v;
                    memcpy(&v, c + 8 * s, 8);
                    reinterpret_cast<uint2 *>(out + base)[s] = v;
                }
            }
        } else {
            for (int k = 0; k < G && base + k < n; ++k) out[base + k] = c[k];
        }
    }
}

__global__ void k_gather_pairs(const int64_t *__restrict__ off, const int *__restrict__ len,
                               const int *__restrict__ first, const int *__restrict__ second, int np,
                               int64_t *__restrict__ qoff, int *__restrict__ qlen, int64_t *__restrict__ toff,
                               int *__restrict__ tlen)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= np) return;
    const int a = first[k], b = second[k];
    qoff[k] = off[a];
    qlen[k] = len[a];
    toff[k] = off[b];
    tlen[k] = len[b];
}

int grid_of(int64_t n)
{
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int64_t want = (n + 255) / 256;
    const int64_t cap = (int64_t)nsm * 8;
    return (int)(want < 1 ? 1 : want < cap ? want : cap);
}

}  // namespace

/* Packs text (n bytes, host) into *d_words (device, padded to whole 4-word
 * groups, zero-filled); *bits is 2, 5 or 8. */
extern "C" int pb_cuda_seqdb_pack(const uint8_t *h_text, int64_t n, uint8_t sep, const int *h_map256, int *bits,
                                  uint32_t **d_words, int64_t *nwords)
{
    if (pb_cuda_init() != 0) return -1;
    uint8_t *T = nullptr;
    int *map = nullptr, *mx = nullptr, hmax = 0;
    int rc = 0;
    *d_words = nullptr;
    *nwords = 0;
    if (cudaMalloc((void **)&T, (size_t)(n > 0 ? n : 1)) != cudaSuccess ||
        cudaMalloc((void **)&map, sizeof(int) * 256) != cudaSuccess ||
        cudaMalloc((void **)&mx, sizeof(int)) != cudaSuccess)
        rc = -1;
    if (rc == 0 && (cudaMemcpy(T, h_text, (size_t)n, cudaMemcpyHostToDevice) != cudaSuccess ||
                    cudaMemcpy(map, h_map256, sizeof(int) * 256, cudaMemcpyHostToDevice) != cudaSuccess ||
                    cudaMemset(mx, 0, sizeof(int)) != cudaSuccess))
        rc = -1;
    if (rc == 0) {
        k_max_code<<<grid_of(n), 256>>>(T, n, sep, map, mx);
        pb_diag_count_launch(1);
        if (cudaMemcpy(&hmax, mx, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) rc = -1;
    }
    if (rc == 0) {
        const int b = hmax < 4 ? 2 : hmax < 32 ? 5 : 8;
        const int per = b == 2 ? 16 : b == 5 ? 6 : 4;
        const int64_t nw = ((n + per - 1) / per + 3) / 4 * 4;
        uint32_t *w = nullptr;
        if (cudaMalloc((void **)&w, sizeof(uint32_t) * (size_t)(nw > 0 ? nw : 4)) != cudaSuccess ||
            cudaMemset(w, 0, sizeof(uint32_t) * (size_t)(nw > 0 ? nw : 4)) != cudaSuccess) {
            if (w) cudaFree(w);
            rc = -1;
        } else {
            k_pack<<<grid_of(nw), 256>>>(T, n, sep, map, b, per, nw, w);
            pb_diag_count_launch(1);
            if (cudaDeviceSynchronize() != cudaSuccess) {
                cudaFree(w);
                rc = -1;
            } else {
                *d_words = w;
                *nwords = nw;
                *bits = b;
            }
        }
    }
    if (T) cudaFree(T);
    if (map) cudaFree(map);
    if (mx) cudaFree(mx);
    return rc;
}

/* One-byte codes of the first n residues of a packed set into d_codes
 * (device, at least n bytes, 16-byte aligned), on `stream`. */
extern "C" int pb_cuda_seqdb_unpack(const uint32_t *d_words, int64_t nwords, int bits, int64_t n, uint8_t *d_codes,
                                    cudaStream_t stream)
{
    const int64_t ng = nwords / 4;
    if (ng <= 0 || n <= 0) return 0;
    const uint4 *g = reinterpret_cast<const uint4 *>(d_words);
    if (bits == 2) k_unpack<2, 16><<<grid_of(ng), 256, 0, stream>>>(g, ng, n, d_codes);
    else if (bits == 5) k_unpack<5, 6><<<grid_of(ng), 256, 0, stream>>>(g, ng, n, d_codes);
    else k_unpack<8, 4><<<grid_of(ng), 256, 0, stream>>>(g, ng, n, d_codes);
    pb_diag_count_launch(1);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

/* per pair k: query = sequence first[k], target = sequence second[k] */
extern "C" int pb_cuda_seqdb_gather(const int64_t *d_off, const int *d_len, const int *d_first, const int *d_second,
                                    int np, int64_t *qoff, int *qlen, int64_t *toff, int *tlen, cudaStream_t stream)
{
    if (np <= 0) return 0;
    k_gather_pairs<<<(np + 255) / 256, 256, 0, stream>>>(d_off, d_len, d_first, d_second, np, qoff, qlen, toff,
                                                          tlen);
    pb_diag_count_launch(1);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
