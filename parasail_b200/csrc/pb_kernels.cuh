/*
 * pb_kernels.cuh -- device-side parameter blocks shared by the CUDA files.
 */
#ifndef PARASAIL_B200_PB_KERNELS_CUH
#define PARASAIL_B200_PB_KERNELS_CUH

#include <cstdint>
#include <cuda_runtime.h>

#include "pb_cuda.h"
#include "pb_resolve.h"

namespace pb {

/* Device copy of one profile's descriptor. */
struct ProfDesc {
    const int32_t *prof;    /* [size][lp] */
    const int8_t *prof8;    /* [size][lp] or nullptr */
    const uint8_t *qcodes;  /* [lp] */
    int qlen, lp, size, pad_;
};

struct ExactParams {
    int alg, sgflags, open, gap, pad_rows, npairs;
    const ProfDesc *profs;
    const int *prof_index;
    const uint8_t *targets;
    const int64_t *toff;
    const int *tlen;
    const int *qlim;
    const int *tlim;
    int *scratch;
    const int64_t *soff;     /* per pair scratch offset in ints */
    pb_pair_out *out;
    /* pairs mode: per-pair query codes scored through a square matrix
     * mat[target letter * msize + query letter] instead of a profile */
    const int32_t *mat;
    int msize;
    const uint8_t *qall;
    const int64_t *qoff;
    const int *qlen;
    /* work item k aligns pair order[k] (nullptr: pair k) */
    const int *order = nullptr;
    /* > 0: pair index = query * nt + target, every query of profs against
     * the same nt targets (outputs query-major); 0: one pair per target */
    int nt = 0;
};

/* the exact kernel with one warp per pair (pb_exact_warp.cu): items
 * order[0..nitems) of p, which uses p.nt query-major pairs */
void launch_exact_warp(const ExactParams &p, int alg, bool stats, int nitems, cudaStream_t st);
/* query rows of one of its passes */
int exact_warp_pass_rows(bool stats);

struct Sw16Query {
    int prof_off;            /* byte offset of the query's int8 profile in shared memory */
    int qlen, lp, posmax;
};

struct Sw16Task {
    int q;                   /* query index */
    int first;               /* first position in the length-sorted target order */
};

struct Sw16Params {
    int open, gap, npairs, nq, ntasks, maxlen;
    int nteam;               /* tasks [0, nteam) are run by a whole block */
    const Sw16Query *queries;
    const int8_t *prof_all;  /* concatenated [size][lp] int8 profiles */
    int prof_bytes;
    const int *order;        /* target ids sorted by length (desc) */
    const Sw16Task *tasks;   /* most cells first */
    const uint8_t *targets;
    const int64_t *toff;
    const int *tlen;
    uint32_t *scratch;       /* per resident warp: [maxlen][32] uint2 */
    pb_pair_out *out;        /* [nq][npairs] */
};

void launch_exact(const ExactParams &p, int alg, bool stats, cudaStream_t st);
/* resolution with the lane-exact rounds (pb_batch.cu) */
int resolve_rounds(const pb_job &job, const pb_lane_args &la, const pb_pair_out *o1, const pb_pair_out *o2,
                   const int *qlen, int qlen_all, const int *tlen, int n, pb_record *rec, cudaStream_t st,
                   void *work, size_t work_bytes);
pb_lane_args lane_args_of(const pb_batch *b, int q, const pb_pair_out *o1);
void launch_sw16(const Sw16Params &p, cudaStream_t st);

}  // namespace pb

#endif
