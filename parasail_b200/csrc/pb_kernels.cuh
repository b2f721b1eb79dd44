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
    /* 1: the vertical gap of the reference's serial scan forms (with or
     * without statistics; exact_pair's SCANF) */
    int scan_vgap = 0;
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
    int nletters;            /* profile alphabet size */
    int bias;                /* k_sw16<true>: H - open in the registers, scores + open */
    const Sw16Query *queries;
    const int8_t *prof_all;  /* concatenated [size][lp] int8 profiles */
    int prof_bytes;
    const int *order;        /* target ids sorted by length (desc) */
    const Sw16Task *tasks;   /* most cells first */
    const uint8_t *targets;
    const int64_t *toff;
    const int *tlen;
    uint32_t *scratch;       /* per resident warp: [maxlen][32] pass boundaries (H, F int16) */
    uint4 *colsave;          /* k_sw16, per resident thread: its strips' best columns (8 x 16 bytes) */
    pb_pair_out *out;        /* [nq][npairs] */
};

/* The int16x2 pair kernels (pb_pair16.cu). Items are pairs (pairs mode:
 * query codes per item scored through an int8 matrix) or query x target
 * products (db mode: item = query * nt + target, int8 profiles). */
struct P16Params {
    int alg, sgflags, open, gap, mmax, mmin;
    int nletters;                 /* alphabet size, <= 32 */
    int nitems;                   /* eligible items: sorted positions [0, nitems) */
    const int *order;             /* sorted position -> item */
    const int *rows, *cols;       /* per item: query rows (or prefix limit) and target columns */
    const int *task_wmax, *task_npass;
    const long long *task_bits;   /* per task: first uint4 of its direction bits in `bits` */
    uint4 *bits;
    const int8_t *mat8;           /* pairs mode: [target letter][query letter] int8, else nullptr */
    const int32_t *mat32;         /* pairs mode: the same in int32 (the statistics walk) */
    const uint8_t *qall;
    const int64_t *qoff;
    const ProfDesc *profs;        /* db mode */
    int nt;                       /* db mode: targets per query; 0 in pairs mode */
    const uint8_t *targets;
    const int64_t *toff;
    uint32_t *scratch;            /* per resident warp [maxlen + 1][32] pass boundaries (H, F int16) */
    uint4 *colsave;               /* SW ends, per resident thread: its strips' best columns (8 x 16 bytes) */
    int maxlen;
    pb_pair_out *out;
    /* traceback paths (optional): per item, steps written backwards into
     * ops[ops_off[item] .. + rows + cols), and path_info[3 * item] = steps,
     * the row and the column where the walk stopped */
    uint8_t *ops;
    const int64_t *ops_off;
    int *path_info;
};

struct P16Setup {
    int alg, open, gap, mmax, mmin, nitems, nt, max_cols;
    const int *qlen;              /* pairs mode, per item */
    const int *prof_qlen;         /* db mode, per query */
    const int *tlen;              /* per target */
    const int *qlim, *tlim;       /* per item limits, or nullptr */
    const int *group;             /* per item query group (pairs mode), or nullptr */
    /* length buckets (bucket b: max(rows, cols) <= 64 << b) whose items go
     * to the intra-task kernel instead (bit b set); 0: none */
    unsigned intra_mask;
};

/* length bucket of a pair for the schedule table */
__host__ __device__ inline int p16_bucket(int rows, int cols)
{
    int m = rows > cols ? rows : cols, b = 0;
    while (b < 31 && (64 << b) < m) ++b;
    return b;
}

/* Runs the items of batch b that fit 16-bit lanes on the pair kernels:
 * scores and ends (prefix = 0), with statistics by the direction-bit walk
 * when the job has them; or (prefix = 1, the FASTSTATS prefix pass, b
 * carrying qlim/tlim) statistics only, walked from the ends in `ends`.
 * Items outside the 16-bit bounds, and items whose width verdicts need
 * exact extremes, are listed in d_rest (*n_rest of them, device memory of
 * at least one int per item) for the exact kernel. group: optional per-item
 * query group (pairs that share a query). Synchronises st. */
int p16_pass(const pb_job &job, const pb_batch *b, int prefix, const pb_pair_out *ends, pb_pair_out *out,
             const int *group, int *d_rest, int *n_rest, cudaStream_t st,
             uint8_t *d_ops = nullptr, const int64_t *d_ops_off = nullptr, int *d_path_info = nullptr,
             unsigned intra_mask = 0);
/* Global score-only pairs (pairs mode) on the intra-task wavefront kernel
 * (pb_nwlong.cu): the listed items of b, scores and ends into out with
 * sound bounds for the width verdicts; items whose verdicts need exact
 * extremes, or that the kernel cannot take, are listed in d_rest2. */
int wave_subset(const pb_job &job, const pb_batch *b, const int *d_list, int n, pb_pair_out *out, int *d_rest2,
                int *n_rest2, cudaStream_t st);
/* can wave_subset take this job? */
bool wave_ok(const pb_job &job, const pb_batch *b);
/* the schedule table's intra-task buckets of global score-only pairs */
unsigned pb_schedule_nw_mask();
/* The exact kernel on the listed items of batch b (pairs or db mode),
 * outputs scattered to out[item]. stats / pad_rows as for the exact kernel. */
int exact_subset(const pb_batch *b, const int *d_list, int n, int stats, int pad_rows, pb_pair_out *out,
                 cudaStream_t st);

void launch_exact(const ExactParams &p, int alg, bool stats, cudaStream_t st);
/* resolution with the lane-exact rounds (pb_batch.cu) */
int resolve_rounds(const pb_job &job, const pb_lane_args &la, const pb_pair_out *o1, const pb_pair_out *o2,
                   const int *qlen, int qlen_all, const int *tlen, int n, pb_record *rec, cudaStream_t st,
                   void *work, size_t work_bytes);
pb_lane_args lane_args_of(const pb_batch *b, int q, const pb_pair_out *o1);
void launch_resolve_plain(const pb_job &job, const pb_pair_out *o1, int qlen_all, const int *tlen, int n,
                          pb_record *rec, int *need, int *counts, cudaStream_t st);
void launch_sw16(const Sw16Params &p, cudaStream_t st);

}  // namespace pb

#endif
