/*
 * pb_cuda.h -- the thin C ABI between the parasail-b200 host library (C) and
 * its CUDA kernels. Plain pointers, sizes and PODs only.
 *
 * Terminology follows parasail: s1 is the query (DP rows, i), s2 the
 * database/reference sequence (DP columns, j); a profile is the query scored
 * against every alphabet letter; a pair is one query/target alignment.
 */
#ifndef PARASAIL_B200_PB_CUDA_H
#define PARASAIL_B200_PB_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { PB_SW = 0, PB_NW = 1, PB_SG = 2 };
/* semi-global free ends; same order as the reference's SG_CASE tuples
 * (src/sg_helper.h:53-63: s1_beg, s1_end, s2_beg, s2_end) */
enum { PB_S1_BEG = 1, PB_S1_END = 2, PB_S2_BEG = 4, PB_S2_END = 8 };

/* Device-resident query profile. prof32[k * lp + i] = score of query
 * position i against alphabet letter k (0 for i >= qlen), the value layout of
 * the reference's striped profile (src/memory_avx2.c:111-127) before
 * striping. prof8 is the same table in int8 when every value fits. */
typedef struct pb_device_profile {
    int qlen;            /* query length (rows) */
    int lp;              /* padded row count, multiple of 64, >= qlen + 32 */
    int size;            /* alphabet size */
    int fits8;           /* 1 when prof8 is valid */
    int mmax, mmin;      /* matrix max / min (parasail_matrix_t.max/min) */
    int32_t *d_prof32;   /* [size][lp] */
    int8_t  *d_prof8;    /* [size][lp] or NULL */
    uint8_t *d_qcodes;   /* [lp], query codes, 255 past qlen */
    int device;          /* CUDA device ordinal the profile lives on */
} pb_device_profile;

/* Per-pair output of the exact kernels. All DP values are exact 32-bit.
 * Predicate statistics: "real" = query rows [0, qlim), pad[k] = padded rows
 * of region k: [qlim, ceil8), [ceil8, ceil16), [ceil16, ceil32) where ceilN
 * rounds qlim up to a multiple of N (the row padding of the reference's
 * 32-, 16- and 8-bit AVX2 layouts). Fields that were not tracked hold
 * INT32_MAX (for minima) or INT32_MIN (for maxima). */
typedef struct pb_pair_out {
    int score, end_query, end_ref;
    int matches, similar, length;
    int max_h;                 /* max H over real and padded rows */
    int min_h_real;
    int max_stat_real;         /* max of matches/similar/length */
    int min_f_real;            /* min vertical-gap value */
    int min_h_pad[3];
    int max_stat_pad[3];
    int min_f_pad[3];
    int status;                /* 0 ok; PB_ST_* bits */
} pb_pair_out;

enum {
    PB_ST_OVERFLOW16 = 1,   /* a 16-bit lane left its exact range: rerun in 32 bits */
    PB_ST_BADCODE = 2,      /* a residue code outside the profile alphabet */
    PB_ST_BOUNDED = 4       /* the extremes fields are sound bounds, not exact values */
};

/* A batch of pairs sharing one alignment mode. Every pointer is DEVICE
 * memory except `prof` (host struct describing device memory). */
typedef struct pb_batch {
    int alg, sgflags, stats;
    int open, gap;
    int pad_rows;              /* 0: real rows only; 8/16/32: also compute the
                                  padded rows up to a multiple of this */
    int npairs;
    const pb_device_profile *const *profs;  /* host array, nprofs entries */
    int nprofs;
    const int *d_prof_index;   /* per pair profile index, or NULL (all use 0) */
    const uint8_t *d_targets;  /* concatenated target codes */
    const int64_t *d_toff;     /* per pair offset into d_targets */
    const int *d_tlen;         /* per pair target length */
    const int *d_qlim;         /* per pair row limit (prefix pass) or NULL */
    const int *d_tlim;         /* per pair column limit or NULL */
    pb_pair_out *d_out;        /* per pair output */
    /* pairs mode (nprofs == 0): per-pair queries scored through a square
     * matrix table on the device, mat[target letter * msize + query letter] */
    const int32_t *d_mat;
    int msize, mmax, mmin;
    const uint8_t *d_qall;
    const int64_t *d_qoff;
    const int *d_qlen;
    /* pairs mode, optional: per-pair query id; pairs with one id share the
     * query (e.g. the rows of an all-vs-all batch) */
    const int *d_qgroup;
    /* 1: the vertical gap of the reference's serial scan forms (src/nw_scan.c
     * etc.: F extends from max(diagonal, E), not from H), score only, on the
     * single-pair exact path */
    int scan_vgap;
} pb_batch;

/* --- device management ------------------------------------------------- */
int pb_cuda_init(void);                     /* 0 ok, <0 no usable GPU */
const char *pb_cuda_last_error(void);
void pb_cuda_set_error(const char *what, const char *detail);
int pb_cuda_device_count(void);

/* --- profiles ------------------------------------------------------------ */
/* table: square (size*size, row = target letter, col = query letter as in
 * the reference profile builder) or pssm (length*size, row = query pos). */
int pb_cuda_profile_create(const int *table, int is_pssm, int size,
                           const uint8_t *qcodes, int qlen, int mmax, int mmin,
                           pb_device_profile *out);
void pb_cuda_profile_destroy(pb_device_profile *p);

/* --- memory helpers (device, stream-ordered on the library stream) -------- */
void *pb_cuda_malloc(size_t bytes);
void pb_cuda_free(void *p);
int pb_cuda_h2d(void *dst, const void *src, size_t bytes);
int pb_cuda_d2h(void *dst, const void *src, size_t bytes);
/* all work on the device, including kernels on the legacy default stream */
int pb_cuda_device_sync(void);
int pb_cuda_memset(void *p, int v, size_t bytes);
/* n host characters to the device, mapped to codes there through mapper256 */
int pb_cuda_h2d_mapped(uint8_t *d_buf, const char *h_chars, int64_t n, const uint8_t *mapper256);
int pb_cuda_sync(void);

/* --- alignment ------------------------------------------------------------- */
/* Exact int32 kernel: any mode, stats, padded-row predicate statistics. */
int pb_cuda_align_exact(const pb_batch *b);
/* every profile of b against every target, one launch, outputs query-major */
int pb_cuda_align_exact_db(const pb_batch *b);
/* Fast Smith-Waterman score-only kernel: two pairs per thread in packed
 * int16x2 lanes. Pairs whose values leave the 16-bit range come back with
 * PB_ST_OVERFLOW16 and must be rerun with pb_cuda_align_exact. Only
 * score/end_query/end_ref/max_h/status are written. */
int pb_cuda_align_sw16(const pb_batch *b);
/* The same for nprofs queries against the same targets in one launch;
 * d_out_all[q * npairs + i]. */
int pb_cuda_align_sw16_multi(const pb_batch *b, pb_pair_out *d_out_all);

/* parasail_nw_banded for one pair: the reference's band recurrence
 * (src/nw_banded.c) on the GPU; h_s2 holds mapped target codes. */
int pb_cuda_nw_banded(const pb_device_profile *dp, const uint8_t *h_s2, int s2Len,
                      int open, int gap, int k, int *score);

/* The batch pipeline: score pass, FASTSTATS prefix pass when the job is SW
 * stats striped, and the reference's width resolution of every pair, all on
 * the device. tmpl carries the device inputs; d_rec receives npairs records.
 * (pb_job and pb_record are defined in pb_resolve.h.) */
struct pb_job;
struct pb_record;
int pb_cuda_batch_run(const struct pb_job *job, const pb_batch *tmpl, struct pb_record *d_rec);
/* The same from host memory: characters are copied and mapped to codes on
 * the device through mapper256 (the matrix mapper as bytes); queries are
 * given in pairs mode only (tmpl->nprofs == 0). */
int pb_cuda_batch_host(const struct pb_job *job, const pb_batch *tmpl, const uint8_t *mapper256,
                       const char *h_targets, const int64_t *h_toff, const int *h_tlen,
                       const char *h_queries, const int64_t *h_qoff, const int *h_qlen,
                       int n, struct pb_record *h_rec);

/* Database-search plans (pb_sw16.cu): SW score-only searches recorded
 * once as a CUDA graph and replayed. */
int pb_cuda_db_plan_create(const struct pb_job *job, const pb_batch *b, struct pb_record *d_rec, void **plan);
int pb_cuda_db_plan_run(void *plan);
int pb_cuda_db_plan_run_host(void *plan, const char *h_chars, size_t nbytes, uint8_t *d_codes,
                             const uint8_t *mapper256, struct pb_record *h_rec);
void pb_cuda_db_plan_free(void *plan);

/* All-vs-all: the upper triangle of n device-resident sequences (codes),
 * pair p = (i, j), i < j, row-major, query i against target j, run as a
 * pairs batch (tmpl in pairs mode: matrix table set, queries unset);
 * d_rec receives n(n-1)/2 records. The host form copies and maps the
 * characters first and copies the records back. */
int pb_cuda_batch_all(const struct pb_job *job, const pb_batch *tmpl, const uint8_t *d_codes,
                      const int64_t *d_off, const int *d_len, int n, struct pb_record *d_rec);
int pb_cuda_batch_all_host(const struct pb_job *job, const pb_batch *tmpl, const uint8_t *mapper256,
                           const char *h_seqs, const int64_t *h_off, const int *h_len, int n,
                           struct pb_record *h_rec);

/* Traceback paths of independent pairs from host memory on the int16x2
 * pair kernels (pb_pair16.cu); see the definition for the outputs. */
int pb_cuda_trace_pairs_host(const struct pb_job *job, const pb_batch *tmpl, const uint8_t *mapper256,
                             const char *h_q, const int64_t *h_qoff, const int *h_qlen,
                             const char *h_t, const int64_t *h_toff, const int *h_tlen, int n,
                             int *h_ends, uint8_t *h_ops, const int64_t *h_ops_off, int *h_info);

/* Lane-exact emulation of the reference's 8/16-bit striped kernels
 * (pb_lane.cu) for the pairs listed in d_list. kind: 0 nw/sg score-only,
 * 1 nw/sg with statistics, 2 the SW statistics kernel on the FASTSTATS prefix
 * [0, o1.end_query] x [0, o1.end_ref], 3 sw score-only, 4/5 the nw/sg
 * trace kernels' saturation flag (striped/scan), 6/7 nw/sg and sw scan
 * score-only, 8 nw/sg scan with statistics. Profile mode (prof, qcodes, lp, qlen)
 * or matrix mode (mat, msize, qall, qoff, qlens). */
/* One lane-exact kernel result; valid = the width of the kernel that
 * wrote it (0: none). */
typedef struct pb_lane_res {
    int score, end_query, end_ref, matches, similar, length, saturated, valid;
} pb_lane_res;

typedef struct pb_lane_args {
    int kind, sgflags, open, gap, mmax, mmin, max_qlen;
    const int32_t *prof; const uint8_t *qcodes; int lp, qlen, size;
    const int32_t *mat; int msize; const uint8_t *qall; const int64_t *qoff; const int *qlens;
    const uint8_t *targets; const int64_t *toff; const int *tlen;
    const pb_pair_out *o1;
} pb_lane_args;

/* scratch: NULL to allocate from the stream's pool, else at least
 * pb_cuda_lane_scratch_per_warp bytes (fewer warps run when it is small).
 * stream: a cudaStream_t. Asynchronous. Returns 0, -1 on a device error or
 * invalid arguments, -3 when the given scratch is smaller than one warp's
 * arrays. */
int pb_cuda_lane_run(int bits, const pb_lane_args *a, const int *d_list, int nlist, pb_lane_res *d_res,
                     void *scratch, size_t scratch_bytes, void *stream);
size_t pb_cuda_lane_scratch_per_warp(int bits, int kind, int max_qlen);
/* One pair from host memory (the single-call entry points): target codes
 * and the score pass's output on the host, result to *res. Synchronous. */
struct pb_mode;
int pb_cuda_lane_pair(int bits, const pb_device_profile *dp, const struct pb_mode *m, const uint8_t *h_codes,
                      int tlen, const pb_pair_out *h_o1, pb_lane_res *h_res);

/* The saturation flag of the reference's 8/16-bit nw/sg trace kernels
 * (kind 4 striped, 5 scan) for the listed pairs of a host batch (host
 * characters, mapped on the device; square matrix h_mat[msize*msize]):
 * sat[k] for pair list[k]. Synchronous. */
int pb_cuda_trace_sat_host(int bits, int kind, int sgflags, int open, int gap, int mmax, int mmin,
                           const int32_t *h_mat, int msize, const uint8_t *map, const char *q, const int64_t *qoff,
                           const int *qlen, const char *t, const int64_t *toff, const int *tlen, const int *list,
                           int nlist, int *sat);

/* One profile against device-resident targets with no device allocation
 * (pb_noalloc.cu): the exact kernel and the width resolution with their
 * scratch in a fixed-size file-scope device array. Jobs that need the
 * FASTSTATS prefix pass are not handled. */
int pb_cuda_noalloc_run(const struct pb_job *job, const pb_batch *b, struct pb_record *d_rec);
size_t pb_cuda_noalloc_capacity(void);
int pb_cuda_noalloc_max_pairs(void);
const char *pb_cuda_noalloc_last_error(void);

/* Global alignment scores of long pairs (pb_nwlong.cu): one warp per pair,
 * device-resident codes, square matrix h_mat (msize x msize, row = target
 * letter, |values| <= 127, msize <= 32); optional per-pair band of
 * diagonals [d_lo, d_hi] (i - j), cells outside it unreachable. */
int pb_cuda_nw_long(int npairs, int open, int gap, const int32_t *h_mat, int msize,
                    const uint8_t *d_q, const int64_t *d_qoff, const int *d_qlen,
                    const uint8_t *d_t, const int64_t *d_toff, const int *d_tlen,
                    const int *d_lo, const int *d_hi, int maxlen, int *d_score);
/* The same with a band per pair and the exactness certificate inside the
 * launch (a = the matrix's largest score): a pair whose banded score fails
 * it is rerun at once, by the same team, on its band widened by the label
 * band of its own cost, which always passes. d_lo/d_hi are updated to the
 * band each pair finally used; d_rounds[i] is set to 2 for those pairs
 * (and left untouched for the others). */
int pb_cuda_nw_long_cert(int npairs, int open, int gap, const int32_t *h_mat, int msize, int a,
                         const uint8_t *d_q, const int64_t *d_qoff, const int *d_qlen,
                         const uint8_t *d_t, const int64_t *d_toff, const int *d_tlen,
                         int *d_lo, int *d_hi, int maxlen, int *d_score, int *d_rounds);

/* diagnostics (pb_diag.cu) */
void pb_diag_count_launch(long n);
void pb_diag_sw16_time(double ms);

/* Host convenience: copy targets to the device, run, copy results back. */
/* Single pairs (the one-pair calls of parasail.h) through a per-thread
 * device arena: one upload, one launch, one download. pb_cuda_exact_single:
 * the exact kernel (qlim/tlim > 0: a prefix). pb_cuda_sw_single: the SW
 * score wavefront kernel (int8 profile required; -2 when dp has none). */
void *pb_cuda_stream(void);   /* the calling thread's stream (a cudaStream_t) */
/* raise (never lower) a kernel's dynamic shared-memory limit; 0 or -1 */
int pb_raise_smem(const void *func, int bytes);
char *pb_single_arena(size_t bytes, size_t host_bytes, char **host);
int pb_cuda_exact_single(const pb_batch *tmpl, const uint8_t *h_codes, int tlen, int qlim, int tlim,
                         pb_pair_out *h_out);
int pb_cuda_sw_single(const pb_device_profile *dp, int open, int gap, const uint8_t *h_codes, int tlen,
                      pb_pair_out *h_out);
int pb_cuda_align_host(int kernel /* 0 exact, 1 sw16 */, const pb_batch *tmpl,
                       const uint8_t *h_targets, const int64_t *h_toff,
                       const int *h_tlen, const int *h_qlim, const int *h_tlim,
                       const int *h_prof_index, int npairs, pb_pair_out *h_out);

#ifdef __cplusplus
}
#endif
#endif
