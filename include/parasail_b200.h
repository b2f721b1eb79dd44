/**
 * @file parasail_b200.h
 *
 * Batch extensions of parasail-b200 (additive; the reference has no batch
 * API). Each call aligns many targets against one query profile in a few
 * GPU launches and returns the same values and flags that the per-pair
 * parasail.h function of the same name returns for each pair.
 *
 * They replace the reference's per-pair driver loops, e.g.
 * apps/parasail_aligner.cpp:1694-1740 (a pfunction called per database
 * sequence under OpenMP) and tests/test_openmp.c:353-378.
 *
 * `funcname` names any in-scope profile function of parasail.h, with or
 * without the "parasail_" prefix: "sw_striped_profile_sat",
 * "parasail_nw_stats_scan_profile_16", "sg_qx_stats_striped_profile_sat", ...
 */
#ifndef PARASAIL_B200_H
#define PARASAIL_B200_H

#include <stdint.h>

#include "parasail.h"

#ifdef __cplusplus
extern "C" {
#endif

/** One pair's result, the fields of parasail_result_t and its stats. */
typedef struct parasail_b200_record {
    int score;
    int end_query;
    int end_ref;
    int flag;       /**< PARASAIL_FLAG_* exactly as the per-pair function sets them */
    int matches;    /**< 0 unless flag has PARASAIL_FLAG_STATS */
    int similar;
    int length;
    int reserved;
} parasail_b200_record_t;

/** Aligns n targets (host memory; target i is targets[offsets[i] ..
 * offsets[i] + lengths[i])) against the profile's query with the profile
 * function `funcname`. Results go to records[0..n). Returns 0 on success,
 * -1 on invalid arguments or a device error (message on stderr).
 * Replaces n calls of the reference pfunction (parasail.h:206-209). */
extern int parasail_b200_batch_profile(
        const char *funcname, const parasail_profile_t *profile,
        const char *targets, const int64_t *offsets, const int *lengths, int n,
        int open, int gap, parasail_b200_record_t *records);

/** As parasail_b200_batch_profile, but with inputs and outputs already in
 * device memory on the current CUDA device: d_codes holds the targets
 * already mapped through profile->matrix->mapper (one byte per residue),
 * d_records receives the results. Asynchronous with respect to the host
 * until it returns; it synchronizes its own stream before returning. */
extern int parasail_b200_batch_profile_device(
        const char *funcname, const parasail_profile_t *profile,
        const uint8_t *d_codes, const int64_t *d_offsets, const int *d_lengths, int n,
        int open, int gap, parasail_b200_record_t *d_records);

/** parasail_b200_batch_profile_device without any device allocation. No
 * counterpart in the reference (its CPU kernels allocate per call with
 * parasail_memalign, src/memory.c); it exists for callers that may not
 * allocate device memory while they run, e.g. a process whose device memory
 * is reserved up front by another allocator, or a latency-bound loop in which
 * a cudaMalloc/cudaFree would synchronise the device.
 *
 * Scratch comes from one fixed file-scope device array of
 * parasail_b200_noalloc_scratch_bytes() bytes (32 MiB) per device; the
 * profile (parasail_profile_create_*), d_codes, d_offsets, d_lengths and
 * d_records are the caller's and must live on the current device. The
 * batch must fit: n <= 190650 pairs, and 88 bytes per pair plus 8 bytes per
 * target residue (32 with statistics), each region rounded up to 256 bytes,
 * within the array (about 3.5 million residues score-only); a larger batch
 * is rejected (-1 and a message naming the bytes it needs), never
 * truncated. Functions that need the two-pass statistics
 * pipeline (sw_stats_striped_*) are rejected. Records equal those of
 * parasail_b200_batch_profile_device.
 *
 * The first call on a device does a one-time set-up (the array's address is
 * looked up with cudaGetSymbolAddress, and a stream is created for the
 * calling thread); make that first call before any stream capture begins.
 * The array is shared by all calls on the device: calls that overlap in time
 * on one device race on it and must be serialised by the caller. It keeps
 * the last call's contents, none of which a later call reads. */
extern int parasail_b200_batch_profile_device_noalloc(
        const char *funcname, const parasail_profile_t *profile,
        const uint8_t *d_codes, const int64_t *d_offsets, const int *d_lengths, int n,
        int open, int gap, parasail_b200_record_t *d_records);

/** Size in bytes of the per-device static scratch array of
 * parasail_b200_batch_profile_device_noalloc. */
extern size_t parasail_b200_noalloc_scratch_bytes(void);

/** Database search: every one of nq query profiles (sharing one matrix)
 * against every target, in one pipeline; a Smith-Waterman score batch runs
 * all queries in a single kernel launch. records[q * n + i] is query q
 * against target i. Replaces the reference aligner's per-query loop
 * (apps/parasail_aligner.cpp:1694-1740). */
extern int parasail_b200_batch_db(
        const char *funcname, const parasail_profile_t *const *profiles, int nq,
        const char *targets, const int64_t *offsets, const int *lengths, int n,
        int open, int gap, parasail_b200_record_t *records);

/** parasail_b200_batch_db with device-resident, already mapped targets and
 * device-resident records (see parasail_b200_batch_profile_device). */
extern int parasail_b200_batch_db_device(
        const char *funcname, const parasail_profile_t *const *profiles, int nq,
        const uint8_t *d_codes, const int64_t *d_offsets, const int *d_lengths, int n,
        int open, int gap, parasail_b200_record_t *d_records);

/** A database-search plan: parasail_b200_batch_db_device prepared once
 * and recorded as a CUDA graph. Creation does the host-side work that
 * depends only on the profiles and the target lengths (the length order of
 * the targets, the task list, the concatenated profiles, every device
 * buffer) and captures the device work of one search -- the int16x2
 * score kernel, the count of pairs past its 16-bit range and the width
 * resolution of the 8 -> 16 -> 32 chain writing d_records -- in one graph.
 * Each parasail_b200_db_plan_run replays it on the current contents of
 * d_codes (same offsets and lengths) and gives the records
 * parasail_b200_batch_db_device would give; a search with a pair past the
 * 16-bit range runs once through the full pipeline instead. Plans hold the
 * Smith-Waterman score-only functions (sw_{striped,scan}_profile_{8,16,32,sat})
 * with open > gap and profiles whose scores fit int8; creation returns NULL
 * for anything else. The buffers must outlive the plan. Replaces the
 * reference aligner's repeated searches of one database
 * (apps/parasail_aligner.cpp:1694-1740) without per-call host work. */
typedef struct parasail_b200_db_plan parasail_b200_db_plan_t;
extern parasail_b200_db_plan_t *parasail_b200_db_plan_create(
        const char *funcname, const parasail_profile_t *const *profiles, int nq,
        const uint8_t *d_codes, const int64_t *d_offsets, const int *d_lengths, int n,
        int open, int gap, parasail_b200_record_t *d_records);
extern int parasail_b200_db_plan_run(parasail_b200_db_plan_t *plan);
/** A plan run from host memory: `targets` holds the targets' characters in
 * the layout of the plan's d_offsets (nbytes of them); they are copied into
 * the plan's d_codes and mapped there through the profiles' matrix, the
 * graph replays, and the records (nq * n, query-major) are copied into the
 * host array `records`. */
extern int parasail_b200_db_plan_run_host(parasail_b200_db_plan_t *plan, const char *targets, size_t nbytes,
                                          parasail_b200_record_t *records);
extern void parasail_b200_db_plan_free(parasail_b200_db_plan_t *plan);

/** Independent pairs: query i against target i, both from host memory,
 * scored with `matrix` by the direct-form function `funcname`
 * ("nw_stats_scan_16", "sg_qx_stats_striped_16", ...). Replaces n calls of
 * the reference's direct function (parasail.h:184-188). */
extern int parasail_b200_batch_pairs(
        const char *funcname, const parasail_matrix_t *matrix,
        const char *queries, const int64_t *qoffsets, const int *qlengths,
        const char *targets, const int64_t *toffsets, const int *tlengths, int n,
        int open, int gap, parasail_b200_record_t *records);

/** parasail_b200_batch_pairs with device-resident, already mapped queries
 * and targets (codes through matrix->mapper, one byte per residue) and
 * device-resident records; query i is d_qcodes[d_qoffsets[i] ..
 * d_qoffsets[i] + d_qlengths[i]). Replaces n calls of the reference's
 * direct function (parasail.h:184-188) with inputs already on the GPU. */
extern int parasail_b200_batch_pairs_device(
        const char *funcname, const parasail_matrix_t *matrix,
        const uint8_t *d_qcodes, const int64_t *d_qoffsets, const int *d_qlengths,
        const uint8_t *d_tcodes, const int64_t *d_toffsets, const int *d_tlengths,
        int n, int open, int gap, parasail_b200_record_t *d_records);

/** All-vs-all: every pair (i, j), i < j, of n sequences (host memory;
 * sequence i is seqs[offsets[i] .. offsets[i] + lengths[i])), sequence i as
 * the query (the profile side) and j as the target, scored with `matrix`
 * by `funcname` (profile or direct form, e.g. "sw_stats_striped_profile_32";
 * both forms return the same results). records[p] receives pair p of the
 * upper triangle in row-major order: p = i*n - i*(i+1)/2 + (j - i - 1), n(n-1)/2
 * records in all. Replaces the reference aligner's all-against-all mode,
 * which enumerates these pairs (apps/parasail_aligner.cpp:1441-1447), builds
 * one profile per query sequence (:1543-1567) and calls the pfunction per
 * pair under OpenMP (:1714-1740). */
extern int parasail_b200_batch_all(
        const char *funcname, const parasail_matrix_t *matrix,
        const char *seqs, const int64_t *offsets, const int *lengths, int n,
        int open, int gap, parasail_b200_record_t *records);

/** parasail_b200_batch_all with device-resident, already mapped sequences
 * and device-resident records. */
extern int parasail_b200_batch_all_device(
        const char *funcname, const parasail_matrix_t *matrix,
        const uint8_t *d_codes, const int64_t *d_offsets, const int *d_lengths, int n,
        int open, int gap, parasail_b200_record_t *d_records);

/** Trace results of n independent pairs (host memory) with a trace
 * function of parasail.h (the names parasail_b200_batch_pairs_cigar takes,
 * and their _profile forms) in one GPU pipeline: results[i] is what the
 * trace function returns for pair i -- usable with
 * parasail_result_get_cigar[_extra], parasail_result_get_traceback[_extra]
 * and parasail_traceback_generic*, freed with parasail_result_free; a
 * saturated 8/16-bit result carries no alignment -- or NULL (with a
 * message) when the pair's scores leave the int16 range of the traceback
 * kernel. Replaces n calls of the trace function (the reference
 * aligner's trace outputs, apps/parasail_aligner.cpp:2210-2550). */
extern int parasail_b200_batch_pairs_trace(
        const char *funcname, const parasail_matrix_t *matrix,
        const char *queries, const int64_t *qoffsets, const int *qlengths,
        const char *targets, const int64_t *toffsets, const int *tlengths, int n,
        int open, int gap, parasail_result_t **results);

/** CIGARs of n independent pairs (host memory) with a trace function of
 * parasail.h: "sw_trace", "nw_trace_scan", "sg_qx_trace_striped_32",
 * "sg_de_trace_scan_16", "nw_trace_striped_sat", ... (serial forms and the
 * striped/scan forms at 8, 16, 32 bits and _sat; with or without the
 * "parasail_" prefix). For pair i: records[i] holds the score, ends and
 * flags the trace function returns; its CIGAR -- the one
 * parasail_result_get_cigar gives for that result (src/cigar.c), BAM
 * encoding -- goes to cigars[o_i ..] with o_i = sum over k < i of
 * qlengths[k] + tlengths[k] (the buffer holds sum over all pairs), its
 * element count to cigar_lengths[i] (-1 when the result is saturated or
 * the pair's scores leave the int16 range of the traceback kernel), and
 * the first aligned positions
 * to beg_query[i], beg_ref[i]. Replaces n calls of a trace function
 * followed by parasail_result_get_cigar. */
extern int parasail_b200_batch_pairs_cigar(
        const char *funcname, const parasail_matrix_t *matrix,
        const char *queries, const int64_t *qoffsets, const int *qlengths,
        const char *targets, const int64_t *toffsets, const int *tlengths, int n,
        int open, int gap, parasail_b200_record_t *records, uint32_t *cigars,
        int *cigar_lengths, int *beg_query, int *beg_ref);

/* ---- long global alignments and the learned band ---------------------- */

/** Global alignment score of each long pair (query i against target i),
 * the value of the reference's parasail_nw_scan_profile_32 for the pair
 * (src/nw_scan_avx2_256_32.c); one warp per pair on the GPU. Square matrix
 * of at most 32 letters with |scores| <= 127. */
extern int parasail_b200_nw_long(
        const parasail_matrix_t *matrix,
        const char *queries, const int64_t *qoffsets, const int *qlengths,
        const char *targets, const int64_t *toffsets, const int *tlengths, int n,
        int open, int gap, int *scores);

/** The learned-band model: a 258 -> 128 -> 128 -> 2 MLP (ReLU, BF16 weights,
 * FP32 accumulation) mapping a pair's k = 8 diagonal-offset histogram (256
 * bins) and both lengths to a band centre and half-width. Bands are placed
 * at the certificate's own centre, (n - m) / 2 diagonals, with the predicted
 * half-width; the centre output is trained but not used for them. */
typedef struct parasail_b200_band_model parasail_b200_band_model_t;

typedef struct parasail_b200_band_stats {
    long long pairs;        /**< pairs aligned */
    long long certified;    /**< pairs whose banded score passed the certificate */
    long long fallback;     /**< pairs whose first band failed the certificate and reran on a wider one */
    double band_cells;      /**< DP cells computed: first bands of all pairs, second bands of the reruns */
} parasail_b200_band_stats_t;

extern parasail_b200_band_model_t *parasail_b200_band_model_new(unsigned seed);
extern void parasail_b200_band_model_free(parasail_b200_band_model_t *model);
/** Sizes of the model: inputs, hidden units, outputs, weight and bias counts. */
extern int parasail_b200_band_model_sizes(int *n_in, int *n_hidden, int *n_out, int *n_weights, int *n_biases);
/** FP32 master weights (w1 [128][258] | w2 [128][128] | w3 [2][128]) and
 * biases (b1 | b2 | b3), to or from host memory. */
extern int parasail_b200_band_model_get(const parasail_b200_band_model_t *model, float *weights, float *biases);
extern int parasail_b200_band_model_set(parasail_b200_band_model_t *model, const float *weights, const float *biases);
/** Input features ([n][258]) of DNA pairs. */
extern int parasail_b200_band_features(
        const parasail_matrix_t *matrix,
        const char *queries, const int64_t *qoffsets, const int *qlengths,
        const char *targets, const int64_t *toffsets, const int *tlengths, int n, float *features);
/** Gradients of the training loss over a batch of features/targets
 * (squared error on the centre, pinball loss with quantile tau on the
 * half-width), computed by the GPU backward kernels; for gradient checks. */
extern int parasail_b200_band_model_gradients(
        const parasail_b200_band_model_t *model, const float *x, const float *target, int n, float tau,
        float *grad_weights, float *grad_biases, float *loss);
/** Trains on the GPU with Adam: labels are the smallest certifiable band of
 * each pair's optimal score from the full-DP kernel. The last tenth of the
 * pairs (when n >= 20) is held out of the gradient steps and then chooses
 * the band scaling: the widen factor (of 1.0 ... 3.0) with the least
 * expected DP work, the band cells of every held-out pair plus, for each
 * pair whose band would fail the certificate, six times the cells of the
 * rerun band (its band joined with its label band; a rerun lengthens its
 * pair's latency, which bounds the launch). */
extern int parasail_b200_band_model_train(
        parasail_b200_band_model_t *model, const parasail_matrix_t *matrix,
        const char *queries, const int64_t *qoffsets, const int *qlengths,
        const char *targets, const int64_t *toffsets, const int *tlengths, int n,
        int open, int gap, int epochs, int batch, float lr, float *final_loss);
/** The band scaling chosen at training (widen factor, slack diagonals). */
extern void parasail_b200_band_model_scaling(const parasail_b200_band_model_t *model, float *widen, int *slack);
/** Global alignment scores through the learned band: predicted band
 * (centred on (n - m) / 2 diagonals, predicted half-width scaled by
 * `widen`, plus `slack` diagonals; widen <= 0 and
 * slack < 0 take the scaling chosen at training), banded DP with the
 * exactness certificate checked inside the launch. A pair whose band fails
 * it reruns at once, in the same launch, on its band widened by the label
 * band of its own banded cost, which always passes. scores[] always equals
 * parasail_b200_nw_long's; band_lo/band_hi receive the band each pair
 * finally used, either may be NULL; stats->fallback counts the reruns and
 * stats->band_cells every DP cell the call computed. */
extern int parasail_b200_nw_learned_band(
        const parasail_b200_band_model_t *model, const parasail_matrix_t *matrix,
        const char *queries, const int64_t *qoffsets, const int *qlengths,
        const char *targets, const int64_t *toffsets, const int *tlengths, int n,
        int open, int gap, float widen, int slack,
        int *scores, int *band_lo, int *band_hi, parasail_b200_band_stats_t *stats);
/** The same scores without a model: every pair starts on the band of
 * half-width w0 around (n - m) / 2 diagonals, and a pair whose banded score
 * fails the exactness certificate reruns on a band twice as wide, until it
 * passes or the band covers the whole matrix. The non-learned baseline of
 * parasail_b200_nw_learned_band; stats as there (fallback = pairs that
 * needed more than one band, band_cells = cells of every round). */
extern int parasail_b200_nw_doubling_band(
        const parasail_matrix_t *matrix,
        const char *queries, const int64_t *qoffsets, const int *qlengths,
        const char *targets, const int64_t *toffsets, const int *tlengths, int n,
        int open, int gap, int w0, int *scores, parasail_b200_band_stats_t *stats);
/** Banded DP with caller-given bands and the certificate, no fallback:
 * certified[i] = 1 when scores[i] is provably the full optimum. */
extern int parasail_b200_nw_banded_certified(
        const parasail_matrix_t *matrix,
        const char *queries, const int64_t *qoffsets, const int *qlengths,
        const char *targets, const int64_t *toffsets, const int *tlengths, int n,
        int open, int gap, const int *band_lo, const int *band_hi, int *scores, int *certified);

/** parasail_nw_banded (parasail.h:293-296) for n independent pairs in one
 * launch: scores[i] is the value parasail_nw_banded(query i, target i,
 * open, gap, k, matrix) returns. The band of src/nw_banded.c:92-97 -- query
 * positions [j + s1Len - s2Len - k, j + k] of target column j when s1Len <=
 * s2Len, [j - k, j + s1Len - s2Len + k] otherwise -- runs as a band of
 * diagonals on the wavefront kernel. Square matrix of at most 32 letters
 * with |scores| <= 127; k > 0. */
extern int parasail_b200_nw_banded_batch(
        const parasail_matrix_t *matrix,
        const char *queries, const int64_t *qoffsets, const int *qlengths,
        const char *targets, const int64_t *toffsets, const int *tlengths, int n,
        int open, int gap, int k, int *scores);

/** The schedule table of global score-only pair batches: bit b set sends
 * the pairs of length bucket b (the longer sequence at most 64 << b
 * residues) to the intra-task wavefront kernel (a team of warps per pair)
 * instead of the inter-task pair kernel (one thread per pair). Read on
 * first use from $PARASAIL_B200_SCHEDULE or from schedule.txt beside the
 * library, which the tuner (parasail_b200/tune.py) writes from measured
 * rates per bucket; the reference has no counterpart (its one-time ISA
 * dispatch, src/sw_dispatch.c:4082-4121, picks kernels by CPU features,
 * not by size). */
extern unsigned parasail_b200_schedule_get(void);
extern void parasail_b200_schedule_set(unsigned intra_mask);

/** A packed sequence set resident on the device: the '$'-separated text of
 * parasail_sequences_pack (every sequence followed by `sentinel`), mapped
 * through `matrix`'s mapper and stored at 2 bits a residue when every code
 * is below 4, 5 bits below 32, else 8 (parasail_b200_seqdb_bits). Sequence
 * k is text[offsets[k] .. offsets[k] + lengths[k]) (host arrays of the
 * set). NULL with a message on failure. The reference keeps the packed
 * text in host memory (apps/parasail_aligner.cpp:1077-1178). */
typedef struct parasail_b200_seqdb parasail_b200_seqdb_t;
extern parasail_b200_seqdb_t *parasail_b200_seqdb_create(
        const char *text, size_t size, char sentinel, const parasail_matrix_t *matrix);
extern void parasail_b200_seqdb_free(parasail_b200_seqdb_t *db);
extern int parasail_b200_seqdb_count(const parasail_b200_seqdb_t *db);
extern int parasail_b200_seqdb_bits(const parasail_b200_seqdb_t *db);
/** text characters of the set, sentinels included */
extern size_t parasail_b200_seqdb_size(const parasail_b200_seqdb_t *db);
/** device bytes of the packed residues */
extern size_t parasail_b200_seqdb_device_bytes(const parasail_b200_seqdb_t *db);
extern const int64_t *parasail_b200_seqdb_offsets(const parasail_b200_seqdb_t *db);
extern const int *parasail_b200_seqdb_lengths(const parasail_b200_seqdb_t *db);
/** One-byte codes of the whole text (parasail_b200_seqdb_size bytes, 16-byte
 * aligned device buffer; sentinels as code 0). */
extern int parasail_b200_seqdb_unpack(const parasail_b200_seqdb_t *db, uint8_t *d_codes);
/** Pairs of a set's sequences: query first[k] against target second[k]
 * with the direct or profile function `funcname` (score-only or stats,
 * any algorithm and width). The pair list is cut into batches whose device
 * footprint (about 512 bytes a pair plus the set's unpacked codes) fits
 * `budget` bytes (0: 4 GiB); records[k] as parasail_b200_batch_pairs gives
 * them. The batch loop of the reference aligner
 * (apps/parasail_aligner.cpp:414-573, :1585-1760). */
extern int parasail_b200_batch_pairs_seqdb(
        const char *funcname, const parasail_matrix_t *matrix, const parasail_b200_seqdb_t *db,
        const int *first, const int *second, size_t npairs, int open, int gap, size_t budget,
        parasail_b200_record_t *records);

/** Candidate pairs of the reference aligner's exact-match filter
 * (apps/parasail_aligner.cpp:1316-1420, :1816-1904, its enhanced suffix
 * array walked for maximal pairs of at least `cutoff` characters): the
 * pairs of sequences of `text` -- every sequence followed by `sentinel`,
 * the text ending with one (parasail_sequences_pack) -- that share a
 * substring of `cutoff` characters, computed on the GPU by sorting every
 * cutoff-window of the text. db_chars < 0: all against all, each pair
 * (smaller id, larger id); db_chars >= 0: the first db_chars characters are
 * the database file and only (query id, database id) pairs are kept, ids
 * counting all sequences of the text. *pairs (malloc'd, freed by the
 * caller) holds 2 * *count ints, the pairs in ascending order: the
 * reference's std::set. Returns 0, or -1 with a message. */
extern int parasail_b200_candidate_pairs(
        const char *text, size_t size, char sentinel, int cutoff, long db_chars,
        int **pairs, size_t *count);

/** Diagnostics: number of this library's kernel launches so far. */
extern long parasail_b200_kernel_launches(void);
/** Diagnostics: summed device time (ms) of the int16x2 Smith-Waterman score
 * kernel, measured with CUDA events on its stream; *launches its count. */
extern double parasail_b200_sw16_kernel_ms(long *launches);
/** Diagnostics: zero the two counters above. */
extern void parasail_b200_reset_counters(void);
/** Host wall time (ms) of the phases of this thread's last
 * parasail_b200_nw_learned_band call: [0] features, MLP and bands, [1]
 * banded DP with the in-launch certificate and reruns, [2] cell counting,
 * [3] unused (0), [4] upload of the pairs. */
extern void parasail_b200_band_phase_ms(double *out5);
/** Measured lane-operations per second of the DPX int16x2 add-max pipe on
 * the current device (the integer roofline of the DP kernels). */
extern double parasail_b200_dpx_peak(void);

#ifdef __cplusplus
}
#endif

#endif /* PARASAIL_B200_H */
