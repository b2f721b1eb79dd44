/*
 * band.c -- long global alignments, full and with a learned band
 * (include/parasail_b200.h), host side.
 *
 * The plain path (parasail_b200_nw_long) returns the global score of every
 * pair, the value the reference's parasail_nw_scan_profile_32 returns. The
 * learned path predicts a band per pair from k-mer diagonal histograms with
 * a small MLP, aligns inside the band, keeps the banded score only when the
 * exactness certificate holds and reruns every other pair on the full DP;
 * its scores therefore always equal the plain path's.
 */
#include <stdlib.h>
#include <time.h>
#include <string.h>

#include "pb_internal.h"
#include "parasail_b200.h"

struct pb_band_model;
struct pb_band_model *pb_cuda_band_model_new(unsigned seed);
void pb_cuda_band_model_free(struct pb_band_model *m);
int pb_cuda_band_model_get(const struct pb_band_model *m, float *w, float *b);
int pb_cuda_band_model_set(struct pb_band_model *m, const float *w, const float *b);
int pb_cuda_band_sizes(int *n_in, int *n_hidden, int *n_out, int *nw, int *nb);
int pb_cuda_band_features(int npairs, const uint8_t *d_q, const int64_t *d_qoff, const int *d_qlen,
                          const uint8_t *d_t, const int64_t *d_toff, const int *d_tlen, float *d_feat);
int pb_cuda_band_forward(const struct pb_band_model *m, int n, const float *d_x, float *d_h1, float *d_h2,
                         float *d_y);
int pb_cuda_band_gradients(const struct pb_band_model *m, int n, const float *d_x, const float *d_target,
                           float tau, float *d_gw, float *d_gb, float *loss_out);
int pb_cuda_band_adam(struct pb_band_model *m, const float *d_gw, const float *d_gb, float lr);
int pb_cuda_band_labels(int npairs, int a, int open, int ext, const int *d_qlen, const int *d_tlen,
                        const int *d_score, float *d_target, int *d_lo, int *d_hi);
int pb_cuda_band_from_pred(int npairs, const int *d_qlen, const int *d_tlen, const float *d_y,
                           float widen, int slack, int *d_lo, int *d_hi);
int pb_cuda_band_certify(int npairs, int a, int open, int ext, const int *d_qlen, const int *d_tlen,
                         const int *d_lo, const int *d_hi, const int *d_score, int *d_cert, int *h_failures);
int pb_cuda_band_tune(struct pb_band_model *m, int n, const float *d_x, const int *d_qlen, const int *d_tlen,
                      const int *d_lab_lo, const int *d_lab_hi, float *chosen);
void pb_cuda_band_scaling(const struct pb_band_model *m, float *widen, int *slack);
int pb_cuda_band_select(int npairs, const int *d_rounds, const int *d_lo, const int *d_hi, int *sel_lo, int *sel_hi);
int pb_cuda_band_cells(int npairs, const int *d_qlen, const int *d_tlen, const int *d_lo, const int *d_hi,
                       unsigned long long *h_cells);

#define BAND_TAU 0.9f

typedef struct dev_pairs {
    uint8_t *q, *t;
    int64_t *qoff, *toff;
    int *qlen, *tlen;
    int n, maxlen;
} dev_pairs;

static void dev_pairs_free(dev_pairs *d)
{
    pb_cuda_free(d->q); pb_cuda_free(d->t); pb_cuda_free(d->qoff); pb_cuda_free(d->toff);
    pb_cuda_free(d->qlen); pb_cuda_free(d->tlen);
    pb_cuda_sync();
    memset(d, 0, sizeof *d);
}

/* host sequences -> device codes through the matrix mapper */
static int dev_pairs_upload(const parasail_matrix_t *matrix, const char *queries, const int64_t *qoff,
                            const int *qlen, const char *targets, const int64_t *toff, const int *tlen,
                            int n, dev_pairs *d)
{
    int64_t qb = 0, tb = 0, k;
    int i;
    uint8_t map[256];
    memset(d, 0, sizeof *d);
    d->n = n;
    for (i = 0; i < n; ++i) {
        if (qlen[i] <= 0 || tlen[i] <= 0) return -1;
        if (qoff[i] + qlen[i] > qb) qb = qoff[i] + qlen[i];
        if (toff[i] + tlen[i] > tb) tb = toff[i] + tlen[i];
        if (tlen[i] > d->maxlen) d->maxlen = tlen[i];
    }
    for (k = 0; k < 256; ++k) map[k] = (uint8_t)matrix->mapper[k];
    d->q = (uint8_t *)pb_cuda_malloc((size_t)qb + 16);
    d->t = (uint8_t *)pb_cuda_malloc((size_t)tb + 16);
    d->qoff = (int64_t *)pb_cuda_malloc(sizeof(int64_t) * n);
    d->toff = (int64_t *)pb_cuda_malloc(sizeof(int64_t) * n);
    d->qlen = (int *)pb_cuda_malloc(sizeof(int) * n);
    d->tlen = (int *)pb_cuda_malloc(sizeof(int) * n);
    if (!d->q || !d->t || !d->qoff || !d->toff || !d->qlen || !d->tlen) {
        dev_pairs_free(d); return -1;
    }
    /* characters go up as they are and are mapped to codes on the device */
    if (pb_cuda_h2d_mapped(d->q, queries, qb, map) != 0 || pb_cuda_h2d_mapped(d->t, targets, tb, map) != 0) {
        dev_pairs_free(d); return -1;
    }
    pb_cuda_h2d(d->qoff, qoff, sizeof(int64_t) * n);
    pb_cuda_h2d(d->toff, toff, sizeof(int64_t) * n);
    pb_cuda_h2d(d->qlen, qlen, sizeof(int) * n);
    pb_cuda_h2d(d->tlen, tlen, sizeof(int) * n);
    pb_cuda_sync();
    return 0;
}

static int long_ok(const char *func, const parasail_matrix_t *matrix, int open, int gap)
{
    if (!matrix) { fprintf(stderr, "%s: missing %s\n", func, "matrix"); return 0; }
    if (matrix->type != PARASAIL_MATRIX_TYPE_SQUARE || matrix->size > 32) {
        fprintf(stderr, "%s: needs a square matrix of at most 32 letters\n", func);
        return 0;
    }
    if (open < 0 || gap < 0) { fprintf(stderr, "%s: open and gap must be >= 0\n", func); return 0; }
    return pb_gpu_ready(func);
}

static int run_full(const parasail_matrix_t *matrix, const dev_pairs *d, int open, int gap, int *d_score)
{
    return pb_cuda_nw_long(d->n, open, gap, matrix->matrix, matrix->size, d->q, d->qoff, d->qlen,
                           d->t, d->toff, d->tlen, NULL, NULL, d->maxlen, d_score);
}

int parasail_b200_nw_long(const parasail_matrix_t *matrix,
                          const char *queries, const int64_t *qoffsets, const int *qlengths,
                          const char *targets, const int64_t *toffsets, const int *tlengths, int n,
                          int open, int gap, int *scores)
{
    dev_pairs d;
    int *d_score;
    int rc;
    if (!long_ok(__func__, matrix, open, gap)) return -1;
    if (n <= 0) return n == 0 ? 0 : -1;
    if (dev_pairs_upload(matrix, queries, qoffsets, qlengths, targets, toffsets, tlengths, n, &d) != 0) {
        fprintf(stderr, "%s: invalid pairs\n", __func__);
        return -1;
    }
    d_score = (int *)pb_cuda_malloc(sizeof(int) * n);
    pb_cuda_sync();
    rc = run_full(matrix, &d, open, gap, d_score);
    if (rc == 0) rc = pb_cuda_d2h(scores, d_score, sizeof(int) * n);
    pb_cuda_free(d_score);
    dev_pairs_free(&d);
    return rc;
}

parasail_b200_band_model_t *parasail_b200_band_model_new(unsigned seed)
{
    if (!pb_gpu_ready(__func__)) return NULL;
    return (parasail_b200_band_model_t *)pb_cuda_band_model_new(seed);
}

void parasail_b200_band_model_free(parasail_b200_band_model_t *model)
{
    pb_cuda_band_model_free((struct pb_band_model *)model);
}

int parasail_b200_band_model_sizes(int *n_in, int *n_hidden, int *n_out, int *n_weights, int *n_biases)
{
    return pb_cuda_band_sizes(n_in, n_hidden, n_out, n_weights, n_biases);
}

int parasail_b200_band_model_get(const parasail_b200_band_model_t *model, float *weights, float *biases)
{
    return model ? pb_cuda_band_model_get((const struct pb_band_model *)model, weights, biases) : -1;
}

void parasail_b200_band_model_scaling(const parasail_b200_band_model_t *model, float *widen, int *slack)
{
    if (model) pb_cuda_band_scaling((const struct pb_band_model *)model, widen, slack);
}

int parasail_b200_band_model_set(parasail_b200_band_model_t *model, const float *weights, const float *biases)
{
    return (model && weights && biases) ? pb_cuda_band_model_set((struct pb_band_model *)model, weights, biases) : -1;
}

int parasail_b200_band_features(const parasail_matrix_t *matrix,
                                const char *queries, const int64_t *qoffsets, const int *qlengths,
                                const char *targets, const int64_t *toffsets, const int *tlengths, int n,
                                float *features)
{
    dev_pairs d;
    float *d_feat;
    int rc, nin, nh, no, nw, nb;
    if (!long_ok(__func__, matrix, 0, 0)) return -1;
    pb_cuda_band_sizes(&nin, &nh, &no, &nw, &nb);
    if (dev_pairs_upload(matrix, queries, qoffsets, qlengths, targets, toffsets, tlengths, n, &d) != 0) return -1;
    d_feat = (float *)pb_cuda_malloc(sizeof(float) * (size_t)n * nin);
    pb_cuda_sync();
    rc = pb_cuda_band_features(n, d.q, d.qoff, d.qlen, d.t, d.toff, d.tlen, d_feat);
    if (rc == 0) rc = pb_cuda_d2h(features, d_feat, sizeof(float) * (size_t)n * nin);
    pb_cuda_free(d_feat);
    dev_pairs_free(&d);
    return rc;
}

int parasail_b200_band_model_gradients(const parasail_b200_band_model_t *model, const float *x,
                                       const float *target, int n, float tau,
                                       float *grad_weights, float *grad_biases, float *loss)
{
    int nin, nh, no, nw, nb, rc;
    float *d_x, *d_t, *d_gw, *d_gb;
    if (!model || n <= 0) return -1;
    pb_cuda_band_sizes(&nin, &nh, &no, &nw, &nb);
    d_x = (float *)pb_cuda_malloc(sizeof(float) * (size_t)n * nin);
    d_t = (float *)pb_cuda_malloc(sizeof(float) * (size_t)n * no);
    d_gw = (float *)pb_cuda_malloc(sizeof(float) * (size_t)nw);
    d_gb = (float *)pb_cuda_malloc(sizeof(float) * (size_t)nb);
    pb_cuda_h2d(d_x, x, sizeof(float) * (size_t)n * nin);
    pb_cuda_h2d(d_t, target, sizeof(float) * (size_t)n * no);
    pb_cuda_sync();
    rc = pb_cuda_band_gradients((const struct pb_band_model *)model, n, d_x, d_t, tau, d_gw, d_gb, loss);
    if (rc == 0) rc = pb_cuda_d2h(grad_weights, d_gw, sizeof(float) * (size_t)nw);
    if (rc == 0) rc = pb_cuda_d2h(grad_biases, d_gb, sizeof(float) * (size_t)nb);
    pb_cuda_free(d_x); pb_cuda_free(d_t); pb_cuda_free(d_gw); pb_cuda_free(d_gb);
    pb_cuda_sync();
    return rc;
}

int parasail_b200_band_model_train(parasail_b200_band_model_t *model, const parasail_matrix_t *matrix,
                                   const char *queries, const int64_t *qoffsets, const int *qlengths,
                                   const char *targets, const int64_t *toffsets, const int *tlengths, int n,
                                   int open, int gap, int epochs, int batch, float lr, float *final_loss)
{
    dev_pairs d;
    int nin, nh, no, nw, nb, rc, e, s, n_tr, n_tune;
    float *d_feat, *d_tgt, *d_gw, *d_gb, loss = 0.0f;
    int *d_score, *d_lab_lo, *d_lab_hi;
    if (!model || !long_ok(__func__, matrix, open, gap)) return -1;
    if (n <= 0 || epochs <= 0 || batch <= 0) return -1;
    pb_cuda_band_sizes(&nin, &nh, &no, &nw, &nb);
    if (dev_pairs_upload(matrix, queries, qoffsets, qlengths, targets, toffsets, tlengths, n, &d) != 0) return -1;
    d_feat = (float *)pb_cuda_malloc(sizeof(float) * (size_t)n * nin);
    d_tgt = (float *)pb_cuda_malloc(sizeof(float) * (size_t)n * no);
    d_score = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
    d_gw = (float *)pb_cuda_malloc(sizeof(float) * (size_t)nw);
    d_gb = (float *)pb_cuda_malloc(sizeof(float) * (size_t)nb);
    d_lab_lo = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
    d_lab_hi = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
    pb_cuda_sync();
    /* the last tenth of the pairs is held out of the gradient steps and
     * chooses the band scaling afterwards */
    n_tune = n >= 20 ? n / 10 : 0;
    n_tr = n - n_tune;
    /* labels: the smallest certifiable band of the full-DP optimum */
    rc = pb_cuda_band_features(n, d.q, d.qoff, d.qlen, d.t, d.toff, d.tlen, d_feat);
    if (rc == 0) rc = run_full(matrix, &d, open, gap, d_score);
    if (rc == 0) rc = pb_cuda_band_labels(n, matrix->max, open, gap, d.qlen, d.tlen, d_score, d_tgt, d_lab_lo, d_lab_hi);
    for (e = 0; rc == 0 && e < epochs; ++e) {
        double tot = 0.0;
        int nbat = 0;
        for (s = 0; rc == 0 && s < n_tr; s += batch) {
            const int bn = (n_tr - s) < batch ? (n_tr - s) : batch;
            float l = 0.0f;
            rc = pb_cuda_band_gradients((const struct pb_band_model *)model, bn, d_feat + (size_t)s * nin,
                                        d_tgt + (size_t)s * no, BAND_TAU, d_gw, d_gb, &l);
            if (rc == 0) rc = pb_cuda_band_adam((struct pb_band_model *)model, d_gw, d_gb, lr);
            tot += l;
            ++nbat;
        }
        loss = (float)(tot / (nbat ? nbat : 1));
    }
    if (rc == 0 && n_tune > 0)
        rc = pb_cuda_band_tune((struct pb_band_model *)model, n_tune, d_feat + (size_t)n_tr * nin, d.qlen + n_tr,
                               d.tlen + n_tr, d_lab_lo + n_tr, d_lab_hi + n_tr, NULL);
    if (final_loss) *final_loss = loss;
    pb_cuda_free(d_feat); pb_cuda_free(d_tgt); pb_cuda_free(d_score); pb_cuda_free(d_gw); pb_cuda_free(d_gb);
    pb_cuda_free(d_lab_lo); pb_cuda_free(d_lab_hi);
    dev_pairs_free(&d);
    return rc;
}

/* shared by the host and device entry points */
/* host wall time of the phases of the last parasail_b200_nw_learned_band
 * call on this thread (diagnostics) */
static __thread double g_phase_ms[5];

static double now_ms(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec * 1e3 + ts.tv_nsec * 1e-6;
}

void parasail_b200_band_phase_ms(double *out)
{
    int k;
    for (k = 0; k < 5; ++k) out[k] = g_phase_ms[k];
}

static int learned_run(const struct pb_band_model *model, const parasail_matrix_t *matrix, const dev_pairs *d,
                       int open, int gap, float widen, int slack, int *d_score, int *d_lo, int *d_hi,
                       parasail_b200_band_stats_t *stats)
{
    int nin, nh, no, nw, nb, rc, nfail = 0;
    float *d_feat, *d_y;
    int *d_cert;
    const int n = d->n;
    pb_cuda_band_sizes(&nin, &nh, &no, &nw, &nb);
    {
        /* widen <= 0 / slack < 0: the scaling tuned at training */
        float tw;
        int ts;
        pb_cuda_band_scaling(model, &tw, &ts);
        if (widen <= 0.0f) widen = tw;
        if (slack < 0) slack = ts;
    }
    d_feat = (float *)pb_cuda_malloc(sizeof(float) * (size_t)n * nin);
    d_y = (float *)pb_cuda_malloc(sizeof(float) * (size_t)n * no);
    d_cert = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);   /* rounds per pair */
    pb_cuda_sync();
    {
        double t0 = now_ms(), t1;
        rc = pb_cuda_band_features(n, d->q, d->qoff, d->qlen, d->t, d->toff, d->tlen, d_feat);
        if (rc == 0) rc = pb_cuda_band_forward(model, n, d_feat, NULL, NULL, d_y);
        if (rc == 0) rc = pb_cuda_band_from_pred(n, d->qlen, d->tlen, d_y, widen, slack, d_lo, d_hi);
        /* the MLP and band kernels run on the default stream, the DP on its
         * own: the bands must be complete before the DP reads them */
        if (rc == 0) rc = pb_cuda_device_sync();
        t1 = now_ms();
        g_phase_ms[0] = t1 - t0;
        /* cells of the first bands (every pair runs them) */
        if (rc == 0 && stats) {
            unsigned long long cells = 0;
            pb_cuda_band_cells(n, d->qlen, d->tlen, d_lo, d_hi, &cells);
            stats->band_cells = (double)cells;
        }
        t0 = now_ms();
        g_phase_ms[2] = t0 - t1;
        /* banded DP with the certificate in the launch: a pair that fails it
         * reruns at once on a band that passes */
        if (rc == 0) rc = pb_cuda_memset(d_cert, 0, sizeof(int) * (size_t)n);
        if (rc == 0) rc = pb_cuda_nw_long_cert(n, open, gap, matrix->matrix, matrix->size, matrix->max, d->q,
                                               d->qoff, d->qlen, d->t, d->toff, d->tlen, d_lo, d_hi, d->maxlen,
                                               d_score, d_cert);
        g_phase_ms[1] = now_ms() - t0;
    }
    g_phase_ms[3] = 0.0;
    if (rc == 0) {
        /* pairs that ran twice: count them, and add their second bands */
        int *hr = (int *)malloc(sizeof(int) * (size_t)n);
        int k;
        rc = hr ? pb_cuda_d2h(hr, d_cert, sizeof(int) * n) : -1;
        for (k = 0; rc == 0 && k < n; ++k) if (hr[k] == 2) ++nfail;
        free(hr);
        if (rc == 0 && stats && nfail > 0) {
            /* second-round cells: the final bands of the pairs that reran */
            int *sel_lo = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
            int *sel_hi = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
            unsigned long long cells = 0;
            rc = pb_cuda_band_select(n, d_cert, d_lo, d_hi, sel_lo, sel_hi);
            if (rc == 0) rc = pb_cuda_band_cells(n, d->qlen, d->tlen, sel_lo, sel_hi, &cells);
            stats->band_cells += (double)cells;
            pb_cuda_free(sel_lo); pb_cuda_free(sel_hi);
        }
    }
    if (stats) {
        stats->pairs = n;
        stats->certified = n - nfail;
        stats->fallback = nfail;
    }
    pb_cuda_free(d_feat); pb_cuda_free(d_y); pb_cuda_free(d_cert);
    pb_cuda_sync();
    return rc;
}

int parasail_b200_nw_learned_band(const parasail_b200_band_model_t *model, const parasail_matrix_t *matrix,
                                  const char *queries, const int64_t *qoffsets, const int *qlengths,
                                  const char *targets, const int64_t *toffsets, const int *tlengths, int n,
                                  int open, int gap, float widen, int slack,
                                  int *scores, int *band_lo, int *band_hi, parasail_b200_band_stats_t *stats)
{
    dev_pairs d;
    int *d_score, *d_lo, *d_hi, rc;
    if (!model || !long_ok(__func__, matrix, open, gap)) return -1;
    if (n <= 0) return n == 0 ? 0 : -1;
    {
        const double tu = now_ms();
        if (dev_pairs_upload(matrix, queries, qoffsets, qlengths, targets, toffsets, tlengths, n, &d) != 0) return -1;
        pb_cuda_sync();
        g_phase_ms[4] = now_ms() - tu;
    }
    d_score = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
    d_lo = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
    d_hi = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
    pb_cuda_sync();
    rc = learned_run((const struct pb_band_model *)model, matrix, &d, open, gap, widen, slack, d_score, d_lo, d_hi,
                     stats);
    if (rc == 0) rc = pb_cuda_d2h(scores, d_score, sizeof(int) * n);
    if (rc == 0 && band_lo) rc = pb_cuda_d2h(band_lo, d_lo, sizeof(int) * n);
    if (rc == 0 && band_hi) rc = pb_cuda_d2h(band_hi, d_hi, sizeof(int) * n);
    pb_cuda_free(d_score); pb_cuda_free(d_lo); pb_cuda_free(d_hi);
    dev_pairs_free(&d);
    return rc;
}

/* band given by the caller (e.g. fixed-width baselines): banded score,
 * certificate, full-DP fallback; the same contract as the learned path */
int parasail_b200_nw_banded_certified(const parasail_matrix_t *matrix,
                                      const char *queries, const int64_t *qoffsets, const int *qlengths,
                                      const char *targets, const int64_t *toffsets, const int *tlengths, int n,
                                      int open, int gap, const int *band_lo, const int *band_hi,
                                      int *scores, int *certified)
{
    dev_pairs d;
    int *d_score, *d_lo, *d_hi, *d_cert, rc, nfail = 0;
    if (!long_ok(__func__, matrix, open, gap)) return -1;
    if (n <= 0) return n == 0 ? 0 : -1;
    if (dev_pairs_upload(matrix, queries, qoffsets, qlengths, targets, toffsets, tlengths, n, &d) != 0) return -1;
    d_score = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
    d_lo = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
    d_hi = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
    d_cert = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
    pb_cuda_h2d(d_lo, band_lo, sizeof(int) * n);
    pb_cuda_h2d(d_hi, band_hi, sizeof(int) * n);
    pb_cuda_sync();
    rc = pb_cuda_nw_long(n, open, gap, matrix->matrix, matrix->size, d.q, d.qoff, d.qlen, d.t, d.toff, d.tlen,
                         d_lo, d_hi, d.maxlen, d_score);
    if (rc == 0) rc = pb_cuda_band_certify(n, matrix->max, open, gap, d.qlen, d.tlen, d_lo, d_hi, d_score, d_cert,
                                           &nfail);
    if (rc == 0) rc = pb_cuda_d2h(scores, d_score, sizeof(int) * n);
    if (rc == 0 && certified) rc = pb_cuda_d2h(certified, d_cert, sizeof(int) * n);
    pb_cuda_free(d_score); pb_cuda_free(d_lo); pb_cuda_free(d_hi); pb_cuda_free(d_cert);
    dev_pairs_free(&d);
    return rc;
}

/* parasail_nw_banded's band (src/nw_banded.c:92-97): query positions
 * [j + low, j + k] of target column j when s1Len <= s2Len (low = s1Len -
 * s2Len - k), [j - k, j + s1Len - s2Len + k] otherwise; as diagonals i - j. */
static void banded_k_band(int s1Len, int s2Len, int k, int *lo, int *hi)
{
    if (s1Len <= s2Len) { *lo = s1Len - s2Len - k; *hi = k; }
    else { *lo = -k; *hi = s1Len - s2Len + k; }
}

int pb_nw_banded_fits_wave(const parasail_matrix_t *matrix)
{
    return matrix && matrix->type == PARASAIL_MATRIX_TYPE_SQUARE && matrix->size <= 32 &&
           matrix->max <= 127 && matrix->min >= -127;
}

int parasail_b200_nw_banded_batch(const parasail_matrix_t *matrix,
                                  const char *queries, const int64_t *qoffsets, const int *qlengths,
                                  const char *targets, const int64_t *toffsets, const int *tlengths, int n,
                                  int open, int gap, int k, int *scores)
{
    dev_pairs d;
    int *d_score, *d_lo, *d_hi, *h_lo, *h_hi, rc, i;
    if (!long_ok(__func__, matrix, open, gap)) return -1;
    if (!pb_nw_banded_fits_wave(matrix)) {
        fprintf(stderr, "%s: needs a square matrix of at most 32 letters with |scores| <= 127\n", __func__);
        return -1;
    }
    if (k <= 0) { fprintf(stderr, "%s: %s must be > 0\n", __func__, "k"); return -1; }
    if (n <= 0) return n == 0 ? 0 : -1;
    if (!scores) { fprintf(stderr, "%s: missing %s\n", __func__, "scores"); return -1; }
    if (dev_pairs_upload(matrix, queries, qoffsets, qlengths, targets, toffsets, tlengths, n, &d) != 0) {
        fprintf(stderr, "%s: invalid pairs\n", __func__);
        return -1;
    }
    h_lo = (int *)malloc(sizeof(int) * (size_t)n);
    h_hi = (int *)malloc(sizeof(int) * (size_t)n);
    if (!h_lo || !h_hi) { free(h_lo); free(h_hi); dev_pairs_free(&d); return -1; }
    for (i = 0; i < n; ++i) banded_k_band(qlengths[i], tlengths[i], k, &h_lo[i], &h_hi[i]);
    d_score = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
    d_lo = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
    d_hi = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
    rc = (!d_score || !d_lo || !d_hi) ? -1 : 0;
    if (rc == 0) rc = pb_cuda_h2d(d_lo, h_lo, sizeof(int) * n);
    if (rc == 0) rc = pb_cuda_h2d(d_hi, h_hi, sizeof(int) * n);
    pb_cuda_sync();
    if (rc == 0)
        rc = pb_cuda_nw_long(n, open, gap, matrix->matrix, matrix->size, d.q, d.qoff, d.qlen, d.t, d.toff, d.tlen,
                             d_lo, d_hi, d.maxlen, d_score);
    if (rc == 0) rc = pb_cuda_d2h(scores, d_score, sizeof(int) * n);
    pb_cuda_free(d_score); pb_cuda_free(d_lo); pb_cuda_free(d_hi);
    free(h_lo); free(h_hi);
    dev_pairs_free(&d);
    return rc;
}

/* Certified banded global alignment without a model: every pair starts on
 * the band of half-width w0 around the certificate's centre (n - m) / 2
 * diagonals (always holding the diagonals between 0 and n - m); a pair whose
 * banded score fails the exactness certificate reruns on a band twice as
 * wide, until the band covers the whole matrix, where the score is the
 * full DP's. Returns the scores of parasail_b200_nw_long. */
int parasail_b200_nw_doubling_band(const parasail_matrix_t *matrix,
                                   const char *queries, const int64_t *qoffsets, const int *qlengths,
                                   const char *targets, const int64_t *toffsets, const int *tlengths, int n,
                                   int open, int gap, int w0, int *scores, parasail_b200_band_stats_t *stats)
{
    dev_pairs d;
    int *act = NULL, *h_lo = NULL, *h_hi = NULL, *h_sc = NULL, *h_cert = NULL, *h_ql = NULL, *h_tl = NULL;
    int64_t *h_qo = NULL, *h_to = NULL;
    int64_t *d_qo = NULL, *d_to = NULL;
    int *d_ql = NULL, *d_tl = NULL, *d_lo = NULL, *d_hi = NULL, *d_sc = NULL, *d_cert = NULL;
    int na = n, i, rc = 0, round = 0, nfail = 0;
    long long w = w0 > 0 ? w0 : 64;
    parasail_b200_band_stats_t st;
    memset(&st, 0, sizeof st);
    if (!long_ok(__func__, matrix, open, gap)) return -1;
    if (n <= 0) return n == 0 ? 0 : -1;
    if (!scores) { fprintf(stderr, "%s: missing %s\n", __func__, "scores"); return -1; }
    if (dev_pairs_upload(matrix, queries, qoffsets, qlengths, targets, toffsets, tlengths, n, &d) != 0) {
        fprintf(stderr, "%s: invalid pairs\n", __func__);
        return -1;
    }
    act = (int *)malloc(sizeof(int) * (size_t)n);
    h_lo = (int *)malloc(sizeof(int) * (size_t)n);
    h_hi = (int *)malloc(sizeof(int) * (size_t)n);
    h_sc = (int *)malloc(sizeof(int) * (size_t)n);
    h_cert = (int *)malloc(sizeof(int) * (size_t)n);
    h_ql = (int *)malloc(sizeof(int) * (size_t)n);
    h_tl = (int *)malloc(sizeof(int) * (size_t)n);
    h_qo = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    h_to = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    d_qo = (int64_t *)pb_cuda_malloc(sizeof(int64_t) * (size_t)n);
    d_to = (int64_t *)pb_cuda_malloc(sizeof(int64_t) * (size_t)n);
    d_ql = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
    d_tl = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
    d_lo = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
    d_hi = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
    d_sc = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
    d_cert = (int *)pb_cuda_malloc(sizeof(int) * (size_t)n);
    if (!act || !h_lo || !h_hi || !h_sc || !h_cert || !h_ql || !h_tl || !h_qo || !h_to || !d_qo || !d_to ||
        !d_ql || !d_tl || !d_lo || !d_hi || !d_sc || !d_cert)
        rc = -1;
    for (i = 0; i < n; ++i) act[i] = i;
    st.pairs = n;
    while (rc == 0 && na > 0) {
        int k, full = 1;
        unsigned long long cells = 0;
        for (k = 0; k < na; ++k) {
            const int p = act[k], qn = qlengths[p], tm = tlengths[p], de = qn - tm;
            long long lo = (de >= 0 ? de / 2 : -((-de + 1) / 2)) - w, hi = (de >= 0 ? (de + 1) / 2 : -((-de) / 2)) + w;
            if (lo > 0) lo = 0;
            if (lo > de) lo = de;
            if (hi < 0) hi = 0;
            if (hi < de) hi = de;
            /* a band past the matrix's corners is the whole matrix */
            if (lo < -(long long)tm) lo = -tm;
            if (hi > qn) hi = qn;
            if (lo > -(long long)tm || hi < qn) full = 0;
            h_lo[k] = (int)lo; h_hi[k] = (int)hi;
            h_qo[k] = qoffsets[p]; h_to[k] = toffsets[p]; h_ql[k] = qn; h_tl[k] = tm;
        }
        (void)full;
        if (pb_cuda_h2d(d_qo, h_qo, sizeof(int64_t) * na) || pb_cuda_h2d(d_to, h_to, sizeof(int64_t) * na) ||
            pb_cuda_h2d(d_ql, h_ql, sizeof(int) * na) || pb_cuda_h2d(d_tl, h_tl, sizeof(int) * na) ||
            pb_cuda_h2d(d_lo, h_lo, sizeof(int) * na) || pb_cuda_h2d(d_hi, h_hi, sizeof(int) * na)) { rc = -1; break; }
        pb_cuda_sync();
        rc = pb_cuda_nw_long(na, open, gap, matrix->matrix, matrix->size, d.q, d_qo, d_ql, d.t, d_to, d_tl,
                             d_lo, d_hi, d.maxlen, d_sc);
        if (rc == 0) rc = pb_cuda_band_certify(na, matrix->max, open, gap, d_ql, d_tl, d_lo, d_hi, d_sc, d_cert, &nfail);
        if (rc == 0) rc = pb_cuda_band_cells(na, d_ql, d_tl, d_lo, d_hi, &cells);
        if (rc == 0) rc = pb_cuda_d2h(h_sc, d_sc, sizeof(int) * na);
        if (rc == 0) rc = pb_cuda_d2h(h_cert, d_cert, sizeof(int) * na);
        if (rc != 0) break;
        st.band_cells += (double)cells;
        {
            int nn = 0;
            for (k = 0; k < na; ++k) {
                /* a band holding the whole matrix is the full DP */
                const int whole = h_lo[k] <= -h_tl[k] && h_hi[k] >= h_ql[k];
                if (h_cert[k] || whole) {
                    scores[act[k]] = h_sc[k];
                    if (round == 0) st.certified += 1;
                } else {
                    act[nn++] = act[k];
                }
            }
            if (round == 0) st.fallback = nn;
            na = nn;
        }
        w *= 2;
        ++round;
    }
    pb_cuda_free(d_qo); pb_cuda_free(d_to); pb_cuda_free(d_ql); pb_cuda_free(d_tl);
    pb_cuda_free(d_lo); pb_cuda_free(d_hi); pb_cuda_free(d_sc); pb_cuda_free(d_cert);
    free(act); free(h_lo); free(h_hi); free(h_sc); free(h_cert); free(h_ql); free(h_tl); free(h_qo); free(h_to);
    dev_pairs_free(&d);
    if (stats) *stats = st;
    return rc;
}
