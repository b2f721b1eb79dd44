/*
 * seqdb.c -- device-resident packed sequence sets (parasail_b200_seqdb_t)
 * and the memory-budgeted batch that aligns pairs of their sequences.
 *
 * A set is built from the '$'-separated text of parasail_sequences_pack
 * (src/parser.c:235-258 of the reference): the sequence offsets and lengths
 * are found on the host, the residues mapped and packed on the GPU
 * (pb_seqdb.cu) at 2, 5 or 8 bits. parasail_b200_batch_pairs_seqdb is the
 * B200 form of the reference aligner's batch loop
 * (apps/parasail_aligner.cpp:414-573 and :1585-1760): the pair list is cut
 * into batches whose device footprint fits a byte budget, and each batch
 * runs as one GPU pipeline over the resident codes.
 */
#include <stdlib.h>
#include <string.h>

#include "pb_internal.h"
#include "parasail_b200.h"

int pb_cuda_seqdb_pack(const uint8_t *h_text, int64_t n, uint8_t sep, const int *h_map256, int *bits,
                       uint32_t **d_words, int64_t *nwords);
int pb_cuda_seqdb_unpack(const uint32_t *d_words, int64_t nwords, int bits, int64_t n, uint8_t *d_codes,
                         void *stream);
int pb_cuda_seqdb_gather(const int64_t *d_off, const int *d_len, const int *d_first, const int *d_second, int np,
                         int64_t *qoff, int *qlen, int64_t *toff, int *tlen, void *stream);

struct parasail_b200_seqdb {
    int nseq;
    int bits;
    int64_t size;           /* text characters, sentinels included */
    uint32_t *d_words;
    int64_t nwords;
    int64_t *h_off, *d_off;
    int *h_len, *d_len;
};

parasail_b200_seqdb_t *parasail_b200_seqdb_create(const char *text, size_t size, char sentinel,
                                                  const parasail_matrix_t *matrix)
{
    parasail_b200_seqdb_t *db;
    size_t i, k = 0, nseq = 0, start = 0;
    if (!text || !matrix) {
        fprintf(stderr, "%s: missing text or matrix\n", __func__);
        return NULL;
    }
    if (size == 0 || text[size - 1] != sentinel) {
        fprintf(stderr, "%s: the text must end with the sentinel '%c'\n", __func__, sentinel);
        return NULL;
    }
    for (i = 0; i < size; ++i) nseq += text[i] == sentinel;
    if (nseq > 0x7fffffffULL) {
        fprintf(stderr, "%s: too many sequences\n", __func__);
        return NULL;
    }
    if (!pb_gpu_ready(__func__)) return NULL;
    db = (parasail_b200_seqdb_t *)calloc(1, sizeof *db);
    if (!db) return NULL;
    db->nseq = (int)nseq;
    db->size = (int64_t)size;
    db->h_off = (int64_t *)malloc(sizeof(int64_t) * nseq);
    db->h_len = (int *)malloc(sizeof(int) * nseq);
    if (!db->h_off || !db->h_len) goto fail;
    for (i = 0; i < size; ++i) {
        if (text[i] == sentinel) {
            db->h_off[k] = (int64_t)start;
            db->h_len[k] = (int)(i - start);
            ++k;
            start = i + 1;
        }
    }
    db->d_off = (int64_t *)pb_cuda_malloc(sizeof(int64_t) * nseq);
    db->d_len = (int *)pb_cuda_malloc(sizeof(int) * nseq);
    if (!db->d_off || !db->d_len) goto fail;
    if (pb_cuda_h2d(db->d_off, db->h_off, sizeof(int64_t) * nseq) != 0 ||
        pb_cuda_h2d(db->d_len, db->h_len, sizeof(int) * nseq) != 0)
        goto fail;
    if (pb_cuda_sync() != 0) goto fail;
    if (pb_cuda_seqdb_pack((const uint8_t *)text, (int64_t)size, (uint8_t)sentinel, matrix->mapper, &db->bits,
                           &db->d_words, &db->nwords) != 0)
        goto fail;
    return db;
fail:
    fprintf(stderr, "%s: failed: %s\n", __func__, pb_cuda_last_error());
    parasail_b200_seqdb_free(db);
    return NULL;
}

void parasail_b200_seqdb_free(parasail_b200_seqdb_t *db)
{
    if (!db) return;
    if (db->d_words) pb_cuda_free(db->d_words);
    if (db->d_off) pb_cuda_free(db->d_off);
    if (db->d_len) pb_cuda_free(db->d_len);
    pb_cuda_sync();
    free(db->h_off);
    free(db->h_len);
    free(db);
}

int parasail_b200_seqdb_count(const parasail_b200_seqdb_t *db) { return db ? db->nseq : 0; }
int parasail_b200_seqdb_bits(const parasail_b200_seqdb_t *db) { return db ? db->bits : 0; }
size_t parasail_b200_seqdb_size(const parasail_b200_seqdb_t *db) { return db ? (size_t)db->size : 0; }
size_t parasail_b200_seqdb_device_bytes(const parasail_b200_seqdb_t *db)
{
    return db ? (size_t)db->nwords * sizeof(uint32_t) : 0;
}
const int64_t *parasail_b200_seqdb_offsets(const parasail_b200_seqdb_t *db) { return db ? db->h_off : NULL; }
const int *parasail_b200_seqdb_lengths(const parasail_b200_seqdb_t *db) { return db ? db->h_len : NULL; }

int parasail_b200_seqdb_unpack(const parasail_b200_seqdb_t *db, uint8_t *d_codes)
{
    if (!db || !d_codes) {
        fprintf(stderr, "%s: missing db or d_codes\n", __func__);
        return -1;
    }
    if (pb_cuda_seqdb_unpack(db->d_words, db->nwords, db->bits, db->size, d_codes, NULL) != 0 ||
        pb_cuda_device_sync() != 0) {
        fprintf(stderr, "%s: CUDA failure: %s\n", __func__, pb_cuda_last_error());
        return -1;
    }
    return 0;
}

/* device bytes one pair of a batch holds: ids, offsets and lengths, the
 * record, and the pipeline's per-item state (ends, limits, sort keys,
 * lists) */
#define PB_SEQDB_BYTES_PER_PAIR 512

int parasail_b200_batch_pairs_seqdb(const char *funcname, const parasail_matrix_t *matrix,
                                    const parasail_b200_seqdb_t *db, const int *first, const int *second,
                                    size_t npairs, int open, int gap, size_t budget,
                                    parasail_b200_record_t *records)
{
    char name[128];
    const char *p;
    uint8_t *d_codes = NULL;
    int *d_ids = NULL;
    int64_t *d_qoff = NULL, *d_toff = NULL;
    int *d_qlen = NULL, *d_tlen = NULL;
    parasail_b200_record_t *d_rec = NULL;
    size_t per, batch, b0, i;
    int rc = -1;
    if (!funcname || !matrix || !db || (npairs && (!first || !second || !records))) {
        fprintf(stderr, "%s: missing arguments\n", __func__);
        return -1;
    }
    if (npairs == 0) return 0;
    for (i = 0; i < npairs; ++i) {
        if (first[i] < 0 || first[i] >= db->nseq || second[i] < 0 || second[i] >= db->nseq) {
            fprintf(stderr, "%s: pair %zu names a sequence outside the set\n", __func__, i);
            return -1;
        }
    }
    /* profile and direct names give the same records: the direct form */
    p = strstr(funcname, "_profile");
    if (strlen(funcname) >= sizeof name) return -1;
    if (p) {
        const size_t k = (size_t)(p - funcname);
        memcpy(name, funcname, k);
        strcpy(name + k, p + 8);
    } else {
        strcpy(name, funcname);
    }
    if (!pb_gpu_ready(__func__)) return -1;
    /* the batch size from the budget left after the resident codes */
    per = PB_SEQDB_BYTES_PER_PAIR;
    if (budget == 0) budget = (size_t)4 << 30;
    batch = budget > (size_t)db->size + per * 1024 ? (budget - (size_t)db->size) / per : 1024;
    if (batch > npairs) batch = npairs;
    if (batch > 0x7fffffffULL) batch = 0x7fffffffULL;
    d_codes = (uint8_t *)pb_cuda_malloc((size_t)db->size + 16);
    d_ids = (int *)pb_cuda_malloc(sizeof(int) * 2 * batch);
    d_qoff = (int64_t *)pb_cuda_malloc(sizeof(int64_t) * batch);
    d_toff = (int64_t *)pb_cuda_malloc(sizeof(int64_t) * batch);
    d_qlen = (int *)pb_cuda_malloc(sizeof(int) * batch);
    d_tlen = (int *)pb_cuda_malloc(sizeof(int) * batch);
    d_rec = (parasail_b200_record_t *)pb_cuda_malloc(sizeof(parasail_b200_record_t) * batch);
    if (!d_codes || !d_ids || !d_qoff || !d_toff || !d_qlen || !d_tlen || !d_rec) goto done;
    /* the allocations (on the library stream) before the unpack and gather
     * kernels (on the default stream) use them */
    if (pb_cuda_sync() != 0) goto done;
    if (pb_cuda_seqdb_unpack(db->d_words, db->nwords, db->bits, db->size, d_codes, NULL) != 0) goto done;
    for (b0 = 0; b0 < npairs; b0 += batch) {
        const int nb = (int)(npairs - b0 < batch ? npairs - b0 : batch);
        if (pb_cuda_device_sync() != 0 ||
            pb_cuda_h2d(d_ids, first + b0, sizeof(int) * nb) != 0 ||
            pb_cuda_h2d(d_ids + batch, second + b0, sizeof(int) * nb) != 0 || pb_cuda_sync() != 0 ||
            pb_cuda_seqdb_gather(db->d_off, db->d_len, d_ids, d_ids + batch, nb, d_qoff, d_qlen, d_toff, d_tlen,
                                 NULL) != 0 ||
            pb_cuda_device_sync() != 0)
            goto done;
        if (parasail_b200_batch_pairs_device(name, matrix, d_codes, d_qoff, d_qlen, d_codes, d_toff, d_tlen, nb,
                                             open, gap, d_rec) != 0)
            goto done;
        if (pb_cuda_d2h(records + b0, d_rec, sizeof(parasail_b200_record_t) * nb) != 0) goto done;
    }
    rc = 0;
done:
    if (rc != 0) fprintf(stderr, "%s: failed: %s\n", __func__, pb_cuda_last_error());
    if (d_codes) pb_cuda_free(d_codes);
    if (d_ids) pb_cuda_free(d_ids);
    if (d_qoff) pb_cuda_free(d_qoff);
    if (d_toff) pb_cuda_free(d_toff);
    if (d_qlen) pb_cuda_free(d_qlen);
    if (d_tlen) pb_cuda_free(d_tlen);
    if (d_rec) pb_cuda_free(d_rec);
    pb_cuda_sync();
    return rc;
}
