/*
 * trace.c -- traceback entry points and CIGAR strings of parasail-b200.
 *
 * A trace result carries the alignment path the reference's trace tables
 * encode, computed on the GPU (pb_pair16.cu: direction bits per cell and a
 * walk from the end cell): the trace functions of the exact widths --
 *   parasail_{alg}_trace, parasail_{alg}_trace_scan        (serial forms,
 *       src/sw_trace.c etc.: flags NOVEC / NOVEC_SCAN, 32 bits, 1 lane)
 *   parasail_{alg}_trace_{striped,scan}[_profile]_32       (the 32-bit
 *       trace kernels, e.g. src/sw_trace_striped_avx2_256_32.c: flags
 *       STRIPED / SCAN, 32 bits, 8 lanes)
 *   parasail_{alg}_trace_{striped,scan}[_profile]_{8,16,sat} (the 8- and
 *       16-bit trace kernels and the _sat chain 8 -> 16 -> 32: a result
 *       equal to the 32-bit one unless the kernel of that width saturates,
 *       which returns score and ends 0 with PARASAIL_FLAG_SATURATED)
 * -- return the score and ends of the alignment with PARASAIL_FLAG_TRACE,
 * and parasail_result_get_cigar builds the CIGAR from the path with the
 * rules of src/cigar_template.c: steps walked back from the end cell
 * (diagonal, vertical gap, horizontal gap, as the trace table's DIAG / DEL /
 * INS and DIAG_E / DIAG_F bits select: src/sw_trace.c:138-147), '=' or 'X'
 * by comparing the characters (upper-cased unless case sensitive, with
 * optional alias pairs), a query residue against a gap written 'I' and a
 * target residue against a gap 'D', the gaps to the matrix edge when the
 * walk reaches row or column -1, and for semi-global alignments the end
 * gaps past the end cell. The CIGAR encoding (length << 4 | op index into
 * "MIDNSHP=XB") is the BAM one the reference uses (src/cigar.c).
 */
#include <ctype.h>
#include <stdlib.h>
#include <string.h>

#include "pb_internal.h"
#include "parasail_b200.h"

/* the path behind a trace result's `extra` pointer */
typedef struct pb_trace_path {
    uint8_t *ops;     /* steps in forward order: 0 diagonal, 1 vertical gap (query residue), 2 horizontal gap */
    int n;
    int stop_i, stop_j;   /* the cell where the walk stopped (row/column; -1 = boundary) */
} pb_trace_path;

void pb_trace_free(parasail_result_t *r)
{
    pb_trace_path *t = (pb_trace_path *)r->extra;
    if (t) {
        free(t->ops);
        free(t);
    }
    r->extra = NULL;
}

/* ---- CIGAR encoding (src/cigar.c) ---------------------------------------- */

static const char cigar_ops[] = "MIDNSHP=XB";

const uint8_t parasail_cigar_encoded_ops[256] = {
    ['M'] = 0, ['I'] = 1, ['D'] = 2, ['N'] = 3, ['S'] = 4, ['H'] = 5, ['P'] = 6, ['='] = 7, ['X'] = 8, ['B'] = 9,
};

uint32_t parasail_cigar_encode(uint32_t length, char op_letter)
{
    return (length << 4) | parasail_cigar_encoded_ops[(unsigned char)op_letter];
}

char parasail_cigar_decode_op(uint32_t cigar_int)
{
    const uint32_t op = cigar_int & 0xfu;
    return op < 10 ? cigar_ops[op] : 'M';
}

uint32_t parasail_cigar_decode_len(uint32_t cigar_int)
{
    return cigar_int >> 4;
}

char *parasail_cigar_decode(parasail_cigar_t *cigar)
{
    size_t cap, used = 0;
    int k;
    char *s;
    if (!cigar) { fprintf(stderr, "%s: missing %s\n", __func__, "cigar"); return NULL; }
    cap = (size_t)cigar->len * 12 + 1;
    s = (char *)malloc(cap);
    if (!s) return NULL;
    s[0] = 0;
    for (k = 0; k < cigar->len; ++k)
        used += (size_t)snprintf(s + used, cap - used, "%u%c", parasail_cigar_decode_len(cigar->seq[k]),
                                 parasail_cigar_decode_op(cigar->seq[k]));
    return s;
}

parasail_cigar_t *parasail_cigar_encode_string(const char *cigar)
{
    parasail_cigar_t *c;
    size_t cap = 16;
    const char *p = cigar;
    if (!cigar) { fprintf(stderr, "%s: missing %s\n", __func__, "cigar"); return NULL; }
    c = (parasail_cigar_t *)calloc(1, sizeof *c);
    if (!c) return NULL;
    c->seq = (uint32_t *)malloc(sizeof(uint32_t) * cap);
    if (!c->seq) { free(c); return NULL; }
    while (*p) {
        char *end;
        const unsigned long len = strtoul(p, &end, 10);
        if (end == p || !*end || !strchr(cigar_ops, *end)) {
            fprintf(stderr, "%s: invalid CIGAR string '%s'\n", __func__, cigar);
            free(c->seq);
            free(c);
            return NULL;
        }
        if ((size_t)c->len == cap) {
            uint32_t *x = (uint32_t *)realloc(c->seq, sizeof(uint32_t) * cap * 2);
            if (!x) { free(c->seq); free(c); return NULL; }
            c->seq = x;
            cap *= 2;
        }
        c->seq[c->len++] = parasail_cigar_encode((uint32_t)len, *end);
        p = end + 1;
    }
    return c;
}

void parasail_cigar_free(parasail_cigar_t *cigar)
{
    if (!cigar) return;
    free(cigar->seq);
    free(cigar);
}

/* ---- CIGAR of a trace result ------------------------------------------------ */

typedef struct cigar_builder {
    parasail_cigar_t *c;
    size_t cap;
    char op;          /* pending run */
    uint32_t run;
} cigar_builder;

static int cb_flush(cigar_builder *b)
{
    if (!b->run) return 0;
    if ((size_t)b->c->len == b->cap) {
        uint32_t *x = (uint32_t *)realloc(b->c->seq, sizeof(uint32_t) * b->cap * 2);
        if (!x) return -1;
        b->c->seq = x;
        b->cap *= 2;
    }
    b->c->seq[b->c->len++] = parasail_cigar_encode(b->run, b->op);
    b->run = 0;
    return 0;
}

static int cb_add(cigar_builder *b, char op, uint32_t n)
{
    if (!n) return 0;
    if (b->run && b->op != op && cb_flush(b) != 0) return -1;
    b->op = op;
    b->run += n;
    return 0;
}

static int same_residue(char a, char b, int case_sensitive, const char *aliases)
{
    size_t k, n;
    if (!case_sensitive) { a = (char)toupper((unsigned char)a); b = (char)toupper((unsigned char)b); }
    if (a == b) return 1;
    if (!aliases) return 0;
    n = strlen(aliases);
    for (k = 0; k + 1 < n; k += 2) {
        char x = aliases[k], y = aliases[k + 1];
        if (!case_sensitive) { x = (char)toupper((unsigned char)x); y = (char)toupper((unsigned char)y); }
        if ((x == a && y == b) || (y == a && x == b)) return 1;
    }
    return 0;
}

parasail_cigar_t *parasail_result_get_cigar_extra(parasail_result_t *result, const char *seqA, int lena,
                                                  const char *seqB, int lenb, const parasail_matrix_t *matrix,
                                                  int case_sensitive, const char *alphabet_aliases)
{
    const pb_trace_path *t;
    cigar_builder b;
    int i, j, k;
    (void)matrix;
    PB_CHECK_NULL(result);
    PB_CHECK_NULL(seqA);
    PB_CHECK_NULL(seqB);
    if (!(result->flag & PARASAIL_FLAG_TRACE) || !result->extra) {
        if (result->flag & PARASAIL_FLAG_SATURATED)
            fprintf(stderr, "%s: the result is saturated and holds no alignment\n", __func__);
        else
            fprintf(stderr, "%s: assert(%s) failed\n", __func__, "parasail_result_is_trace(result)");
        return NULL;
    }
    if (alphabet_aliases && strlen(alphabet_aliases) % 2 != 0) {
        fprintf(stderr, "%s: alphabet aliases must come in pairs\n", __func__);
        return NULL;
    }
    t = (const pb_trace_path *)result->extra;
    memset(&b, 0, sizeof b);
    b.c = (parasail_cigar_t *)calloc(1, sizeof *b.c);
    b.cap = (size_t)(t->n + 4);
    if (!b.c || !(b.c->seq = (uint32_t *)malloc(sizeof(uint32_t) * b.cap))) { free(b.c); return NULL; }
    i = t->stop_i;
    j = t->stop_j;
    b.c->beg_query = i + 1;
    b.c->beg_ref = j + 1;
    /* the walk reached the matrix edge: the rest of the other sequence
     * aligns against gaps and the alignment begins at 0, 0
     * (src/cigar_template.c:145-163) */
    if (i < 0 && j >= 0) { cb_add(&b, 'D', (uint32_t)(j + 1)); b.c->beg_ref = 0; }
    else if (j < 0 && i >= 0) { cb_add(&b, 'I', (uint32_t)(i + 1)); b.c->beg_query = 0; }
    /* the path's first step starts at (stop_i + 1, stop_j + 1) */
    i += 1;
    j += 1;
    for (k = 0; k < t->n; ++k) {
        const uint8_t op = t->ops[k];
        int rc;
        if (op == 0) {
            if (i >= lena || j >= lenb) break;
            rc = cb_add(&b, same_residue(seqA[i], seqB[j], case_sensitive, alphabet_aliases) ? '=' : 'X', 1);
            ++i;
            ++j;
        } else if (op == 1) {
            rc = cb_add(&b, 'I', 1);
            ++i;
        } else {
            rc = cb_add(&b, 'D', 1);
            ++j;
        }
        if (rc != 0) { parasail_cigar_free(b.c); return NULL; }
    }
    /* semi-global: the end gaps past the end cell (src/cigar_template.c:124-142) */
    if (result->flag & PARASAIL_FLAG_SG) {
        if (result->end_query + 1 == lena) cb_add(&b, 'D', (uint32_t)(lenb - 1 - result->end_ref));
        else if (result->end_ref + 1 == lenb) cb_add(&b, 'I', (uint32_t)(lena - 1 - result->end_query));
        else { parasail_cigar_free(b.c); return NULL; }
    }
    if (cb_flush(&b) != 0) { parasail_cigar_free(b.c); return NULL; }
    return b.c;
}

parasail_cigar_t *parasail_result_get_cigar(parasail_result_t *result, const char *seqA, int lena,
                                            const char *seqB, int lenb, const parasail_matrix_t *matrix)
{
    return parasail_result_get_cigar_extra(result, seqA, lena, seqB, lenb, matrix, 0, NULL);
}

/* ---- traceback strings and the printed alignment (src/traceback.c,
 *      src/traceback_template.c) ---------------------------------------------- */

/* the three rows of an alignment in forward order: query residues or '-',
 * the comparison characters (match / pos / neg, ' ' against a gap), target
 * residues or '-'; c_ins and c_del count the target and query residues
 * aligned against gaps */
typedef struct {
    char *q, *a, *d;
    int64_t len, c_ins, c_del;
} tb_rows;

/* the comparison character of a query and a target residue
 * (src/traceback.c:19-70): equal (upper-cased unless case sensitive), or
 * equal through an alias -- the alias table is upper-cased and scanned at
 * every offset, pairing each character with the next, against the residues
 * as they are -- gives match; otherwise the substitution score (the PSSM row
 * of the query position for a PSSM) > 0 gives pos, else neg */
static char tb_match_char(const char *seqA, int ai, const char *seqB, int bi, const parasail_matrix_t *m,
                          char match, char pos, char neg, int cs, const char *al, size_t nal)
{
    const char a = seqA ? seqA[ai] : '*';
    const char b = seqB[bi];
    int same = cs ? a == b : toupper((unsigned char)a) == toupper((unsigned char)b);
    size_t k;
    int sub;
    for (k = 0; al && k < nal; ++k) {
        const char next = k + 1 < nal ? al[k + 1] : '\0';
        if (al[k] == a) same |= next == b;
        else if (next == a) same |= al[k] == b;
    }
    if (same) return match;
    if (m->type == PARASAIL_MATRIX_TYPE_SQUARE)
        sub = m->matrix[m->mapper[(unsigned char)a] * m->size + m->mapper[(unsigned char)b]];
    else
        sub = m->matrix[ai * m->size + m->mapper[(unsigned char)b]];
    return sub > 0 ? pos : neg;
}

static void tb_rows_free(tb_rows *r)
{
    free(r->q);
    free(r->a);
    free(r->d);
}

/* The rows of a trace result: the walk of src/traceback_template.c:57-174
 * read from the result's path -- gaps to the matrix edge first (not for SW),
 * then the path's steps, then a semi-global alignment's end gaps past the
 * end cell. Returns 0, or -1 (message printed) for an unusable result. */
static int tb_build(const char *who, parasail_result_t *result, const char *seqA, int lena, const char *seqB,
                    int lenb, const parasail_matrix_t *matrix, char match, char pos, char neg, int cs,
                    const char *aliases_in, tb_rows *out)
{
    const pb_trace_path *t;
    char al[256];
    size_t nal = 0, k;
    int64_t n = 0, cap, i, j, s;
    memset(out, 0, sizeof *out);
    if (!result || !(result->flag & PARASAIL_FLAG_TRACE) || !result->extra) {
        fprintf(stderr, "%s: assert(%s) failed\n", who, "parasail_result_is_trace(result)");
        return -1;
    }
    if (aliases_in) {
        nal = strlen(aliases_in);
        if (!(nal % 2 == 0 && nal < 256)) {
            fprintf(stderr, "%s: assert(%s) failed\n", who, "aliases_size % 2 == 0 && aliases_size < 256");
            return -1;
        }
        for (k = 0; k < nal; ++k) al[k] = cs ? aliases_in[k] : (char)toupper((unsigned char)aliases_in[k]);
    }
    t = (const pb_trace_path *)result->extra;
    cap = (int64_t)lena + lenb + 1;
    out->q = (char *)malloc((size_t)cap);
    out->a = (char *)malloc((size_t)cap);
    out->d = (char *)malloc((size_t)cap);
    if (!out->q || !out->a || !out->d) { tb_rows_free(out); return -1; }
#define TB_PUT(qc, ac, dc) do { if (n + 1 >= cap) goto overflow; out->q[n] = (qc); out->a[n] = (ac); out->d[n] = (dc); ++n; } while (0)
    if (!(result->flag & PARASAIL_FLAG_SW)) {
        if (t->stop_i < 0 && t->stop_j >= 0)
            for (j = 0; j <= t->stop_j; ++j) { TB_PUT('-', ' ', seqB[j]); ++out->c_ins; }
        else if (t->stop_j < 0 && t->stop_i >= 0)
            for (i = 0; i <= t->stop_i; ++i) { TB_PUT(seqA ? seqA[i] : '*', ' ', '-'); ++out->c_del; }
    }
    i = t->stop_i + 1;
    j = t->stop_j + 1;
    for (s = 0; s < t->n; ++s) {
        const uint8_t op = t->ops[s];
        if (op == 0) {
            if (i >= lena || j >= lenb) break;
            TB_PUT(seqA ? seqA[i] : '*', tb_match_char(seqA, (int)i, seqB, (int)j, matrix, match, pos, neg, cs,
                                                         aliases_in ? al : NULL, nal), seqB[j]);
            ++i;
            ++j;
        } else if (op == 1) {
            TB_PUT(seqA ? seqA[i] : '*', ' ', '-');
            ++out->c_del;
            ++i;
        } else {
            TB_PUT('-', ' ', seqB[j]);
            ++out->c_ins;
            ++j;
        }
    }
    if (result->flag & PARASAIL_FLAG_SG) {
        if (result->end_query + 1 == lena) {
            for (j = result->end_ref + 1; j < lenb; ++j) { TB_PUT('-', ' ', seqB[j]); ++out->c_ins; }
        } else if (result->end_ref + 1 == lenb) {
            for (i = result->end_query + 1; i < lena; ++i) { TB_PUT(seqA ? seqA[i] : '*', ' ', '-'); ++out->c_del; }
        } else {
            fprintf(stderr, "%s: assert(%s) failed\n", who, "0 && \"internal error\"");
            tb_rows_free(out);
            return -1;
        }
    }
#undef TB_PUT
    out->q[n] = out->a[n] = out->d[n] = '\0';
    out->len = n;
    return 0;
overflow:
    fprintf(stderr, "%s: path longer than the sequences\n", who);
    tb_rows_free(out);
    return -1;
}

parasail_traceback_t *parasail_result_get_traceback_extra(parasail_result_t *result, const char *seqA, int lena,
                                                          const char *seqB, int lenb,
                                                          const parasail_matrix_t *matrix, char match, char pos,
                                                          char neg, int case_sensitive,
                                                          const char *alphabet_aliases)
{
    tb_rows r;
    parasail_traceback_t *tb;
    if (tb_build(__func__, result, seqA, lena, seqB, lenb, matrix, match, pos, neg, case_sensitive,
                 alphabet_aliases, &r) != 0)
        return NULL;
    tb = (parasail_traceback_t *)malloc(sizeof *tb);
    if (!tb) { tb_rows_free(&r); return NULL; }
    tb->query = r.q;
    tb->comp = r.a;
    tb->ref = r.d;
    return tb;
}

parasail_traceback_t *parasail_result_get_traceback(parasail_result_t *result, const char *seqA, int lena,
                                                    const char *seqB, int lenb, const parasail_matrix_t *matrix,
                                                    char match, char pos, char neg)
{
    return parasail_result_get_traceback_extra(result, seqA, lena, seqB, lenb, matrix, match, pos, neg, 0, NULL);
}

void parasail_traceback_free(parasail_traceback_t *traceback)
{
    if (!traceback) return;
    free(traceback->query);
    free(traceback->comp);
    free(traceback->ref);
    free(traceback);
}

/* a name cut or padded to w characters */
static void tb_name(FILE *f, const char *name, int w)
{
    const int64_t nl = name ? (int64_t)strlen(name) : 0;
    int64_t k;
    for (k = 0; k < w; ++k) fputc(k < nl ? name[k] : ' ', f);
}

/* The printed alignment (src/traceback_template.c:188-489): blocks of
 * `width` columns, each a target line (name, first and last residue
 * positions), the comparison line and a query line; positions count from 1,
 * offset by where a local alignment begins; then, with use_stats, length,
 * identity, similarity, gaps and score. */
void parasail_traceback_generic_extra2(const char *seqA, int lena, const char *seqB, int lenb, const char *nameA,
                                       const char *nameB, const parasail_matrix_t *matrix,
                                       parasail_result_t *result, char match, char pos, char neg, int width,
                                       int name_width, int use_stats, int int_width, FILE *stream,
                                       int case_sensitive, const char *alphabet_aliases)
{
    tb_rows r;
    char tmp[32];
    int64_t qp, dp, mch = 0, sim = 0, gap = 0, c, col;
    int need;
    if (tb_build(__func__, result, seqA, lena, seqB, lenb, matrix, match, pos, neg, case_sensitive,
                 alphabet_aliases, &r) != 0)
        return;
    need = snprintf(tmp, sizeof tmp, "%llu", (unsigned long long)lena + (unsigned long long)lenb);
    if (int_width < need) int_width = need;
    if (result->flag & PARASAIL_FLAG_SW) {
        qp = result->end_query + 1 - r.len + r.c_ins;
        dp = result->end_ref + 1 - r.len + r.c_del;
    } else {
        qp = dp = 0;
    }
    for (col = 0; col < r.len; col += width) {
        const int64_t stop = col + width < r.len ? col + width : r.len;
        fprintf(stream, "\n");
        tb_name(stream, nameB, name_width);
        fprintf(stream, " %*lld ", int_width, (long long)dp + 1);
        for (c = col; c < stop; ++c) {
            if (r.d[c] != '-') ++dp;
            fputc(r.d[c], stream);
        }
        fprintf(stream, " %*lld\n", int_width, (long long)dp);
        for (c = 0; c < name_width + 1 + int_width + 1; ++c) fputc(' ', stream);
        for (c = col; c < stop; ++c) {
            const char x = r.a[c];
            if (x == match) { ++mch; ++sim; }
            else if (x == pos) ++sim;
            else if (x == neg) { }
            else if (x == ' ') ++gap;
            else {
                fprintf(stderr, "bad char in traceback '%c'\n", x);
                fprintf(stderr, "%s: assert(%s) failed\n", __func__, "0 && \"internal error\"");
                tb_rows_free(&r);
                return;
            }
            fputc(x, stream);
        }
        fprintf(stream, "\n");
        tb_name(stream, nameA, name_width);
        fprintf(stream, " %*lld ", int_width, (long long)qp + 1);
        for (c = col; c < stop; ++c) {
            if (r.q[c] != '-') ++qp;
            fputc(r.q[c], stream);
        }
        fprintf(stream, " %*lld\n", int_width, (long long)qp);
    }
    if (use_stats) {
        const long long L = (long long)r.len;
        fprintf(stream, "\n");
        fprintf(stream, "Length: %lld\n", L);
        fprintf(stream, "Identity:   %*lld/%lld (%4.1f%%)\n", int_width, (long long)mch, L, 100.0 * mch / L);
        fprintf(stream, "Similarity: %*lld/%lld (%4.1f%%)\n", int_width, (long long)sim, L, 100.0 * sim / L);
        fprintf(stream, "Gaps:       %*lld/%lld (%4.1f%%)\n", int_width, (long long)gap, L, 100.0 * gap / L);
        fprintf(stream, "Score: %d\n", result->score);
    }
    tb_rows_free(&r);
}

void parasail_traceback_generic_extra(const char *seqA, int lena, const char *seqB, int lenb, const char *nameA,
                                      const char *nameB, const parasail_matrix_t *matrix,
                                      parasail_result_t *result, char match, char pos, char neg, int width,
                                      int name_width, int use_stats, int int_width, FILE *stream)
{
    parasail_traceback_generic_extra2(seqA, lena, seqB, lenb, nameA, nameB, matrix, result, match, pos, neg,
                                      width, name_width, use_stats, int_width, stream, 0, NULL);
}

void parasail_traceback_generic(const char *seqA, int lena, const char *seqB, int lenb, const char *nameA,
                                const char *nameB, const parasail_matrix_t *matrix, parasail_result_t *result,
                                char match, char pos, char neg, int width, int name_width, int use_stats)
{
    parasail_traceback_generic_extra2(seqA, lena, seqB, lenb, nameA, nameB, matrix, result, match, pos, neg,
                                      width, name_width, use_stats, 7, stdout, 0, NULL);
}

/* ---- paths on the GPU ------------------------------------------------------- */

static int trace_job(int alg, int sgflags, const parasail_matrix_t *matrix, int open, int gap, pb_job *job)
{
    memset(job, 0, sizeof *job);
    job->mode.alg = alg; job->mode.sgflags = sgflags; job->mode.stats = 0; job->mode.striped = 0;
    job->mode.open = open; job->mode.gap = gap; job->mode.mmax = matrix->max; job->mode.mmin = matrix->min;
    job->bits = -1;     /* exact values, no width verdicts */
    return 0;
}

static void mapper_of(const parasail_matrix_t *m, uint8_t *out)
{
    int c;
    for (c = 0; c < 256; ++c) out[c] = (uint8_t)m->mapper[c];
}

/* Paths of n pairs (host characters). ends[3k..] score, end_query,
 * end_ref; paths[k] allocated here (NULL when the pair has no path: it is
 * outside the 16-bit bounds of the pair kernels). */
static int trace_pairs(int alg, int sgflags, const parasail_matrix_t *matrix, int open, int gap,
                       const char *q, const int64_t *qoff, const int *qlen,
                       const char *t, const int64_t *toff, const int *tlen, int n,
                       int *ends, pb_trace_path **paths)
{
    pb_job job;
    pb_batch b;
    uint8_t map[256];
    int32_t *d_mat;
    int64_t *ooff;
    uint8_t *ops;
    int *info;
    int64_t total = 0;
    int k, rc;
    if (matrix->type != PARASAIL_MATRIX_TYPE_SQUARE) return -2;
    trace_job(alg, sgflags, matrix, open, gap, &job);
    ooff = (int64_t *)malloc(sizeof(int64_t) * (size_t)n);
    info = (int *)malloc(sizeof(int) * 3 * (size_t)n);
    if (!ooff || !info) { free(ooff); free(info); return -1; }
    for (k = 0; k < n; ++k) { ooff[k] = total; total += (int64_t)qlen[k] + tlen[k]; }
    ops = (uint8_t *)malloc((size_t)total + 16);
    d_mat = (int32_t *)pb_cuda_malloc(sizeof(int32_t) * (size_t)matrix->size * matrix->size);
    if (!ops || !d_mat) { free(ooff); free(info); free(ops); pb_cuda_free(d_mat); return -1; }
    rc = pb_cuda_h2d(d_mat, matrix->matrix, sizeof(int32_t) * (size_t)matrix->size * matrix->size);
    pb_cuda_sync();
    memset(&b, 0, sizeof b);
    b.alg = alg; b.sgflags = sgflags; b.open = open; b.gap = gap;
    b.d_mat = d_mat; b.msize = matrix->size; b.mmax = matrix->max; b.mmin = matrix->min;
    mapper_of(matrix, map);
    if (rc == 0)
        rc = pb_cuda_trace_pairs_host(&job, &b, map, q, qoff, qlen, t, toff, tlen, n, ends, ops, ooff, info);
    pb_cuda_free(d_mat);
    pb_cuda_sync();
    for (k = 0; k < n; ++k) paths[k] = NULL;
    for (k = 0; rc == 0 && k < n; ++k) {
        const int steps = info[3 * k];
        const int64_t cap = (int64_t)qlen[k] + tlen[k];
        pb_trace_path *p;
        if (steps < 0) continue;
        p = (pb_trace_path *)calloc(1, sizeof *p);
        if (!p || !(p->ops = (uint8_t *)malloc((size_t)steps + 1))) { free(p); rc = -1; break; }
        memcpy(p->ops, ops + ooff[k] + cap - steps, (size_t)steps);
        p->n = steps;
        p->stop_i = info[3 * k + 1];
        p->stop_j = info[3 * k + 2];
        paths[k] = p;
    }
    free(ooff);
    free(info);
    free(ops);
    return rc;
}

static int alg_flags(int alg, int sgflags)
{
    int f = alg == PB_SW ? PARASAIL_FLAG_SW : alg == PB_NW ? PARASAIL_FLAG_NW : PARASAIL_FLAG_SG;
    if (alg == PB_SG) {
        if (sgflags & PB_S1_BEG) f |= PARASAIL_FLAG_SG_S1_BEG;
        if (sgflags & PB_S1_END) f |= PARASAIL_FLAG_SG_S1_END;
        if (sgflags & PB_S2_BEG) f |= PARASAIL_FLAG_SG_S2_BEG;
        if (sgflags & PB_S2_END) f |= PARASAIL_FLAG_SG_S2_END;
    }
    return f;
}

/* ---- widths of the vector trace forms ------------------------------------ */

/* A trace form: serial (kind 0) or serial scan (1), or a vector form,
 * striped (2) or scan (3), at 8, 16 or 32 bits or the _sat chain (bits 0). */
typedef struct trace_form {
    int alg, sgf, kind, bits;
} trace_form;

/* the reference's BITS / LANES flags of its AVX2 trace kernels */
static int width_flags(int w)
{
    return w == 8 ? PARASAIL_FLAG_BITS_8 | PARASAIL_FLAG_LANES_32
         : w == 16 ? PARASAIL_FLAG_BITS_16 | PARASAIL_FLAG_LANES_16
         : PARASAIL_FLAG_BITS_32 | PARASAIL_FLAG_LANES_8;
}

static int form_flags(const trace_form *f, int width)
{
    const int fl = alg_flags(f->alg, f->sgf) | PARASAIL_FLAG_TRACE;
    if (f->kind == 0) return fl | PARASAIL_FLAG_NOVEC | PARASAIL_FLAG_BITS_32 | PARASAIL_FLAG_LANES_1;
    if (f->kind == 1) return fl | PARASAIL_FLAG_NOVEC_SCAN | PARASAIL_FLAG_BITS_32 | PARASAIL_FLAG_LANES_1;
    return fl | (f->kind == 2 ? PARASAIL_FLAG_STRIPED : PARASAIL_FLAG_SCAN) | width_flags(width);
}

/* A sound verdict that the w-bit nw/sg trace kernel (striped or scan) does
 * not saturate: every value it checks stays inside [NEG_LIMIT, POS_LIMIT]
 * (constants of e.g. src/nw_trace_striped_avx2_256_8.c:170-171). Every H
 * is at least the least boundary value (-open - gap * (rows or columns))
 * plus min(matrix, 0) per diagonal step, every checked E and F at least
 * that minus open, every H at most max(matrix, 0) per aligned pair; the SG
 * scan kernels also check the gap ramp -open - segLen * gap. Penalties
 * that wrap in the lane are never clean. */
static int nwsg_clean(int w, int qlen, int tlen, int open, int gap, int mmax, int mmin)
{
    const int64_t imin = w == 8 ? INT8_MIN : INT16_MIN, imax = w == 8 ? INT8_MAX : INT16_MAX;
    const int64_t neg = ((-(int64_t)open < mmin) ? imin + open : imin - mmin) + 1;
    const int64_t pos = imax - mmax - 1;
    const int64_t lanes = 256 / w, seg = (qlen + lanes - 1) / lanes, pad = seg * lanes;
    const int64_t far = (pad > tlen ? pad : tlen) - 1, diag = (pad < tlen ? pad : tlen) + 1;
    const int64_t lb = -(int64_t)open - (int64_t)gap * far + (mmin < 0 ? (int64_t)mmin * diag : 0);
    if (open > imax || gap > imax) return 0;
    if (lb - open - gap < neg) return 0;
    if (-(int64_t)open - (int64_t)gap * seg < neg) return 0;
    return (int64_t)(mmax > 0 ? mmax : 0) * (qlen < tlen ? qlen : tlen) <= pos;
}

/* Per pair, the width whose trace kernel gives a vector form's result and
 * whether that kernel saturated (the _sat dispatchers of src/satcheck.c
 * run 8, then 16, then 32 bits while the result saturates). A kernel of any
 * width that does not saturate returns the exact result the path
 * describes. SW: the 8/16-bit trace kernels (unbiased lanes; src/
 * sw_trace_striped_avx2_256_8.c:398-418, sw_trace_scan_avx2_256_8.c:
 * 352-359) saturate exactly when the alignment score exceeds
 * INT_MAX_w - max(matrix) - 1 (penalties that wrap in the lane are taken
 * as saturating). NW/SG: clean by nwsg_clean, else the lane-exact
 * emulation of the kernel on the GPU decides (pb_lane.cuh). sat[k] is -1
 * for a SW pair with no path: its score, and so its width, is unknown. */
static int trace_widths(const trace_form *f, const parasail_matrix_t *matrix, int open, int gap, const char *q,
                        const int64_t *qoff, const int *qlen, const char *t, const int64_t *toff, const int *tlen,
                        int n, const int *ends, pb_trace_path *const *paths, int *width, int *sat)
{
    static const int chain[3] = {8, 16, 32};
    const int first = f->bits == 16 ? 1 : f->bits == 32 ? 2 : 0;
    const int last = f->bits == 0 ? 2 : first;
    int *pending = (int *)malloc(sizeof(int) * (size_t)n);
    int *list = (int *)malloc(sizeof(int) * (size_t)n);
    int *lsat = (int *)malloc(sizeof(int) * (size_t)n);
    uint8_t map[256];
    int np = 0, c, i, k, rc = 0;
    if (!pending || !list || !lsat) { free(pending); free(list); free(lsat); return -1; }
    for (k = 0; k < n; ++k) pending[np++] = k;
    mapper_of(matrix, map);
    for (c = first; c <= last && np > 0 && rc == 0; ++c) {
        const int w = chain[c];
        const int64_t imax = w == 8 ? INT8_MAX : INT16_MAX;
        int nl = 0, nn = 0;
        for (i = 0; i < np; ++i) {
            k = pending[i];
            width[k] = w;
            sat[k] = 0;
            if (w == 32) continue;
            if (f->alg == PB_SW) {
                if (open > imax || gap > imax) sat[k] = 1;
                else if (!paths[k]) sat[k] = -1;
                else sat[k] = ends[3 * k] > imax - matrix->max - 1;
            } else if (!nwsg_clean(w, qlen[k], tlen[k], open, gap, matrix->max, matrix->min)) {
                list[nl++] = k;
            }
        }
        if (nl > 0) {
            rc = pb_cuda_trace_sat_host(w, f->kind == 2 ? 4 : 5, f->sgf, open, gap, matrix->max, matrix->min,
                                        matrix->matrix, matrix->size, map, q, qoff, qlen, t, toff, tlen, list, nl,
                                        lsat);
            for (i = 0; rc == 0 && i < nl; ++i) sat[list[i]] = lsat[i];
        }
        for (i = 0; i < np; ++i) if (sat[pending[i]] == 1) pending[nn++] = pending[i];
        if (c < last) np = nn;
    }
    free(pending);
    free(list);
    free(lsat);
    return rc;
}

/* Trace results of n pairs (host characters): results[k] NULL, with a
 * message, for a pair whose result needs a path that the 16-bit pair
 * kernels cannot give. Returns 0, or -1 (message printed, no results). */
static int trace_results(const char *who, const trace_form *f, const parasail_matrix_t *matrix, int open, int gap,
                         const char *q, const int64_t *qoff, const int *qlen, const char *t, const int64_t *toff,
                         const int *tlen, int n, parasail_result_t **results)
{
    int *ends = (int *)malloc(sizeof(int) * 3 * (size_t)n);
    int *width = (int *)malloc(sizeof(int) * (size_t)n);
    int *sat = (int *)malloc(sizeof(int) * (size_t)n);
    pb_trace_path **paths = (pb_trace_path **)calloc((size_t)n, sizeof *paths);
    int k, rc;
    for (k = 0; k < n; ++k) results[k] = NULL;
    if (!ends || !width || !sat || !paths) { free(ends); free(width); free(sat); free(paths); return -1; }
    rc = trace_pairs(f->alg, f->sgf, matrix, open, gap, q, qoff, qlen, t, toff, tlen, n, ends, paths);
    if (rc == -2) fprintf(stderr, "%s: traceback needs a square matrix\n", who);
    else if (rc != 0) fprintf(stderr, "%s: GPU alignment failed: %s\n", who, pb_cuda_last_error());
    for (k = 0; k < n; ++k) { width[k] = 32; sat[k] = 0; }
    if (rc == 0 && f->kind >= 2 && f->bits != 32) {
        rc = trace_widths(f, matrix, open, gap, q, qoff, qlen, t, toff, tlen, n, ends, paths, width, sat);
        if (rc != 0) fprintf(stderr, "%s: GPU alignment failed: %s\n", who, pb_cuda_last_error());
    }
    for (k = 0; rc == 0 && k < n; ++k) {
        parasail_result_t *r;
        if (sat[k] != 1 && !paths[k]) {
            fprintf(stderr, "%s: pair %d leaves the range of the traceback kernel (int16)\n", who, k);
            continue;
        }
        if (!(r = pb_result_new(0))) { rc = -1; break; }
        r->flag = form_flags(f, width[k]);
        if (sat[k] == 1) {
            /* the saturated kernel's result (e.g. src/nw_trace_striped_avx2_256_8.c:431-437) */
            r->flag |= PARASAIL_FLAG_SATURATED;
        } else {
            r->score = ends[3 * k];
            r->end_query = ends[3 * k + 1];
            r->end_ref = ends[3 * k + 2];
            r->extra = paths[k];
            paths[k] = NULL;
        }
        results[k] = r;
    }
    for (k = 0; k < n; ++k) if (paths[k]) { free(paths[k]->ops); free(paths[k]); }
    if (rc != 0)
        for (k = 0; k < n; ++k) if (results[k]) { parasail_result_free(results[k]); results[k] = NULL; }
    free(ends);
    free(width);
    free(sat);
    free(paths);
    return rc;
}

static parasail_result_t *trace_one(const char *func, int alg, int sgflags, int kind, int bits, const char *s1,
                                    int s1Len, const char *s2, int s2Len, int open, int gap,
                                    const parasail_matrix_t *matrix)
{
    const trace_form f = {alg, sgflags, kind, bits};
    const int64_t zero = 0;
    parasail_result_t *r = NULL;
    if (!pb_gpu_ready(func)) return NULL;
    if (trace_results(func, &f, matrix, open, gap, s1, &zero, &s1Len, s2, &zero, &s2Len, 1, &r) != 0) return NULL;
    return r;
}

/* the reference's checks and messages (parasail/memory.h:46-80) */
#define TRACE_CHECKS()            \
    PB_CHECK_NULL(s1);            \
    PB_CHECK_GT0(s1Len);          \
    PB_CHECK_NULL(s2);            \
    PB_CHECK_GT0(s2Len);          \
    PB_CHECK_GE0(open);           \
    PB_CHECK_GE0(gap);            \
    PB_CHECK_NULL(matrix)

#define PCHECKS()                                                         \
    PB_CHECK_NULL(profile);                                               \
    PB_CHECK_NULL(profile->matrix);                                       \
    PB_CHECK_NULL(s2);                                                    \
    PB_CHECK_GT0(s2Len);                                                  \
    PB_CHECK_GE0(open);                                                   \
    PB_CHECK_GE0(gap)

/* one vector trace form at one width (W = 8, 16, 32 or sat; BITS 0 = sat),
 * direct and profile */
#define TRACE_VEC(name, ALG, SGF, SCHEME, KIND, W, BITS)                                                       \
    parasail_result_t *parasail_##name##_trace_##SCHEME##_##W(const char *const restrict s1, const int s1Len,   \
                                                              const char *const restrict s2, const int s2Len,    \
                                                              const int open, const int gap,                    \
                                                              const parasail_matrix_t *matrix)                  \
    {                                                                                                           \
        TRACE_CHECKS();                                                                                         \
        return trace_one(__func__, ALG, SGF, KIND, BITS, s1, s1Len, s2, s2Len, open, gap, matrix);             \
    }                                                                                                           \
    parasail_result_t *parasail_##name##_trace_##SCHEME##_profile_##W(                                          \
        const parasail_profile_t *const restrict profile, const char *const restrict s2, const int s2Len,       \
        const int open, const int gap)                                                                          \
    {                                                                                                           \
        PCHECKS();                                                                                              \
        return trace_one(__func__, ALG, SGF, KIND, BITS, profile->s1, profile->s1Len, s2, s2Len, open, gap,    \
                         profile->matrix);                                                                      \
    }

#define TRACE_FAMILY(name, ALG, SGF)                                                                           \
    parasail_result_t *parasail_##name##_trace(const char *const restrict s1, const int s1Len,                  \
                                               const char *const restrict s2, const int s2Len, const int open,   \
                                               const int gap, const parasail_matrix_t *matrix)                  \
    {                                                                                                           \
        TRACE_CHECKS();                                                                                         \
        return trace_one(__func__, ALG, SGF, 0, 32, s1, s1Len, s2, s2Len, open, gap, matrix);                  \
    }                                                                                                           \
    parasail_result_t *parasail_##name##_trace_scan(const char *const restrict s1, const int s1Len,             \
                                                    const char *const restrict s2, const int s2Len,              \
                                                    const int open, const int gap,                              \
                                                    const parasail_matrix_t *matrix)                            \
    {                                                                                                           \
        TRACE_CHECKS();                                                                                         \
        return trace_one(__func__, ALG, SGF, 1, 32, s1, s1Len, s2, s2Len, open, gap, matrix);                  \
    }                                                                                                           \
    TRACE_VEC(name, ALG, SGF, striped, 2, 8, 8)                                                                 \
    TRACE_VEC(name, ALG, SGF, striped, 2, 16, 16)                                                               \
    TRACE_VEC(name, ALG, SGF, striped, 2, 32, 32)                                                               \
    TRACE_VEC(name, ALG, SGF, striped, 2, sat, 0)                                                               \
    TRACE_VEC(name, ALG, SGF, scan, 3, 8, 8)                                                                    \
    TRACE_VEC(name, ALG, SGF, scan, 3, 16, 16)                                                                  \
    TRACE_VEC(name, ALG, SGF, scan, 3, 32, 32)                                                                  \
    TRACE_VEC(name, ALG, SGF, scan, 3, sat, 0)

TRACE_FAMILY(sw, PB_SW, 0)
TRACE_FAMILY(nw, PB_NW, 0)
TRACE_FAMILY(sg, PB_SG, PB_S1_BEG | PB_S1_END | PB_S2_BEG | PB_S2_END)
TRACE_FAMILY(sg_qb, PB_SG, PB_S1_BEG)
TRACE_FAMILY(sg_qe, PB_SG, PB_S1_END)
TRACE_FAMILY(sg_qx, PB_SG, PB_S1_BEG | PB_S1_END)
TRACE_FAMILY(sg_db, PB_SG, PB_S2_BEG)
TRACE_FAMILY(sg_de, PB_SG, PB_S2_END)
TRACE_FAMILY(sg_dx, PB_SG, PB_S2_BEG | PB_S2_END)
TRACE_FAMILY(sg_qb_de, PB_SG, PB_S1_BEG | PB_S2_END)
TRACE_FAMILY(sg_qe_db, PB_SG, PB_S1_END | PB_S2_BEG)
TRACE_FAMILY(sg_qb_db, PB_SG, PB_S1_BEG | PB_S2_BEG)
TRACE_FAMILY(sg_qe_de, PB_SG, PB_S1_END | PB_S2_END)

/* ---- batch CIGARs (include/parasail_b200.h) ------------------------------- */

/* the trace form a function name gives ("sw_trace", "nw_trace_scan_16",
 * "sg_qx_trace_striped_profile_sat", ...; the profile forms give the
 * results of the direct forms); -1 when it names none */
static int parse_trace_name(const char *funcname, trace_form *f)
{
    static const struct { const char *name; int alg, sgf; } algs[] = {
        {"sw", PB_SW, 0}, {"nw", PB_NW, 0},
        {"sg_qb_de", PB_SG, PB_S1_BEG | PB_S2_END}, {"sg_qe_db", PB_SG, PB_S1_END | PB_S2_BEG},
        {"sg_qb_db", PB_SG, PB_S1_BEG | PB_S2_BEG}, {"sg_qe_de", PB_SG, PB_S1_END | PB_S2_END},
        {"sg_qb", PB_SG, PB_S1_BEG}, {"sg_qe", PB_SG, PB_S1_END}, {"sg_qx", PB_SG, PB_S1_BEG | PB_S1_END},
        {"sg_db", PB_SG, PB_S2_BEG}, {"sg_de", PB_SG, PB_S2_END}, {"sg_dx", PB_SG, PB_S2_BEG | PB_S2_END},
        {"sg", PB_SG, PB_S1_BEG | PB_S1_END | PB_S2_BEG | PB_S2_END},
    };
    static const struct { const char *w; int bits; } widths[] = {{"8", 8}, {"16", 16}, {"32", 32}, {"sat", 0}};
    const char *s = funcname;
    size_t a;
    if (!s) return -1;
    memset(f, 0, sizeof *f);
    f->alg = -1;
    if (0 == strncmp(s, "parasail_", 9)) s += 9;
    for (a = 0; a < sizeof algs / sizeof algs[0]; ++a) {
        const size_t l = strlen(algs[a].name);
        if (0 == strncmp(s, algs[a].name, l) && 0 == strncmp(s + l, "_trace", 6)) {
            f->alg = algs[a].alg; f->sgf = algs[a].sgf; s += l + 6; break;
        }
    }
    if (f->alg < 0) return -1;
    f->bits = 32;
    if (!*s) { f->kind = 0; return 0; }
    if (!strcmp(s, "_scan")) { f->kind = 1; return 0; }
    if (0 == strncmp(s, "_striped_", 9)) { f->kind = 2; s += 9; }
    else if (0 == strncmp(s, "_scan_", 6)) { f->kind = 3; s += 6; }
    else return -1;
    if (0 == strncmp(s, "profile_", 8)) s += 8;
    for (a = 0; a < sizeof widths / sizeof widths[0]; ++a)
        if (!strcmp(s, widths[a].w)) { f->bits = widths[a].bits; return 0; }
    return -1;
}

/* Trace results of n independent pairs (host characters) in one GPU
 * pipeline; results[k] NULL for a pair whose result needs a path outside
 * the traceback kernels' 16-bit bounds (a message names it). */
int parasail_b200_batch_pairs_trace(const char *funcname, const parasail_matrix_t *matrix,
                                    const char *queries, const int64_t *qoffsets, const int *qlengths,
                                    const char *targets, const int64_t *toffsets, const int *tlengths, int n,
                                    int open, int gap, parasail_result_t **results)
{
    trace_form f;
    int k;
    if (!matrix || !queries || !qoffsets || !qlengths || !targets || !toffsets || !tlengths || !results) {
        fprintf(stderr, "%s: missing arguments\n", __func__);
        return -1;
    }
    if (n < 0 || open < 0 || gap < 0) { fprintf(stderr, "%s: invalid n/open/gap\n", __func__); return -1; }
    if (parse_trace_name(funcname, &f) != 0) {
        fprintf(stderr, "%s: unknown trace function '%s'\n", __func__, funcname ? funcname : "(null)");
        return -1;
    }
    if (n == 0) return 0;
    for (k = 0; k < n; ++k) {
        results[k] = NULL;
        if (qlengths[k] <= 0 || tlengths[k] <= 0) { fprintf(stderr, "%s: pair %d has an empty sequence\n", __func__, k); return -1; }
    }
    if (!pb_gpu_ready(__func__)) return -1;
    return trace_results(__func__, &f, matrix, open, gap, queries, qoffsets, qlengths, targets, toffsets, tlengths,
                         n, results);
}

int parasail_b200_batch_pairs_cigar(const char *funcname, const parasail_matrix_t *matrix,
                                    const char *queries, const int64_t *qoffsets, const int *qlengths,
                                    const char *targets, const int64_t *toffsets, const int *tlengths, int n,
                                    int open, int gap, parasail_b200_record_t *records, uint32_t *cigars,
                                    int *cigar_lengths, int *beg_query, int *beg_ref)
{
    trace_form f;
    parasail_result_t **res;
    int64_t off = 0;
    int k, rc;
    if (!matrix || !queries || !qoffsets || !qlengths || !targets || !toffsets || !tlengths || !records || !cigars ||
        !cigar_lengths || !beg_query || !beg_ref || !funcname) {
        fprintf(stderr, "%s: missing arguments\n", __func__);
        return -1;
    }
    if (n < 0 || open < 0 || gap < 0) { fprintf(stderr, "%s: invalid n/open/gap\n", __func__); return -1; }
    if (n == 0) return 0;
    if (parse_trace_name(funcname, &f) != 0) {
        fprintf(stderr, "%s: unknown trace function '%s'\n", __func__, funcname);
        return -1;
    }
    for (k = 0; k < n; ++k)
        if (qlengths[k] <= 0 || tlengths[k] <= 0) { fprintf(stderr, "%s: pair %d has an empty sequence\n", __func__, k); return -1; }
    if (!pb_gpu_ready(__func__)) return -1;
    res = (parasail_result_t **)calloc((size_t)n, sizeof *res);
    if (!res) return -1;
    rc = trace_results(__func__, &f, matrix, open, gap, queries, qoffsets, qlengths, targets, toffsets, tlengths, n,
                       res);
    for (k = 0; rc == 0 && k < n; off += (int64_t)qlengths[k] + tlengths[k], ++k) {
        parasail_b200_record_t *rec = &records[k];
        parasail_cigar_t *c;
        memset(rec, 0, sizeof *rec);
        cigar_lengths[k] = -1;
        beg_query[k] = beg_ref[k] = 0;
        if (!res[k]) continue;
        rec->score = res[k]->score; rec->end_query = res[k]->end_query; rec->end_ref = res[k]->end_ref;
        rec->flag = res[k]->flag;
        if (!res[k]->extra) continue;    /* saturated: no alignment */
        c = parasail_result_get_cigar(res[k], queries + qoffsets[k], qlengths[k], targets + toffsets[k], tlengths[k],
                                      matrix);
        if (c) {
            memcpy(cigars + off, c->seq, sizeof(uint32_t) * (size_t)c->len);
            cigar_lengths[k] = c->len;
            beg_query[k] = c->beg_query;
            beg_ref[k] = c->beg_ref;
            parasail_cigar_free(c);
        }
    }
    for (k = 0; k < n; ++k) if (res[k]) parasail_result_free(res[k]);
    free(res);
    return rc;
}
