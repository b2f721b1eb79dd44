/*
 * io.c -- FASTA / FASTQ files, the '$'-separated packed text, and matrices
 * read from files: the reference's parasail/io.h API (jeffdaily/parasail
 * v2.6.2, src/io.c and src/parser.c) with the same results on the same
 * bytes.
 *
 * Record parsing (parasail_sequences_from_file) follows the rules of the
 * kseq reader the reference uses (contrib/kseq.h, "Last Modified:
 * 05MAR2012", read through parser.c:120-176):
 *   - a record starts at the first '>' or '@' (later records at the header
 *     character that ended the previous sequence);
 *   - name: the header up to the first white-space character; comment: the
 *     rest of that line when the name did not end at '\n';
 *   - sequence: every following line not starting with '>', '+' or '@',
 *     empty lines skipped, the line ends removed (and one '\r' at the end of
 *     the text read so far when that text is longer than one character);
 *   - '+' after the sequence makes it FASTQ: the '+' line is skipped and
 *     quality lines are read until the quality is as long as the sequence;
 *     a missing or short quality ends the file (parser.c keeps the records
 *     read before it).
 * The scanners of src/io.c (stat / pack of FASTA and FASTQ buffers) are
 * restated with the same acceptance rules, the same counters and Welford
 * statistics (parasail/stats.h), but every read is bounded by the buffer
 * size, where the reference's skip_line may read past the end of a file
 * without a final newline.
 */
#include <ctype.h>
#include <errno.h>
#include <fcntl.h>
#include <limits.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include "parasail.h"
#include "parasail/io.h"

/* ---- running statistics (the Welford update of parasail/stats.h) -------- */

typedef struct {
    unsigned long n;
    double mean, m2, lo, hi;
} pb_stats;

static void st_add(pb_stats *s, double x)
{
    double d;
    if (s->n == 0) { s->lo = x; s->hi = x; }
    else { s->lo = s->lo < x ? s->lo : x; s->hi = s->hi > x ? s->hi : x; }
    s->n += 1;
    d = x - s->mean;
    s->mean += d / (double)s->n;
    s->m2 += d * (x - s->mean);
}

static double st_stddev(const pb_stats *s) { return sqrt(s->m2 / (double)(s->n - 1UL)); }

/* ---- files ------------------------------------------------------------------ */

parasail_file_t *parasail_open(const char *fname)
{
    parasail_file_t *pf;
    struct stat fs;
    void *buf;
    int fd;
    if (NULL == fname) {
        fprintf(stderr, "parasail_open: NULL filename\n");
        return NULL;
    }
    fd = open(fname, O_RDONLY);
    if (fd == -1) {
        perror("open");
        fprintf(stderr, "parasail_open: cannot open input file `%s'\n", fname);
        return NULL;
    }
    if (fstat(fd, &fs) == -1) {
        perror("fstat");
        fprintf(stderr, "parasail_open: cannont stat input file `%s'\n", fname);
        close(fd);
        return NULL;
    }
    buf = mmap(NULL, (size_t)fs.st_size, PROT_READ, MAP_SHARED, fd, 0);
    if (buf == MAP_FAILED) {
        perror("mmap");
        fprintf(stderr, "parasail_open: cannont mmap input file `%s'\n", fname);
        close(fd);
        return NULL;
    }
    pf = (parasail_file_t *)malloc(sizeof *pf);
    if (!pf) {
        perror("malloc");
        fprintf(stderr, "parasail_open: cannont allocate parasail_file_t\n");
        munmap(buf, (size_t)fs.st_size);
        close(fd);
        return NULL;
    }
    pf->fd = fd;
    pf->size = fs.st_size;
    pf->buf = (const char *)buf;
    return pf;
}

void parasail_close(parasail_file_t *pf)
{
    if (NULL == pf) {
        fprintf(stderr, "parasail_close: NULL file\n");
        return;
    }
    if (munmap((void *)pf->buf, (size_t)pf->size) == -1) {
        perror("munmap");
        fprintf(stderr, "parasail_close: cannot munmap file buffer\n");
    }
    if (close(pf->fd) == -1) {
        perror("close");
        fprintf(stderr, "parasail_close: cannot close file descriptor\n");
    }
    free(pf);
}

int parasail_is_fasta_buffer(const char *buf, off_t size)
{
    if (NULL == buf) {
        fprintf(stderr, "parasail_is_fasta_buffer: NULL pointer\n");
        return -1;
    }
    return size > 0 && buf[0] == '>';
}

int parasail_is_fastq_buffer(const char *buf, off_t size)
{
    if (NULL == buf) {
        fprintf(stderr, "parasail_is_fastq_buffer: NULL pointer\n");
        return -1;
    }
    return size > 0 && buf[0] == '@';
}

int parasail_is_fasta(const parasail_file_t *pf)
{
    if (NULL == pf) {
        fprintf(stderr, "parasail_is_fasta: NULL pointer\n");
        return -1;
    }
    return parasail_is_fasta_buffer(pf->buf, pf->size);
}

int parasail_is_fastq(const parasail_file_t *pf)
{
    if (NULL == pf) {
        fprintf(stderr, "parasail_is_fastq: NULL pointer\n");
        return -1;
    }
    return parasail_is_fastq_buffer(pf->buf, pf->size);
}

/* ---- the buffer scanners of src/io.c ------------------------------------------ */

static int is_eol(char c) { return c == '\n' || c == '\r'; }

/* index of the newline ending the line at i (one further for a "\r\n" or
 * "\n\r" pair); the size when the line has no newline (src/io.c:265-278) */
static off_t line_end(const char *T, off_t i, off_t size)
{
    while (i < size && !is_eol(T[i])) ++i;
    if (i + 1 < size && is_eol(T[i + 1])) ++i;
    return i;
}

static parasail_file_stat_t *new_stat(unsigned long seqs, unsigned long chars, const pb_stats *st,
                                      const char *who)
{
    parasail_file_stat_t *p = (parasail_file_stat_t *)malloc(sizeof *p);
    if (!p) {
        perror("malloc");
        fprintf(stderr, "%s: cannont allocate parasail_file_stat_t", who);
        return NULL;
    }
    p->sequences = seqs;
    p->characters = chars;
    p->shortest = (unsigned long)st->lo;
    p->longest = (unsigned long)st->hi;
    p->mean = (float)st->mean;
    p->stddev = (float)st_stddev(st);
    return p;
}

/* One pass over a FASTA buffer (src/io.c:291-365, :607-681): letters are
 * kept, line ends skipped, a '>' line starts the next sequence, any other
 * character is an error. With out != NULL the letters are written with a
 * '$' after each sequence. Returns 0, or -1 after printing the error. */
static int scan_fasta(const char *T, off_t size, const char *who, unsigned long *seqs,
                      unsigned long *chars, pb_stats *st, char *out, long *w)
{
    off_t i = 0;
    unsigned long c = 0;
    if (size <= 0 || T[0] != '>') {
        fprintf(stderr, "%s: poorly formatted FASTA file\n", who);
        return -1;
    }
    i = line_end(T, 0, size) + 1;
    *seqs = 1;
    while (i < size) {
        const unsigned char ch = (unsigned char)T[i];
        if (ch == '>') {
            ++*seqs;
            st_add(st, (double)c);
            c = 0;
            if (out) out[(*w)++] = '$';
            i = line_end(T, i, size);
        } else if (isalpha(ch)) {
            ++c;
            ++*chars;
            if (out) out[(*w)++] = (char)ch;
        } else if (is_eol((char)ch)) {
            if (i + 1 < size && is_eol(T[i + 1])) ++i;
        } else if (isprint(ch)) {
            fprintf(stderr, "%s: non-alpha character ('%c')\n", who, ch);
            return -1;
        } else {
            fprintf(stderr, "%s: non-printing character ('%d')\n", who, (int)(char)ch);
            return -1;
        }
        ++i;
    }
    if (c == 0) {
        fprintf(stderr, "%s: empty sequence at end of input\n", who);
        return -1;
    }
    st_add(st, (double)c);
    if (out) out[(*w)++] = '$';
    return 0;
}

/* One pass over a FASTQ buffer (src/io.c:379-470, :697-789): four lines a
 * record, '@' header, sequence line, '+' line, quality line. The length
 * statistics take each sequence length after its line and again when the
 * next record starts, and the character count stays 0, as in the
 * reference's scanner. With out != NULL the sequence lines are written,
 * joined by '$' and ended by one. */
static int scan_fastq(const char *T, off_t size, const char *who, unsigned long *seqs,
                      unsigned long *chars, pb_stats *st, char *out, long *w)
{
    off_t i = 0;
    unsigned long c = 0, line = 0;
    int first = 1;
    (void)chars;
    while (i < size) {
        if (T[i] != '@') {
            fprintf(stderr, "%s: poorly formatted FASTQ file, line %lu\n", who, line);
            return -1;
        }
        ++*seqs;
        if (first) first = 0;
        else {
            st_add(st, (double)c);
            if (out) out[(*w)++] = '$';
        }
        c = 0;
        i = line_end(T, i, size) + 1;
        ++line;
        while (i < size && !is_eol(T[i])) {
            if (out) out[(*w)++] = T[i];
            ++c;
            ++i;
        }
        if (i + 1 < size && is_eol(T[i + 1])) ++i;
        st_add(st, (double)c);
        ++i;
        ++line;
        if (i >= size || T[i] != '+') {
            fprintf(stderr, "%s: poorly formatted FASTQ file, line %lu\n", who, line);
            return -1;
        }
        i = line_end(T, i, size) + 1;
        ++line;
        i = line_end(T, i, size) + 1;
        ++line;
    }
    if (out) out[(*w)++] = '$';
    return 0;
}

parasail_file_stat_t *parasail_stat_fasta_buffer(const char *T, off_t size)
{
    unsigned long seqs = 0, chars = 0;
    pb_stats st;
    memset(&st, 0, sizeof st);
    if (NULL == T) {
        fprintf(stderr, "parasail_stat_fasta_buffer: NULL pointer\n");
        return NULL;
    }
    if (scan_fasta(T, size, "parasail_stat_fasta_buffer", &seqs, &chars, &st, NULL, NULL) != 0) return NULL;
    return new_stat(seqs, chars, &st, "parasail_stat_fasta_buffer");
}

parasail_file_stat_t *parasail_stat_fastq_buffer(const char *T, off_t size)
{
    unsigned long seqs = 0, chars = 0;
    pb_stats st;
    memset(&st, 0, sizeof st);
    if (NULL == T) {
        fprintf(stderr, "parasail_stat_fastq_buffer: NULL pointer\n");
        return NULL;
    }
    if (scan_fastq(T, size, "parasail_stat_fastq_buffer", &seqs, &chars, &st, NULL, NULL) != 0) return NULL;
    return new_stat(seqs, chars, &st, "parasail_stat_fastq_buffer");
}

parasail_file_stat_t *parasail_stat_buffer(const char *buf, off_t size)
{
    parasail_file_stat_t *s = NULL;
    if (NULL == buf) {
        fprintf(stderr, "parasail_stat_buffer: NULL pointer\n");
        return NULL;
    }
    if (1 == parasail_is_fasta_buffer(buf, size)) s = parasail_stat_fasta_buffer(buf, size);
    else if (1 == parasail_is_fastq_buffer(buf, size)) s = parasail_stat_fastq_buffer(buf, size);
    else {
        fprintf(stderr, "parasail_stat: cannot determine file format\n");
        return NULL;
    }
    if (!s) fprintf(stderr, "parasail_stat_buffer: failed\n");
    return s;
}

parasail_file_stat_t *parasail_stat_fasta(const parasail_file_t *pf)
{
    if (NULL == pf) {
        fprintf(stderr, "parasail_stat_fasta: NULL pointer\n");
        return NULL;
    }
    return parasail_stat_fasta_buffer(pf->buf, pf->size);
}

parasail_file_stat_t *parasail_stat_fastq(const parasail_file_t *pf)
{
    if (NULL == pf) {
        fprintf(stderr, "parasail_stat_fastq: NULL pointer\n");
        return NULL;
    }
    return parasail_stat_fastq_buffer(pf->buf, pf->size);
}

parasail_file_stat_t *parasail_stat(const parasail_file_t *pf)
{
    parasail_file_stat_t *s = NULL;
    if (NULL == pf) {
        fprintf(stderr, "parasail_stat: NULL pointer\n");
        return NULL;
    }
    if (1 == parasail_is_fasta(pf)) s = parasail_stat_fasta(pf);
    else if (1 == parasail_is_fastq(pf)) s = parasail_stat_fastq(pf);
    else {
        fprintf(stderr, "parasail_stat: cannot determine file format\n");
        return NULL;
    }
    if (!s) fprintf(stderr, "parasail_stat: failed\n");
    return s;
}

char *parasail_read(const parasail_file_t *pf, long *size)
{
    char *b;
    if (NULL == pf) {
        fprintf(stderr, "parasail_read: NULL pointer\n");
        return NULL;
    }
    if (NULL == size) {
        fprintf(stderr, "parasail_read: NULL size pointer\n");
        return NULL;
    }
    b = (char *)malloc((size_t)pf->size + 1);
    if (!b) {
        perror("malloc");
        fprintf(stderr, "parasail_read: cannont malloc buffer for input file");
        return NULL;
    }
    memcpy(b, pf->buf, (size_t)pf->size);
    b[pf->size] = '\0';
    *size = (long)pf->size;
    return b;
}

/* packed text of a buffer: a counting pass sizes the output exactly */
static char *pack_with(int fastq, const char *T, off_t size, long *packed_size, const char *who)
{
    unsigned long seqs = 0, chars = 0;
    pb_stats st;
    char *P;
    long w = 0;
    off_t cap;
    if (NULL == T) {
        fprintf(stderr, "%s: NULL pointer\n", who);
        return NULL;
    }
    if (NULL == packed_size) {
        fprintf(stderr, "%s: NULL size pointer\n", who);
        return NULL;
    }
    memset(&st, 0, sizeof st);
    if ((fastq ? scan_fastq : scan_fasta)(T, size, who, &seqs, &chars, &st, NULL, NULL) != 0) {
        fprintf(stderr, fastq ? "parasail_stat_fastq_buffer: fastq stat failed\n"
                              : "parasail_stat_fasta_buffer: fasta stat failed\n");
        return NULL;
    }
    /* at most every byte plus a '$' per record and the NUL */
    cap = size + (off_t)seqs + 2;
    P = (char *)malloc((size_t)cap);
    if (!P) {
        perror("malloc");
        fprintf(stderr, "%s: malloc failed\n", who);
        return NULL;
    }
    seqs = chars = 0;
    memset(&st, 0, sizeof st);
    (fastq ? scan_fastq : scan_fasta)(T, size, who, &seqs, &chars, &st, P, &w);
    P[w] = '\0';
    *packed_size = w;
    return P;
}

char *parasail_pack_fasta_buffer(const char *T, off_t size, long *packed_size)
{
    return pack_with(0, T, size, packed_size, "parasail_pack_fasta_buffer");
}

char *parasail_pack_fastq_buffer(const char *T, off_t size, long *packed_size)
{
    return pack_with(1, T, size, packed_size, "parasail_pack_fastq_buffer");
}

char *parasail_pack_buffer(const char *buf, off_t size, long *packed_size)
{
    char *p = NULL;
    if (NULL == buf) {
        fprintf(stderr, "parasail_pack_buffer: NULL pointer\n");
        return NULL;
    }
    if (NULL == packed_size) {
        fprintf(stderr, "parasail_pack_buffer: NULL size pointer\n");
        return NULL;
    }
    if (1 == parasail_is_fasta_buffer(buf, size)) p = parasail_pack_fasta_buffer(buf, size, packed_size);
    else if (1 == parasail_is_fastq_buffer(buf, size)) p = parasail_pack_fastq_buffer(buf, size, packed_size);
    else {
        fprintf(stderr, "parasail_pack: cannot determine file format\n");
        return NULL;
    }
    if (!p) fprintf(stderr, "parasail_pack_buffer: failed\n");
    return p;
}

char *parasail_pack_fasta(const parasail_file_t *pf, long *size)
{
    if (NULL == pf) {
        fprintf(stderr, "parasail_pack_fasta: NULL pointer\n");
        return NULL;
    }
    if (NULL == size) {
        fprintf(stderr, "parasail_pack_fasta: NULL size pointer\n");
        return NULL;
    }
    return parasail_pack_fasta_buffer(pf->buf, pf->size, size);
}

char *parasail_pack_fastq(const parasail_file_t *pf, long *size)
{
    if (NULL == pf) {
        fprintf(stderr, "parasail_pack_fastq: NULL pointer\n");
        return NULL;
    }
    if (NULL == size) {
        fprintf(stderr, "parasail_pack_fastq: NULL size pointer\n");
        return NULL;
    }
    return parasail_pack_fastq_buffer(pf->buf, pf->size, size);
}

char *parasail_pack(const parasail_file_t *pf, long *size)
{
    char *p = NULL;
    if (NULL == pf) {
        fprintf(stderr, "parasail_pack: NULL pointer\n");
        return NULL;
    }
    if (NULL == size) {
        fprintf(stderr, "parasail_pack: NULL size pointer\n");
        return NULL;
    }
    if (1 == parasail_is_fasta(pf)) p = parasail_pack_fasta(pf, size);
    else if (1 == parasail_is_fastq(pf)) p = parasail_pack_fastq(pf, size);
    else {
        fprintf(stderr, "parasail_pack: cannot determine file format\n");
        return NULL;
    }
    if (!p) fprintf(stderr, "parasail_pack: failed\n");
    return p;
}

/* ---- records (parasail_sequences_from_file) ------------------------------------ */

typedef struct {
    const unsigned char *p;
    size_t n, i;
} rd_t;

typedef struct {
    char *s;
    size_t l, m;
} sbuf;

static int sb_put(sbuf *b, const unsigned char *src, size_t k)
{
    if (b->l + k + 1 > b->m) {
        size_t m = b->m ? b->m : 64;
        char *q;
        while (m < b->l + k + 1) m *= 2;
        q = (char *)realloc(b->s, m);
        if (!q) return -1;
        b->s = q;
        b->m = m;
    }
    memcpy(b->s + b->l, src, k);
    b->l += k;
    b->s[b->l] = '\0';
    return 0;
}

static int rd_getc(rd_t *r) { return r->i < r->n ? (int)r->p[r->i++] : -1; }

/* the rest of a line (up to and without '\n') appended to b; one trailing
 * '\r' of b is then dropped when b is longer than one character. Returns -1
 * when nothing was left to read, -2 when out of memory. */
static int rd_line(rd_t *r, sbuf *b)
{
    size_t j = r->i;
    if (r->i >= r->n) return -1;
    while (j < r->n && r->p[j] != '\n') ++j;
    if (sb_put(b, r->p + r->i, j - r->i) != 0) return -2;
    r->i = j < r->n ? j + 1 : j;
    if (b->l > 1 && b->s[b->l - 1] == '\r') b->s[--b->l] = '\0';
    return 0;
}

/* one record; returns its sequence length, -1 at the end of the input, -2
 * on a truncated quality, -3 when out of memory */
static long rd_record(rd_t *r, int *last_char, sbuf *name, sbuf *comment, sbuf *seq, sbuf *qual)
{
    int c;
    size_t j;
    if (*last_char == 0) {
        while ((c = rd_getc(r)) >= 0 && c != '>' && c != '@') {
        }
        if (c < 0) return -1;
        *last_char = c;
    }
    name->l = comment->l = seq->l = qual->l = 0;
    if (name->s) name->s[0] = '\0';
    if (comment->s) comment->s[0] = '\0';
    if (seq->s) seq->s[0] = '\0';
    if (qual->s) qual->s[0] = '\0';
    /* name: up to the first white space, which is consumed */
    if (r->i >= r->n) return -1;
    j = r->i;
    while (j < r->n && !isspace(r->p[j])) ++j;
    if (sb_put(name, r->p + r->i, j - r->i) != 0) return -3;
    c = j < r->n ? (int)r->p[j] : 0;
    r->i = j < r->n ? j + 1 : j;
    if (c != '\n' && rd_line(r, comment) == -2) return -3;
    /* sequence lines */
    while ((c = rd_getc(r)) >= 0 && c != '>' && c != '+' && c != '@') {
        const unsigned char ch = (unsigned char)c;
        if (c == '\n') continue;
        if (sb_put(seq, &ch, 1) != 0) return -3;
        if (rd_line(r, seq) == -2) return -3;
    }
    if (c == '>' || c == '@') *last_char = c;
    if (c != '+') return (long)seq->l;
    /* FASTQ: skip the '+' line, then quality lines up to the sequence length */
    while ((c = rd_getc(r)) >= 0 && c != '\n') {
    }
    if (c < 0) return -2;
    for (;;) {
        const int k = rd_line(r, qual);
        if (k == -2) return -3;
        if (k < 0 || qual->l >= seq->l) break;
    }
    *last_char = 0;
    if (seq->l != qual->l) return -2;
    return (long)seq->l;
}

static char *dup_or_null(const sbuf *b)
{
    char *s;
    if (b->l == 0) return NULL;
    s = (char *)calloc(b->l + 1, 1);
    if (s) memcpy(s, b->s, b->l);
    return s;
}

/* the whole input in memory */
static unsigned char *slurp(const char *filename, size_t *n)
{
    int fd;
    size_t cap = 1 << 20, len = 0;
    unsigned char *buf;
    const int is_stdin = 0 == strncmp("stdin", filename, 5);
    fd = is_stdin ? 0 : open(filename, O_RDONLY);
    if (fd < 0) {
        perror("fopen");
        return NULL;
    }
    buf = (unsigned char *)malloc(cap);
    while (buf) {
        ssize_t k;
        if (len == cap) {
            unsigned char *q = (unsigned char *)realloc(buf, cap * 2);
            if (!q) { free(buf); buf = NULL; break; }
            buf = q;
            cap *= 2;
        }
        k = read(fd, buf + len, cap - len);
        if (k < 0) {
            if (errno == EINTR) continue;
            free(buf);
            buf = NULL;
            break;
        }
        if (k == 0) break;
        len += (size_t)k;
    }
    if (!is_stdin) close(fd);
    *n = len;
    return buf;
}

parasail_sequences_t *parasail_sequences_from_file(const char *filename)
{
    parasail_sequences_t *ret;
    parasail_sequence_t *v;
    size_t count = 0, cap = 1000, chars = 0;
    sbuf name = {0, 0, 0}, comment = {0, 0, 0}, seq = {0, 0, 0}, qual = {0, 0, 0};
    pb_stats st;
    rd_t r;
    int last_char = 0, err = 0;
    long l;
    if (NULL == filename) {
        fprintf(stderr, "parasail_sequences_from_file: failed\n");
        return NULL;
    }
    memset(&st, 0, sizeof st);
    ret = (parasail_sequences_t *)malloc(sizeof *ret);
    v = (parasail_sequence_t *)malloc(sizeof *v * cap);
    if (!ret || !v) {
        perror("malloc");
        fprintf(stderr, "parasail_sequences_from_file: failed\n");
        free(ret);
        free(v);
        return NULL;
    }
    r.p = slurp(filename, &r.n);
    r.i = 0;
    if (!r.p) {
        fprintf(stderr, "parasail_sequences_from_file: failed\n");
        free(ret);
        free(v);
        return NULL;
    }
    while ((l = rd_record(&r, &last_char, &name, &comment, &seq, &qual)) >= 0) {
        parasail_sequence_t *e = &v[count];
        e->name.l = name.l; e->comment.l = comment.l; e->seq.l = seq.l; e->qual.l = qual.l;
        e->name.s = dup_or_null(&name);
        e->comment.s = dup_or_null(&comment);
        e->seq.s = dup_or_null(&seq);
        e->qual.s = dup_or_null(&qual);
        st_add(&st, (double)seq.l);
        chars += seq.l;
        ++count;
        if ((name.l && !e->name.s) || (comment.l && !e->comment.s) || (seq.l && !e->seq.s) ||
            (qual.l && !e->qual.s)) {
            err = 1;
            break;
        }
        if (count >= cap) {
            parasail_sequence_t *q = (parasail_sequence_t *)realloc(v, sizeof *v * cap * 2);
            if (!q) { err = 1; break; }
            v = q;
            cap *= 2;
        }
    }
    if (l == -3) err = 1;
    free((void *)r.p);
    free(name.s); free(comment.s); free(seq.s); free(qual.s);
    ret->seqs = v;
    ret->l = count;
    ret->characters = chars;
    ret->shortest = (size_t)st.lo;
    ret->longest = (size_t)st.hi;
    ret->mean = (float)st.mean;
    ret->stddev = (float)st_stddev(&st);
    if (err) {
        fprintf(stderr, "parasail_sequences_from_file: failed\n");
        parasail_sequences_free(ret);
        return NULL;
    }
    return ret;
}

void parasail_sequences_free(parasail_sequences_t *sequences)
{
    size_t i;
    if (!sequences) return;
    for (i = 0; i < sequences->l; ++i) {
        free(sequences->seqs[i].name.s);
        free(sequences->seqs[i].comment.s);
        free(sequences->seqs[i].seq.s);
        free(sequences->seqs[i].qual.s);
    }
    free(sequences->seqs);
    free(sequences);
}

char *parasail_sequences_pack(const parasail_sequences_t *sequences, size_t *size)
{
    size_t i, off = 0;
    char *p;
    if (!sequences || !size) {
        fprintf(stderr, "parasail_sequences_pack: failed\n");
        return NULL;
    }
    p = (char *)malloc(sequences->characters + sequences->l + 1);
    if (!p) {
        perror("malloc");
        fprintf(stderr, "parasail_sequences_pack: failed\n");
        return NULL;
    }
    for (i = 0; i < sequences->l; ++i) {
        if (sequences->seqs[i].seq.l) memcpy(p + off, sequences->seqs[i].seq.s, sequences->seqs[i].seq.l);
        off += sequences->seqs[i].seq.l;
        p[off++] = '$';
    }
    p[off] = '\0';
    *size = off;
    return p;
}

/* ---- matrices from files (src/io.c:960-1179) ------------------------------------ */

/* a signed decimal of at most 9 digits after optional spaces/tabs
 * (src/io.c:794-835); 1 with *i past it, -1 when there is none */
static int read_int(const char *T, off_t size, off_t *i_, int *out)
{
    off_t i = *i_;
    char tok[10];
    int p;
    while (i < size && (T[i] == ' ' || T[i] == '\t')) ++i;
    if (i >= size || !(isdigit((unsigned char)T[i]) || T[i] == '-')) return -1;
    tok[0] = T[i++];
    for (p = 1; p < 10; ++p) {
        if (i < size && isdigit((unsigned char)T[i])) tok[p] = T[i++];
        else break;
    }
    if (p == 10) return -1;
    tok[p] = '\0';
    if (sscanf(tok, "%d", out) != 1) return -1;
    *i_ = i;
    return 1;
}

/* the letters (and '*') of the header line at i; NULL when the line holds
 * anything else or no letter (src/io.c:838-893) */
static char *read_alphabet(const char *T, off_t i, off_t size)
{
    size_t count = 0;
    off_t k;
    char *a;
    for (k = i; k < size && T[k] != '\n' && T[k] != '\r' && T[k] != '#'; ++k) {
        if (T[k] == ' ' || T[k] == '\t') continue;
        if (isalpha((unsigned char)T[k]) || T[k] == '*') ++count;
        else return NULL;
    }
    if (count == 0) return NULL;
    a = (char *)malloc(count + 1);
    if (!a) return NULL;
    count = 0;
    for (k = i; k < size && T[k] != '\n' && T[k] != '\r' && T[k] != '#'; ++k)
        if (T[k] != ' ' && T[k] != '\t') a[count++] = T[k];
    a[count] = '\0';
    return a;
}

static parasail_matrix_t *matrix_from_file(const char *filename, int case_sensitive)
{
    const char *who = "parasail_matrix_from_file";
    parasail_file_t *pf;
    const char *T;
    off_t i = 0, size;
    char *alphabet = NULL, *query = NULL;
    int *values = NULL, *mapper = NULL;
    size_t asize = 0, nq = 0, qcap = 0, nv = 0, vcap = 0, rows = 0, c;
    int mx = INT_MIN, mn = INT_MAX, type = PARASAIL_MATRIX_TYPE_SQUARE;
    const char *err = NULL;
    parasail_matrix_t *m;
    if (NULL == filename) {
        fprintf(stderr, "%s: NULL pointer\n", who);
        return NULL;
    }
    pf = parasail_open(filename);
    if (!pf) {
        fprintf(stderr, "%s: parasail_open(%s) failed\n", who, filename);
        return NULL;
    }
    T = pf->buf;
    size = pf->size;
    while (i < size && !err) {
        const unsigned char ch = (unsigned char)T[i];
        if (ch == '#') {
            i = line_end(T, i, size);
        } else if (isalnum(ch) || ch == '*' || ch == '-') {
            if (!alphabet) {
                alphabet = read_alphabet(T, i, size);
                if (!alphabet) { err = "poorly formed matrix file alphabet"; break; }
                asize = strlen(alphabet);
                vcap = asize * asize;
                qcap = asize;
                values = (int *)malloc(sizeof(int) * vcap);
                query = (char *)malloc(qcap + 1);
                if (!values || !query) { err = "cannont malloc buffer for matrix"; break; }
                i = line_end(T, i, size);
            } else {
                size_t j;
                if (nq >= qcap) {
                    char *q = (char *)realloc(query, qcap * 2 + 1);
                    if (!q) { err = "couldn't grow query size"; break; }
                    query = q;
                    qcap *= 2;
                }
                ++rows;
                /* a row may omit its letter (a PSSM row): recorded as '*' */
                if (isalpha(ch) || ch == '*') { query[nq++] = (char)ch; ++i; }
                else query[nq++] = '*';
                for (j = 0; j < asize; ++j) {
                    int v = 0;
                    if (read_int(T, size, &i, &v) != 1) { err = "poorly formed matrix file"; break; }
                    if (nv >= vcap) {
                        int *q = (int *)realloc(values, sizeof(int) * vcap * 2);
                        if (!q) { err = "couldn't grow matrix size"; break; }
                        values = q;
                        vcap *= 2;
                    }
                    values[nv++] = v;
                    mx = v > mx ? v : mx;
                    mn = v < mn ? v : mn;
                }
                if (err) break;
            }
        } else if (ch == '\n' || ch == '\r') {
            if (i + 1 < size && (T[i + 1] == '\n' || T[i + 1] == '\r')) ++i;
        } else if (ch == ' ' || ch == '\t') {
        } else if (isprint(ch)) {
            fprintf(stderr, "%s: non-alpha character in matrix file ('%c')\n", who, ch);
            err = "";
            break;
        } else {
            fprintf(stderr, "%s: non-printing character in matrix file ('%d')\n", who, (int)(char)ch);
            err = "";
            break;
        }
        ++i;
    }
    parasail_close(pf);
    if (!err && !alphabet) err = "poorly formed matrix file alphabet";
    if (!err) {
        query[nq] = '\0';
        if (asize == nq && 0 == strcmp(alphabet, query)) {
            if (nv != asize * asize) err = "matrix is missing values";
            else if (rows != asize) err = "matrix is missing rows";
        } else {
            type = PARASAIL_MATRIX_TYPE_PSSM;
            if (nv != asize * rows) err = "matrix is missing values";
        }
    }
    if (!err) {
        mapper = (int *)malloc(sizeof(int) * 256);
        m = (parasail_matrix_t *)malloc(sizeof *m);
        if (!mapper || !m) {
            free(mapper);
            free(m);
            err = "cannont malloc mapper buffer for matrix file";
        }
    }
    if (err) {
        if (*err) fprintf(stderr, "%s: %s\n", who, err);
        free(alphabet);
        free(query);
        free(values);
        return NULL;
    }
    for (c = 0; c < 256; ++c) mapper[c] = (int)asize - 1;
    for (c = 0; c < asize; ++c) {
        const unsigned char a = (unsigned char)alphabet[c];
        if (case_sensitive) mapper[a] = (int)c;
        else {
            mapper[toupper(a)] = (int)c;
            mapper[tolower(a)] = (int)c;
        }
    }
    m->name = filename;
    m->matrix = values;
    m->mapper = mapper;
    m->size = (int)asize;
    m->max = mx;
    m->min = mn;
    m->user_matrix = values;
    m->type = type;
    m->length = (int)rows;
    m->alphabet = alphabet;
    m->query = query;
    return m;
}

parasail_matrix_t *parasail_matrix_from_file(const char *filename)
{
    return matrix_from_file(filename, 0);
}

parasail_matrix_t *parasail_matrix_from_file_case_sensitive(const char *filename)
{
    return matrix_from_file(filename, 1);
}
