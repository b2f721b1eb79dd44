/*
 * matrix.c -- substitution matrices: built-in lookup, simple and PSSM
 * creation, copy, conversion, modification and release.
 *
 * Behaviour follows the reference (jeffdaily/parasail v2.6.2):
 * parasail_matrix_lookup src/matrix_lookup.c:16-33, create src/memory.c:336-407,
 * pssm create :420-494, copy :496-548, convert :550-600, set_value :602-620,
 * free :622-640. The built-in tables are the published BLOSUM/PAM/NUC data
 * (matrices_data.inc); each is parsed once, on first lookup, into a static
 * parasail_matrix_t whose user_matrix is NULL (built-ins cannot be freed or
 * modified, as in the reference).
 */
#include <ctype.h>
#include <limits.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "pb_internal.h"

static const char *const pb_matrix_text =
#include "matrices_data.inc"
    ;

#define PB_MAX_BUILTIN 96

typedef struct builtin {
    parasail_matrix_t m;
    char name[32];
    char alphabet[40];
    int mapper[256];
    int *values;
} builtin;

static builtin g_builtins[PB_MAX_BUILTIN];
static int g_nbuiltins = 0;
static pthread_once_t g_once = PTHREAD_ONCE_INIT;

/* Mapper rule of every built-in and created matrix: each alphabet letter in
 * both cases maps to its index, everything else to the last index (the
 * trailing '*' column, or the last letter when there is no '*'). */
static void fill_mapper(int *mapper, const char *alphabet, int size, int case_sensitive)
{
    int i;
    for (i = 0; i < 256; ++i) mapper[i] = size - 1;
    for (i = 0; alphabet[i]; ++i) {
        unsigned char c = (unsigned char)alphabet[i];
        if (case_sensitive) {
            mapper[c] = i;
        } else {
            mapper[toupper(c)] = i;
            mapper[tolower(c)] = i;
        }
    }
}

static void parse_builtins(void)
{
    const char *p = pb_matrix_text;
    while (*p && g_nbuiltins < PB_MAX_BUILTIN) {
        builtin *b = &g_builtins[g_nbuiltins];
        int mx, mn, size, k, n = 0;
        char *end;
        if (sscanf(p, "%31s %39s %d %d%n", b->name, b->alphabet, &mx, &mn, &n) != 4) break;
        p += n;
        size = (int)strlen(b->alphabet);
        b->values = (int *)malloc(sizeof(int) * size * size);
        if (!b->values) break;
        for (k = 0; k < size * size; ++k) {
            b->values[k] = (int)strtol(p, &end, 10);
            p = end;
        }
        while (*p == ' ' || *p == '\n') ++p;
        fill_mapper(b->mapper, b->alphabet, size, 0);
        b->m.name = b->name;
        b->m.matrix = b->values;
        b->m.mapper = b->mapper;
        b->m.size = size;
        b->m.max = mx;
        b->m.min = mn;
        b->m.user_matrix = NULL;
        b->m.type = PARASAIL_MATRIX_TYPE_SQUARE;
        b->m.length = size;
        b->m.alphabet = b->alphabet;
        b->m.query = NULL;
        ++g_nbuiltins;
    }
}

const parasail_matrix_t *parasail_matrix_lookup(const char *matrixname)
{
    int k;
    if (!matrixname) return NULL;
    pthread_once(&g_once, parse_builtins);
    for (k = 0; k < g_nbuiltins; ++k) {
        if (0 == strcmp(matrixname, g_builtins[k].name)) return &g_builtins[k].m;
    }
    return NULL;
}

static parasail_matrix_t *new_matrix(int size, int rows, int with_mapper)
{
    parasail_matrix_t *m = (parasail_matrix_t *)calloc(1, sizeof *m);
    int *values = (int *)calloc((size_t)size * rows, sizeof(int));
    int *mapper = with_mapper ? (int *)calloc(256, sizeof(int)) : NULL;
    char *alphabet = (char *)calloc((size_t)size + 2, 1);
    if (!m || !values || (with_mapper && !mapper) || !alphabet) {
        fprintf(stderr, "%s: failed to malloc\n", __func__);
        free(m); free(values); free(mapper); free(alphabet);
        return NULL;
    }
    m->matrix = values;
    m->user_matrix = values;
    m->mapper = mapper;
    m->alphabet = alphabet;
    m->size = size;
    m->length = rows;
    m->name = "";
    return m;
}

static parasail_matrix_t *create_internal(const char *alphabet, int match, int mismatch,
                                          int case_sensitive)
{
    parasail_matrix_t *m;
    size_t size;
    int size1, i, j;
    PB_CHECK_NULL(alphabet);
    size = strlen(alphabet);
    if (size >= INT_MAX) {
        fprintf(stderr, "%s: alphabet is too large\n", __func__);
        return NULL;
    }
    size1 = (int)size + 1;
    m = new_matrix(size1, size1, 1);
    if (!m) return NULL;
    /* src/memory.c:359-372: match on the diagonal, mismatch elsewhere, a
     * trailing row and column of zeros for the '*' letter */
    for (i = 0; i < (int)size; ++i)
        for (j = 0; j < (int)size; ++j)
            m->user_matrix[i * size1 + j] = i == j ? match : mismatch;
    memcpy((char *)m->alphabet, alphabet, size);
    ((char *)m->alphabet)[size] = '*';
    fill_mapper((int *)m->mapper, alphabet, size1, case_sensitive);
    m->max = match > mismatch ? match : mismatch;
    m->min = match > mismatch ? mismatch : match;
    m->type = PARASAIL_MATRIX_TYPE_SQUARE;
    return m;
}

parasail_matrix_t *parasail_matrix_create(const char *alphabet, const int match, const int mismatch)
{
    return create_internal(alphabet, match, mismatch, 0);
}

parasail_matrix_t *parasail_matrix_create_case_sensitive(const char *alphabet, const int match,
                                                         const int mismatch)
{
    return create_internal(alphabet, match, mismatch, 1);
}

static parasail_matrix_t *pssm_internal(const char *alphabet, const int *values, int length,
                                        int case_sensitive)
{
    parasail_matrix_t *m;
    size_t size;
    int size1, i, j, mn = INT_MAX, mx = INT_MIN;
    PB_CHECK_NULL(alphabet);
    PB_CHECK_NULL(values);
    if (length <= 0) {
        fprintf(stderr, "%s: length must be > 0\n", __func__);
        return NULL;
    }
    size = strlen(alphabet);
    if (size >= INT_MAX) {
        fprintf(stderr, "%s: alphabet is too large\n", __func__);
        return NULL;
    }
    size1 = (int)size + 1;
    for (i = 0; i < (int)size * length; ++i) {
        mn = values[i] < mn ? values[i] : mn;
        mx = values[i] > mx ? values[i] : mx;
    }
    m = new_matrix(size1, length, 1);
    if (!m) return NULL;
    /* src/memory.c:452-458: each position's row, then the minimum for '*' */
    for (i = 0; i < length; ++i) {
        for (j = 0; j < (int)size; ++j) m->user_matrix[i * size1 + j] = values[i * size + j];
        m->user_matrix[i * size1 + size] = mn;
    }
    memcpy((char *)m->alphabet, alphabet, size);
    ((char *)m->alphabet)[size] = '*';
    fill_mapper((int *)m->mapper, alphabet, size1, case_sensitive);
    m->max = mx;
    m->min = mn;
    m->type = PARASAIL_MATRIX_TYPE_PSSM;
    m->length = length;
    return m;
}

parasail_matrix_t *parasail_matrix_pssm_create(const char *alphabet, const int *values,
                                               const int length)
{
    return pssm_internal(alphabet, values, length, 0);
}

parasail_matrix_t *parasail_matrix_pssm_create_case_sensitive(const char *alphabet,
                                                              const int *values, const int length)
{
    return pssm_internal(alphabet, values, length, 1);
}

parasail_matrix_t *parasail_matrix_copy(const parasail_matrix_t *matrix)
{
    parasail_matrix_t *m;
    size_t nvals;
    PB_CHECK_NULL(matrix);
    nvals = matrix->type == PARASAIL_MATRIX_TYPE_PSSM
                ? (size_t)matrix->size * matrix->length
                : (size_t)matrix->size * matrix->size;
    m = new_matrix(matrix->size,
                   matrix->type == PARASAIL_MATRIX_TYPE_PSSM ? matrix->length : matrix->size, 1);
    if (!m) return NULL;
    memcpy(m->user_matrix, matrix->matrix, sizeof(int) * nvals);
    memcpy((int *)m->mapper, matrix->mapper, sizeof(int) * 256);
    {
        size_t al = strlen(matrix->alphabet);
        memcpy((char *)m->alphabet, matrix->alphabet, al <= (size_t)matrix->size + 1 ? al : (size_t)matrix->size + 1);
    }
    m->name = matrix->name;
    m->max = matrix->max;
    m->min = matrix->min;
    m->type = matrix->type;
    m->length = matrix->length;
    if (matrix->query) {
        size_t ql = strlen(matrix->query);
        char *q = (char *)malloc(ql + 1);
        if (!q) { parasail_matrix_free(m); return NULL; }
        memcpy(q, matrix->query, ql + 1);
        m->query = q;
    }
    return m;
}

parasail_matrix_t *parasail_matrix_convert_square_to_pssm(const parasail_matrix_t *matrix,
                                                          const char *s1, int s1Len)
{
    parasail_matrix_t *m;
    char *q;
    int i;
    PB_CHECK_NULL(matrix);
    if (matrix->type != PARASAIL_MATRIX_TYPE_SQUARE) {
        fprintf(stderr, "%s: attempted to convert non-square matrix to pssm\n", __func__);
        return NULL;
    }
    PB_CHECK_NULL(s1);
    PB_CHECK_GT0(s1Len);
    m = new_matrix(matrix->size, s1Len, 1);
    if (!m) return NULL;
    q = (char *)malloc((size_t)s1Len + 1);
    if (!q) { parasail_matrix_free(m); return NULL; }
    /* src/memory.c:578-583: row i is the matrix row of query letter s1[i] */
    for (i = 0; i < s1Len; ++i) {
        memcpy(m->user_matrix + (size_t)matrix->size * i,
               matrix->matrix + (size_t)matrix->size * matrix->mapper[(unsigned char)s1[i]],
               sizeof(int) * matrix->size);
    }
    memcpy(q, s1, (size_t)s1Len);
    q[s1Len] = '\0';
    memcpy((int *)m->mapper, matrix->mapper, sizeof(int) * 256);
    memcpy((char *)m->alphabet, matrix->alphabet, strlen(matrix->alphabet));
    m->name = matrix->name;
    m->max = matrix->max;
    m->min = matrix->min;
    m->type = PARASAIL_MATRIX_TYPE_PSSM;
    m->length = s1Len;
    m->query = q;
    return m;
}

void parasail_matrix_set_value(parasail_matrix_t *matrix, int row, int col, int value)
{
    if (!matrix) {
        fprintf(stderr, "%s: missing %s\n", __func__, "matrix");
        return;
    }
    if (NULL == matrix->user_matrix) {
        fprintf(stderr, "%s: attempted to set value of built-in matrix '%s'\n", __func__,
                matrix->name);
        return;
    }
    matrix->user_matrix[row * matrix->size + col] = value;
    if (value > matrix->max) matrix->max = value;
    if (value < matrix->min) matrix->min = value;
}

void parasail_matrix_free(parasail_matrix_t *matrix)
{
    if (!matrix) {
        fprintf(stderr, "%s: missing %s\n", __func__, "matrix");
        return;
    }
    if (NULL != matrix->user_matrix) {
        free((void *)matrix->matrix);
        free((void *)matrix->mapper);
        free((void *)matrix->alphabet);
        if (matrix->query) free((void *)matrix->query);
        free(matrix);
    } else {
        fprintf(stderr, "%s: attempted to free built-in matrix '%s'\n", __func__, matrix->name);
    }
}
