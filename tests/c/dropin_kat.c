/*
 * dropin_kat.c -- a C program written against the drop-in headers only
 * (include/parasail.h, include/parasail/matrices/*.h), linked with
 * libparasail_b200.so. It checks what a user of the reference's C API
 * relies on: the static matrix objects, direct and profile forms, the
 * statistics accessors, the _sat chains, the name lookups and
 * parasail_nw_banded. Known answers: parasail_sw("asdf", "asdf") scores
 * 20 with BLOSUM62 and 27 with PAM50 (open 10, extend 1), and 4 for "acgt"
 * against itself with a +1/-1 matrix (the reference's tests/test_basic.c
 * cases). Exit status 0 when every check passes.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <parasail.h>
#include <parasail/matrices/blosum62.h>
#include <parasail/matrices/pam50.h>
#include <parasail/matrices/nuc44.h>

static int failures = 0;

#define EXPECT(cond, ...) do { if (!(cond)) { printf("FAIL: " __VA_ARGS__); printf("\n"); ++failures; } } while (0)

static int score_of(parasail_result_t *r)
{
    int s = r ? r->score : -999999;
    if (r) parasail_result_free(r);
    return s;
}

int main(void)
{
    const char *q = "MKTAYIAKQRQISFVKSHFSRQLEERLGLIEVQAPILSRVGDGTQDNLSGAEKAVQVKVKALPDAQ";
    const char *t = "MKTAYIAKQRQISFVKSHFSRQDILDLWIYHTQGYFPDWQNYTPGPGIRYPLTFGWCYKLVPVEP";
    const char *dq = "ACGTTGCAACGTAGCTAGCTAGGATCCAGT", *dt = "ACGTTGCTACGTAGCAGCTAGGATCCTAGT";
    parasail_matrix_t *acgt;
    parasail_profile_t *prof;
    parasail_result_t *r, *r2;
    int major = 0, minor = 0, patch = 0;

    parasail_version(&major, &minor, &patch);
    EXPECT(major == 2, "version %d.%d.%d", major, minor, patch);

    /* the static matrix objects and their library twins */
    {
        const parasail_matrix_t *lk = parasail_matrix_lookup("blosum62");
        EXPECT(lk && lk->size == parasail_blosum62.size &&
               0 == memcmp(lk->matrix, parasail_blosum62.matrix, sizeof(int) * 24 * 24) &&
               0 == memcmp(lk->mapper, parasail_blosum62.mapper, sizeof(int) * 256),
               "blosum62 header object differs from parasail_matrix_lookup");
        lk = parasail_matrix_lookup("nuc44");
        EXPECT(lk && 0 == memcmp(lk->matrix, parasail_nuc44.matrix, sizeof(int) * 15 * 15) &&
               0 == strcmp(lk->alphabet, parasail_nuc44.alphabet), "nuc44 header object");
    }

    /* known answers */
    EXPECT(score_of(parasail_sw("asdf", 4, "asdf", 4, 10, 1, &parasail_blosum62)) == 20, "sw blosum62");
    EXPECT(score_of(parasail_sw("asdf", 4, "asdf", 4, 10, 1, &parasail_pam50)) == 27, "sw pam50");
    acgt = parasail_matrix_create("acgt", 1, -1);
    EXPECT(score_of(parasail_sw("acgt", 4, "acgt", 4, 10, 1, acgt)) == 4, "sw acgt");
    prof = parasail_profile_create_8("asdf", 4, &parasail_blosum62);
    EXPECT(prof != NULL, "profile_create_8");
    EXPECT(score_of(parasail_sw_striped_profile_8(prof, "asdf", 4, 10, 1)) == 20, "sw_striped_profile_8");
    parasail_profile_free(prof);

    /* direct form == profile form == serial form, with statistics */
    prof = parasail_profile_create_stats_sat(q, (int)strlen(q), &parasail_blosum62);
    EXPECT(prof != NULL, "profile_create_stats_sat");
    r = parasail_sw_stats_striped_profile_sat(prof, t, (int)strlen(t), 11, 1);
    r2 = parasail_sw_stats(q, (int)strlen(q), t, (int)strlen(t), 11, 1, &parasail_blosum62);
    EXPECT(r && r2 && parasail_result_is_stats(r) && parasail_result_is_sw(r), "sw stats results");
    if (r && r2) {
        EXPECT(r->score == r2->score && r->end_query == r2->end_query && r->end_ref == r2->end_ref,
               "sw stats striped vs serial: %d %d %d / %d %d %d", r->score, r->end_query, r->end_ref,
               r2->score, r2->end_query, r2->end_ref);
        EXPECT(parasail_result_get_matches(r) == parasail_result_get_matches(r2) &&
               parasail_result_get_similar(r) == parasail_result_get_similar(r2) &&
               parasail_result_get_length(r) == parasail_result_get_length(r2), "sw stats counts");
        EXPECT(parasail_result_get_matches(r) > 20 && parasail_result_get_length(r) >= 22, "sw stats values");
    }
    parasail_result_free(r);
    parasail_result_free(r2);
    parasail_profile_free(prof);

    /* global and semi-global, striped and scan, 16 bits and the chain */
    {
        const char *names[] = {"parasail_nw_stats_striped_16", "parasail_nw_stats_scan_16",
                               "parasail_sg_qx_stats_striped_16", "parasail_sg_qx_stats_scan_sat"};
        const char *serial[] = {"parasail_nw_stats", "parasail_nw_stats", "parasail_sg_qx_stats", "parasail_sg_qx_stats"};
        int k;
        for (k = 0; k < 4; ++k) {
            parasail_function_t *f = parasail_lookup_function(names[k]);
            parasail_function_t *g = parasail_lookup_function(serial[k]);
            EXPECT(f && g, "lookup %s", names[k]);
            if (!f || !g) continue;
            r = f(dq, (int)strlen(dq), dt, (int)strlen(dt), 5, 2, acgt);
            r2 = g(dq, (int)strlen(dq), dt, (int)strlen(dt), 5, 2, acgt);
            EXPECT(r && r2 && r->score == r2->score && r->end_query == r2->end_query &&
                   r->end_ref == r2->end_ref &&
                   parasail_result_get_matches(r) == parasail_result_get_matches(r2) &&
                   parasail_result_get_length(r) == parasail_result_get_length(r2),
                   "%s vs %s", names[k], serial[k]);
            EXPECT(r && (parasail_result_is_striped(r) || parasail_result_is_scan(r)), "%s flags", names[k]);
            parasail_result_free(r);
            parasail_result_free(r2);
        }
    }

    /* banded global alignment equals full global alignment for a wide band */
    r = parasail_nw_banded(dq, (int)strlen(dq), dt, (int)strlen(dt), 5, 2, 30, acgt);
    r2 = parasail_nw(dq, (int)strlen(dq), dt, (int)strlen(dt), 5, 2, acgt);
    EXPECT(r && r2 && r->score == r2->score, "nw_banded vs nw");
    parasail_result_free(r);
    parasail_result_free(r2);
    parasail_matrix_free(acgt);

    printf("%s (%d failures)\n", failures ? "failed" : "pass", failures);
    return failures ? EXIT_FAILURE : 0;
}
