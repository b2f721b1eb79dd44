/*
 * lookup.c -- function lookup by name (parasail_lookup_function and friends).
 *
 * Same contract as the reference (src/function_lookup.c:16-118): a linear
 * search of a name table, retried with a "parasail_" prefix when the caller
 * omitted it; info records carry the reference's field values for the
 * dispatcher-level names (isa "disp", lanes -1) and the serial names
 * (type "orig"/"scan", bits "32", lanes 1; parasail/function_lookup.h).
 */
#include <stdlib.h>
#include <string.h>

#include "pb_internal.h"

#define SER(base, algname, st)                                                        \
    {base, #base, algname, "orig", "NA", "32", "32", 1, 0, 0, 0, st, 1},              \
    {base##_scan, #base "_scan", algname, "scan", "NA", "32", "32", 1, 0, 0, 0, st, 0},
#define DIR1(base, algname, st, scheme, w)                                            \
    {base##_##scheme##_##w, #base "_" #scheme "_" #w, algname, #scheme, "disp", "NA", #w, -1, 0, 0, 0, st, 0},
#define DIR(base, algname, st)                                                        \
    DIR1(base, algname, st, striped, 8) DIR1(base, algname, st, striped, 16)          \
    DIR1(base, algname, st, striped, 32) DIR1(base, algname, st, striped, sat)        \
    DIR1(base, algname, st, scan, 8) DIR1(base, algname, st, scan, 16)                \
    DIR1(base, algname, st, scan, 32) DIR1(base, algname, st, scan, sat)
#define FAM(base, algname, st) SER(base, algname, st) DIR(base, algname, st)
#define BOTH(base, algname)                                                           \
    FAM(base, algname, 0) FAM(base##_stats, algname "_stats", 1)
/* the trace forms: serial, and striped/scan at 8/16/32 bits and _sat
 * (is_trace set, as parasail/function_lookup.h:8184-8277 records them) */
#define TDIR1(base, algname, scheme, w)                                               \
    {base##_trace_##scheme##_##w, #base "_trace_" #scheme "_" #w, algname, #scheme, "disp", "NA", #w, -1, 0, 0, 1, 0, 0},
#define TRACE(base, algname)                                                          \
    {base##_trace, #base "_trace", algname, "orig", "NA", "32", "32", 1, 0, 0, 1, 0, 1}, \
    {base##_trace_scan, #base "_trace_scan", algname, "scan", "NA", "32", "32", 1, 0, 0, 1, 0, 0}, \
    TDIR1(base, algname, striped, 8) TDIR1(base, algname, striped, 16)                \
    TDIR1(base, algname, striped, 32) TDIR1(base, algname, striped, sat)              \
    TDIR1(base, algname, scan, 8) TDIR1(base, algname, scan, 16)                      \
    TDIR1(base, algname, scan, 32) TDIR1(base, algname, scan, sat)

static const parasail_function_info_t functions[] = {
    BOTH(parasail_sw, "sw")
    BOTH(parasail_nw, "nw")
    BOTH(parasail_sg, "sg")
    BOTH(parasail_sg_qb, "sg_qb")
    BOTH(parasail_sg_qe, "sg_qe")
    BOTH(parasail_sg_qx, "sg_qx")
    BOTH(parasail_sg_db, "sg_db")
    BOTH(parasail_sg_de, "sg_de")
    BOTH(parasail_sg_dx, "sg_dx")
    BOTH(parasail_sg_qb_de, "sg_qb_de")
    BOTH(parasail_sg_qe_db, "sg_qe_db")
    BOTH(parasail_sg_qb_db, "sg_qb_db")
    BOTH(parasail_sg_qe_de, "sg_qe_de")
    TRACE(parasail_sw, "sw") TRACE(parasail_nw, "nw") TRACE(parasail_sg, "sg")
    TRACE(parasail_sg_qb, "sg_qb") TRACE(parasail_sg_qe, "sg_qe") TRACE(parasail_sg_qx, "sg_qx")
    TRACE(parasail_sg_db, "sg_db") TRACE(parasail_sg_de, "sg_de") TRACE(parasail_sg_dx, "sg_dx")
    TRACE(parasail_sg_qb_de, "sg_qb_de") TRACE(parasail_sg_qe_db, "sg_qe_db")
    TRACE(parasail_sg_qb_db, "sg_qb_db") TRACE(parasail_sg_qe_de, "sg_qe_de")
    {NULL, "NULL", "NULL", "NULL", "NULL", "NULL", "NULL", 0, 0, 0, 0, 0, 0},
};

#define PF1(base, algname, st, scheme, w, creator)                                     \
    {base##_##scheme##_profile_##w, creator, #base "_" #scheme "_profile_" #w, algname, \
     #scheme "_profile", "disp", "NA", #w, -1, 0, 0, 0, st, 0},
#define PFS(base, algname, st, scheme, pre)                                             \
    PF1(base, algname, st, scheme, 8, pre##_8) PF1(base, algname, st, scheme, 16, pre##_16) \
    PF1(base, algname, st, scheme, 32, pre##_32) PF1(base, algname, st, scheme, sat, pre##_sat)
#define PBOTH(base, algname)                                                            \
    PFS(base, algname, 0, striped, parasail_profile_create)                             \
    PFS(base, algname, 0, scan, parasail_profile_create)                                \
    PFS(base##_stats, algname "_stats", 1, striped, parasail_profile_create_stats)      \
    PFS(base##_stats, algname "_stats", 1, scan, parasail_profile_create_stats)

#define PT1(base, algname, scheme, w)                                                   \
    {base##_trace_##scheme##_profile_##w, parasail_profile_create_##w, #base "_trace_" #scheme "_profile_" #w, \
     algname, #scheme "_profile", "disp", "NA", #w, -1, 0, 0, 1, 0, 0},
#define PTRACE(base, algname)                                                           \
    PT1(base, algname, scan, 8) PT1(base, algname, scan, 16) PT1(base, algname, scan, 32) \
    PT1(base, algname, scan, sat) PT1(base, algname, striped, 8)                        \
    PT1(base, algname, striped, 16) PT1(base, algname, striped, 32) PT1(base, algname, striped, sat)

static const parasail_pfunction_info_t pfunctions[] = {
    PBOTH(parasail_sw, "sw")
    PBOTH(parasail_nw, "nw")
    PBOTH(parasail_sg, "sg")
    PBOTH(parasail_sg_qb, "sg_qb")
    PBOTH(parasail_sg_qe, "sg_qe")
    PBOTH(parasail_sg_qx, "sg_qx")
    PBOTH(parasail_sg_db, "sg_db")
    PBOTH(parasail_sg_de, "sg_de")
    PBOTH(parasail_sg_dx, "sg_dx")
    PBOTH(parasail_sg_qb_de, "sg_qb_de")
    PBOTH(parasail_sg_qe_db, "sg_qe_db")
    PBOTH(parasail_sg_qb_db, "sg_qb_db")
    PBOTH(parasail_sg_qe_de, "sg_qe_de")
    PTRACE(parasail_sw, "sw") PTRACE(parasail_nw, "nw") PTRACE(parasail_sg, "sg")
    PTRACE(parasail_sg_qb, "sg_qb") PTRACE(parasail_sg_qe, "sg_qe") PTRACE(parasail_sg_qx, "sg_qx")
    PTRACE(parasail_sg_db, "sg_db") PTRACE(parasail_sg_de, "sg_de") PTRACE(parasail_sg_dx, "sg_dx")
    PTRACE(parasail_sg_qb_de, "sg_qb_de") PTRACE(parasail_sg_qe_db, "sg_qe_db")
    PTRACE(parasail_sg_qb_db, "sg_qb_db") PTRACE(parasail_sg_qe_de, "sg_qe_de")
    {NULL, NULL, "NULL", "NULL", "NULL", "NULL", "NULL", "NULL", 0, 0, 0, 0, 0, 0},
};

#define FIND(table, funcname, out)                                                     \
    do {                                                                               \
        int k_;                                                                        \
        out = NULL;                                                                    \
        if (!(funcname)) break;                                                        \
        for (k_ = 0; table[k_].pointer; ++k_)                                          \
            if (0 == strcmp((funcname), table[k_].name)) { out = &table[k_]; break; }  \
        if (!out) {                                                                    \
            const char *prefix_ = "parasail_";                                         \
            char *nn_ = (char *)malloc(strlen(prefix_) + strlen(funcname) + 1);        \
            if (!nn_) break;                                                           \
            strcpy(nn_, prefix_);                                                      \
            strcat(nn_, (funcname));                                                   \
            for (k_ = 0; table[k_].pointer; ++k_)                                      \
                if (0 == strcmp(nn_, table[k_].name)) { out = &table[k_]; break; }     \
            free(nn_);                                                                 \
        }                                                                              \
    } while (0)

const parasail_function_info_t *parasail_lookup_function_info(const char *funcname)
{
    const parasail_function_info_t *f;
    FIND(functions, funcname, f);
    return f;
}

const parasail_pfunction_info_t *parasail_lookup_pfunction_info(const char *funcname)
{
    const parasail_pfunction_info_t *f;
    FIND(pfunctions, funcname, f);
    return f;
}

parasail_function_t *parasail_lookup_function(const char *funcname)
{
    const parasail_function_info_t *f = parasail_lookup_function_info(funcname);
    return f ? f->pointer : NULL;
}

parasail_pfunction_t *parasail_lookup_pfunction(const char *funcname)
{
    const parasail_pfunction_info_t *f = parasail_lookup_pfunction_info(funcname);
    return f ? f->pointer : NULL;
}

parasail_pcreator_t *parasail_lookup_pcreator(const char *funcname)
{
    const parasail_pfunction_info_t *f = parasail_lookup_pfunction_info(funcname);
    return f ? f->creator : NULL;
}
