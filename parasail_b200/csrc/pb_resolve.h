/*
 * pb_resolve.h -- which of parasail's 8/16/32-bit results a pair gets.
 *
 * The reference runs a pair in 8-bit lanes and, when that kernel reports
 * saturation, reruns it in 16 and then 32 bits (src/satcheck.c, e.g.
 * :41520-41538). A non-saturated result at any width equals the exact DP
 * result, so the GPU computes exact values once and this file decides, per
 * width, whether the reference's kernel of that width would have flagged the
 * pair. The reference's checks (constants from the kernels' preambles, e.g.
 * src/nw_scan_avx2_256_16.c:205-206, src/sw_striped_avx2_256_16.c:205-210):
 *
 *   NEG_LIMIT = (-open < min ? INT_MIN_w + open : INT_MIN_w - min) + 1
 *   POS_LIMIT = INT_MAX_w - max - 1
 *   SW striped 8/16 (biased lanes): max H > INT_MAX_w - max - 1 - INT_MIN_w
 *   SW striped 32:                  max H > INT32_MAX - max - 1
 *   scan, all:   any H outside [NEG_LIMIT, POS_LIMIT]; sg also any F below
 *                NEG_LIMIT and the gap ramp -open - segLen*gap
 *                (src/sg_scan_avx2_256_16.c:293-301, :355-360)
 *   stats:       additionally matches/similar/length above POS_LIMIT
 *   striped nw/sg: min also over E and the first-pass F and H
 *                (src/nw_striped_avx2_256_16.c:278-283)
 *   SW stats striped (src/sw_stats_striped_avx2_256_16.c:694-730): a score
 *                pass with the SW striped check, then a stats pass on the
 *                prefix [0,end_query]x[0,end_ref] that saturates when a count
 *                reaches INT_MAX_w - INT_MIN_w.
 *
 * Every check reads all rows of the AVX2 layout, including the padded query
 * rows up to ceil(qlen/lanes)*lanes (lanes = 32, 16, 8 for 8, 16, 32 bits);
 * the exact kernel reports those rows' extremes separately. Checks that read
 * the striped first pass (values before the lazy-F correction) are decided
 * here from sound bounds where the bounds show a CLEAN run; any other verdict
 * of an 8/16-bit striped kernel comes from the lane-exact restatement of that
 * kernel (pb_lane.cuh), which also reproduces the reference's results in the
 * cases where its narrow kernels return unflagged wrong values.
 */
#ifndef PARASAIL_B200_PB_RESOLVE_H
#define PARASAIL_B200_PB_RESOLVE_H

#include <stdint.h>

#include "parasail.h"
#include "pb_cuda.h"

#ifdef __CUDACC__
#define PB_HD __host__ __device__
#else
#define PB_HD
#endif

enum { PB_CLEAN = 0, PB_SAT = 1, PB_AMBIG = 2 };

typedef struct pb_mode {
    int alg, sgflags, stats, striped;
    int open, gap, mmax, mmin;
} pb_mode;

PB_HD static inline int64_t int_min_w(int bits) { return bits == 8 ? INT8_MIN : bits == 16 ? INT16_MIN : INT32_MIN; }
PB_HD static inline int64_t int_max_w(int bits) { return bits == 8 ? INT8_MAX : bits == 16 ? INT16_MAX : INT32_MAX; }

/* number of padded-row regions that belong to the layout of `bits` */
PB_HD static inline int pad_regions(int bits) { return bits == 32 ? 1 : bits == 16 ? 2 : 3; }
PB_HD static inline int lanes_of(int bits) { return 256 / bits; }

PB_HD static inline int64_t boundary_h(const pb_mode *m, int idx, int is_row)
{
    if (idx < 0) return 0;
    if (m->alg == PB_SW) return 0;
    if (m->alg == PB_SG && (m->sgflags & (is_row ? PB_S2_BEG : PB_S1_BEG))) return 0;
    return -(int64_t)m->open - (int64_t)idx * m->gap;
}

PB_HD static inline int pb_resolve_faststats_pass1(const pb_mode *m, int bits, const pb_pair_out *o)
{
    if (bits == 32) return (int64_t)o->max_h > (int64_t)INT32_MAX - m->mmax - 1 ? PB_SAT : PB_CLEAN;
    return (int64_t)o->max_h > int_max_w(bits) - m->mmax - 1 - int_min_w(bits) ? PB_SAT : PB_CLEAN;
}

PB_HD static inline int pb_resolve_tier(const pb_mode *m, int bits, const pb_pair_out *o, int qlim, int tlim)
{
    const int64_t imin = int_min_w(bits), imax = int_max_w(bits);
    const int64_t neg = ((-(int64_t)m->open < m->mmin) ? imin + m->open : imin - m->mmin) + 1;
    const int64_t pos = imax - m->mmax - 1;
    const int L = lanes_of(bits);
    const int64_t seglen = (qlim + L - 1) / L;
    const int64_t padlen = seglen * L;
    int64_t min_h = o->min_h_real, max_st = o->max_stat_real, min_f = o->min_f_real;
    const int64_t max_h = o->max_h;
    int k;
    for (k = 0; k < pad_regions(bits); ++k) {
        if (o->min_h_pad[k] < min_h) min_h = o->min_h_pad[k];
        if (o->max_stat_pad[k] > max_st) max_st = o->max_stat_pad[k];
        if (o->min_f_pad[k] < min_f) min_f = o->min_f_pad[k];
    }

    if (m->alg == PB_SW && !m->stats) {
        if (m->striped) return pb_resolve_faststats_pass1(m, bits, o);
        return max_h > pos ? PB_SAT : PB_CLEAN;
    }
    if (m->alg == PB_SW && m->stats && !m->striped) {
        return (max_h > pos || max_st > pos) ? PB_SAT : PB_CLEAN;
    }
    if (m->alg == PB_SW && m->stats && m->striped) {
        /* prefix stats pass of the FASTSTATS wrapper; o describes the prefix */
        const int64_t lim = bits == 32 ? INT32_MAX : imax - imin;
        if (bits == 32) return PB_CLEAN;
        if (max_st >= lim) return PB_SAT;
        if (padlen + tlim < lim) return PB_CLEAN;
        return PB_AMBIG;
    }
    /* NW and SG */
    if (!m->striped) {
        if (max_h > pos || min_h < neg) return PB_SAT;
        if (m->stats && max_st > pos) return PB_SAT;
        if (!m->stats && m->alg == PB_SG) {
            int64_t ramp = -(int64_t)m->open - seglen * m->gap;
            if (ramp < imin) ramp = imin;
            if (min_f < neg || ramp < neg) return PB_SAT;
        }
        return PB_CLEAN;
    }
    /* striped NW/SG. The first pass starts every stripe's F at NEG_LIMIT,
     * which lifts an underflowing H back into range; the E and F checks of
     * the non-stats kernels usually catch it one step later, but not when a
     * stripe has a single segment and the low cell sits in the last column,
     * and the stats kernels do not check E and F at all (the reference then
     * returns a wrong, unflagged score). Only an overflowing maximum is a
     * certain flag; pairs with values near NEG_LIMIT go to the lane-exact
     * kernel. */
    if (max_h > pos) return PB_SAT;
    if (!m->stats && boundary_h(m, (int)padlen - 1, 0) - m->open < neg) {
        /* column 0 loads E = H(i,-1) - open for every row of the layout
         * (src/nw_striped_avx2_256_16.c:243-258), and E is range-checked */
        return PB_SAT;
    }
    {
        int64_t minb = 0, lb;
        const int64_t top = boundary_h(m, tlim - 1, 1), left = boundary_h(m, (int)padlen - 1, 0);
        if (top < minb) minb = top;
        if (left < minb) minb = left;
        lb = (min_h < minb ? min_h : minb) + (m->mmin < 0 ? m->mmin : 0);
        if (!m->stats) lb -= m->open;   /* E and the first-pass F are also checked */
        else lb -= 1;                   /* strict: H == NEG_LIMIT ties the F floor */
        if (lb >= neg && (!m->stats || padlen + tlim <= pos)) return PB_CLEAN;
    }
    return PB_AMBIG;
}

/* One alignment request: mode + width (8/16/32, or 0 for the 8->16->32
 * chain) + the family flags the reference sets (algorithm, semi-global
 * ends, STRIPED or SCAN; for serial forms NOVEC/NOVEC_SCAN with bits = -1). */
typedef struct pb_job {
    pb_mode mode;
    int bits;
    int base_flags;
} pb_job;

/* Compact per-pair result. `ambig`: 0 when every width was decided
 * exactly; PB_REC_FALLBACK when a scan or 32-bit verdict came from the
 * bounds' fallback rule (pb_ambig_fallback); 8 or 16 while the pair still
 * waits for the lane-exact kernel of that width (never in a finished
 * record). */
typedef struct pb_record {
    int score, end_query, end_ref, flag;
    int matches, similar, length, ambig;
} pb_record;

enum { PB_REC_FALLBACK = 1 };

/* Widths at which the reference's striped kernel computes something other
 * than the exact DP for every pair, so that only the lane-exact kernel
 * gives its result: a penalty that wraps in the lane width (set1 of open or
 * gap above INT_w_MAX), in the score-only kernels open <= gap (their lazy-F
 * loop stops on a tie between F - gap and H - open, which open <= gap makes
 * common), and in the statistics kernels open < gap (they continue on ties,
 * and agree with the exact DP at open == gap). The SW statistics kernels of
 * the FASTSTATS wrapper are not emulated in these regimes. The scan
 * kernels, score-only and statistics alike, depart from the exact DP at
 * open < gap (their prefix scan of F assumes F - gap >= F - open) and with
 * a wrapped penalty, and agree with it at open == gap. The SW statistics
 * scan kernel is not emulated in these regimes (its restatement,
 * pb_lane.cuh scan_stats<SW>, is pinned on the host only). */
PB_HD static inline int pb_lane_forced(const pb_mode *m, int bits)
{
    const int wrapped = bits < 32 && (m->open > int_max_w(bits) || m->gap > int_max_w(bits));
    if (!m->striped) return (!m->stats || m->alg != PB_SW) && (m->open < m->gap || wrapped);
    if (m->alg == PB_SW && m->stats) return 0;
    if (wrapped) return 1;
    return m->stats ? m->open < m->gap : m->open <= m->gap;
}

/* Widths whose verdict the lane-exact kernels (pb_lane.cuh) give: the
 * 8/16-bit striped nw/sg kernels and the 8/16-bit SW statistics kernel of
 * the FASTSTATS wrapper whenever the exact values do not show a CLEAN run,
 * and every width pb_lane_forced names (striped or scan). */
PB_HD static inline int pb_lane_applies(const pb_mode *m, int bits)
{
    if (!m->striped) return pb_lane_forced(m, bits);
    if (m->alg == PB_SW) return m->stats ? (bits == 8 || bits == 16) : pb_lane_forced(m, bits);
    return bits == 8 || bits == 16 || pb_lane_forced(m, bits);
}

/* lane kernel kind for a mode (pb_lane_args.kind) */
PB_HD static inline int pb_lane_kind(const pb_mode *m)
{
    if (!m->striped) return m->alg == PB_SW ? 7 : (m->stats ? 8 : 6);   /* scan */
    return m->alg == PB_SW ? (m->stats ? 2 : 3) : (m->stats ? 1 : 0);
}

PB_HD static inline int pb_bits_flag(int bits)
{
    return bits == 8 ? PARASAIL_FLAG_BITS_8 : bits == 16 ? PARASAIL_FLAG_BITS_16 : PARASAIL_FLAG_BITS_32;
}

PB_HD static inline int pb_lanes_flag(int bits)
{
    return bits == 8 ? PARASAIL_FLAG_LANES_32 : bits == 16 ? PARASAIL_FLAG_LANES_16 : PARASAIL_FLAG_LANES_8;
}

PB_HD static inline int pb_job_is_faststats(const pb_job *j)
{
    return j->bits >= 0 && j->mode.alg == PB_SW && j->mode.stats && j->mode.striped;
}

/* Widths the chain tries: [first, last] indices into {8, 16, 32}. */
PB_HD static inline void pb_job_widths(const pb_job *j, int *first, int *last)
{
    const int b = j->bits;
    *first = (b == 0 || b == 8) ? 0 : b == 16 ? 1 : 2;
    *last = b == 0 ? 2 : *first;
}

/* FASTSTATS: does any width pass the score check, so that the prefix stats
 * pass is needed? */
PB_HD static inline int pb_needs_pass2(const pb_job *j, const pb_pair_out *o1)
{
    int f, l, t;
    const int w3[3] = {8, 16, 32};
    if (!pb_job_is_faststats(j)) return 0;
    pb_job_widths(j, &f, &l);
    for (t = f; t <= l; ++t)
        if (pb_resolve_faststats_pass1(&j->mode, w3[t], o1) != PB_SAT) return 1;
    return 0;
}

/* Rule for PB_AMBIG pairs when the lane-exact kernel is not run: the
 * width's check evaluated on the exact final values. */
PB_HD static inline int pb_ambig_fallback(const pb_mode *m, int bits, const pb_pair_out *o,
                                          int qlim, int tlim)
{
    if (m->alg == PB_SW && m->stats && m->striped) {
        int64_t st = o->max_stat_real;
        int k;
        for (k = 0; k < pad_regions(bits); ++k) if (o->max_stat_pad[k] > st) st = o->max_stat_pad[k];
        return st >= int_max_w(bits) - int_min_w(bits) ? PB_SAT : PB_CLEAN;
    }
    {
        pb_mode s = *m;
        s.striped = 0;
        return pb_resolve_tier(&s, bits, o, qlim, tlim) == PB_SAT ? PB_SAT : PB_CLEAN;
    }
}

/* The result the reference returns for one pair (src/satcheck.c chains,
 * the kernels' sentinel values, the FASTSTATS wrapper). o2 is the prefix
 * pass (FASTSTATS only, may be NULL when pb_needs_pass2 said no). e8, e16
 * and e32 the lane-exact kernels' results for the pair (NULL or not valid when they
 * have not run); when a width needs one that is missing, the returned record
 * has ambig = that width and nothing else in it is final. */
PB_HD static inline pb_record pb_chain_resolve(const pb_job *j, const pb_pair_out *o1,
                                               const pb_pair_out *o2, int qlen, int tlen,
                                               const pb_lane_res *e8, const pb_lane_res *e16,
                                               const pb_lane_res *e32)
{
    const int w3[3] = {8, 16, 32};
    const pb_mode *m = &j->mode;
    pb_record r;
    int f, l, t, fallback = 0;
    r.score = r.end_query = r.end_ref = r.matches = r.similar = r.length = 0;
    r.ambig = 0;
    r.flag = 0;
    if (j->bits < 0) {   /* serial forms: exact 32-bit, flags given */
        r.score = o1->score; r.end_query = o1->end_query; r.end_ref = o1->end_ref;
        r.matches = o1->matches; r.similar = o1->similar; r.length = o1->length;
        r.flag = j->base_flags | (m->stats ? PARASAIL_FLAG_STATS : 0);
        return r;
    }
    pb_job_widths(j, &f, &l);
    for (t = f; t <= l; ++t) {
        const int w = w3[t];
        const int fl = j->base_flags | pb_bits_flag(w) | pb_lanes_flag(w);
        const pb_lane_res *e = w == 8 ? e8 : w == 16 ? e16 : e32;
        int v;
        if (pb_job_is_faststats(j)) {
            if (pb_resolve_faststats_pass1(m, w, o1) == PB_SAT) {
                if (t < l) continue;
                /* the score-only pass's saturated result, without stats */
                r.score = w == 8 ? 255 : w == 16 ? 65535 : 0x7fffffff;
                r.flag = fl | PARASAIL_FLAG_SATURATED;
                r.ambig = fallback;
                return r;
            }
            v = pb_resolve_tier(m, w, o2, o1->end_query + 1, o1->end_ref + 1);
            if (v != PB_CLEAN && pb_lane_applies(m, w)) {
                /* the prefix kernel's own result, ends from the score pass */
                if (!e || !e->valid) { r.ambig = w; return r; }
                if (e->saturated && t < l) continue;
                r.score = e->score; r.end_query = o1->end_query; r.end_ref = o1->end_ref;
                r.matches = e->matches; r.similar = e->similar; r.length = e->length;
                r.flag = fl | PARASAIL_FLAG_STATS | (e->saturated ? PARASAIL_FLAG_SATURATED : 0);
                r.ambig = fallback;
                return r;
            }
            if (v == PB_AMBIG) { fallback = PB_REC_FALLBACK; v = pb_ambig_fallback(m, w, o2, o1->end_query + 1, o1->end_ref + 1); }
            if (v == PB_SAT) {
                if (t < l) continue;
                r.end_query = o1->end_query; r.end_ref = o1->end_ref;
                r.flag = fl | PARASAIL_FLAG_SATURATED | PARASAIL_FLAG_STATS;
                r.ambig = fallback;
                return r;
            }
            r.score = o1->score; r.end_query = o1->end_query; r.end_ref = o1->end_ref;
            r.matches = o2->matches; r.similar = o2->similar; r.length = o2->length;
            r.flag = fl | PARASAIL_FLAG_STATS;
            r.ambig = fallback;
            return r;
        }
        v = pb_resolve_tier(m, w, o1, qlen, tlen);
        if ((v != PB_CLEAN || pb_lane_forced(m, w)) && pb_lane_applies(m, w)) {
            if (!e || !e->valid) { r.ambig = w; return r; }
            if (e->saturated) {
                if (t < l) continue;
                /* the kernel's saturated result: zeros, or the SW sentinel */
                r.score = e->score; r.end_query = e->end_query; r.end_ref = e->end_ref;
                r.flag = fl | PARASAIL_FLAG_SATURATED | (m->stats ? PARASAIL_FLAG_STATS : 0);
                r.ambig = fallback;
                return r;
            }
            r.score = e->score; r.end_query = e->end_query; r.end_ref = e->end_ref;
            if (m->stats) { r.matches = e->matches; r.similar = e->similar; r.length = e->length; }
            r.flag = fl | (m->stats ? PARASAIL_FLAG_STATS : 0);
            r.ambig = fallback;
            return r;
        }
        if (v == PB_AMBIG) { fallback = PB_REC_FALLBACK; v = pb_ambig_fallback(m, w, o1, qlen, tlen); }
        if (v == PB_SAT) {
            if (t < l) continue;
            if (m->alg == PB_SW && m->striped && !m->stats)
                r.score = w == 8 ? 255 : w == 16 ? 65535 : 0x7fffffff;
            r.flag = fl | PARASAIL_FLAG_SATURATED | (m->stats ? PARASAIL_FLAG_STATS : 0);
            r.ambig = fallback;
            return r;
        }
        r.score = o1->score; r.end_query = o1->end_query; r.end_ref = o1->end_ref;
        r.matches = o1->matches; r.similar = o1->similar; r.length = o1->length;
        r.flag = fl | (m->stats ? PARASAIL_FLAG_STATS : 0);
        r.ambig = fallback;
        return r;
    }
    return r;
}

#endif
