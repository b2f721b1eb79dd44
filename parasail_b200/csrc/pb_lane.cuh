/*
 * pb_lane.cuh -- lane-exact restatement of the reference's 8- and 16-bit
 * AVX2 striped kernels, for the pairs whose narrow-width result the exact
 * DP values cannot settle.
 *
 * A narrow striped kernel computes with saturating W-bit lanes, starts every
 * stripe's vertical gap at NEG_LIMIT and checks only some of its values
 * against the limits, so near the limits its result (score, statistics and
 * whether it reports saturation) is a function of its own arithmetic, not of
 * the exact DP. This file restates that arithmetic step by step:
 *
 *   nw/sg score-only:  util/templates/nw_striped.c:186-300,
 *                      util/templates/sg_striped.c (column maximum, s1_end
 *                      scan of the last column in memory order, ends)
 *   nw/sg statistics:  util/templates/nw_stats_striped.c:226-470,
 *                      util/templates/sg_stats_striped.c (vMaxH* blends)
 *   sw statistics:     util/templates/sw_stats_striped_bias.c:226-637 (the
 *                      biased kernel the FASTSTATS wrapper :644-730 runs on
 *                      the prefix [0, end_query] x [0, end_ref])
 *   scan forms:        util/templates/{nw,sg,sw}_scan.c and
 *                      {nw,sg,sw}_stats_scan.c (open < gap, wrapped
 *                      penalties: the prefix scan of F is not the DP's)
 *   nw/sg trace:       util/templates/{nw,sg}_trace_striped.c (the
 *                      score-only passes, lazy-F loop on >=) and
 *                      {nw,sg}_trace_scan.c (saturation flag only)
 *
 * with the profile of src/memory_avx2.c:28-253 / :255-528 (values truncated
 * to W bits, padded rows 0; similar = truncated value > 0).
 *
 * The code is written against a vector policy P: the device policy maps one
 * AVX2 lane to one lane of a warp (lane shift = warp shuffle, movemask = warp
 * vote), so a warp runs one pair with the reference's own data movement.
 */
#ifndef PARASAIL_B200_PB_LANE_CUH
#define PARASAIL_B200_PB_LANE_CUH

#include <stdint.h>

#ifdef __CUDACC__
#define PB_LHD __host__ __device__ __forceinline__
#else
#define PB_LHD inline
#endif

namespace pb {
namespace lane {

template <int W> struct Lim {
    static constexpr int LANES = 256 / W;
    static constexpr int MIN = W == 8 ? -128 : W == 16 ? -32768 : (int)0x80000000;
    static constexpr int MAX = W == 8 ? 127 : W == 16 ? 32767 : 0x7fffffff;
};

/* (intW_t)x: two's-complement wrap, as a C conversion to int8/16/32_t */
template <int W> PB_LHD int wrap(long long x)
{
    return W == 8 ? (int)(int8_t)(uint8_t)(x & 0xff)
         : W == 16 ? (int)(int16_t)(uint16_t)(x & 0xffff)
                   : (int)(uint32_t)(x & 0xffffffffll);
}

template <int W> PB_LHD int clampw(long long x)
{
    return x < Lim<W>::MIN ? Lim<W>::MIN : (x > Lim<W>::MAX ? Lim<W>::MAX : (int)x);
}

/* lane add/subtract of the W-bit kernels: saturating at 8 and 16 bits
 * (_mm256_adds/subs_epi8/16), wrapping at 32 (_mm256_add/sub_epi32) */
template <int W> PB_LHD int lane_arith(long long x)
{
    return W == 32 ? wrap<W>(x) : clampw<W>(x);
}

/* One pair as the emulation sees it. Profile values come from the exact
 * 32-bit profile (vector orientation: prof[k * lp + row], k = target code),
 * queries' codes for the match plane. */
struct Problem {
    int qlen, tlen;                /* s1Len, s2Len of the kernel call */
    int open, gap, mmax, mmin;
    int s1_beg, s1_end, s2_beg, s2_end;
    const int32_t *prof;           /* [size][lp], or nullptr in matrix mode */
    const uint8_t *qcodes;         /* [>= qlen] */
    int lp;
    const int32_t *mat;            /* matrix mode: mat[k * msize + query code] */
    int msize;
    int size;                      /* alphabet size: codes >= size read as code 0 */
    const uint8_t *t;              /* target codes */
};

/* profile value of target code k at query row `row` (row < qlen); an
 * out-of-alphabet code reads as code 0, as in the exact kernel */
PB_LHD int prof_value(const Problem &pr, int k, int row)
{
    if (k >= pr.size) k = 0;
    if (pr.mat) {
        int c = pr.qcodes[row];
        if (c >= pr.msize) c = 0;
        return pr.mat[k * pr.msize + c];
    }
    return pr.prof[(size_t)k * pr.lp + row];
}

struct Out {
    int score, end_query, end_ref, matches, similar, length, saturated;
};

/* ---- nw / sg, score only (NW == SG with no free ends) ----
 * TRACE: the trace kernels (util/templates/nw_trace_striped.c,
 * sg_trace_striped.c) run the same passes and checks; their lazy-F loop
 * continues while F - gap >= H - open in some lane
 * (src/nw_trace_striped_avx2_256_8.c:418-423) where the score kernel's
 * continues on >. */
template <class P, int W, bool TRACE = false>
PB_LHD void striped_nwsg(P &v, const Problem &pr, Out &o)
{
    typedef typename P::V V;
    constexpr int L = Lim<W>::LANES;
    const int s1Len = pr.qlen, s2Len = pr.tlen;
    const int segLen = (s1Len + L - 1) / L;
    const int offset = (s1Len - 1) % segLen;
    const int lastLane = (s1Len - 1) / segLen;          /* lane of row s1Len-1 */
    const int open = pr.open, gap = pr.gap;
    const int NEG_LIMIT = wrap<W>((-open < pr.mmin ? (long long)Lim<W>::MIN + open : (long long)Lim<W>::MIN - pr.mmin) + 1);
    const int POS_LIMIT = wrap<W>((long long)Lim<W>::MAX - pr.mmax - 1);
    const V vGapO = v.set1(wrap<W>(open)), vGapE = v.set1(wrap<W>(gap));
    const V vNegLimit = v.set1(NEG_LIMIT), vPosLimit = v.set1(POS_LIMIT);
    V vSatMin = vPosLimit, vSatMax = vNegLimit, vMaxH = vNegLimit;
    const V vPosMask = v.lane_eq(lastLane);
    int end_query = s1Len - 1, end_ref = s2Len - 1;
    int score = NEG_LIMIT;

    typename P::Arr hs = v.arr(0, segLen), hl = v.arr(1, segLen), pe = v.arr(2, segLen);
    /* initialize H and E */
    for (int i = 0; i < segLen; ++i) {
        V h, e;
        v.template init_he<W>(h, e, i, segLen, pr.s1_beg, open, gap);
        v.store(hs, i, h);
        v.store(pe, i, e);
    }
    for (int j = 0; j < s2Len; ++j) {
        const int bj = v.template boundary<W>(pr, j), bj1 = v.template boundary<W>(pr, j + 1);
        const int k_t = pr.t[j];
        V vE;
        V vF = vNegLimit;
        V vH = v.shift1(v.load(hs, segLen - 1));
        { typename P::Arr tmp = hl; hl = hs; hs = tmp; }
        vH = v.insert0(vH, bj);
        for (int i = 0; i < segLen; ++i) {
            vH = v.template adds<W>(vH, v.template prof<W>(pr, k_t, i, segLen));
            vE = v.load(pe, i);
            vH = v.max(vH, vE);
            vH = v.max(vH, vF);
            v.store(hs, i, vH);
            vSatMax = v.max(vSatMax, vH);
            vSatMin = v.min(vSatMin, vH);
            vSatMin = v.min(vSatMin, vE);
            vSatMin = v.min(vSatMin, vF);
            vH = v.template subs<W>(vH, vGapO);
            vE = v.template subs<W>(vE, vGapE);
            vE = v.max(vE, vH);
            v.store(pe, i, vE);
            vF = v.template subs<W>(vF, vGapE);
            vF = v.max(vF, vH);
            vH = v.load(hl, i);
        }
        {
            long long tmp = pr.s2_beg ? -(long long)open : (long long)bj1 - open;
            const int tmp2 = tmp < Lim<W>::MIN ? Lim<W>::MIN : wrap<W>(tmp);
            bool done = false;
            for (int k = 0; k < L && !done; ++k) {
                vF = v.insert0(v.shift1(vF), tmp2);
                for (int i = 0; i < segLen; ++i) {
                    vH = v.load(hs, i);
                    vH = v.max(vH, vF);
                    v.store(hs, i, vH);
                    vSatMin = v.min(vSatMin, vH);
                    vSatMax = v.max(vSatMax, vH);
                    vH = v.template subs<W>(vH, vGapO);
                    vF = v.template subs<W>(vF, vGapE);
                    const V go = TRACE ? v.or_(v.cmpgt(vF, vH), v.cmpeq(vF, vH)) : v.cmpgt(vF, vH);
                    if (!v.any(go)) { done = true; break; }
                }
            }
        }
        {
            vH = v.load(hs, offset);
            const V vCompare = v.and_(vPosMask, v.cmpgt(vH, vMaxH));
            vMaxH = v.max(vH, vMaxH);
            if (v.any(vCompare)) end_ref = j;
        }
        /* the limit checks only accumulate: once one trips, the kernel's
         * result is the saturated one whatever follows */
        if (v.any(v.or_(v.cmpgt(vNegLimit, vSatMin), v.cmpgt(vSatMax, vPosLimit)))) break;
    }
    if (pr.s2_end) {
        score = v.extract(vMaxH, lastLane);
        end_query = s1Len - 1;
    }
    if (pr.s1_end) {
        /* the last column in memory order: segment-major, lane-minor */
        for (int i = 0; i < segLen; ++i) {
            for (int l = 0; l < L; ++l) {
                const int temp = i + l * segLen;
                if (temp >= s1Len) continue;
                const int t = v.extract(v.load(hs, i), l);
                if (t > score) {
                    score = t; end_query = temp; end_ref = s2Len - 1;
                } else if (t == score && end_ref == s2Len - 1 && temp < end_query) {
                    end_query = temp;
                }
            }
        }
    }
    if (!pr.s1_end && !pr.s2_end) {
        score = v.extract(v.load(hs, offset), lastLane);
        end_ref = s2Len - 1;
        end_query = s1Len - 1;
    }
    o.saturated = v.any(v.or_(v.cmpgt(vNegLimit, vSatMin), v.cmpgt(vSatMax, vPosLimit))) ? 1 : 0;
    if (o.saturated) { score = 0; end_query = 0; end_ref = 0; }
    o.score = score; o.end_query = end_query; o.end_ref = end_ref;
    o.matches = o.similar = o.length = 0;
}

/* ---- nw / sg with statistics ---- */
template <class P, int W>
PB_LHD void striped_nwsg_stats(P &v, const Problem &pr, Out &o)
{
    typedef typename P::V V;
    constexpr int L = Lim<W>::LANES;
    const int s1Len = pr.qlen, s2Len = pr.tlen;
    const int segLen = (s1Len + L - 1) / L;
    const int offset = (s1Len - 1) % segLen;
    const int lastLane = (s1Len - 1) / segLen;
    const int open = pr.open, gap = pr.gap;
    const int NEG_LIMIT = wrap<W>((-open < pr.mmin ? (long long)Lim<W>::MIN + open : (long long)Lim<W>::MIN - pr.mmin) + 1);
    const int POS_LIMIT = wrap<W>((long long)Lim<W>::MAX - pr.mmax - 1);
    const V vGapO = v.set1(wrap<W>(open)), vGapE = v.set1(wrap<W>(gap));
    const V vZero = v.set1(0), vOne = v.set1(1);
    const V vNegLimit = v.set1(NEG_LIMIT), vPosLimit = v.set1(POS_LIMIT);
    V vSatMin = vPosLimit, vSatMax = vNegLimit;
    V vMaxH = vNegLimit, vMaxHM = vNegLimit, vMaxHS = vNegLimit, vMaxHL = vNegLimit;
    const V vPosMask = v.lane_eq(lastLane);
    int end_query = s1Len - 1, end_ref = s2Len - 1;
    int score = NEG_LIMIT, matches = 0, similar = 0, length = 0;

    typename P::Arr hs = v.arr(0, segLen), hl = v.arr(1, segLen);
    typename P::Arr hms = v.arr(2, segLen), hml = v.arr(3, segLen);
    typename P::Arr hss = v.arr(4, segLen), hsl = v.arr(5, segLen);
    typename P::Arr hls = v.arr(6, segLen), hll = v.arr(7, segLen);
    typename P::Arr pe = v.arr(8, segLen), pem = v.arr(9, segLen), pes = v.arr(10, segLen), pel = v.arr(11, segLen);
    for (int i = 0; i < segLen; ++i) {
        v.store(hms, i, vZero); v.store(hss, i, vZero); v.store(hls, i, vZero);
        v.store(pem, i, vZero); v.store(pes, i, vZero); v.store(pel, i, vOne);
        V h, e;
        v.template init_he<W>(h, e, i, segLen, pr.s1_beg, open, gap);
        v.store(hs, i, h);
        v.store(pe, i, e);
    }
    for (int j = 0; j < s2Len; ++j) {
        const int bj = v.template boundary<W>(pr, j), bj1 = v.template boundary<W>(pr, j + 1);
        const int k_t = pr.t[j];
        V vF = vNegLimit, vFM = vZero, vFS = vZero, vFL = vOne;
        V vH = v.shift1(v.load(hs, segLen - 1));
        V vHM = v.shift1(v.load(hms, segLen - 1));
        V vHS = v.shift1(v.load(hss, segLen - 1));
        V vHL = v.shift1(v.load(hls, segLen - 1));
        vH = v.insert0(vH, bj);
        { typename P::Arr t0 = hl; hl = hs; hs = t0; }
        { typename P::Arr t0 = hml; hml = hms; hms = t0; }
        { typename P::Arr t0 = hsl; hsl = hss; hss = t0; }
        { typename P::Arr t0 = hll; hll = hls; hls = t0; }
        for (int i = 0; i < segLen; ++i) {
            V vE = v.load(pe, i), vEM = v.load(pem, i), vES = v.load(pes, i), vEL = v.load(pel, i);
            const V vH_dag = v.template adds<W>(vH, v.template prof<W>(pr, k_t, i, segLen));
            vH = v.max(vH_dag, vE);
            vH = v.max(vH, vF);
            v.store(hs, i, vH);
            V case1 = v.cmpeq(vH, vH_dag);
            const V case2 = v.cmpeq(vH, vF);
            vHM = v.blend(v.blend(vEM, vFM, case2), v.template adds<W>(vHM, v.template match<W>(pr, k_t, i, segLen)), case1);
            v.store(hms, i, vHM);
            vHS = v.blend(v.blend(vES, vFS, case2), v.template adds<W>(vHS, v.template similar<W>(pr, k_t, i, segLen)), case1);
            v.store(hss, i, vHS);
            vHL = v.blend(v.blend(vEL, vFL, case2), v.template adds<W>(vHL, vOne), case1);
            v.store(hls, i, vHL);
            vSatMin = v.min(vSatMin, vH);
            vSatMax = v.max(vSatMax, vH);
            vSatMax = v.max(vSatMax, vHM);
            vSatMax = v.max(vSatMax, vHS);
            vSatMax = v.max(vSatMax, vHL);
            const V vEF_opn = v.template subs<W>(vH, vGapO);
            const V vE_ext = v.template subs<W>(vE, vGapE);
            vE = v.max(vEF_opn, vE_ext);
            case1 = v.cmpgt(vEF_opn, vE_ext);
            vEM = v.blend(vEM, vHM, case1);
            vES = v.blend(vES, vHS, case1);
            vEL = v.blend(v.template adds<W>(vEL, vOne), v.template adds<W>(vHL, vOne), case1);
            v.store(pe, i, vE); v.store(pem, i, vEM); v.store(pes, i, vES); v.store(pel, i, vEL);
            const V vF_ext = v.template subs<W>(vF, vGapE);
            vF = v.max(vEF_opn, vF_ext);
            case1 = v.cmpgt(vEF_opn, vF_ext);
            vFM = v.blend(vFM, vHM, case1);
            vFS = v.blend(vFS, vHS, case1);
            vFL = v.blend(v.template adds<W>(vFL, vOne), v.template adds<W>(vHL, vOne), case1);
            vH = v.load(hl, i); vHM = v.load(hml, i); vHS = v.load(hsl, i); vHL = v.load(hll, i);
        }
        {
            long long tmp = pr.s2_beg ? -(long long)open : (long long)bj1 - open;
            const int tmp2 = tmp < Lim<W>::MIN ? Lim<W>::MIN : wrap<W>(tmp);
            bool done = false;
            for (int k = 0; k < L && !done; ++k) {
                V vHp = v.shift1(v.load(hl, segLen - 1));
                vF = v.shift1(vF); vFM = v.shift1(vFM); vFS = v.shift1(vFS); vFL = v.shift1(vFL);
                vHp = v.insert0(vHp, bj);
                vF = v.insert0(vF, tmp2);
                vFL = v.insert0(vFL, 1);
                for (int i = 0; i < segLen; ++i) {
                    vHp = v.template adds<W>(vHp, v.template prof<W>(pr, k_t, i, segLen));
                    vH = v.load(hs, i);
                    vH = v.max(vH, vF);
                    v.store(hs, i, vH);
                    const V case1 = v.cmpeq(vH, vHp);
                    const V case2 = v.cmpeq(vH, vF);
                    V cond = v.andnot(case1, case2);
                    vHM = v.blend(v.load(hms, i), vFM, cond); v.store(hms, i, vHM);
                    vHS = v.blend(v.load(hss, i), vFS, cond); v.store(hss, i, vHS);
                    vHL = v.blend(v.load(hls, i), vFL, cond); v.store(hls, i, vHL);
                    vSatMin = v.min(vSatMin, vH);
                    vSatMax = v.max(vSatMax, vH);
                    vSatMax = v.max(vSatMax, vHM);
                    vSatMax = v.max(vSatMax, vHS);
                    vSatMax = v.max(vSatMax, vHL);
                    const V vEF_opn = v.template subs<W>(vH, vGapO);
                    const V vF_ext = v.template subs<W>(vF, vGapE);
                    if (!v.any(v.or_(v.cmpgt(vF_ext, vEF_opn), v.cmpeq(vF_ext, vEF_opn)))) { done = true; break; }
                    vF = vF_ext;
                    cond = v.cmpgt(vEF_opn, vF_ext);
                    vFM = v.blend(vFM, vHM, cond);
                    vFS = v.blend(vFS, vHS, cond);
                    vFL = v.blend(v.template adds<W>(vFL, vOne), v.template adds<W>(vHL, vOne), cond);
                    vHp = v.load(hl, i);
                }
            }
        }
        {
            vH = v.load(hs, offset); vHM = v.load(hms, offset); vHS = v.load(hss, offset); vHL = v.load(hls, offset);
            const V cond_max = v.cmpgt(vH, vMaxH);
            vMaxH = v.blend(vMaxH, vH, cond_max);
            vMaxHM = v.blend(vMaxHM, vHM, cond_max);
            vMaxHS = v.blend(vMaxHS, vHS, cond_max);
            vMaxHL = v.blend(vMaxHL, vHL, cond_max);
            if (v.any(v.and_(vPosMask, cond_max))) end_ref = j;
        }
        if (v.any(v.or_(v.cmpgt(vNegLimit, vSatMin), v.cmpgt(vSatMax, vPosLimit)))) break;
    }
    if (pr.s2_end) {
        end_query = s1Len - 1;
        score = v.extract(vMaxH, lastLane);
        matches = v.extract(vMaxHM, lastLane);
        similar = v.extract(vMaxHS, lastLane);
        length = v.extract(vMaxHL, lastLane);
    }
    if (pr.s1_end) {
        for (int i = 0; i < segLen; ++i) {
            const V th = v.load(hs, i), tm = v.load(hms, i), ts = v.load(hss, i), tl = v.load(hls, i);
            for (int l = 0; l < L; ++l) {
                const int temp = i + l * segLen;
                if (temp >= s1Len) continue;
                const int t = v.extract(th, l);
                if (t > score) {
                    score = t; end_query = temp; end_ref = s2Len - 1;
                    matches = v.extract(tm, l); similar = v.extract(ts, l); length = v.extract(tl, l);
                } else if (t == score && end_ref == s2Len - 1 && temp < end_query) {
                    end_query = temp;
                    matches = v.extract(tm, l); similar = v.extract(ts, l); length = v.extract(tl, l);
                }
            }
        }
    }
    if (!pr.s1_end && !pr.s2_end) {
        score = v.extract(v.load(hs, offset), lastLane);
        matches = v.extract(v.load(hms, offset), lastLane);
        similar = v.extract(v.load(hss, offset), lastLane);
        length = v.extract(v.load(hls, offset), lastLane);
        end_ref = s2Len - 1;
        end_query = s1Len - 1;
    }
    o.saturated = v.any(v.or_(v.cmpgt(vNegLimit, vSatMin), v.cmpgt(vSatMax, vPosLimit))) ? 1 : 0;
    if (o.saturated) { score = matches = similar = length = 0; end_query = end_ref = 0; }
    o.score = score; o.end_query = end_query; o.end_ref = end_ref;
    o.matches = matches; o.similar = similar; o.length = length;
}

/* ---- sw with statistics, biased lanes (the FASTSTATS prefix kernel) ---- */
template <class P, int W>
PB_LHD void striped_sw_stats_bias(P &v, const Problem &pr, Out &o)
{
    typedef typename P::V V;
    constexpr int L = Lim<W>::LANES;
    const int s1Len = pr.qlen, s2Len = pr.tlen;
    const int segLen = (s1Len + L - 1) / L;
    const int open = pr.open, gap = pr.gap;
    const int bias = Lim<W>::MIN;
    const V vGapO = v.set1(wrap<W>(open)), vGapE = v.set1(wrap<W>(gap));
    const V vOne = v.set1(1);
    const V vBias = v.set1(bias);
    const V vBias1 = v.template adds<W>(vBias, vOne);
    const V insert_mask = v.lane_eq(0);
    const V vPosLimit = v.set1(Lim<W>::MAX);
    const int maxp = wrap<W>((long long)Lim<W>::MAX - wrap<W>((long long)pr.mmax + 1));
    V vMaxH = vBias, vMaxHUnit = vBias, vSatMax = vBias;
    int score = bias, matches = bias, similar = bias, length = bias;
    int end_query = 0, end_ref = 0;
    int saturated = 0;

    typename P::Arr hs = v.arr(0, segLen), hl = v.arr(1, segLen), hx = v.arr(2, segLen);
    typename P::Arr hms = v.arr(3, segLen), hml = v.arr(4, segLen), hmx = v.arr(5, segLen);
    typename P::Arr hss = v.arr(6, segLen), hsl = v.arr(7, segLen), hsx = v.arr(8, segLen);
    typename P::Arr hls = v.arr(9, segLen), hll = v.arr(10, segLen), hlx = v.arr(11, segLen);
    typename P::Arr pe = v.arr(12, segLen), pem = v.arr(13, segLen), pes = v.arr(14, segLen), pel = v.arr(15, segLen);
    for (int i = 0; i < segLen; ++i) {
        v.store(hs, i, vBias); v.store(hms, i, vBias); v.store(hss, i, vBias); v.store(hls, i, vBias);
        v.store(pe, i, vBias); v.store(pem, i, vBias); v.store(pes, i, vBias); v.store(pel, i, vBias1);
    }
    int j;
    for (j = 0; j < s2Len; ++j) {
        const int k_t = pr.t[j];
        V vF = vBias, vFM = vBias, vFS = vBias, vFL = vBias1;
        V vH = v.blend(v.shift1(v.load(hs, segLen - 1)), vBias, insert_mask);
        V vHM = v.blend(v.shift1(v.load(hms, segLen - 1)), vBias, insert_mask);
        V vHS = v.blend(v.shift1(v.load(hss, segLen - 1)), vBias, insert_mask);
        V vHL = v.blend(v.shift1(v.load(hls, segLen - 1)), vBias, insert_mask);
        if (end_ref == j - 2) {
            /* SWAP3(Max, Load, Store): Max <- Load, Load <- Store, Store <- old Max */
            typename P::Arr t0;
            t0 = hx; hx = hl; hl = hs; hs = t0;
            t0 = hmx; hmx = hml; hml = hms; hms = t0;
            t0 = hsx; hsx = hsl; hsl = hss; hss = t0;
            t0 = hlx; hlx = hll; hll = hls; hls = t0;
        } else {
            typename P::Arr t0;
            t0 = hl; hl = hs; hs = t0;
            t0 = hml; hml = hms; hms = t0;
            t0 = hsl; hsl = hss; hss = t0;
            t0 = hll; hll = hls; hls = t0;
        }
        for (int i = 0; i < segLen; ++i) {
            V vE = v.load(pe, i), vEM = v.load(pem, i), vES = v.load(pes, i), vEL = v.load(pel, i);
            const V vH_dag = v.template adds<W>(vH, v.template prof<W>(pr, k_t, i, segLen));
            vH = v.max(vH_dag, vE);
            vH = v.max(vH, vF);
            v.store(hs, i, vH);
            const V cond_zero = v.cmpeq(vH, vBias);
            V case1 = v.cmpeq(vH, vH_dag);
            const V case2 = v.cmpeq(vH, vF);
            vHM = v.blend(v.blend(vEM, vFM, case2), v.template adds<W>(vHM, v.template match<W>(pr, k_t, i, segLen)), case1);
            vHM = v.blend(vHM, vBias, cond_zero);
            v.store(hms, i, vHM);
            vHS = v.blend(v.blend(vES, vFS, case2), v.template adds<W>(vHS, v.template similar<W>(pr, k_t, i, segLen)), case1);
            vHS = v.blend(vHS, vBias, cond_zero);
            v.store(hss, i, vHS);
            vHL = v.blend(v.blend(vEL, vFL, case2), v.template adds<W>(vHL, vOne), case1);
            vHL = v.blend(vHL, vBias, cond_zero);
            v.store(hls, i, vHL);
            vSatMax = v.max(vSatMax, vHM);
            vSatMax = v.max(vSatMax, vHS);
            vSatMax = v.max(vSatMax, vHL);
            vMaxH = v.max(vH, vMaxH);
            const V vEF_opn = v.template subs<W>(vH, vGapO);
            const V vE_ext = v.template subs<W>(vE, vGapE);
            vE = v.max(vEF_opn, vE_ext);
            case1 = v.cmpgt(vEF_opn, vE_ext);
            vEM = v.blend(vEM, vHM, case1);
            vES = v.blend(vES, vHS, case1);
            vEL = v.blend(v.template adds<W>(vEL, vOne), v.template adds<W>(vHL, vOne), case1);
            v.store(pe, i, vE); v.store(pem, i, vEM); v.store(pes, i, vES); v.store(pel, i, vEL);
            const V vF_ext = v.template subs<W>(vF, vGapE);
            vF = v.max(vEF_opn, vF_ext);
            case1 = v.cmpgt(vEF_opn, vF_ext);
            vFM = v.blend(vFM, vHM, case1);
            vFS = v.blend(vFS, vHS, case1);
            vFL = v.blend(v.template adds<W>(vFL, vOne), v.template adds<W>(vHL, vOne), case1);
            vH = v.load(hl, i); vHM = v.load(hml, i); vHS = v.load(hsl, i); vHL = v.load(hll, i);
        }
        {
            bool done = false;
            for (int k = 0; k < L && !done; ++k) {
                V vHp = v.shift1(v.load(hl, segLen - 1));
                vF = v.shift1(vF); vFM = v.shift1(vFM); vFS = v.shift1(vFS); vFL = v.shift1(vFL);
                vHp = v.blend(vHp, vBias, insert_mask);
                vF = v.blend(vF, vBias, insert_mask);
                vFM = v.blend(vFM, vBias, insert_mask);
                vFS = v.blend(vFS, vBias, insert_mask);
                vFL = v.blend(vFL, vBias1, insert_mask);
                for (int i = 0; i < segLen; ++i) {
                    vHp = v.template adds<W>(vHp, v.template prof<W>(pr, k_t, i, segLen));
                    vH = v.load(hs, i);
                    vH = v.max(vH, vF);
                    v.store(hs, i, vH);
                    const V case1 = v.cmpeq(vH, vHp);
                    const V case2 = v.cmpeq(vH, vF);
                    V cond = v.andnot(case1, case2);
                    vHM = v.blend(v.load(hms, i), vFM, cond); v.store(hms, i, vHM);
                    vHS = v.blend(v.load(hss, i), vFS, cond); v.store(hss, i, vHS);
                    vHL = v.blend(v.load(hls, i), vFL, cond); v.store(hls, i, vHL);
                    vSatMax = v.max(vSatMax, vHM);
                    vSatMax = v.max(vSatMax, vHS);
                    vSatMax = v.max(vSatMax, vHL);
                    vMaxH = v.max(vH, vMaxH);
                    const V vEF_opn = v.template subs<W>(vH, vGapO);
                    const V vF_ext = v.template subs<W>(vF, vGapE);
                    if (!v.any(v.or_(v.cmpgt(vF_ext, vEF_opn),
                                     v.and_(v.cmpeq(vF_ext, vEF_opn), v.cmpgt(vF_ext, vBias))))) { done = true; break; }
                    vF = vF_ext;
                    cond = v.cmpgt(vEF_opn, vF_ext);
                    vFM = v.blend(vFM, vHM, cond);
                    vFS = v.blend(vFS, vHS, cond);
                    vFL = v.blend(v.template adds<W>(vFL, vOne), v.template adds<W>(vHL, vOne), cond);
                    vHp = v.load(hl, i);
                }
            }
        }
        if (v.any(v.cmpgt(vMaxH, vMaxHUnit))) {
            score = v.hmax(vMaxH);
            if (score > maxp) { saturated = 1; break; }
            vMaxHUnit = v.set1(score);
            end_ref = j;
        }
        if (v.any(v.cmpeq(vSatMax, vPosLimit))) { saturated = 1; break; }
    }
    if (score == Lim<W>::MAX || v.any(v.cmpeq(vSatMax, vPosLimit))) saturated = 1;
    if (saturated) {
        score = end_query = end_ref = matches = similar = length = 0;
    } else {
        typename P::Arr tx = hx, tmx = hmx, tsx = hsx, tlx = hlx;
        if (end_ref == j - 1) { tx = hs; tmx = hms; tsx = hss; tlx = hls; }
        else if (end_ref == j - 2) { tx = hl; tmx = hml; tsx = hsl; tlx = hll; }
        end_query = s1Len;
        for (int i = 0; i < segLen; ++i) {
            const V th = v.load(tx, i), tm = v.load(tmx, i), ts = v.load(tsx, i), tl = v.load(tlx, i);
            for (int l = 0; l < L; ++l) {
                if (v.extract(th, l) == score) {
                    const int temp = i + l * segLen;
                    if (temp < end_query) {
                        end_query = temp;
                        matches = v.extract(tm, l); similar = v.extract(ts, l); length = v.extract(tl, l);
                    }
                }
            }
        }
    }
    o.saturated = saturated;
    o.score = score - bias;
    o.end_query = end_query;
    o.end_ref = end_ref;
    o.matches = matches - bias;
    o.similar = similar - bias;
    o.length = length - bias;
}

/* ---- sw, score only: biased lanes at 8/16 bits (util/templates/
 * sw_striped_bias.c), plain lanes with an explicit 0 floor at 32
 * (util/templates/sw_striped.c) ---- */
template <class P, int W>
PB_LHD void striped_sw(P &v, const Problem &pr, Out &o)
{
    typedef typename P::V V;
    constexpr int L = Lim<W>::LANES;
    constexpr bool BIAS = W != 32;
    const int s1Len = pr.qlen, s2Len = pr.tlen;
    const int segLen = (s1Len + L - 1) / L;
    const int open = pr.open, gap = pr.gap;
    const int bias = BIAS ? Lim<W>::MIN : 0;
    const int neg_inf = BIAS ? Lim<W>::MIN : Lim<W>::MIN / 2;
    const V vGapO = v.set1(wrap<W>(open)), vGapE = v.set1(wrap<W>(gap));
    const V vZero = v.set1(0);
    const V vBias = v.set1(bias);
    const V insert_mask = v.lane_eq(0);
    const int maxp = wrap<W>((long long)Lim<W>::MAX - wrap<W>((long long)pr.mmax + 1));
    V vMaxH = v.set1(BIAS ? bias : neg_inf), vMaxHUnit = vMaxH;
    int score = BIAS ? bias : neg_inf;
    int end_query = 0, end_ref = 0, saturated = 0;

    typename P::Arr hs = v.arr(0, segLen), hl = v.arr(1, segLen), hx = v.arr(2, segLen), pe = v.arr(3, segLen);
    const V e0 = BIAS ? vBias : v.set1(wrap<W>(-(long long)open));
    for (int i = 0; i < segLen; ++i) {
        v.store(hs, i, BIAS ? vBias : vZero);
        v.store(pe, i, e0);
    }
    int j;
    for (j = 0; j < s2Len; ++j) {
        const int k_t = pr.t[j];
        V vE;
        V vF = BIAS ? vBias : vZero;
        V vH = v.shift1(v.load(hs, segLen - 1));
        if (BIAS) vH = v.blend(vH, vBias, insert_mask);
        if (end_ref == j - 2) {
            typename P::Arr t0 = hx; hx = hl; hl = hs; hs = t0;
        } else {
            typename P::Arr t0 = hl; hl = hs; hs = t0;
        }
        for (int i = 0; i < segLen; ++i) {
            vH = v.template adds<W>(vH, v.template prof<W>(pr, k_t, i, segLen));
            vE = v.load(pe, i);
            vH = v.max(vH, vE);
            vH = v.max(vH, vF);
            if (!BIAS) vH = v.max(vH, vZero);
            v.store(hs, i, vH);
            vMaxH = v.max(vH, vMaxH);
            vH = v.template subs<W>(vH, vGapO);
            vE = v.template subs<W>(vE, vGapE);
            vE = v.max(vE, vH);
            v.store(pe, i, vE);
            vF = v.template subs<W>(vF, vGapE);
            vF = v.max(vF, vH);
            vH = v.load(hl, i);
        }
        {
            bool done = false;
            for (int k = 0; k < L && !done; ++k) {
                vF = v.shift1(vF);
                if (BIAS) vF = v.blend(vF, vBias, insert_mask);
                for (int i = 0; i < segLen; ++i) {
                    vH = v.load(hs, i);
                    vH = v.max(vH, vF);
                    v.store(hs, i, vH);
                    vMaxH = v.max(vH, vMaxH);
                    vH = v.template subs<W>(vH, vGapO);
                    vF = v.template subs<W>(vF, vGapE);
                    if (!v.any(v.cmpgt(vF, vH))) { done = true; break; }
                }
            }
        }
        if (v.any(v.cmpgt(vMaxH, vMaxHUnit))) {
            score = v.hmax(vMaxH);
            if (score > maxp) { saturated = 1; break; }
            vMaxHUnit = v.set1(score);
            end_ref = j;
        }
    }
    if (score == Lim<W>::MAX) saturated = 1;
    if (saturated) {
        score = Lim<W>::MAX;
        end_query = 0;
        end_ref = 0;
    } else {
        typename P::Arr tx = hx;
        if (end_ref == j - 1) tx = hs;
        else if (end_ref == j - 2) tx = hl;
        end_query = s1Len - 1;
        for (int i = 0; i < segLen; ++i) {
            const V th = v.load(tx, i);
            for (int l = 0; l < L; ++l) {
                if (v.extract(th, l) == score) {
                    const int temp = i + l * segLen;
                    if (temp < end_query) end_query = temp;
                }
            }
        }
    }
    o.saturated = saturated;
    o.score = (int)((long long)score - bias);
    o.end_query = end_query;
    o.end_ref = end_ref;
    o.matches = o.similar = o.length = 0;
}

/* ---- nw / sg trace, scan: the saturation flag of util/templates/
 * nw_trace_scan.c and sg_trace_scan.c (src/nw_trace_scan_avx2_256_8.c:
 * 238-350, src/sg_trace_scan_avx2_256_8.c:255-262). The checks cover E as
 * the first loop updates it, H and F of the final loop, and for SG the
 * gap ramp of pvGapper; the prefix scan adds set1(-segLen*gap), which the
 * lane width truncates. A non-saturated trace result is the exact DP's, so
 * only the flag is produced. ---- */
template <int W> PB_LHD int gapper_at(int open, int gap, int segLen, int i)
{
    /* pvGapper[i]: 0 - open, then segLen-1-i subtractions of gap in the
     * lane's arithmetic (saturating at 8/16 bits: a constant saturating step
     * stays clamped once it clamps; wrapping at 32) */
    const long long x0 = lane_arith<W>(-(long long)wrap<W>(open));
    return lane_arith<W>(x0 - (long long)(segLen - 1 - i) * wrap<W>(gap));
}

template <class P, int W>
PB_LHD void scan_nwsg_trace(P &v, const Problem &pr, Out &o)
{
    typedef typename P::V V;
    constexpr int L = Lim<W>::LANES;
    const int s1Len = pr.qlen, s2Len = pr.tlen;
    const int segLen = (s1Len + L - 1) / L;
    const int open = pr.open, gap = pr.gap;
    const bool sg = pr.s1_beg || pr.s1_end || pr.s2_beg || pr.s2_end;
    const int NEG_LIMIT = wrap<W>((-open < pr.mmin ? (long long)Lim<W>::MIN + open : (long long)Lim<W>::MIN - pr.mmin) + 1);
    const int POS_LIMIT = wrap<W>((long long)Lim<W>::MAX - pr.mmax - 1);
    const V vGapO = v.set1(wrap<W>(open)), vGapE = v.set1(wrap<W>(gap));
    const V vNegLimit = v.set1(NEG_LIMIT), vPosLimit = v.set1(POS_LIMIT);
    const V vNegInfFront = v.insert0(v.set1(0), NEG_LIMIT);
    const V vSegLenXgap = v.template adds<W>(vNegInfFront, v.shift1(v.set1(wrap<W>(-(long long)segLen * gap))));
    const V vGapper0 = v.set1(gapper_at<W>(open, gap, segLen, 0));
    V vSatMin = vPosLimit, vSatMax = vNegLimit;
    if (sg) {
        /* the ramp's values after each step, monotone: its two ends */
        const long long x0 = clampw<W>(-(long long)wrap<W>(open));
        const int a = clampw<W>(x0 - wrap<W>(gap)), b = clampw<W>(x0 - (long long)segLen * wrap<W>(gap));
        vSatMin = v.min(vSatMin, v.set1(a < b ? a : b));
    }

    typename P::Arr pe = v.arr(0, segLen), pht = v.arr(1, segLen), ph = v.arr(2, segLen);
    for (int i = 0; i < segLen; ++i) {
        V h, e;
        v.template init_he<W>(h, e, i, segLen, pr.s1_beg, open, gap);
        v.store(ph, i, h);
        v.store(pe, i, e);
    }
    for (int j = 0; j < s2Len; ++j) {
        const int bj = v.template boundary<W>(pr, j), bj1 = v.template boundary<W>(pr, j + 1);
        const int k_t = pr.t[j];
        V vHp = v.insert0(v.shift1(v.load(ph, segLen - 1)), bj);
        V vHt = v.template subs<W>(vNegLimit, vGapper0);
        V vF = vNegLimit;
        for (int i = 0; i < segLen; ++i) {
            const V vH = v.load(ph, i);
            V vE = v.load(pe, i);
            vE = v.max(v.template subs<W>(vH, vGapO), v.template subs<W>(vE, vGapE));
            vSatMin = v.min(vSatMin, vE);
            vF = v.max(vF, v.template adds<W>(vHt, v.set1(gapper_at<W>(open, gap, segLen, i))));
            vHp = v.template adds<W>(vHp, v.template prof<W>(pr, k_t, i, segLen));
            vHt = v.max(vE, vHp);
            v.store(pe, i, vE);
            v.store(pht, i, vHt);
            v.store(ph, i, vHp);
            vHp = vH;
        }
        /* pseudo prefix scan on F */
        vHt = v.insert0(v.shift1(vHt), bj1);
        vF = v.max(vF, v.template adds<W>(vHt, vGapper0));
        for (int k = 0; k < L - 2; ++k) vF = v.max(vF, v.template adds<W>(v.shift1(vF), vSegLenXgap));
        vF = v.template adds<W>(v.shift1(vF), vNegInfFront);
        V vH = v.max(vF, vHt);
        for (int i = 0; i < segLen; ++i) {
            vF = v.max(v.template subs<W>(vH, vGapO), v.template subs<W>(vF, vGapE));
            vH = v.max(v.load(pht, i), vF);
            v.store(ph, i, vH);
            vSatMin = v.min(vSatMin, vH);
            vSatMin = v.min(vSatMin, vF);
            vSatMax = v.max(vSatMax, vH);
        }
        if (v.any(v.or_(v.cmpgt(vNegLimit, vSatMin), v.cmpgt(vSatMax, vPosLimit)))) break;
    }
    o.saturated = v.any(v.or_(v.cmpgt(vNegLimit, vSatMin), v.cmpgt(vSatMax, vPosLimit))) ? 1 : 0;
    o.score = o.end_query = o.end_ref = 0;
    o.matches = o.similar = o.length = 0;
}

/* ---- nw / sg scan, score only: util/templates/nw_scan.c and sg_scan.c
 * (src/nw_scan_avx2_256_16.c:255-394, src/sg_scan_avx2_256_16.c:270-444):
 * E and the H of the diagonal in a first loop over the segments, F by a
 * pseudo prefix scan across the lanes, final H and F in a second loop.
 * Checked: H (and for SG F and the gap ramp of pvGapper). Ends as in the
 * striped kernels (column maxima of the last row, the last column in memory
 * order). ---- */
template <class P, int W>
PB_LHD void scan_nwsg(P &v, const Problem &pr, Out &o)
{
    typedef typename P::V V;
    constexpr int L = Lim<W>::LANES;
    const int s1Len = pr.qlen, s2Len = pr.tlen;
    const int segLen = (s1Len + L - 1) / L;
    const int offset = (s1Len - 1) % segLen;
    const int lastLane = (s1Len - 1) / segLen;
    const int open = pr.open, gap = pr.gap;
    const bool sg = pr.s1_beg || pr.s1_end || pr.s2_beg || pr.s2_end;
    const int NEG_LIMIT = wrap<W>((-open < pr.mmin ? (long long)Lim<W>::MIN + open : (long long)Lim<W>::MIN - pr.mmin) + 1);
    const int POS_LIMIT = wrap<W>((long long)Lim<W>::MAX - pr.mmax - 1);
    const V vGapO = v.set1(wrap<W>(open)), vGapE = v.set1(wrap<W>(gap));
    const V vNegLimit = v.set1(NEG_LIMIT), vPosLimit = v.set1(POS_LIMIT);
    const V vNegInfFront = v.insert0(v.set1(0), NEG_LIMIT);
    const V vSegLenXgap = v.template adds<W>(vNegInfFront, v.shift1(v.set1(wrap<W>(-(long long)segLen * gap))));
    const V vGapper0 = v.set1(gapper_at<W>(open, gap, segLen, 0));
    const V vPosMask = v.lane_eq(lastLane);
    V vSatMin = vPosLimit, vSatMax = vNegLimit, vMaxH = vNegLimit;
    if (sg) {
        const long long x0 = lane_arith<W>(-(long long)wrap<W>(open));
        const int a = lane_arith<W>(x0 - wrap<W>(gap)), b = lane_arith<W>(x0 - (long long)segLen * wrap<W>(gap));
        vSatMin = v.min(vSatMin, v.set1(a < b ? a : b));
    }
    int end_query = s1Len - 1, end_ref = s2Len - 1;
    int score = NEG_LIMIT;

    typename P::Arr pe = v.arr(0, segLen), pht = v.arr(1, segLen), ph = v.arr(2, segLen);
    for (int i = 0; i < segLen; ++i) {
        V h, e;
        v.template init_he<W>(h, e, i, segLen, pr.s1_beg, open, gap);
        v.store(ph, i, h);
        v.store(pe, i, e);
    }
    for (int j = 0; j < s2Len; ++j) {
        const int bj = v.template boundary<W>(pr, j), bj1 = v.template boundary<W>(pr, j + 1);
        const int k_t = pr.t[j];
        V vHp = v.insert0(v.shift1(v.load(ph, segLen - 1)), bj);
        V vHt = v.template subs<W>(vNegLimit, vGapper0);
        V vF = vNegLimit;
        for (int i = 0; i < segLen; ++i) {
            const V vH = v.load(ph, i);
            V vE = v.load(pe, i);
            vE = v.max(v.template subs<W>(vE, vGapE), v.template subs<W>(vH, vGapO));
            vHp = v.template adds<W>(vHp, v.template prof<W>(pr, k_t, i, segLen));
            vF = v.max(vF, v.template adds<W>(vHt, v.set1(gapper_at<W>(open, gap, segLen, i))));
            vHt = v.max(vE, vHp);
            v.store(pe, i, vE);
            v.store(pht, i, vHt);
            vHp = vH;
        }
        vHt = v.insert0(v.shift1(vHt), bj1);
        vF = v.max(vF, v.template adds<W>(vHt, vGapper0));
        for (int k = 0; k < L - 2; ++k) vF = v.max(vF, v.template adds<W>(v.shift1(vF), vSegLenXgap));
        vF = v.template adds<W>(v.shift1(vF), vNegInfFront);
        V vH = v.max(vHt, vF);
        for (int i = 0; i < segLen; ++i) {
            vF = v.max(v.template subs<W>(vF, vGapE), v.template subs<W>(vH, vGapO));
            vH = v.max(v.load(pht, i), vF);
            v.store(ph, i, vH);
            vSatMin = v.min(vSatMin, vH);
            if (sg) vSatMin = v.min(vSatMin, vF);
            vSatMax = v.max(vSatMax, vH);
        }
        {
            vH = v.load(ph, offset);
            const V vCompare = v.and_(vPosMask, v.cmpgt(vH, vMaxH));
            vMaxH = v.max(vH, vMaxH);
            if (v.any(vCompare)) end_ref = j;
        }
        if (v.any(v.or_(v.cmpgt(vNegLimit, vSatMin), v.cmpgt(vSatMax, vPosLimit)))) break;
    }
    if (pr.s2_end) {
        score = v.extract(vMaxH, lastLane);
        end_query = s1Len - 1;
    }
    if (pr.s1_end) {
        for (int i = 0; i < segLen; ++i) {
            for (int l = 0; l < L; ++l) {
                const int temp = i + l * segLen;
                if (temp >= s1Len) continue;
                const int t = v.extract(v.load(ph, i), l);
                if (t > score) {
                    score = t; end_query = temp; end_ref = s2Len - 1;
                } else if (t == score && end_ref == s2Len - 1 && temp < end_query) {
                    end_query = temp;
                }
            }
        }
    }
    if (!pr.s1_end && !pr.s2_end) {
        score = v.extract(v.load(ph, offset), lastLane);
        end_ref = s2Len - 1;
        end_query = s1Len - 1;
    }
    o.saturated = v.any(v.or_(v.cmpgt(vNegLimit, vSatMin), v.cmpgt(vSatMax, vPosLimit))) ? 1 : 0;
    if (o.saturated) { score = 0; end_query = 0; end_ref = 0; }
    o.score = score; o.end_query = end_query; o.end_ref = end_ref;
    o.matches = o.similar = o.length = 0;
}

/* ---- sw scan, score only: util/templates/sw_scan.c
 * (src/sw_scan_avx2_256_16.c:226-380): the scan passes with H clamped at 0,
 * the column maxima folded into vMaxH, the column of a new maximum copied,
 * and the smallest row of the best score found in that copy (padded rows
 * included). Checked: H. ---- */
template <class P, int W>
PB_LHD void scan_sw(P &v, const Problem &pr, Out &o)
{
    typedef typename P::V V;
    constexpr int L = Lim<W>::LANES;
    const int s1Len = pr.qlen, s2Len = pr.tlen;
    const int segLen = (s1Len + L - 1) / L;
    const int open = pr.open, gap = pr.gap;
    const int NEG_LIMIT = wrap<W>((-open < pr.mmin ? (long long)Lim<W>::MIN + open : (long long)Lim<W>::MIN - pr.mmin) + 1);
    const int POS_LIMIT = wrap<W>((long long)Lim<W>::MAX - pr.mmax - 1);
    const V vGapO = v.set1(wrap<W>(open)), vGapE = v.set1(wrap<W>(gap));
    const V vZero = v.set1(0);
    const V vNegLimit = v.set1(NEG_LIMIT), vPosLimit = v.set1(POS_LIMIT);
    const V vNegInfFront = v.insert0(vZero, NEG_LIMIT);
    const V vSegLenXgap = v.template adds<W>(vNegInfFront, v.shift1(v.set1(wrap<W>(-(long long)segLen * gap))));
    const V vGapper0 = v.set1(gapper_at<W>(open, gap, segLen, 0));
    V vSatMin = vPosLimit, vSatMax = vNegLimit, vMaxH = vNegLimit, vMaxHUnit = vNegLimit;
    int score = NEG_LIMIT, end_ref = 0, end_query = 0;

    typename P::Arr pe = v.arr(0, segLen), pht = v.arr(1, segLen), ph = v.arr(2, segLen), pmax = v.arr(3, segLen);
    for (int i = 0; i < segLen; ++i) {
        v.store(ph, i, vZero);
        v.store(pe, i, vNegLimit);
    }
    for (int j = 0; j < s2Len; ++j) {
        const int k_t = pr.t[j];
        V vHp = v.shift1(v.load(ph, segLen - 1));
        V vHt = vZero;
        V vF = vNegLimit;
        for (int i = 0; i < segLen; ++i) {
            const V vH = v.load(ph, i);
            V vE = v.load(pe, i);
            vE = v.max(v.template subs<W>(vE, vGapE), v.template subs<W>(vH, vGapO));
            vHp = v.template adds<W>(vHp, v.template prof<W>(pr, k_t, i, segLen));
            vF = v.max(vF, v.template adds<W>(vHt, v.set1(gapper_at<W>(open, gap, segLen, i))));
            vHt = v.max(vE, vHp);
            v.store(pe, i, vE);
            v.store(pht, i, vHt);
            vHp = vH;
        }
        vHt = v.shift1(vHt);
        vF = v.max(vF, v.template adds<W>(vHt, vGapper0));
        for (int k = 0; k < L - 2; ++k) vF = v.max(vF, v.template adds<W>(v.shift1(vF), vSegLenXgap));
        vF = v.template adds<W>(v.shift1(vF), vNegInfFront);
        V vH = v.max(v.max(vHt, vF), vZero);
        for (int i = 0; i < segLen; ++i) {
            vF = v.max(v.template subs<W>(vF, vGapE), v.template subs<W>(vH, vGapO));
            vH = v.max(v.max(v.load(pht, i), vF), vZero);
            v.store(ph, i, vH);
            vSatMin = v.min(vSatMin, vH);
            vSatMax = v.max(vSatMax, vH);
            vMaxH = v.max(vH, vMaxH);
        }
        if (v.any(v.cmpgt(vMaxH, vMaxHUnit))) {
            score = v.hmax(vMaxH);
            vMaxHUnit = v.set1(score);
            end_ref = j;
            for (int i = 0; i < segLen; ++i) v.store(pmax, i, v.load(ph, i));
        }
        if (v.any(v.or_(v.cmpgt(vNegLimit, vSatMin), v.cmpgt(vSatMax, vPosLimit)))) break;
    }
    /* the smallest row holding the score in the copied column (memory order,
     * padded rows included: src/sw_scan_avx2_256_16.c:356-368) */
    end_query = s1Len;
    for (int i = 0; i < segLen; ++i)
        for (int l = 0; l < L; ++l)
            if (v.extract(v.load(pmax, i), l) == score && i + l * segLen < end_query) end_query = i + l * segLen;
    o.saturated = v.any(v.or_(v.cmpgt(vNegLimit, vSatMin), v.cmpgt(vSatMax, vPosLimit))) ? 1 : 0;
    if (o.saturated) { score = 0; end_query = 0; end_ref = 0; }
    o.score = score; o.end_query = end_query; o.end_ref = end_ref;
    o.matches = o.similar = o.length = 0;
}

/* ---- nw / sg / sw scan with statistics: util/templates/nw_stats_scan.c,
 * sg_stats_scan.c, sw_stats_scan.c (src/nw_stats_scan_avx2_256_16.c:
 * 310-600, src/sg_stats_scan_avx2_256_16.c:615-675, src/sw_stats_scan_
 * avx2_256_16.c:319-612). First loop: E with its counts, the diagonal H
 * (stored in place of H) and Ht = max(E, diagonal), the running F of the
 * gap ramp pvGapper with its length ramp pvGapperL. Prefix scan of F over
 * the lanes, ties to the shifted value. Final loop: F from H, H = max of
 * diagonal, E and F with counts by diagonal > F > E (SW: clamped at 0 and
 * counts zeroed there). Checked: H and its three counts, every column, no
 * early exit. SW keeps a copy of the column where the lane maximum grew;
 * its end row is the smallest row of that copy holding the score, padded
 * rows included. The first-loop F blend reads Ht's counts before the loop
 * has set them; it can only pick them when F is still the gap ramp, whose
 * counts never reach a result, and they start at zero here. ---- */
template <class P, int W, bool SW>
PB_LHD void scan_stats(P &v, const Problem &pr, Out &o)
{
    typedef typename P::V V;
    constexpr int L = Lim<W>::LANES;
    const int s1Len = pr.qlen, s2Len = pr.tlen;
    const int segLen = (s1Len + L - 1) / L;
    const int offset = (s1Len - 1) % segLen;
    const int lastLane = (s1Len - 1) / segLen;
    const int open = pr.open, gap = pr.gap;
    const int NEG_LIMIT = wrap<W>((-open < pr.mmin ? (long long)Lim<W>::MIN + open : (long long)Lim<W>::MIN - pr.mmin) + 1);
    const int POS_LIMIT = wrap<W>((long long)Lim<W>::MAX - pr.mmax - 1);
    const V vGapO = v.set1(wrap<W>(open)), vGapE = v.set1(wrap<W>(gap));
    const V vZero = v.set1(0), vOne = v.set1(1);
    const V vNegLimit = v.set1(NEG_LIMIT), vPosLimit = v.set1(POS_LIMIT);
    const V vNegInfFront = v.insert0(vZero, NEG_LIMIT);
    const V vSegLenXgap = v.template adds<W>(vNegInfFront, v.shift1(v.set1(wrap<W>(-(long long)segLen * gap))));
    const V vSegLen = v.shift1(v.set1(wrap<W>(segLen)));
    const V vPosMask = v.lane_eq(lastLane);
    V vSatMin = vPosLimit, vSatMax = vNegLimit;
    V vMaxH = vNegLimit, vMaxM = vNegLimit, vMaxS = vNegLimit, vMaxL = vNegLimit, vMaxHUnit = vNegLimit;
    int end_query = SW ? 0 : s1Len - 1, end_ref = SW ? 0 : s2Len - 1;
    int score = NEG_LIMIT, matches = 0, similar = 0, length = 0;

    typename P::Arr pe = v.arr(0, segLen), pem = v.arr(1, segLen), pes = v.arr(2, segLen), pel = v.arr(3, segLen);
    typename P::Arr ph = v.arr(4, segLen), phm = v.arr(5, segLen), phs = v.arr(6, segLen), phl = v.arr(7, segLen);
    typename P::Arr px = SW ? v.arr(8, segLen) : ph, pxm = SW ? v.arr(9, segLen) : ph;
    typename P::Arr pxs = SW ? v.arr(10, segLen) : ph, pxl = SW ? v.arr(11, segLen) : ph;
    for (int i = 0; i < segLen; ++i) {
        v.store(phm, i, vZero); v.store(phs, i, vZero); v.store(phl, i, vZero);
        v.store(pe, i, vNegLimit); v.store(pem, i, vZero); v.store(pes, i, vZero); v.store(pel, i, vZero);
        if (SW) {
            v.store(ph, i, vZero);
        } else {
            V h, e;
            v.template init_he<W>(h, e, i, segLen, pr.s1_beg, open, gap);
            v.store(ph, i, h);
        }
    }
    for (int j = 0; j < s2Len; ++j) {
        const int k_t = pr.t[j];
        V vHp = v.shift1(v.load(ph, segLen - 1));
        V vHpM = v.shift1(v.load(phm, segLen - 1));
        V vHpS = v.shift1(v.load(phs, segLen - 1));
        V vHpL = v.shift1(v.load(phl, segLen - 1));
        if (!SW) vHp = v.insert0(vHp, v.template boundary<W>(pr, j));
        V vHt = SW ? vZero : v.template subs<W>(vNegLimit, v.set1(gapper_at<W>(open, gap, segLen, 0)));
        V vHtM = vZero, vHtS = vZero, vHtL = vZero;
        V vF = vNegLimit, vFM = vZero, vFS = vZero, vFL = vZero;
        for (int i = 0; i < segLen; ++i) {
            const V vH = v.load(ph, i), vHM = v.load(phm, i), vHS = v.load(phs, i), vHL = v.load(phl, i);
            V vE = v.load(pe, i), vEM = v.load(pem, i), vES = v.load(pes, i), vEL = v.load(pel, i);
            /* pvGapperL[i]: 1, then segLen-1-i lane additions of one */
            const V vGapperL = v.set1(lane_arith<W>((long long)segLen - i));
            const V vE_opn = v.template subs<W>(vH, vGapO);
            const V vE_ext = v.template subs<W>(vE, vGapE);
            V case1 = v.cmpgt(vE_opn, vE_ext);
            vE = v.max(vE_opn, vE_ext);
            vEM = v.blend(vEM, vHM, case1);
            vES = v.blend(vES, vHS, case1);
            vEL = v.template adds<W>(v.blend(vEL, vHL, case1), vOne);
            const V vGapper = v.template adds<W>(vHt, v.set1(gapper_at<W>(open, gap, segLen, i)));
            case1 = v.or_(v.cmpgt(vF, vGapper), v.cmpeq(vF, vGapper));
            vF = v.max(vF, vGapper);
            vFM = v.blend(vHtM, vFM, case1);
            vFS = v.blend(vHtS, vFS, case1);
            vFL = v.blend(v.template adds<W>(vHtL, vGapperL), vFL, case1);
            vHp = v.template adds<W>(vHp, v.template prof<W>(pr, k_t, i, segLen));
            vHpM = v.template adds<W>(vHpM, v.template match<W>(pr, k_t, i, segLen));
            vHpS = v.template adds<W>(vHpS, v.template similar<W>(pr, k_t, i, segLen));
            vHpL = v.template adds<W>(vHpL, vOne);
            case1 = v.cmpgt(vE, vHp);
            vHt = v.max(vE, vHp);
            vHtM = v.blend(vHpM, vEM, case1);
            vHtS = v.blend(vHpS, vES, case1);
            vHtL = v.blend(vHpL, vEL, case1);
            v.store(pe, i, vE); v.store(pem, i, vEM); v.store(pes, i, vES); v.store(pel, i, vEL);
            v.store(ph, i, vHp); v.store(phm, i, vHpM); v.store(phs, i, vHpS); v.store(phl, i, vHpL);
            vHp = vH; vHpM = vHM; vHpS = vHS; vHpL = vHL;
        }
        /* pseudo prefix scan on F and H */
        vHt = v.shift1(vHt); vHtM = v.shift1(vHtM); vHtS = v.shift1(vHtS); vHtL = v.shift1(vHtL);
        if (!SW) vHt = v.insert0(vHt, v.template boundary<W>(pr, j + 1));
        {
            const V vGapper = v.template adds<W>(vHt, v.set1(gapper_at<W>(open, gap, segLen, 0)));
            const V vGapperL = v.set1(lane_arith<W>((long long)segLen));
            const V case1 = v.or_(v.cmpgt(vGapper, vF), v.cmpeq(vGapper, vF));
            vF = v.max(vF, vGapper);
            vFM = v.blend(vFM, vHtM, case1);
            vFS = v.blend(vFS, vHtS, case1);
            vFL = v.blend(vFL, v.template adds<W>(vHtL, vGapperL), case1);
        }
        for (int k = 0; k < L - 2; ++k) {
            V vFt = v.shift1(vF);
            const V vFtM = v.shift1(vFM), vFtS = v.shift1(vFS), vFtL = v.shift1(vFL);
            vFt = v.template adds<W>(vFt, vSegLenXgap);
            const V case1 = v.or_(v.cmpgt(vFt, vF), v.cmpeq(vFt, vF));
            vF = v.max(vF, vFt);
            vFM = v.blend(vFM, vFtM, case1);
            vFS = v.blend(vFS, vFtS, case1);
            vFL = v.blend(vFL, v.template adds<W>(vFtL, vSegLen), case1);
        }
        /* final H */
        vF = v.shift1(vF); vFM = v.shift1(vFM); vFS = v.shift1(vFS); vFL = v.shift1(vFL);
        vF = v.template adds<W>(vF, vNegInfFront);
        V vH, vHM, vHS, vHL;
        {
            const V case1 = v.cmpgt(vF, vHt);
            vH = v.max(vF, vHt);
            vHM = v.blend(vHtM, vFM, case1);
            vHS = v.blend(vHtS, vFS, case1);
            vHL = v.blend(vHtL, vFL, case1);
        }
        for (int i = 0; i < segLen; ++i) {
            const V vHq = v.load(ph, i), vHqM = v.load(phm, i), vHqS = v.load(phs, i), vHqL = v.load(phl, i);
            const V vE = v.load(pe, i), vEM = v.load(pem, i), vES = v.load(pes, i), vEL = v.load(pel, i);
            const V vF_opn = v.template subs<W>(vH, vGapO);
            const V vF_ext = v.template subs<W>(vF, vGapE);
            vF = v.max(vF_opn, vF_ext);
            V case1 = v.cmpgt(vF_opn, vF_ext);
            vFM = v.blend(vFM, vHM, case1);
            vFS = v.blend(vFS, vHS, case1);
            vFL = v.template adds<W>(v.blend(vFL, vHL, case1), vOne);
            vH = v.max(v.max(vHq, vE), vF);
            if (SW) vH = v.max(vH, vZero);
            case1 = v.cmpeq(vH, vHq);
            const V case2 = v.cmpeq(vH, vF);
            vHM = v.blend(v.blend(vEM, vFM, case2), vHqM, case1);
            vHS = v.blend(v.blend(vES, vFS, case2), vHqS, case1);
            vHL = v.blend(v.blend(vEL, vFL, case2), vHqL, case1);
            if (SW) {
                const V case0 = v.cmpeq(vH, vZero);
                vHM = v.blend(vHM, vZero, case0);
                vHS = v.blend(vHS, vZero, case0);
                vHL = v.blend(vHL, vZero, case0);
            }
            v.store(ph, i, vH); v.store(phm, i, vHM); v.store(phs, i, vHS); v.store(phl, i, vHL);
            vSatMin = v.min(vSatMin, vH);
            vSatMax = v.max(vSatMax, vH);
            vSatMax = v.max(vSatMax, vHM);
            vSatMax = v.max(vSatMax, vHS);
            vSatMax = v.max(vSatMax, vHL);
            if (SW) {
                const V cond_max = v.cmpgt(vH, vMaxH);
                vMaxH = v.max(vH, vMaxH);
                vMaxM = v.blend(vMaxM, vHM, cond_max);
                vMaxS = v.blend(vMaxS, vHS, cond_max);
                vMaxL = v.blend(vMaxL, vHL, cond_max);
            }
        }
        if (SW) {
            if (v.any(v.cmpgt(vMaxH, vMaxHUnit))) {
                score = v.hmax(vMaxH);
                vMaxHUnit = v.set1(score);
                end_ref = j;
                for (int i = 0; i < segLen; ++i) {
                    v.store(px, i, v.load(ph, i)); v.store(pxm, i, v.load(phm, i));
                    v.store(pxs, i, v.load(phs, i)); v.store(pxl, i, v.load(phl, i));
                }
            }
        } else {
            const V vHo = v.load(ph, offset);
            const V cond_max = v.cmpgt(vHo, vMaxH);
            vMaxH = v.max(vMaxH, vHo);
            vMaxM = v.blend(vMaxM, v.load(phm, offset), cond_max);
            vMaxS = v.blend(vMaxS, v.load(phs, offset), cond_max);
            vMaxL = v.blend(vMaxL, v.load(phl, offset), cond_max);
            if (v.any(v.and_(vPosMask, cond_max))) end_ref = j;
        }
    }
    if (SW) {
        end_query = s1Len;
        for (int i = 0; i < segLen; ++i) {
            const V th = v.load(px, i), tm = v.load(pxm, i), ts = v.load(pxs, i), tl = v.load(pxl, i);
            for (int l = 0; l < L; ++l) {
                const int temp = i + l * segLen;
                if (v.extract(th, l) == score && temp < end_query) {
                    end_query = temp;
                    matches = v.extract(tm, l); similar = v.extract(ts, l); length = v.extract(tl, l);
                }
            }
        }
    } else {
        if (pr.s2_end) {
            end_query = s1Len - 1;
            score = v.extract(vMaxH, lastLane);
            matches = v.extract(vMaxM, lastLane);
            similar = v.extract(vMaxS, lastLane);
            length = v.extract(vMaxL, lastLane);
        }
        if (pr.s1_end) {
            for (int i = 0; i < segLen; ++i) {
                const V th = v.load(ph, i), tm = v.load(phm, i), ts = v.load(phs, i), tl = v.load(phl, i);
                for (int l = 0; l < L; ++l) {
                    const int temp = i + l * segLen;
                    if (temp >= s1Len) continue;
                    const int t = v.extract(th, l);
                    if (t > score) {
                        score = t; end_query = temp; end_ref = s2Len - 1;
                        matches = v.extract(tm, l); similar = v.extract(ts, l); length = v.extract(tl, l);
                    } else if (t == score && end_ref == s2Len - 1 && temp < end_query) {
                        end_query = temp;
                        matches = v.extract(tm, l); similar = v.extract(ts, l); length = v.extract(tl, l);
                    }
                }
            }
        }
        if (!pr.s1_end && !pr.s2_end) {
            score = v.extract(v.load(ph, offset), lastLane);
            matches = v.extract(v.load(phm, offset), lastLane);
            similar = v.extract(v.load(phs, offset), lastLane);
            length = v.extract(v.load(phl, offset), lastLane);
            end_ref = s2Len - 1;
            end_query = s1Len - 1;
        }
    }
    o.saturated = v.any(v.or_(v.cmpgt(vNegLimit, vSatMin), v.cmpgt(vSatMax, vPosLimit))) ? 1 : 0;
    if (o.saturated) { score = matches = similar = length = 0; end_query = end_ref = 0; }
    o.score = score; o.end_query = end_query; o.end_ref = end_ref;
    o.matches = matches; o.similar = similar; o.length = length;
}

}  // namespace lane
}  // namespace pb

#endif
