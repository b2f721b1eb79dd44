/*
 * Host build of the lane-exact striped emulation (parasail_b200/csrc/
 * pb_lane.cuh) for the CPU tests: the same templates, with a vector policy
 * that loops over the AVX2 lanes instead of mapping them to a warp. Test
 * infrastructure only; the library runs the device policy.
 */
#include <stdint.h>
#include <string.h>
#include <vector>

#include "pb_lane.cuh"

namespace {

using namespace pb::lane;

template <int W> struct HostVec {
    static constexpr int L = Lim<W>::LANES;
    struct V { int v[32]; };
    typedef V *Arr;
    std::vector<V> mem[16];

    Arr arr(int a, int segLen) { mem[a].assign(segLen, V()); return mem[a].data(); }
    V load(Arr a, int i) { return a[i]; }
    void store(Arr a, int i, const V &x) { a[i] = x; }
    V set1(int x) { V r; for (int l = 0; l < 32; ++l) r.v[l] = x; return r; }
    template <int W2> V adds(const V &a, const V &b) { V r; for (int l = 0; l < 32; ++l) r.v[l] = lane_arith<W2>((long long)a.v[l] + b.v[l]); return r; }
    template <int W2> V subs(const V &a, const V &b) { V r; for (int l = 0; l < 32; ++l) r.v[l] = lane_arith<W2>((long long)a.v[l] - b.v[l]); return r; }
    V max(const V &a, const V &b) { V r; for (int l = 0; l < 32; ++l) r.v[l] = a.v[l] > b.v[l] ? a.v[l] : b.v[l]; return r; }
    V min(const V &a, const V &b) { V r; for (int l = 0; l < 32; ++l) r.v[l] = a.v[l] < b.v[l] ? a.v[l] : b.v[l]; return r; }
    V cmpgt(const V &a, const V &b) { V r; for (int l = 0; l < 32; ++l) r.v[l] = a.v[l] > b.v[l] ? -1 : 0; return r; }
    V cmpeq(const V &a, const V &b) { V r; for (int l = 0; l < 32; ++l) r.v[l] = a.v[l] == b.v[l] ? -1 : 0; return r; }
    V blend(const V &a, const V &b, const V &m) { V r; for (int l = 0; l < 32; ++l) r.v[l] = m.v[l] ? b.v[l] : a.v[l]; return r; }
    V and_(const V &a, const V &b) { V r; for (int l = 0; l < 32; ++l) r.v[l] = a.v[l] & b.v[l]; return r; }
    V or_(const V &a, const V &b) { V r; for (int l = 0; l < 32; ++l) r.v[l] = a.v[l] | b.v[l]; return r; }
    V andnot(const V &a, const V &b) { V r; for (int l = 0; l < 32; ++l) r.v[l] = ~a.v[l] & b.v[l]; return r; }
    V shift1(const V &a) { V r = a; for (int l = L - 1; l >= 1; --l) r.v[l] = a.v[l - 1]; r.v[0] = 0; return r; }
    V insert0(const V &a, int x) { V r = a; r.v[0] = x; return r; }
    bool any(const V &m) { for (int l = 0; l < L; ++l) if (m.v[l]) return true; return false; }
    int extract(const V &a, int l) { return a.v[l]; }
    int hmax(const V &a) { int m = a.v[0]; for (int l = 1; l < L; ++l) m = a.v[l] > m ? a.v[l] : m; return m; }
    V lane_eq(int k) { V r; for (int l = 0; l < 32; ++l) r.v[l] = l == k ? -1 : 0; return r; }
    template <int W2> void init_he(V &h, V &e, int i, int segLen, int s1_beg, int open, int gap)
    {
        for (int l = 0; l < 32; ++l) {
            long long tmp = s1_beg ? 0 : (-(long long)open - (long long)gap * (l * segLen + i));
            h.v[l] = tmp < Lim<W2>::MIN ? Lim<W2>::MIN : (int)tmp;
            tmp = tmp - open;
            e.v[l] = tmp < Lim<W2>::MIN ? Lim<W2>::MIN : (int)tmp;
        }
    }
    template <int W2> int boundary(const Problem &pr, int j)
    {
        if (j == 0) return 0;
        long long tmp = pr.s2_beg ? 0 : (-(long long)pr.open - (long long)pr.gap * (j - 1));
        return tmp < Lim<W2>::MIN ? Lim<W2>::MIN : (int)tmp;
    }
    template <int W2> V prof(const Problem &pr, int k, int i, int segLen)
    {
        V r;
        for (int l = 0; l < 32; ++l) {
            const int row = l * segLen + i;
            r.v[l] = (l < L && row < pr.qlen) ? wrap<W2>(prof_value(pr, k, row)) : 0;
        }
        return r;
    }
    template <int W2> V match(const Problem &pr, int k, int i, int segLen)
    {
        V r;
        for (int l = 0; l < 32; ++l) {
            const int row = l * segLen + i;
            r.v[l] = (l < L && row < pr.qlen) ? (k == pr.qcodes[row]) : 0;
        }
        return r;
    }
    template <int W2> V similar(const Problem &pr, int k, int i, int segLen)
    {
        V r = prof<W2>(pr, k, i, segLen);
        for (int l = 0; l < 32; ++l) r.v[l] = r.v[l] > 0;
        return r;
    }
};

template <int W> void run(int kind, const Problem &pr, Out &o)
{
    HostVec<W> v;
    if (kind == 0) striped_nwsg<HostVec<W>, W>(v, pr, o);
    else if (kind == 1) striped_nwsg_stats<HostVec<W>, W>(v, pr, o);
    else if (kind == 2) striped_sw_stats_bias<HostVec<W>, W>(v, pr, o);
    else if (kind == 3) striped_sw<HostVec<W>, W>(v, pr, o);
    else if (kind == 4) striped_nwsg<HostVec<W>, W, true>(v, pr, o);
    else if (kind == 5) scan_nwsg_trace<HostVec<W>, W>(v, pr, o);
    else if (kind == 6) scan_nwsg<HostVec<W>, W>(v, pr, o);
    else if (kind == 7) scan_sw<HostVec<W>, W>(v, pr, o);
    else if (kind == 8) scan_stats<HostVec<W>, W, false>(v, pr, o);
    else scan_stats<HostVec<W>, W, true>(v, pr, o);
}

}  // namespace

/* kind: 0 nw/sg score-only, 1 nw/sg statistics, 2 sw statistics (biased),
 * 3 sw score-only, 4 nw/sg striped trace, 5 nw/sg scan trace (flag only),
 * 6 nw/sg scan score-only, 7 sw scan score-only, 8 nw/sg scan statistics,
 * 9 sw scan statistics;
 * sg = {s1_beg, s1_end, s2_beg, s2_end}; out = {score, end_query, end_ref,
 * matches, similar, length, saturated} */
extern "C" int lane_host_run(int kind, int bits, const int32_t *prof, int size, int lp, const uint8_t *qcodes, int qlen,
                             const uint8_t *t, int tlen, int open, int gap, int mmax, int mmin, const int *sg,
                             int *out)
{
    Problem pr;
    pr.qlen = qlen; pr.tlen = tlen; pr.open = open; pr.gap = gap; pr.mmax = mmax; pr.mmin = mmin;
    pr.s1_beg = sg[0]; pr.s1_end = sg[1]; pr.s2_beg = sg[2]; pr.s2_end = sg[3];
    pr.prof = prof; pr.qcodes = qcodes; pr.lp = lp; pr.t = t;
    pr.mat = nullptr; pr.msize = 0; pr.size = size;
    Out o;
    if (bits == 8) run<8>(kind, pr, o);
    else if (bits == 16) run<16>(kind, pr, o);
    else if (bits == 32 && kind != 2 && kind != 5) run<32>(kind, pr, o);
    else return -1;
    out[0] = o.score; out[1] = o.end_query; out[2] = o.end_ref;
    out[3] = o.matches; out[4] = o.similar; out[5] = o.length; out[6] = o.saturated;
    return 0;
}
