/*
 * esa_pairs.cpp -- TEST INFRASTRUCTURE (the oracle of the candidate-pair
 * filter): the reference aligner's enhanced-suffix-array filter restated
 * on the CPU, with the suffix and LCP arrays built by the reference's own
 * contrib/sais-lite-lcp/sais.c (compiled from where it lies by
 * oracle/Makefile into oracle/_ref/libesa_ref.so).
 *
 * Follows apps/parasail_aligner.cpp of jeffdaily/parasail v2.6.2:
 *   - sequence ids, begin/end and database flags of the '$'-separated text
 *     (:1206-1268);
 *   - SA + LCP by sais, a naive BWT, the LCP clamp at each suffix's
 *     sentinel (:1316-1345);
 *   - which end of the SA the sentinels sort to (:1353-1368);
 *   - the bottom-up traversal of the lcp-interval tree (Abouelhoda et al.)
 *     with a stack of (lcp, lb, rb, children) intervals (:1371-1410);
 *   - process(): intervals of lcp >= cutoff pair the suffixes of different
 *     child intervals (:1865-1904);
 *   - pair_check(): a left-maximal pair (different preceding characters, or
 *     a sentinel) of suffixes of different sequences (and, with a query
 *     file, of one database and one query sequence) adds the pair
 *     (smaller, larger) or (query, database) to a set (:1816-1853).
 * The result is the set in ascending order, as the aligner iterates it.
 * Nothing in the product links or loads this file.
 */
#include <algorithm>
#include <climits>
#include <cstdint>
#include <cstdlib>
#include <stack>
#include <vector>

extern "C" int sais(const unsigned char *T, int *SA, int *LCP, int n);

namespace {

struct Interval {
    int lcp, lb, rb;
    std::vector<Interval> children;
    Interval() : lcp(0), lb(0), rb(INT_MAX) {}
    Interval(int l, int b, int r) : lcp(l), lb(b), rb(r) {}
    bool empty() const { return rb == INT_MAX; }
};

struct Ctx {
    const int *SA, *SID;
    const unsigned char *BWT;
    const std::vector<int> *DB;
    unsigned char sentinel;
    int cutoff;
    std::vector<uint64_t> pairs;
};

void check_pair(Ctx &c, int i, int j)
{
    const int si = c.SID[c.SA[i]], sj = c.SID[c.SA[j]];
    if (!(c.BWT[i] != c.BWT[j] || c.BWT[i] == c.sentinel)) return;
    if (si == sj) return;
    int a, b;
    if (c.DB->empty()) {
        a = si < sj ? si : sj;
        b = si < sj ? sj : si;
    } else {
        if ((*c.DB)[si] == (*c.DB)[sj]) return;
        a = si > sj ? si : sj;
        b = si > sj ? sj : si;
    }
    c.pairs.push_back(((uint64_t)(uint32_t)a << 32) | (uint32_t)b);
}

void process(Ctx &c, const Interval &q)
{
    if (q.lcp < c.cutoff) return;
    const size_t nch = q.children.size();
    size_t ci = 0;
    if (nch) {
        for (int i = q.lb; i <= q.rb; ++i) {
            int j = i + 1;
            if (ci < nch && i >= q.children[ci].lb) {
                j = q.children[ci].rb + 1;
                if (i >= q.children[ci].rb) ++ci;
            }
            for (; j <= q.rb; ++j) check_pair(c, i, j);
        }
    } else {
        for (int i = q.lb; i <= q.rb; ++i)
            for (int j = i + 1; j <= q.rb; ++j) check_pair(c, i, j);
    }
}

}  // namespace

/*
 * T[0..n): the text the aligner builds (sequences each followed by the
 * sentinel). db_chars: the number of leading text characters that belong to
 * the database file, or -1 without a query file. Writes up to `cap` pairs
 * as (first, second) int pairs into out and returns the number of distinct
 * pairs, or -1 on an error.
 */
extern "C" long esa_pairs(const unsigned char *T, int n, unsigned char sentinel, int cutoff, long db_chars,
                          int *out, long cap)
{
    if (n <= 0) return 0;
    std::vector<int> SID(n), SA(n + 1), LCP(n + 1);
    std::vector<long> BEG, END;
    std::vector<int> DB;
    std::vector<unsigned char> BWT(n + 1);
    int sid = 0;
    BEG.push_back(0);
    for (int i = 0; i < n; ++i) {
        SID[i] = sid;
        if (T[i] == sentinel) {
            END.push_back(i);
            BEG.push_back(i + 1);
            DB.push_back(i < db_chars);
            ++sid;
        }
    }
    if (db_chars < 0) DB.clear();
    if (sid == 0) return -1;
    if (sais(T, SA.data(), LCP.data(), n) != 0) return -1;
    for (int i = 0; i < n; ++i) BWT[i] = SA[i] > 0 ? T[SA[i] - 1] : sentinel;
    for (int i = 0; i < n; ++i) {
        const int len = (int)(END[SID[SA[i]]] - SA[i]);
        if (LCP[i] > len) LCP[i] = len;
    }
    int bup_start, bup_stop;
    if (T[SA[0]] == sentinel) {
        bup_start = sid + 1;
        bup_stop = n;
    } else if (T[SA[n - 1]] == sentinel) {
        bup_start = 1;
        bup_stop = n - sid;
    } else {
        return -1;
    }
    Ctx c;
    c.SA = SA.data();
    c.SID = SID.data();
    c.BWT = BWT.data();
    c.DB = &DB;
    c.sentinel = sentinel;
    c.cutoff = cutoff;
    LCP[n] = 0;
    std::stack<Interval> st;
    Interval last;
    st.push(Interval());
    for (int i = bup_start; i <= bup_stop; ++i) {
        int lb = i - 1;
        while (LCP[i] < st.top().lcp) {
            st.top().rb = i - 1;
            last = st.top();
            st.pop();
            process(c, last);
            lb = last.lb;
            if (LCP[i] <= st.top().lcp) {
                last.children.clear();
                st.top().children.push_back(last);
                last = Interval();
            }
        }
        if (LCP[i] > st.top().lcp) {
            if (!last.empty()) {
                last.children.clear();
                Interval q(LCP[i], lb, INT_MAX);
                q.children.push_back(last);
                st.push(q);
                last = Interval();
            } else {
                st.push(Interval(LCP[i], lb, INT_MAX));
            }
        }
    }
    st.top().rb = bup_stop - 1;
    process(c, st.top());
    std::sort(c.pairs.begin(), c.pairs.end());
    c.pairs.erase(std::unique(c.pairs.begin(), c.pairs.end()), c.pairs.end());
    const long np = (long)c.pairs.size();
    for (long k = 0; k < np && k < cap; ++k) {
        out[2 * k] = (int)(c.pairs[k] >> 32);
        out[2 * k + 1] = (int)(uint32_t)c.pairs[k];
    }
    return np;
}
