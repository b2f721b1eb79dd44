/*
 * pb_cert.cuh -- the exactness certificate of a banded global alignment, in
 * cost form (host and device).
 *
 * With a = the matrix's largest score, any global alignment of lengths n
 * (query) and m (target) has cost C = a(n+m)/2 - score, a sum of
 * non-negative terms: a - s per aligned pair, a/2 + ext per gap column and
 * open - ext per gap (open >= ext and a + 2 ext > 0 required). A path that
 * reaches diagonal hi+1 (i - j, above the band) needs at least
 * 2(hi+1) - d_end gap columns in at least two gaps, d_end = n - m, so its
 * cost is at least C_up = (2(hi+1) - d_end)(a/2 + ext) + 2(open - ext);
 * below the band, C_dn = (d_end - 2(lo-1))(a/2 + ext) + 2(open - ext). If a
 * banded optimum's cost is <= min(C_up, C_dn), no path leaving the band
 * scores more, so the banded score is the full optimum. label_band gives
 * the smallest band that passes this test for a cost C.
 */
#ifndef PARASAIL_B200_PB_CERT_CUH
#define PARASAIL_B200_PB_CERT_CUH

namespace pb {

struct CostModel { int a, open, ext; };

/* doubled minimum cost of any path leaving [lo, hi] */
__host__ __device__ inline long long exit_cost2(const CostModel &c, int n, int m, int lo, int hi)
{
    const long long dend = (long long)n - m;
    const long long unit2 = c.a + 2LL * c.ext;           /* 2 (a/2 + ext) */
    const long long up = (2LL * (hi + 1) - dend) * unit2 + 4LL * (c.open - c.ext);
    const long long dn = (dend - 2LL * (lo - 1)) * unit2 + 4LL * (c.open - c.ext);
    return up < dn ? up : dn;
}

__host__ __device__ inline long long floor_div(long long x, long long d)
{
    long long q = x / d;
    if ((x % d != 0) && ((x < 0) != (d < 0))) --q;
    return q;
}

/* smallest band whose exit cost covers the doubled optimal cost c2 */
__host__ __device__ inline void label_band(const CostModel &c, int n, int m, long long c2, int *lo, int *hi)
{
    const long long dend = (long long)n - m;
    const long long unit2 = c.a + 2LL * c.ext;
    const long long need = c2 - 4LL * (c.open - c.ext);
    /* g = fewest gap columns an exit must have: (2(hi+1) - dend) >= g */
    const long long g = need <= 0 ? 0 : -floor_div(-need, unit2);
    long long h = -floor_div(-(g + dend), 2) - 1;       /* ceil((g + dend)/2) - 1 */
    long long l = floor_div(dend + 2 - g, 2);           /* (dend - 2(lo-1)) >= g */
    const long long lmin = dend < 0 ? dend : 0, hmax = dend > 0 ? dend : 0;
    if (h < hmax) h = hmax;
    if (l > lmin) l = lmin;
    *lo = (int)(l < -(long long)m - 1 ? -(long long)m - 1 : l);
    *hi = (int)(h > (long long)n + 1 ? (long long)n + 1 : h);
}

/* doubled cost of a global alignment score */
__host__ __device__ inline long long cost2_of(const CostModel &c, int n, int m, int score)
{
    return (long long)c.a * (n + m) - 2LL * score;
}

/* the certificate's preconditions on the scoring */
__host__ __device__ inline bool cert_valid(const CostModel &c)
{
    return c.open >= c.ext && c.a + 2 * c.ext > 0;
}

}  // namespace pb

#endif
