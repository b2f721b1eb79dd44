/*
 * pb_exact.cu -- exact 32-bit alignment kernel (any mode, optional stats).
 *
 * One thread aligns one pair. The query rows are processed in strips of R
 * rows held in registers; the thread sweeps the whole target for each strip
 * and hands the strip's bottom row (H, F and their statistics) to the next
 * strip through a per-pair buffer in global memory.
 *
 * Semantics follow the reference's serial dynamic programs exactly
 * (jeffdaily/parasail v2.6.2 src/sw.c:131-158, src/nw.c:131-156,
 * src/sg.c:142-242 and the _stats twins src/sw_stats.c:183-262,
 * src/nw_stats.c:165-228, src/sg_stats.c), which the reference's striped and
 * scan kernels reproduce for every non-saturated result. The kernel also
 * records the statistics that the reference's vector kernels use to decide
 * saturation: extreme values over the real query rows and over the padded
 * rows of the 8-, 16- and 32-lane layouts.
 */
#include "pb_exact_core.cuh"

namespace pb {

template <int ALG, bool STATS, int R, bool SCANF>
__global__ void __launch_bounds__(128)
k_exact(ExactParams p)
{
    const int pid = blockIdx.x * blockDim.x + threadIdx.x;
    if (pid >= p.npairs) return;
    exact_pair<ALG, STATS, R, SCANF>(p, pid);
}

template <int ALG, bool STATS, bool SCANF = false>
static void launch_alg(const ExactParams &p, cudaStream_t st)
{
    /* score-only: 32-row strips (34 vs 29 GCUPS for NW against 16 rows,
     * 128 registers); statistics: 8 (the row loop stays rolled there) */
    constexpr int R = STATS ? 8 : 32;
    const int threads = 128;
    const int blocks = (p.npairs + threads - 1) / threads;
    k_exact<ALG, STATS, R, SCANF><<<blocks, threads, 0, st>>>(p);
}

void launch_exact(const ExactParams &p, int alg, bool stats, cudaStream_t st)
{
    if (p.npairs <= 0) return;
    if (p.scan_vgap) {
        /* the serial scan forms' vertical gap */
        if (stats) {
            if (alg == PB_SW) launch_alg<PB_SW, true, true>(p, st);
            else if (alg == PB_NW) launch_alg<PB_NW, true, true>(p, st);
            else launch_alg<PB_SG, true, true>(p, st);
        } else {
            if (alg == PB_SW) launch_alg<PB_SW, false, true>(p, st);
            else if (alg == PB_NW) launch_alg<PB_NW, false, true>(p, st);
            else launch_alg<PB_SG, false, true>(p, st);
        }
        return;
    }
    if (alg == PB_SW) { if (stats) launch_alg<PB_SW, true>(p, st); else launch_alg<PB_SW, false>(p, st); }
    else if (alg == PB_NW) { if (stats) launch_alg<PB_NW, true>(p, st); else launch_alg<PB_NW, false>(p, st); }
    else { if (stats) launch_alg<PB_SG, true>(p, st); else launch_alg<PB_SG, false>(p, st); }
}

}  // namespace pb
