// yk_gofr.cuh -- the pair-distance histogram of the two-particle correlation
// function g(r) (subroutine g, g.f:55-66; the reference has the routine but
// its calls are commented out, md.F:64, 154, 184).
//
// For every unique pair: rr = pdist(i, j) (gen_utils.f:115-128: per axis
// min(|d|, xl - |d|), the root of the sum of squares, plus the REAL*4 literal
// 1.e-15), and bin ii = min(nbin, int(fac2 rr + 1)), fac2 = 2.*float(nbin) /
// sqrt(3.) / xlmin.  Every operation is the reference's, correctly rounded and
// unfused, so each pair lands in the same bin as in the reference's loop; the
// counts are integers, exact in any order.
//
// Work: units (target tile R, source tile C >= R) of 128 x 128 slot pairs,
// spread over a fixed grid; each CTA keeps one histogram in shared memory over
// all its units (32-bit counters, at most 128 x 128 x units-per-CTA pairs,
// far below 2^32) and adds it to the 64-bit global histogram once at the end.
#pragma once

#include "yk_force.cuh"

namespace yk {

constexpr int GOFR_BLOCK = 128;
constexpr int GOFR_MAX_BINS = 8192;          // 32 KB of shared counters

struct GofrArgs {
    double xl[3];
    double fac2;                             // (double)(REAL*4 2*nbin/sqrt(3)) / xlmin
    double tiny;                             // (double)1.e-15f
    int nbin, n, M;                          // bins, particles, 128-slot tiles
};

static __global__ void __launch_bounds__(GOFR_BLOCK)
k_gofr(const double4* __restrict__ pos, GofrArgs g, unsigned long long* __restrict__ hist)
{
    extern __shared__ __align__(16) unsigned char gsm[];
    double4* tile = reinterpret_cast<double4*>(gsm);
    unsigned* h = reinterpret_cast<unsigned*>(gsm + GOFR_BLOCK * sizeof(double4));
    const int tid = threadIdx.x;
    for (int b = tid; b < g.nbin; b += GOFR_BLOCK) h[b] = 0u;
    const long long units = (long long)g.M * (g.M + 1) / 2;
    for (long long u = blockIdx.x; u < units; u += gridDim.x) {
        // u = C (C + 1) / 2 + R with 0 <= R <= C
        int C = (int)((sqrt(8.0 * (double)u + 1.0) - 1.0) * 0.5);
        while ((long long)(C + 1) * (C + 2) / 2 <= u) ++C;
        while ((long long)C * (C + 1) / 2 > u) --C;
        const int R = (int)(u - (long long)C * (C + 1) / 2);
        __syncthreads();                     // the previous unit's tile is no longer read
        const int j0 = C * GOFR_BLOCK;
        const int cnt = min(GOFR_BLOCK, g.n - j0);
        if (tid < cnt) tile[tid] = pos[j0 + tid];
        __syncthreads();
        const int i = R * GOFR_BLOCK + tid;
        if (i >= g.n) continue;
        const double4 pi = pos[i];
        const double ci[3] = {pi.x, pi.y, pi.z};
        const int jstart = (C == R) ? tid + 1 : 0;
        for (int jj = jstart; jj < cnt; ++jj) {
            const double4 pj = tile[jj];
            const double cj[3] = {pj.x, pj.y, pj.z};
            double rr = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                double yy = fabs(__dsub_rn(ci[k], cj[k]));
                yy = fmin(yy, __dsub_rn(g.xl[k], yy));
                rr = __dadd_rn(rr, __dmul_rn(yy, yy));
            }
            rr = __dadd_rn(__dsqrt_rn(rr), g.tiny);
            const int ii = min(g.nbin, __double2int_rz(__dadd_rn(__dmul_rn(g.fac2, rr), 1.0)));
            atomicAdd(&h[ii - 1], 1u);
        }
    }
    __syncthreads();
    for (int b = tid; b < g.nbin; b += GOFR_BLOCK)
        if (h[b]) atomicAdd(&hist[b], (unsigned long long)h[b]);
}

}  // namespace yk
