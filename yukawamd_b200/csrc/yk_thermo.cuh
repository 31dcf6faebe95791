// yk_thermo.cuh -- the per-step O(N) host passes of the reference driver,
// on the device (gen_utils.f:40-110, strain.f:73-79).
//
//   ttot         eka = (0.5 xmass sum_i aii |v_i|^2) / float(n)
//   tnorm        v = v / sqrt(eka / (1.5 kT))
//   cancel_vcom  v = v - (sum aii v)/(sum aii), then tnorm
//   strain       x = x - xl(k) where x > xl(k) (after the host updates xl)
//
// Sums are per-block partials reduced by one block in a fixed order, so the
// results are reproducible; the scale and shift are computed on the device
// from those sums, with the reference's formulas and operation order, so
// none of these steps needs the host.
#pragma once

#include "yk_common.cuh"

namespace yk {

constexpr int TBLOCK = 256;
constexpr int NVSUM = 5;      // sum aii, sum aii v (3), sum aii |v|^2

static __global__ void __launch_bounds__(TBLOCK)
k_vsums(const double* __restrict__ v, const double* __restrict__ aii, int n, double* __restrict__ part)
{
    __shared__ double red[32 * NVSUM];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double t[NVSUM] = {0.0, 0.0, 0.0, 0.0, 0.0};
    if (i < n) {
        const double m = aii[i];
        const double v1 = v[3 * i], v2 = v[3 * i + 1], v3 = v[3 * i + 2];
        t[0] = m;
        t[1] = m * v1;
        t[2] = m * v2;
        t[3] = m * v3;
        // ekx = ekx + aii(i)*(v(1,i)**2+v(2,i)**2+v(3,i)**2)   (gen_utils.f:49)
        t[4] = m * __dadd_rn(__dadd_rn(__dmul_rn(v1, v1), __dmul_rn(v2, v2)), __dmul_rn(v3, v3));
    }
    block_sum_store<NVSUM>(t, red, part + (size_t)blockIdx.x * NVSUM);
}

static __global__ void __launch_bounds__(TBLOCK)
k_vreduce(const double* __restrict__ part, int nb, double* __restrict__ sums)
{
    __shared__ double red[32 * NVSUM];
    double t[NVSUM] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < NVSUM; ++k) t[k] += part[(size_t)b * NVSUM + k];
    block_sum_store<NVSUM>(t, red, sums);
}

// v = v - vcom, vcom = ptot / mtot (gen_utils.f:102-106)
static __global__ void k_vshift(double* __restrict__ v, int n, const double* __restrict__ sums)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 3 * n) return;
    const double vcom = __ddiv_rn(sums[1 + e % 3], sums[0]);
    v[e] = __dsub_rn(v[e], vcom);
}

// v = v / fac, fac = sqrt(eka / (1.5 kT)), eka = (0.5 xmass ekx) / float(n)
// (gen_utils.f:52, 69-73)
static __global__ void k_vscale(double* __restrict__ v, int n, const double* __restrict__ sums, double xmass,
                                double f_n, double kT)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 3 * n) return;
    const double eka = __ddiv_rn(__dmul_rn(__dmul_rn(0.5, xmass), sums[4]), f_n);
    const double fac = __dsqrt_rn(__ddiv_rn(eka, __dmul_rn(1.5, kT)));
    v[e] = __ddiv_rn(v[e], fac);
}

// strain.f:73-79: wrap coordinates pushed outside the (shrunk) box
static __global__ void k_strain_wrap(double* __restrict__ x, int n, double l0, double l1, double l2)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 3 * n) return;
    const int k = e % 3;
    const double L = k == 0 ? l0 : (k == 1 ? l1 : l2);
    if (x[e] > L) x[e] = __dsub_rn(x[e], L);
}

}  // namespace yk
