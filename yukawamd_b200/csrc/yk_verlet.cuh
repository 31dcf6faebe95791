// yk_verlet.cuh -- velocity-Verlet kernels and the scalar finish.
//
// Reference integrators (all O(N), HBM-bound):
//   vel_verlet_2.f:18-120  drift + wrap, vold = v, v += dt a, accel,
//                          B-field term, v = (v + vold + dt a)/2, ek and P
//   vel_verlet_1.f:16-89   drift + wrap, v += dt/2 a, accel, v += dt/2 a
//   vel_verlet_3.f:20-100  Spreiter-Walter magnetic Verlet
//
// Arrays keep the Fortran layout x(3,0:n-1).  The VV1/VV2 drifts take one
// thread per element (each warp access is 256 contiguous bytes); the kernels
// that mix a particle's components take one thread per particle and load all
// of its values before the first store.  Every element update uses
// explicitly rounded operations (__dadd_rn / __dmul_rn) so that nothing is
// contracted into an FMA: positions and velocities come out bit-identical to
// the reference's arithmetic (which is compiled without FMA) given the same
// accelerations.  After a drift, k_pack_slots gathers the FP64 positions with
// the per-particle weight (zii) into the slot-ordered double4 array and the
// FP32 shadow that the force kernels stream.
#pragma once

#include "yk_force.cuh"

namespace yk {

constexpr int VBLOCK = 256;
constexpr int NKIN = 6;             // vxx vxy vxz vyy vyz vzz

struct StepArgs {
    double xl[3];
    double dt, afac, halfdt;
    double bfield;
    double lorentz_c;               // 3.218404d-20 (VV2) or REAL*4 3.218404e-20 (VV3)
    int n;
    int pack_w;                     // 1: pos.w = zii; 0: pos.w = 0
};

__device__ __forceinline__ double wrap_once(double x, double L)
{
    // vel_verlet_2.f:39-40: if (x < 0) x += L; if (x > L) x -= L
    if (x < 0.0) x = __dadd_rn(x, L);
    if (x > L) x = __dsub_rn(x, L);
    return x;
}

// Slot `slot` of the FP64 positions and of their FP32 shadow (screening).
__device__ __forceinline__ void store_pos(double4* pos, float* posf, int slot, const double (&xn)[3],
                                          double w)
{
    pos[slot] = make_double4(xn[0], xn[1], xn[2], w);
    store_shadow(posf, slot, xn[0], xn[1], xn[2], (float)w);
}

// The slot-ordered FP64 positions and FP32 shadow after a drift, a thread
// per slot: the position is gathered through perm and each slot's words are
// written in slot order (a warp writes contiguous runs).  The drift kernels
// themselves only touch the caller-order arrays, all coalesced; writing the
// slot copies from them would scatter every 4-byte shadow word through the
// permutation, one 32-byte sector each.
static __global__ void k_pack_slots(const int* __restrict__ perm, const double* __restrict__ x,
                                    const double* __restrict__ zii, double4* __restrict__ pos,
                                    float* __restrict__ posf, int n, int pack_w)
{
    const int sl = blockIdx.x * blockDim.x + threadIdx.x;
    if (sl >= n) return;
    const int o = perm[sl];
    const double xn[3] = {x[3 * o], x[3 * o + 1], x[3 * o + 2]};
    store_pos(pos, posf, sl, xn, pack_w ? zii[o] : 0.0);
}

// x = x + v dt + afac a, wrapped once (vel_verlet_2.f:36-42)
__device__ __forceinline__ double drift1(double x, double v, double a, const StepArgs& s, int k)
{
    return wrap_once(__dadd_rn(__dadd_rn(x, __dmul_rn(v, s.dt)), __dmul_rn(s.afac, a)), s.xl[k]);
}

// VV2 first half: drift, vold = v, v += dt a; one thread per element
// (component e % 3 of particle e / 3).
static __global__ void k_drift_vv2(double* __restrict__ x, double* __restrict__ v, double* __restrict__ vold,
                            const double* __restrict__ a, StepArgs s)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 3 * s.n) return;
    const double xi = x[e], vi = v[e], ai = a[e];
    x[e] = drift1(xi, vi, ai, s, e % 3);
    vold[e] = vi;
    v[e] = __dadd_rn(vi, __dmul_rn(s.dt, ai));
}

// VV1 first half: drift, v += dt/2 a (vel_verlet_1.f:148-166); one thread
// per element.
static __global__ void k_drift_vv1(double* __restrict__ x, double* __restrict__ v,
                            const double* __restrict__ a, StepArgs s)
{
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= 3 * s.n) return;
    const double xi = x[e], vi = v[e], ai = a[e];
    x[e] = drift1(xi, vi, ai, s, e % 3);
    v[e] = __dadd_rn(vi, __dmul_rn(s.halfdt, ai));
}

// VV3 first half: drift and the first Spreiter-Walter stage
// (vel_verlet_3.f:255-262; v(2,i) reads the already updated v(1,i)).
static __global__ void k_drift_vv3(double* __restrict__ x, double* __restrict__ v,
                            const double* __restrict__ a, const double* __restrict__ zii,
                            const double* __restrict__ aii, StepArgs s)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= s.n) return;
    const double x1 = x[3 * i], x2 = x[3 * i + 1], x3 = x[3 * i + 2];
    const double a1 = a[3 * i], a2 = a[3 * i + 1], a3 = a[3 * i + 2];
    double v1 = v[3 * i], v2 = v[3 * i + 1], v3 = v[3 * i + 2];
    const double zi = zii[i], ai = aii[i];
    x[3 * i] = drift1(x1, v1, a1, s, 0);
    x[3 * i + 1] = drift1(x2, v2, a2, s, 1);
    x[3 * i + 2] = drift1(x3, v3, a3, s, 2);
    const double omega = __ddiv_rn(__dmul_rn(__dmul_rn(s.lorentz_c, zi), s.bfield), ai);
    const double w = __dmul_rn(s.halfdt, omega);
    const double w2 = __dmul_rn(w, w);
    v1 = __dadd_rn(__dadd_rn(__dmul_rn(__dsub_rn(1.0, w2), v1), __dmul_rn(__dmul_rn(2.0, w), v2)),
                   __dmul_rn(s.halfdt, __dadd_rn(a1, __dmul_rn(w, a2))));
    v2 = __dadd_rn(__dsub_rn(__dmul_rn(__dsub_rn(1.0, w2), v2), __dmul_rn(__dmul_rn(2.0, w), v1)),
                   __dmul_rn(s.halfdt, __dsub_rn(a2, __dmul_rn(w, a1))));
    v3 = __dadd_rn(v3, __dmul_rn(s.halfdt, a3));
    v[3 * i] = v1;
    v[3 * i + 1] = v2;
    v[3 * i + 2] = v3;
}

template <bool KIN>
__device__ __forceinline__ void kin_sums(double (&t)[NKIN], double am, double v1, double v2, double v3)
{
    if constexpr (KIN) {
        // vxx = vxx + aii(i)*v(1,i)*v(1,i) ... (vel_verlet_2.f:88-93)
        const double m1 = am * v1, m2 = am * v2;
        t[0] = m1 * v1;
        t[1] = m1 * v2;
        t[2] = m1 * v3;
        t[3] = m2 * v2;
        t[4] = m2 * v3;
        t[5] = __dmul_rn(am, v3) * v3;
    }
}

// VV2 second half: B-field term (vel_verlet_2.f:61-69), corrector average
// (:75-79), kinetic tensor partial sums when measuring (:84-95).
template <bool KIN, bool BFIELD>
__global__ void __launch_bounds__(VBLOCK)
k_post_vv2(double* __restrict__ v, const double* __restrict__ vold, double* __restrict__ a,
           const double* __restrict__ zii, const double* __restrict__ aii,
           double* __restrict__ kpart, StepArgs s)
{
    __shared__ double red[32 * NKIN];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double t[NKIN] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (i < s.n) {
        double vv[3], aa[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            vv[k] = v[3 * i + k];
            aa[k] = a[3 * i + k];
        }
        if constexpr (BFIELD) {
            const double omega = __ddiv_rn(__dmul_rn(__dmul_rn(s.lorentz_c, zii[i]), s.bfield), aii[i]);
            aa[0] = __dadd_rn(aa[0], __dmul_rn(vv[1], omega));
            aa[1] = __dsub_rn(aa[1], __dmul_rn(vv[0], omega));
            a[3 * i] = aa[0];
            a[3 * i + 1] = aa[1];
        }
        const double vo[3] = {vold[3 * i], vold[3 * i + 1], vold[3 * i + 2]};
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double vp = __dadd_rn(vo[k], __dmul_rn(s.dt, aa[k]));
            vv[k] = __dmul_rn(0.5, __dadd_rn(vv[k], vp));
            v[3 * i + k] = vv[k];
        }
        kin_sums<KIN>(t, aii[i], vv[0], vv[1], vv[2]);
    }
    if constexpr (KIN) block_sum_store<NKIN>(t, red, kpart + (size_t)blockIdx.x * NKIN);
}

// VV1 second half: v += dt/2 a; kinetic sums always (vel_verlet_1.f:177-188).
static __global__ void __launch_bounds__(VBLOCK)
k_post_vv1(double* __restrict__ v, const double* __restrict__ a, const double* __restrict__ aii,
           double* __restrict__ kpart, StepArgs s)
{
    __shared__ double red[32 * NKIN];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double t[NKIN] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (i < s.n) {
        double vv[3], aa[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            vv[k] = v[3 * i + k];
            aa[k] = a[3 * i + k];
        }
        const double am = aii[i];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            vv[k] = __dadd_rn(vv[k], __dmul_rn(s.halfdt, aa[k]));
            v[3 * i + k] = vv[k];
        }
        kin_sums<true>(t, am, vv[0], vv[1], vv[2]);
    }
    block_sum_store<NKIN>(t, red, kpart + (size_t)blockIdx.x * NKIN);
}

// VV3 second half: second Spreiter-Walter stage (vel_verlet_3.f:274-287).
static __global__ void __launch_bounds__(VBLOCK)
k_post_vv3(double* __restrict__ v, const double* __restrict__ a, const double* __restrict__ zii,
           const double* __restrict__ aii, double* __restrict__ kpart, StepArgs s)
{
    __shared__ double red[32 * NKIN];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double t[NKIN] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (i < s.n) {
        const double omega = __ddiv_rn(__dmul_rn(__dmul_rn(s.lorentz_c, zii[i]), s.bfield), aii[i]);
        const double w = __dmul_rn(s.halfdt, omega);
        const double den = __dadd_rn(1.0, __dmul_rn(w, w));
        const double a1 = a[3 * i], a2 = a[3 * i + 1], a3 = a[3 * i + 2];
        double v1 = v[3 * i], v2 = v[3 * i + 1], v3 = v[3 * i + 2];
        v1 = __ddiv_rn(__dadd_rn(v1, __dmul_rn(s.halfdt, __dadd_rn(a1, __dmul_rn(w, a2)))), den);
        v2 = __ddiv_rn(__dadd_rn(v2, __dmul_rn(s.halfdt, __dsub_rn(a2, __dmul_rn(w, a1)))), den);
        v3 = __dadd_rn(v3, __dmul_rn(s.halfdt, a3));
        v[3 * i] = v1;
        v[3 * i + 1] = v2;
        v[3 * i + 2] = v3;
        kin_sums<true>(t, aii[i], v1, v2, v3);
    }
    block_sum_store<NKIN>(t, red, kpart + (size_t)blockIdx.x * NKIN);
}

// Device copy of the md_globals scalars, kept between calls so that the
// B-field case can leave ev / px / pp untouched as the reference does.
struct DevScalars {
    double ev, vir, px, ek, pp[9];
};

struct FinishArgs {
    int n;
    int nfp;              // force partial rows (0 = none)
    int nkp;              // kinetic partial rows (0 = none)
    int force_mode;       // 0: keep previous ev/vir/px/pp (B-field); 1: from partials
    int do_meas;          // measurement force call
    int kin_mode;         // 0: accel only (ek, pp untouched); 1: ek=0, pp=0; 2: add kinetic
    double half;          // factor on the force partials (1/2: each pair counted twice)
    double coef;          // frp zi^2 vc / frp vc / 1
    double rho, kT, xmass, vol;
    double f_n, f_3n;     // float(n), 3.0*n as the reference's REAL*4
};

// Sums the per-CTA partials in a fixed order, writes the packed raw sums to
// a(:,n..n+2) (int_ion_pure.f:217-225) and the md_globals scalars
// (int_ion_pure.f:232-248, vel_verlet_2.f:96-110).  Called by one block of
// 256 threads; `series` (13 doubles) may be null.
__device__ __forceinline__ void finish_body(const double* __restrict__ fpart, const double* __restrict__ kpart,
                                            const FinishArgs& fz, double* __restrict__ a,
                                            DevScalars* __restrict__ ds, double* __restrict__ series)
{
    __shared__ double red[32 * 8];
    __shared__ double tot[8 + NKIN];
    double fs[8];
    double ks[NKIN];
#pragma unroll
    for (int k = 0; k < 8; ++k) fs[k] = 0.0;
#pragma unroll
    for (int k = 0; k < NKIN; ++k) ks[k] = 0.0;
    for (int b = threadIdx.x; b < fz.nfp; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < 8; ++k) fs[k] += fpart[(size_t)b * 8 + k];
    for (int b = threadIdx.x; b < fz.nkp; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < NKIN; ++k) ks[k] += kpart[(size_t)b * NKIN + k];
    block_sum_store<8>(fs, red, tot);
    __syncthreads();
    block_sum_store<NKIN>(ks, red, tot + 8);
    __syncthreads();
    if (threadIdx.x != 0) return;

    const int n = fz.n;
    DevScalars s = *ds;
    if (fz.force_mode == 1) {
        double raw[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) raw[k] = fz.do_meas ? fz.half * tot[k] : 0.0;
        // raw: U, W, Pxx, Pxy, Pxz, Pyy, Pyz, Pzz
        a[3 * n + 0] = raw[0];
        a[3 * n + 1] = raw[1];
        a[3 * n + 2] = 0.0;
        a[3 * n + 3] = raw[2];
        a[3 * n + 4] = raw[3];
        a[3 * n + 5] = raw[4];
        a[3 * n + 6] = raw[5];
        a[3 * n + 7] = raw[6];
        a[3 * n + 8] = raw[7];
        if (fz.do_meas) {
            s.ev = fz.coef * raw[0];
            s.vir = fz.coef * raw[1];
            s.pp[0] = fz.coef * raw[2];
            s.pp[3] = fz.coef * raw[3];
            s.pp[6] = fz.coef * raw[4];
            s.pp[4] = fz.coef * raw[5];
            s.pp[7] = fz.coef * raw[6];
            s.pp[8] = fz.coef * raw[7];
            s.pp[1] = s.pp[3];
            s.pp[2] = s.pp[6];
            s.pp[5] = s.pp[7];
            s.ev = s.ev / fz.f_n;
            s.px = fz.rho * (fz.kT + s.vir / fz.f_3n);
        } else {
            s.ev = s.vir = s.px = 0.0;
#pragma unroll
            for (int k = 0; k < 9; ++k) s.pp[k] = 0.0;
        }
    }
    if (fz.kin_mode == 1) {
        s.ek = 0.0;
#pragma unroll
        for (int k = 0; k < 9; ++k) s.pp[k] = 0.0;
    } else if (fz.kin_mode == 2) {
        const double* v = tot + 8;
        s.ek = (0.5 * fz.xmass) * (v[0] + v[3] + v[5]) / fz.f_n;
        s.pp[0] = s.pp[0] + fz.xmass * v[0];
        s.pp[3] = s.pp[3] + fz.xmass * v[1];
        s.pp[6] = s.pp[6] + fz.xmass * v[2];
        s.pp[4] = s.pp[4] + fz.xmass * v[3];
        s.pp[7] = s.pp[7] + fz.xmass * v[4];
        s.pp[8] = s.pp[8] + fz.xmass * v[5];
        s.pp[1] = s.pp[3];
        s.pp[2] = s.pp[6];
        s.pp[5] = s.pp[7];
#pragma unroll
        for (int k = 0; k < 9; ++k) s.pp[k] = s.pp[k] / fz.vol;
    }
    *ds = s;
    if (series) {
        series[0] = s.ev;
        series[1] = s.vir;
        series[2] = s.px;
        series[3] = s.ek;
#pragma unroll
        for (int k = 0; k < 9; ++k) series[4 + k] = s.pp[k];
    }
}

// Single box: one block of 256; the series slot is taken from *series_idx.
static __global__ void __launch_bounds__(256)
k_finish(const double* __restrict__ fpart, const double* __restrict__ kpart, FinishArgs fz,
         double* __restrict__ a, DevScalars* __restrict__ ds, double* __restrict__ series,
         int* __restrict__ series_idx)
{
    double* slot = nullptr;
    if (series) slot = series + (size_t)(*series_idx) * 13;
    finish_body(fpart, kpart, fz, a, ds, slot);
    if (series && threadIdx.x == 0) *series_idx += 1;
}

}  // namespace yk
