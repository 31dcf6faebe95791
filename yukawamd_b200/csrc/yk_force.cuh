// yk_force.cuh -- O(N^2) minimum-image pair-force kernels.
//
// Reference routines (one pass over all pairs per force call):
//   accel_ion_pure  int_ion_pure.f:98-254   screened Coulomb, one species
//   accel_ion_mix   int_ion_mix.f:105-295   screened Coulomb, Z_i Z_j weights
//   accel_nn        int_nn.f:130-345        HPP Gaussians + p-p screened Coulomb
//
// Kernel k_force_rows ("row" form): every thread owns one target particle i
// and keeps its position and its force / energy / virial / pressure-tensor
// sums in registers; the CTA streams the whole source array through shared
// memory in tiles of FTILE particles, each tile a single 1-D TMA bulk copy
// (double-buffered on two mbarriers).  Each pair is evaluated from both
// sides (N(N-1) evaluations), so no thread ever writes another particle's
// force: forces need no atomics and no scratch, and every per-particle sum
// runs in the fixed order j = 0..n-1.  The scalar sums (U, virial, P) are
// reduced per CTA into a partials array and finished by k_finalize.
//
// Physics per pair (d = x_i - x_j after minimum image, r = |d|):
//   ion:  u = e^{-mu r}/r - evcut,  f = (1 + mu r) e^{-mu r}/r^3   (x Z_j for
//         the mixture), F_i += f d, W += f r^2, P += d (f d)
//   nn:   nuclear (r^2 <= rncut^2): e = exp(-r^2/(2 Lambda)),
//         u = (aa e + B) e, f = (2 aa e + B) e / Lambda, B = bb +/- cc by
//         species equality; Coulomb (p-p, r^2 <= rccut^2): vc x the ion terms.
//
// PREC_FP64: all FP64 (exp(), rsqrt() from the CUDA math library).
// PREC_MIXED: displacement and minimum image in FP64, then cast to FP32;
// the r^2, rsqrt, exp and force terms in FP32; per-particle force sums in
// compensated FP32 (two-sum), folded to FP64 in the epilogue.
#pragma once

#include <type_traits>

#include "yk_common.cuh"

namespace yk {

constexpr int SIM_NUCLEON = 1, SIM_PURE = 2, SIM_MIX = 3;
constexpr int PREC_FP64 = 0, PREC_MIXED = 1;
constexpr int FBLOCK = 128;          // threads per CTA = target particles per CTA
constexpr int FTILE = 128;           // source particles per shared-memory tile
constexpr int NSCAL = 8;             // U, W, Pxx, Pxy, Pxz, Pyy, Pyz, Pzz

struct ForceArgs {
    double xl[3];
    long long hlb[3];                // bit patterns of xl/2
    double rc2, rn2;                 // rccut^2, rncut^2
    double xmuc, evcut, vc;          // evcut already includes vc for nucleons
    double xpi, xp2i;                // 1/Lambda, 1/(2 Lambda)
    double aa, aa2, bpc, bmc;        // aa, 2 aa, bb+cc, bb-cc
    double coef;                     // pure: frp zi^2 vc; mix: frp vc; nn: 1
    double xmass, ai_xmass;          // xmass; pure: ai*xmass
    float rc2f, rn2f, xmucf, evcutf, vcf, xpif, xp2if, aaf, aa2f, bpcf, bmcf;
    int n, nuclear_on, coulomb_on, mix_compat;
};

// ---- FP64 accumulators -------------------------------------------------
template <bool MEAS>
struct Acc64 {
    double f[3];
    double s[NSCAL];
    __device__ __forceinline__ Acc64()
    {
        f[0] = f[1] = f[2] = 0.0;
#pragma unroll
        for (int k = 0; k < NSCAL; ++k) s[k] = 0.0;
    }
    __device__ __forceinline__ void add(double fs, double dx, double dy, double dz,
                                        double u, double w)
    {
        const double fx = fs * dx, fy = fs * dy, fz = fs * dz;
        f[0] += fx;
        f[1] += fy;
        f[2] += fz;
        if constexpr (MEAS) {
            s[0] += u;
            s[1] += w;
            s[2] += dx * fx;
            s[3] += dx * fy;
            s[4] += dx * fz;
            s[5] += dy * fy;
            s[6] += dy * fz;
            s[7] += dz * fz;
        }
    }
};

// ---- compensated FP32 accumulators --------------------------------------
template <bool MEAS>
struct AccMixed {
    cf32 f[3];
    cf32 s[MEAS ? NSCAL : 1];
    __device__ __forceinline__ void add(float fs, float dx, float dy, float dz, float u, float w)
    {
        const float fx = fs * dx, fy = fs * dy, fz = fs * dz;
        f[0].add(fx);
        f[1].add(fy);
        f[2].add(fz);
        if constexpr (MEAS) {
            s[0].add(u);
            s[1].add(w);
            s[2].add(dx * fx);
            s[3].add(dx * fy);
            s[4].add(dx * fz);
            s[5].add(dy * fy);
            s[6].add(dy * fz);
            s[7].add(dz * fz);
        }
    }
};

// ---- one directed pair, FP64 --------------------------------------------
template <int SIM, bool MEAS>
__device__ __forceinline__ void pair_eval(const ForceArgs& fa, const double4& pi, const double4& pj,
                                          bool distinct, Acc64<MEAS>& acc)
{
    const double dx = min_image(__dsub_rn(pi.x, pj.x), fa.xl[0], fa.hlb[0]);
    const double dy = min_image(__dsub_rn(pi.y, pj.y), fa.xl[1], fa.hlb[1]);
    const double dz = min_image(__dsub_rn(pi.z, pj.z), fa.xl[2], fa.hlb[2]);
    const double r2 = dx * dx + dy * dy + dz * dz;
    if constexpr (SIM == SIM_PURE || SIM == SIM_MIX) {
        if (distinct && r2 <= fa.rc2) {
            const double rinv = rsqrt(r2);
            const double r = r2 * rinv;
            const double mr = fa.xmuc * r;
            const double er = exp(-mr) * rinv;               // e^{-mu r}/r
            double fs = (1.0 + mr) * er * (rinv * rinv);      // (1+mu r) e^{-mu r}/r^3
            double u = 0.0, w = 0.0;
            if (MEAS) {
                u = er - fa.evcut;
                w = fs * r2;
            }
            if constexpr (SIM == SIM_MIX) {
                fs *= pj.w;
                if constexpr (MEAS) {
                    u *= pj.w;
                    w *= pj.w;
                }
            }
            acc.add(fs, dx, dy, dz, u, w);
        }
    } else {
        if (!distinct) return;
        double fs = 0.0, u = 0.0, w = 0.0;
        bool hit = false;
        if (fa.nuclear_on && r2 <= fa.rn2) {
            const double e = exp(-(r2 * fa.xp2i));
            const double B = (pi.w == pj.w) ? fa.bpc : fa.bmc;
            const double fn = fa.xpi * (fa.aa2 * e + B) * e;
            fs = fn;
            if (MEAS) {
                u = (fa.aa * e + B) * e;
                w = fn * r2;
            }
            hit = true;
        }
        if (fa.coulomb_on && pi.w == 1.0 && pj.w == 1.0 && r2 <= fa.rc2) {
            const double rinv = rsqrt(r2);
            const double r = r2 * rinv;
            const double mr = fa.xmuc * r;
            const double er = fa.vc * exp(-mr) * rinv;        // vc e^{-mu r}/r
            const double fc = (1.0 + mr) * er * (rinv * rinv);
            fs += fc;
            if (MEAS) {
                u += er - fa.evcut;
                w += fc * r2;
            }
            hit = true;
        }
        if (hit) acc.add(fs, dx, dy, dz, u, w);
    }
}

// ---- one directed pair, mixed ------------------------------------------
template <int SIM, bool MEAS>
__device__ __forceinline__ void pair_eval(const ForceArgs& fa, const double4& pi, const double4& pj,
                                           bool distinct, AccMixed<MEAS>& acc)
{
    const float dx = __double2float_rn(min_image(__dsub_rn(pi.x, pj.x), fa.xl[0], fa.hlb[0]));
    const float dy = __double2float_rn(min_image(__dsub_rn(pi.y, pj.y), fa.xl[1], fa.hlb[1]));
    const float dz = __double2float_rn(min_image(__dsub_rn(pi.z, pj.z), fa.xl[2], fa.hlb[2]));
    const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    if constexpr (SIM == SIM_PURE || SIM == SIM_MIX) {
        if (distinct && r2 <= fa.rc2f) {
            const float rinv = rsqrt_f32(r2);
            const float r = r2 * rinv;
            const float mr = fa.xmucf * r;
            const float er = exp_neg_f32(mr) * rinv;
            float fs = (1.0f + mr) * er * (rinv * rinv);
            float u = 0.f, w = 0.f;
            if (MEAS) {
                u = er - fa.evcutf;
                w = fs * r2;
            }
            if constexpr (SIM == SIM_MIX) {
                const float zj = (float)pj.w;
                fs *= zj;
                if constexpr (MEAS) {
                    u *= zj;
                    w *= zj;
                }
            }
            acc.add(fs, dx, dy, dz, u, w);
        }
    } else {
        if (!distinct) return;
        float fs = 0.f, u = 0.f, w = 0.f;
        bool hit = false;
        if (fa.nuclear_on && r2 <= fa.rn2f) {
            const float e = exp_neg_f32(r2 * fa.xp2if);
            const float B = (pi.w == pj.w) ? fa.bpcf : fa.bmcf;
            const float fn = fa.xpif * fmaf(fa.aa2f, e, B) * e;
            fs = fn;
            if (MEAS) {
                u = fmaf(fa.aaf, e, B) * e;
                w = fn * r2;
            }
            hit = true;
        }
        if (fa.coulomb_on && pi.w == 1.0 && pj.w == 1.0 && r2 <= fa.rc2f) {
            const float rinv = rsqrt_f32(r2);
            const float r = r2 * rinv;
            const float mr = fa.xmucf * r;
            const float er = fa.vcf * exp_neg_f32(mr) * rinv;
            const float fc = (1.0f + mr) * er * (rinv * rinv);
            fs += fc;
            if (MEAS) {
                u += er - fa.evcutf;
                w += fc * r2;
            }
            hit = true;
        }
        if (hit) acc.add(fs, dx, dy, dz, u, w);
    }
}

// ---- epilogue: scale to accelerations (int_ion_pure.f:227-231,
// int_ion_mix.f:273-277 with the fold of :201, int_nn.f:318-322) ----------
template <int SIM>
__device__ __forceinline__ void store_accel(const ForceArgs& fa, int i, double wi, const double* aii,
                                            double F[3], double* a_out)
{
    if constexpr (SIM == SIM_PURE) {
#pragma unroll
        for (int k = 0; k < 3; ++k) a_out[3 * i + k] = fa.coef * F[k] / fa.ai_xmass;
    } else if constexpr (SIM == SIM_MIX) {
        // Reference fold fj(:,i) = zii(i)*(...) runs only for i <= n-2.
        const bool fold = !(fa.mix_compat && i == fa.n - 1);
        const double am = aii[i] * fa.xmass;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double f = fold ? wi * F[k] : F[k];
            a_out[3 * i + k] = fa.coef * f / am;
        }
    } else {
#pragma unroll
        for (int k = 0; k < 3; ++k) a_out[3 * i + k] = F[k] / fa.xmass;
    }
}

// Shared memory of k_force_rows: 2 stages of FTILE double4, 2 mbarriers,
// and the block-reduction scratch.
constexpr int FORCE_SMEM = 2 * FTILE * (int)sizeof(double4) + 16 + 32 * NSCAL * (int)sizeof(double);

template <int SIM, int PREC, bool MEAS>
__global__ void __launch_bounds__(FBLOCK)
k_force_rows(const double4* __restrict__ pos, const double* __restrict__ aii, ForceArgs fa,
             double* __restrict__ a_out, double* __restrict__ part, unsigned* __restrict__ err)
{
    extern __shared__ __align__(128) unsigned char smem[];
    double4* tile = reinterpret_cast<double4*>(smem);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 2 * FTILE * sizeof(double4));
    double* red = reinterpret_cast<double*>(smem + 2 * FTILE * sizeof(double4) + 16);
    __shared__ int s_abort;

    const int n = fa.n;
    const int i = blockIdx.x * FBLOCK + threadIdx.x;
    const bool active = i < n;
    const double4 pi = active ? pos[i] : make_double4(0.0, 0.0, 0.0, 0.0);
    const int ntiles = (n + FTILE - 1) / FTILE;

    if (threadIdx.x == 0) {
        s_abort = 0;
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    auto issue = [&](int t) {
        const int j0 = t * FTILE;
        const int cnt = min(FTILE, n - j0);
        const unsigned bytes = (unsigned)cnt * (unsigned)sizeof(double4);
        uint64_t* b = &bar[t & 1];
        mbar_arrive_expect_tx(b, bytes);
        bulk_g2s(tile + (t & 1) * FTILE, pos + j0, bytes, b);
    };
    if (threadIdx.x == 0) {
        issue(0);
        if (ntiles > 1) issue(1);
    }

    using Acc = std::conditional_t<PREC == PREC_FP64, Acc64<MEAS>, AccMixed<MEAS>>;
    Acc acc;

    for (int t = 0; t < ntiles; ++t) {
        const int st = t & 1;
        const bool ok = mbar_wait_bounded(&bar[st], (unsigned)((t >> 1) & 1), err);
        if (__syncthreads_or(!ok)) {
            // A copy never completed: wait (bounded) for the other stage's
            // copy, if one was issued, and leave without touching outputs.
            if (threadIdx.x == 0 && t + 1 < ntiles)
                mbar_wait_bounded(&bar[st ^ 1], (unsigned)(((t + 1) >> 1) & 1), err);
            return;
        }
        const int j0 = t * FTILE;
        const int cnt = min(FTILE, n - j0);
        const double4* tl = tile + st * FTILE;
        if (active) {
#pragma unroll 2
            for (int jj = 0; jj < cnt; ++jj)
                pair_eval<SIM, MEAS>(fa, pi, tl[jj], (j0 + jj) != i, acc);
        }
        __syncthreads();                      // every thread is done with stage st
        if (threadIdx.x == 0 && t + 2 < ntiles) issue(t + 2);
    }

    double F[3], S[NSCAL];
#pragma unroll
    for (int k = 0; k < NSCAL; ++k) S[k] = 0.0;
    if constexpr (PREC == PREC_FP64) {
#pragma unroll
        for (int k = 0; k < 3; ++k) F[k] = acc.f[k];
        if constexpr (MEAS) {
#pragma unroll
            for (int k = 0; k < NSCAL; ++k) S[k] = acc.s[k];
        }
    } else {
#pragma unroll
        for (int k = 0; k < 3; ++k) F[k] = acc.f[k].value();
        if constexpr (MEAS) {
#pragma unroll
            for (int k = 0; k < NSCAL; ++k) S[k] = acc.s[k].value();
        }
    }
    if (active) store_accel<SIM>(fa, i, pi.w, aii, F, a_out);
    if constexpr (MEAS) {
        if constexpr (SIM == SIM_MIX) {
#pragma unroll
            for (int k = 0; k < NSCAL; ++k) S[k] *= pi.w;    // ev += zii(i)*evx ...
        }
        if (!active) {
#pragma unroll
            for (int k = 0; k < NSCAL; ++k) S[k] = 0.0;
        }
        block_sum_store<NSCAL>(S, red, part + (size_t)blockIdx.x * NSCAL);
    }
}

}  // namespace yk
