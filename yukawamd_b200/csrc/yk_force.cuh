// yk_force.cuh -- pair physics and the "row" force kernel.
//
// Reference routines (one pass over all pairs per force call):
//   accel_ion_pure  int_ion_pure.f:98-254   screened Coulomb, one species
//   accel_ion_mix   int_ion_mix.f:105-295   screened Coulomb, Z_i Z_j weights
//   accel_nn        int_nn.f:130-345        HPP Gaussians + p-p screened Coulomb
//
// Physics per pair (d = x_i - x_j after minimum image, r = |d|); the pair
// functions return the scalar fs with F_i += fs d, plus u and w = fs r^2 for
// measurements:
//   ion:  u = e^{-mu r}/r - evcut,  fs = (1 + mu r) e^{-mu r}/r^3
//         (the mixture's Z_j / Z_i weights are applied by the caller, exactly
//         where int_ion_mix.f:179-180 applies them)
//   nn:   nuclear (r^2 <= rncut^2): e = exp(-r^2/(2 Lambda)),
//         u = (aa e + B) e, fs = (2 aa e + B) e / Lambda, B = bb +/- cc by
//         species equality; Coulomb (p-p, r^2 <= rccut^2): vc x the ion terms.
//
// PREC_FP64: all FP64 (exp(), rsqrt() from the CUDA math library; rsqrt
// replaces the reference's sqrt and divide, 1/(r r^2) = rinv^3).
// PREC_MIXED: displacement and minimum image in FP64, then cast to FP32; the
// r^2, rsqrt, exp and force terms in FP32.
//
// Particles are addressed by "slot": the engine keeps them in a Morton
// (space-filling-curve) order so that the 32 targets of a warp are close in
// space and mostly leave or enter the cutoff sphere together.  perm[slot] is
// the caller's particle index; outputs are scattered back through it.
//
// Kernel k_force_rows: every thread owns one target slot and sums over all
// N-1 sources (each pair evaluated from both sides, no scratch).  The
// default engine kernel is k_force_pairs in yk_pairs.cuh.
#pragma once

#include <type_traits>

#include "yk_common.cuh"

namespace yk {

constexpr int SIM_NUCLEON = 1, SIM_PURE = 2, SIM_MIX = 3;
constexpr int PREC_FP64 = 0, PREC_MIXED = 1;
constexpr int FBLOCK = 128;          // threads per CTA of the row kernel
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

template <typename R>
struct PairOut {
    R fs, u, w;
    R dx, dy, dz;
    bool hit;
};

// ---- one pair, FP64 -------------------------------------------------------
template <int SIM, bool MEAS>
__device__ __forceinline__ void pair64(const ForceArgs& fa, const double4& pi, const double4& pj,
                                       bool valid, PairOut<double>& o)
{
    o.dx = min_image(__dsub_rn(pi.x, pj.x), fa.xl[0], fa.hlb[0]);
    o.dy = min_image(__dsub_rn(pi.y, pj.y), fa.xl[1], fa.hlb[1]);
    o.dz = min_image(__dsub_rn(pi.z, pj.z), fa.xl[2], fa.hlb[2]);
    const double r2 = o.dx * o.dx + o.dy * o.dy + o.dz * o.dz;
    o.fs = 0.0;
    o.u = 0.0;
    o.w = 0.0;
    o.hit = false;
    if constexpr (SIM == SIM_PURE || SIM == SIM_MIX) {
        if (valid && r2 <= fa.rc2) {
            const double rinv = rsqrt(r2);
            const double r = r2 * rinv;
            const double mr = fa.xmuc * r;
            const double er = exp(-mr) * rinv;                // e^{-mu r}/r
            o.fs = (1.0 + mr) * er * (rinv * rinv);           // (1+mu r) e^{-mu r}/r^3
            if constexpr (MEAS) {
                o.u = er - fa.evcut;
                o.w = o.fs * r2;
            }
            o.hit = true;
        }
    } else {
        if (!valid) return;
        if (fa.nuclear_on && r2 <= fa.rn2) {
            const double e = exp(-(r2 * fa.xp2i));
            const double B = (pi.w == pj.w) ? fa.bpc : fa.bmc;
            const double fn = fa.xpi * (fa.aa2 * e + B) * e;
            o.fs = fn;
            if constexpr (MEAS) {
                o.u = (fa.aa * e + B) * e;
                o.w = fn * r2;
            }
            o.hit = true;
        }
        if (fa.coulomb_on && pi.w == 1.0 && pj.w == 1.0 && r2 <= fa.rc2) {
            const double rinv = rsqrt(r2);
            const double r = r2 * rinv;
            const double mr = fa.xmuc * r;
            const double er = fa.vc * exp(-mr) * rinv;         // vc e^{-mu r}/r
            const double fc = (1.0 + mr) * er * (rinv * rinv);
            o.fs += fc;
            if constexpr (MEAS) {
                o.u += er - fa.evcut;
                o.w += fc * r2;
            }
            o.hit = true;
        }
    }
}

// ---- one pair, mixed ---------------------------------------------------------
template <int SIM, bool MEAS>
__device__ __forceinline__ void pair32(const ForceArgs& fa, const double4& pi, const double4& pj,
                                       bool valid, PairOut<float>& o)
{
    o.dx = __double2float_rn(min_image(__dsub_rn(pi.x, pj.x), fa.xl[0], fa.hlb[0]));
    o.dy = __double2float_rn(min_image(__dsub_rn(pi.y, pj.y), fa.xl[1], fa.hlb[1]));
    o.dz = __double2float_rn(min_image(__dsub_rn(pi.z, pj.z), fa.xl[2], fa.hlb[2]));
    const float r2 = fmaf(o.dx, o.dx, fmaf(o.dy, o.dy, o.dz * o.dz));
    o.fs = 0.f;
    o.u = 0.f;
    o.w = 0.f;
    o.hit = false;
    if constexpr (SIM == SIM_PURE || SIM == SIM_MIX) {
        if (valid && r2 <= fa.rc2f) {
            const float rinv = rsqrt_f32(r2);
            const float r = r2 * rinv;
            const float mr = fa.xmucf * r;
            const float er = exp_neg_f32(mr) * rinv;
            o.fs = (1.0f + mr) * er * (rinv * rinv);
            if constexpr (MEAS) {
                o.u = er - fa.evcutf;
                o.w = o.fs * r2;
            }
            o.hit = true;
        }
    } else {
        if (!valid) return;
        if (fa.nuclear_on && r2 <= fa.rn2f) {
            const float e = exp_neg_f32(r2 * fa.xp2if);
            const float B = (pi.w == pj.w) ? fa.bpcf : fa.bmcf;
            const float fn = fa.xpif * fmaf(fa.aa2f, e, B) * e;
            o.fs = fn;
            if constexpr (MEAS) {
                o.u = fmaf(fa.aaf, e, B) * e;
                o.w = fn * r2;
            }
            o.hit = true;
        }
        if (fa.coulomb_on && pi.w == 1.0 && pj.w == 1.0 && r2 <= fa.rc2f) {
            const float rinv = rsqrt_f32(r2);
            const float r = r2 * rinv;
            const float mr = fa.xmucf * r;
            const float er = fa.vcf * exp_neg_f32(mr) * rinv;
            const float fc = (1.0f + mr) * er * (rinv * rinv);
            o.fs += fc;
            if constexpr (MEAS) {
                o.u += er - fa.evcutf;
                o.w += fc * r2;
            }
            o.hit = true;
        }
    }
}

// ---- per-target accumulators --------------------------------------------
// FP64 form: plain double sums.  Mixed form: Knuth two-sum FP32 sums.
template <int PREC, bool MEAS>
struct TargetAcc;

template <bool MEAS>
struct TargetAcc<PREC_FP64, MEAS> {
    double f[3];
    double s[MEAS ? NSCAL : 1];
    __device__ __forceinline__ void zero()
    {
        f[0] = f[1] = f[2] = 0.0;
#pragma unroll
        for (int k = 0; k < (MEAS ? NSCAL : 1); ++k) s[k] = 0.0;
    }
    // weight: Z_j for the mixture (int_ion_mix.f:179), 1 otherwise
    __device__ __forceinline__ void add(const PairOut<double>& o, double weight)
    {
        const double fs = o.fs * weight;
        const double fx = fs * o.dx, fy = fs * o.dy, fz = fs * o.dz;
        f[0] += fx;
        f[1] += fy;
        f[2] += fz;
        if constexpr (MEAS) {
            s[0] += o.u * weight;
            s[1] += o.w * weight;
            s[2] += o.dx * fx;
            s[3] += o.dx * fy;
            s[4] += o.dx * fz;
            s[5] += o.dy * fy;
            s[6] += o.dy * fz;
            s[7] += o.dz * fz;
        }
    }
    __device__ __forceinline__ double force(int k) const { return f[k]; }
    __device__ __forceinline__ double scal(int k) const
    {
        if constexpr (MEAS) return s[k];
        return 0.0;
    }
};

template <bool MEAS>
struct TargetAcc<PREC_MIXED, MEAS> {
    cf32 f[3];
    cf32 s[MEAS ? NSCAL : 1];
    __device__ __forceinline__ void zero()
    {
        f[0] = f[1] = f[2] = cf32();
#pragma unroll
        for (int k = 0; k < (MEAS ? NSCAL : 1); ++k) s[k] = cf32();
    }
    __device__ __forceinline__ void add(const PairOut<float>& o, float weight)
    {
        const float fs = o.fs * weight;
        const float fx = fs * o.dx, fy = fs * o.dy, fz = fs * o.dz;
        f[0].add(fx);
        f[1].add(fy);
        f[2].add(fz);
        if constexpr (MEAS) {
            s[0].add(o.u * weight);
            s[1].add(o.w * weight);
            s[2].add(o.dx * fx);
            s[3].add(o.dx * fy);
            s[4].add(o.dx * fz);
            s[5].add(o.dy * fy);
            s[6].add(o.dy * fz);
            s[7].add(o.dz * fz);
        }
    }
    __device__ __forceinline__ double force(int k) const { return f[k].value(); }
    __device__ __forceinline__ double scal(int k) const
    {
        if constexpr (MEAS) return s[k].value();
        return 0.0;
    }
};

template <int PREC>
using real_t = std::conditional_t<PREC == PREC_FP64, double, float>;

template <int SIM, int PREC, bool MEAS>
__device__ __forceinline__ void pair_eval(const ForceArgs& fa, const double4& pi, const double4& pj,
                                          bool valid, PairOut<real_t<PREC>>& o)
{
    if constexpr (PREC == PREC_FP64) pair64<SIM, MEAS>(fa, pi, pj, valid, o);
    else pair32<SIM, MEAS>(fa, pi, pj, valid, o);
}

// ---- scaling to accelerations (int_ion_pure.f:227-231, int_ion_mix.f:273-277
// with the fold fj(:,i) = zii(i)*(fj(:,i)+fi(:)) of :201, int_nn.f:318-322).
// F is the sum of Z_j-weighted terms (mixture) or plain terms.  orig is the
// caller's particle index; the fold is skipped for orig = n-1 in compat mode
// because the reference's i loop ends at n-2 (int_ion_mix.f:158).
template <int SIM>
__device__ __forceinline__ void store_accel(const ForceArgs& fa, int orig, double zi,
                                            const double* __restrict__ aii, const double F[3],
                                            double* __restrict__ a_out)
{
    if constexpr (SIM == SIM_PURE) {
#pragma unroll
        for (int k = 0; k < 3; ++k) a_out[3 * orig + k] = fa.coef * F[k] / fa.ai_xmass;
    } else if constexpr (SIM == SIM_MIX) {
        const bool fold = !(fa.mix_compat && orig == fa.n - 1);
        const double am = aii[orig] * fa.xmass;
#pragma unroll
        for (int k = 0; k < 3; ++k) a_out[3 * orig + k] = fa.coef * (fold ? zi * F[k] : F[k]) / am;
    } else {
#pragma unroll
        for (int k = 0; k < 3; ++k) a_out[3 * orig + k] = F[k] / fa.xmass;
    }
}

// Shared memory of k_force_rows: 2 stages of FTILE double4, 2 mbarriers and
// the block-reduction scratch.
constexpr int FORCE_SMEM = 2 * FTILE * (int)sizeof(double4) + 16 + 32 * NSCAL * (int)sizeof(double);

template <int SIM, int PREC, bool MEAS>
__global__ void __launch_bounds__(FBLOCK)
k_force_rows(const double4* __restrict__ pos, const int* __restrict__ perm,
             const double* __restrict__ aii, ForceArgs fa, double* __restrict__ a_out,
             double* __restrict__ part, unsigned* __restrict__ err)
{
    extern __shared__ __align__(128) unsigned char smem[];
    double4* tile = reinterpret_cast<double4*>(smem);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 2 * FTILE * sizeof(double4));
    double* red = reinterpret_cast<double*>(smem + 2 * FTILE * sizeof(double4) + 16);

    const int n = fa.n;
    const int i = blockIdx.x * FBLOCK + threadIdx.x;
    const bool active = i < n;
    const double4 pi = active ? pos[i] : make_double4(0.0, 0.0, 0.0, 0.0);
    const int ntiles = (n + FTILE - 1) / FTILE;

    if (threadIdx.x == 0) {
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

    TargetAcc<PREC, MEAS> acc;
    acc.zero();
    PairOut<real_t<PREC>> o;

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
            for (int jj = 0; jj < cnt; ++jj) {
                const double4 pj = tl[jj];
                pair_eval<SIM, PREC, MEAS>(fa, pi, pj, (j0 + jj) != i, o);
                if (o.hit) acc.add(o, SIM == SIM_MIX ? (real_t<PREC>)pj.w : (real_t<PREC>)1);
            }
        }
        __syncthreads();                      // every thread is done with stage st
        if (threadIdx.x == 0 && t + 2 < ntiles) issue(t + 2);
    }

    double S[NSCAL];
#pragma unroll
    for (int k = 0; k < NSCAL; ++k) S[k] = (MEAS && active) ? acc.scal(k) : 0.0;
    if (active) {
        const double F[3] = {acc.force(0), acc.force(1), acc.force(2)};
        store_accel<SIM>(fa, perm[i], pi.w, aii, F, a_out);
    }
    if constexpr (MEAS) {
        if constexpr (SIM == SIM_MIX) {
#pragma unroll
            for (int k = 0; k < NSCAL; ++k) S[k] *= pi.w;    // ev += zii(i)*evx ...
        }
        block_sum_store<NSCAL>(S, red, part + (size_t)blockIdx.x * NSCAL);
    }
}

}  // namespace yk
