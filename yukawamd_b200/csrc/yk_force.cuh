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
// PREC_FP64: all FP64 (exp_neg_f64, our table-driven exp; for ions
// rsqrt_nr64, a second-order correction of the FP32 hardware estimate, for the
// nucleon Coulomb term the library rsqrt; the reciprocal root replaces the
// reference's sqrt and divide, 1/(r r^2) = rinv^3).
// PREC_MIXED: the r^2, rsqrt, exp and force terms in FP32.  Pairs take their
// displacement from the shadow's hi/lo parts (screen_d_x2: exact FP32 hi-part
// differences plus a lo correction, no FP64 arithmetic) when the box allows it
// (ions: fa.lo; nucleons: fa.hilo, with the pairs near |d| = L/2 on the FP64
// minimum image) and e^{-mu r} from the hardware base-2 exponential;
// otherwise the displacement and minimum image are FP64, then cast to FP32.
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
    // FP32 pre-screen (screen_r2_x2): box, 1/box and squared screening radii
    // widened by a margin that covers the FP32 rounding of the shadow
    // positions, so no pair inside a cutoff is ever screened out.
    float Lf[3], invLf[3];
    float scr_c2, scr_n2;
    int n, nuclear_on, coulomb_on, mix_compat;
    int img_k;                       // the screen's image integers are exact (see setup)
    int nn_short;                    // nucleons: the nuclear screening radius is below L/2 - 2^-5 fm
                                     // on every axis (or the nuclear term is off), so a pair near
                                     // |d| = L/2 on some axis is out of nuclear range in either image
    int exp_ok;                      // mu max(r_c, 1) <= 690: every exponent of an ion pair
                                     // (masked pairs take r = 1) is inside exp_neg_f64's range
    // mixed form, ions: the displacement from the hi/lo shadow parts
    // (screen_d_x2); Lh = box on the SHADOW_Q grid, Ll = box - Lh
    float Lh[3], Ll[3];
    int lo;                          // img_k and every box length below SHADOW_EXACT / 2
    // mixed form, nucleons: hi/lo displacement with the screen's image
    // integers (every box length below SHADOW_EXACT / 2); a pair whose hi-part
    // displacement after the image shift is hLm or more from 0 on some axis
    // (hLm = L/2 - 2^-7 fm, rounded down) takes the reference's exact FP64
    // minimum image instead (pair_group_nn_lo)
    int hilo;
    float hLm[3];
    float hLmin;                     // the smallest hLm (a flag test against it flags a superset)
    int coul_all;                    // the p-p Coulomb cutoff is beyond every FP32 distance (rc2f = inf)
};

// FP32 shadow positions ("posf") are stored tile by tile: tile t (slots
// 128t .. 128t+127) is a contiguous block of SHADOW_FLOATS = 1664 floats:
//   [0, 768)      hi parts of x, y, z, one 256-float section per coordinate
//   [768, 896)    w[128] (charge / species word)
//   [896, 1664)   lo parts of x, y, z, one 256-float section per coordinate
// Within a coordinate's section each group of 4 slots s0..s3 takes 8 floats
// in the order
//     s0 s1 s1 s0 s2 s3 s3 s2
// so that (a) two neighbouring slots (j, j+1), j even, are one aligned
// float2 at offset 2j, and (b) every ordered pair of a group's halves that
// the half-pair kernel's lane swizzle needs -- (s0,s1) (s1,s0) (s2,s3)
// (s3,s2) -- is one aligned float2 at offset 2q, q = 0..3, in the block.
//
// hi = x rounded to the grid of SHADOW_Q = 2^-9 fm, lo = x - hi (|lo| <=
// 2^-10, rounded to FP32).  On that grid every coordinate, box length and
// difference below SHADOW_EXACT = 2^24 SHADOW_Q = 32768 fm is an FP32 number,
// so the hi-part displacement x_j - x_i and its image shift by the grid box
// length are exact FP32 operations; the mixed form adds the lo parts to get
// the displacement to FP32 precision without any FP64 arithmetic
// (screen_d_x2).  The screen and the FP64 form read only the first 896 floats
// (one 3.5 KB bulk copy per tile); the mixed form also copies the lo part.
constexpr int SHADOW_TILE = 128;
constexpr int SHADOW_HI_FLOATS = 7 * SHADOW_TILE;
constexpr int SHADOW_LO_FLOATS = 6 * SHADOW_TILE;
constexpr int SHADOW_FLOATS = SHADOW_HI_FLOATS + SHADOW_LO_FLOATS;
constexpr double SHADOW_Q = 1.0 / 512.0;
constexpr double SHADOW_EXACT = 32768.0;
__host__ __device__ __forceinline__ int shadow_off(int j, int comp)
{
    // comp 0..2: hi x, y, z; 3: w; 4..6: lo x, y, z
    const int paired = 8 * (j >> 2) + ((j & 1) | ((j & 2) << 1));
    return comp < 3 ? comp * 2 * SHADOW_TILE + paired
                    : comp == 3 ? 6 * SHADOW_TILE + j : SHADOW_HI_FLOATS + (comp - 4) * 2 * SHADOW_TILE + paired;
}
// index of slot's (first) copy of component comp; the second copy of a
// coordinate part (comp != 3) is at shadow_index ^ 3
__host__ __device__ __forceinline__ long long shadow_index(int slot, int comp)
{
    return (long long)(slot >> 7) * SHADOW_FLOATS + shadow_off(slot & (SHADOW_TILE - 1), comp);
}

// hi part of a coordinate: the nearest multiple of SHADOW_Q (exact FP64
// arithmetic: scaling by a power of two and rint)
__host__ __device__ __forceinline__ double shadow_hi(double x)
{
    return rint(x * (1.0 / SHADOW_Q)) * SHADOW_Q;
}

__device__ __forceinline__ void store_shadow(float* __restrict__ posf, int slot, double x, double y, double z,
                                             float w)
{
    const double v[3] = {x, y, z};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const double h = shadow_hi(v[c]);
        const float hf = __double2float_rn(h);
        const float lf = __double2float_rn(__dsub_rn(v[c], h));
        const long long k = shadow_index(slot, c);
        posf[k] = hf;
        posf[k ^ 3] = hf;
        const long long kl = shadow_index(slot, 4 + c);
        posf[kl] = lf;
        posf[kl ^ 3] = lf;
    }
    posf[shadow_index(slot, 3)] = w;
}

// Target-side constants of the FP32 screen (negated shadow position).
struct ScreenI {
    float nx, ny, nz, w;
};

__device__ __forceinline__ ScreenI load_screen_i(const float* __restrict__ posf, int slot)
{
    ScreenI s;
    s.nx = -posf[shadow_index(slot, 0)];
    s.ny = -posf[shadow_index(slot, 1)];
    s.nz = -posf[shadow_index(slot, 2)];
    s.w = posf[shadow_index(slot, 3)];
    return s;
}

// FP32 squared distances from the target to sources j and j+1 of a shadow
// tile, two at a time with the packed FP32x2 instructions; the minimum image
// is d - L*rint(d/L) with rint by the 1.5*2^23 magic-number add.  Used only
// to decide which pairs need the exact FP64 test.
__device__ __forceinline__ float2 screen_r2_x2(const ForceArgs& fa, const ScreenI& si,
                                               const float* __restrict__ t, int j)
{
    const float2 MAG = make_float2(12582912.0f, 12582912.0f);
    const float2 NMAG = make_float2(-12582912.0f, -12582912.0f);
    float2 d[3];
    const float ni[3] = {si.nx, si.ny, si.nz};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float2 xj = *reinterpret_cast<const float2*>(t + c * 2 * SHADOW_TILE + 2 * j);
        float2 dc = __fadd2_rn(xj, make_float2(ni[c], ni[c]));
        const float2 k = __fadd2_rn(__ffma2_rn(dc, make_float2(fa.invLf[c], fa.invLf[c]), MAG), NMAG);
        d[c] = __ffma2_rn(make_float2(-fa.Lf[c], -fa.Lf[c]), k, dc);
    }
    float2 r2 = __fmul2_rn(d[2], d[2]);
    r2 = __ffma2_rn(d[1], d[1], r2);
    return __ffma2_rn(d[0], d[0], r2);
}

// Scalar form of the same screen for one source j of a shadow tile.
__device__ __forceinline__ float screen_r2_1(const ForceArgs& fa, const ScreenI& si,
                                            const float* __restrict__ t, int j)
{
    const float MAGIC = 12582912.0f;
    float dx = t[shadow_off(j, 0)] + si.nx, dy = t[shadow_off(j, 1)] + si.ny, dz = t[shadow_off(j, 2)] + si.nz;
    dx = fmaf(-fa.Lf[0], fmaf(dx, fa.invLf[0], MAGIC) - MAGIC, dx);
    dy = fmaf(-fa.Lf[1], fmaf(dy, fa.invLf[1], MAGIC) - MAGIC, dy);
    dz = fmaf(-fa.Lf[2], fmaf(dz, fa.invLf[2], MAGIC) - MAGIC, dz);
    return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
}

// The packed screen for the ordered source pair stored at offset off (0, 2,
// 4 or 6) of group g's blocks, also returning the image integers
// k = rint(d/L) per axis (as floats: -1, 0 or 1 for a pair in the box).
__device__ __forceinline__ float2 screen_r2k_x2(const ForceArgs& fa, const ScreenI& si,
                                                const float* __restrict__ t, int g, int off, float2 (&k)[3])
{
    const float2 MAG = make_float2(12582912.0f, 12582912.0f);
    const float2 NMAG = make_float2(-12582912.0f, -12582912.0f);
    float2 d[3];
    const float ni[3] = {si.nx, si.ny, si.nz};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float2 xj = *reinterpret_cast<const float2*>(t + c * 2 * SHADOW_TILE + 8 * g + off);
        float2 dc = __fadd2_rn(xj, make_float2(ni[c], ni[c]));
        k[c] = __fadd2_rn(__ffma2_rn(dc, make_float2(fa.invLf[c], fa.invLf[c]), MAG), NMAG);
        d[c] = __ffma2_rn(make_float2(-fa.Lf[c], -fa.Lf[c]), k[c], dc);
    }
    float2 r2 = __fmul2_rn(d[2], d[2]);
    r2 = __ffma2_rn(d[1], d[1], r2);
    return __ffma2_rn(d[0], d[0], r2);
}

// The mixed form's displacement for the ordered source pair at offset off
// of group g (the order of screen_r2k_x2): d = x_j - x_i in the minimum
// image, to FP32 precision, without FP64 arithmetic.  The hi-part difference
// dc and its image shift dc - k Lh are exact (every value is a multiple of
// SHADOW_Q below SHADOW_EXACT); the lo parts and the box's lo part go into
// one correction term, and the sum is the one rounding.  t is the hi tile, tl
// the lo tile (x, y, z sections of 256 paired floats); nli holds the target's
// negated lo parts.  Returns r^2.
__device__ __forceinline__ float2 screen_d_x2(const ForceArgs& fa, const ScreenI& si, const float (&nli)[3],
                                              const float* __restrict__ t, const float* __restrict__ tl, int g,
                                              int off, float2 (&d)[3])
{
    const float2 MAG = make_float2(12582912.0f, 12582912.0f);
    const float2 NMAG = make_float2(-12582912.0f, -12582912.0f);
    const float ni[3] = {si.nx, si.ny, si.nz};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float2 xj = *reinterpret_cast<const float2*>(t + c * 2 * SHADOW_TILE + 8 * g + off);
        const float2 lj = *reinterpret_cast<const float2*>(tl + c * 2 * SHADOW_TILE + 8 * g + off);
        const float2 dc = __fadd2_rn(xj, make_float2(ni[c], ni[c]));
        const float2 k = __fadd2_rn(__ffma2_rn(dc, make_float2(fa.invLf[c], fa.invLf[c]), MAG), NMAG);
        const float2 d1 = __ffma2_rn(make_float2(-fa.Lh[c], -fa.Lh[c]), k, dc);
        float2 e = __fadd2_rn(lj, make_float2(nli[c], nli[c]));
        e = __ffma2_rn(make_float2(-fa.Ll[c], -fa.Ll[c]), k, e);
        d[c] = __fadd2_rn(d1, e);
    }
    float2 r2 = __fmul2_rn(d[2], d[2]);
    r2 = __ffma2_rn(d[1], d[1], r2);
    return __ffma2_rn(d[0], d[0], r2);
}

// screen_d_x2 for nucleons, also flagging (bits 0, 1 of flag for the two
// pairs) the pairs whose hi-part displacement after the image shift is hLmin
// or more from 0 on some axis: the image decision of those pairs is close to
// the reference's boundary |d| = L/2, and they take the exact FP64 image.
__device__ __forceinline__ float2 screen_d_flag_x2(const ForceArgs& fa, const ScreenI& si, const float (&nli)[3],
                                                   const float* __restrict__ t, const float* __restrict__ tl,
                                                   int g, int off, float2 (&d)[3], unsigned& flag)
{
    const float2 MAG = make_float2(12582912.0f, 12582912.0f);
    const float2 NMAG = make_float2(-12582912.0f, -12582912.0f);
    const float ni[3] = {si.nx, si.ny, si.nz};
    float2 mx = make_float2(0.f, 0.f);           // the largest |hi-part displacement| over the axes
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float2 xj = *reinterpret_cast<const float2*>(t + c * 2 * SHADOW_TILE + 8 * g + off);
        const float2 lj = *reinterpret_cast<const float2*>(tl + c * 2 * SHADOW_TILE + 8 * g + off);
        const float2 dc = __fadd2_rn(xj, make_float2(ni[c], ni[c]));
        const float2 k = __fadd2_rn(__ffma2_rn(dc, make_float2(fa.invLf[c], fa.invLf[c]), MAG), NMAG);
        const float2 d1 = __ffma2_rn(make_float2(-fa.Lh[c], -fa.Lh[c]), k, dc);       // exact
        mx = make_float2(fmaxf(mx.x, fabsf(d1.x)), fmaxf(mx.y, fabsf(d1.y)));
        float2 e = __fadd2_rn(lj, make_float2(nli[c], nli[c]));
        e = __ffma2_rn(make_float2(-fa.Ll[c], -fa.Ll[c]), k, e);
        d[c] = __fadd2_rn(d1, e);
    }
    // against the smallest axis margin: in a box with unequal edges this also
    // flags some pairs that do not need the exact image, which is only slower
    flag = (mx.x >= fa.hLmin ? 1u : 0u) | (mx.y >= fa.hLmin ? 2u : 0u);
    float2 r2 = __fmul2_rn(d[2], d[2]);
    r2 = __ffma2_rn(d[1], d[1], r2);
    return __ffma2_rn(d[0], d[0], r2);
}

// screen_d_x2 when the image of every reachable source of the tile is the
// same, k per axis, and has been folded into the target's coordinates once
// per tile: th = -(x_i hi part) - k Lh (exact on the SHADOW_Q grid), tl2 =
// -(x_i lo part) - k Ll.  Per axis the exact hi-part difference plus the lo
// correction, one rounding: d = x_j - x_i - k L to FP32 precision.  Returns
// r^2.
__device__ __forceinline__ float2 disp_tile_x2(const float2 (&th)[3], const float2 (&tl2)[3],
                                               const float* __restrict__ t, const float* __restrict__ tl, int g,
                                               int off, float2 (&d)[3])
{
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float2 xj = *reinterpret_cast<const float2*>(t + c * 2 * SHADOW_TILE + 8 * g + off);
        const float2 lj = *reinterpret_cast<const float2*>(tl + c * 2 * SHADOW_TILE + 8 * g + off);
        d[c] = __fadd2_rn(__fadd2_rn(xj, th[c]), __fadd2_rn(lj, tl2[c]));
    }
    float2 r2 = __fmul2_rn(d[2], d[2]);
    r2 = __ffma2_rn(d[1], d[1], r2);
    return __ffma2_rn(d[0], d[0], r2);
}

// Squared screening radius of a pair.  Ions: rccut.  Nucleons: rncut for the
// nuclear force, or rccut for a p-p pair (Coulomb).
template <int SIM>
__device__ __forceinline__ float screen_lim(const ForceArgs& fa, float wi, float wj)
{
    if constexpr (SIM == SIM_PURE || SIM == SIM_MIX) {
        return fa.scr_c2;
    } else {
        const bool pp = (wi == 1.0f) && (wj == 1.0f);
        return (pp && fa.coulomb_on) ? fmaxf(fa.scr_c2, fa.scr_n2) : fa.scr_n2;
    }
}

template <typename R>
struct PairOut {
    R fs, u, w;
    R dx, dy, dz;
    bool hit;
};

// ---- one pair, FP64 -------------------------------------------------------
// phys64: the pair terms from a minimum-image displacement already in o.dx,
// o.dy, o.dz; wi, wj are the species / charge words of the two particles.
template <int SIM, bool MEAS>
__device__ __forceinline__ void phys64(const ForceArgs& fa, double wi, double wj, bool valid, PairOut<double>& o)
{
    const double r2 = o.dx * o.dx + o.dy * o.dy + o.dz * o.dz;
    o.fs = 0.0;
    o.u = 0.0;
    o.w = 0.0;
    o.hit = false;
    if constexpr (SIM == SIM_PURE || SIM == SIM_MIX) {
        if (valid && r2 <= fa.rc2) {
            const double rinv = rsqrt_nr64(r2);
            const double r = r2 * rinv;
            const double mr = fa.xmuc * r;
            const double er = exp_neg_f64(mr) * rinv;                // e^{-mu r}/r
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
            const double e = exp_neg_f64(r2 * fa.xp2i);
            const double B = (wi == wj) ? fa.bpc : fa.bmc;
            const double fn = fa.xpi * (fa.aa2 * e + B) * e;
            o.fs = fn;
            if constexpr (MEAS) {
                o.u = (fa.aa * e + B) * e;
                o.w = fn * r2;
            }
            o.hit = true;
        }
        if (fa.coulomb_on && wi == 1.0 && wj == 1.0 && r2 <= fa.rc2) {
            // the library root: on this branchy single-pair path the longer
            // dependency chain of two Newton steps from the FP32 estimate
            // made the 51,200-nucleon step 3.5 % slower (the ion paths
            // interleave four pairs and gained 2 %)
            const double rinv = rsqrt(r2);
            const double r = r2 * rinv;
            const double mr = fa.xmuc * r;
            const double er = fa.vc * exp_neg_f64(mr) * rinv;         // vc e^{-mu r}/r
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

template <int SIM, bool MEAS>
__device__ __forceinline__ void pair64(const ForceArgs& fa, const double4& pi, const double4& pj,
                                       bool valid, PairOut<double>& o)
{
    o.dx = min_image(__dsub_rn(pi.x, pj.x), fa.xl[0], fa.hlb[0]);
    o.dy = min_image(__dsub_rn(pi.y, pj.y), fa.xl[1], fa.hlb[1]);
    o.dz = min_image(__dsub_rn(pi.z, pj.z), fa.xl[2], fa.hlb[2]);
    phys64<SIM, MEAS>(fa, pi.w, pj.w, valid, o);
}

// ---- one pair, mixed ---------------------------------------------------------
// phys32: the FP32 pair terms from the cast displacement in o.dx, o.dy, o.dz.
template <int SIM, bool MEAS>
__device__ __forceinline__ void phys32(const ForceArgs& fa, double wi, double wj, bool valid, PairOut<float>& o)
{
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
            const float B = (wi == wj) ? fa.bpcf : fa.bmcf;
            const float fn = fa.xpif * fmaf(fa.aa2f, e, B) * e;
            o.fs = fn;
            if constexpr (MEAS) {
                o.u = fmaf(fa.aaf, e, B) * e;
                o.w = fn * r2;
            }
            o.hit = true;
        }
        if (fa.coulomb_on && wi == 1.0 && wj == 1.0 && r2 <= fa.rc2f) {
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

// The reference's conditional minimum image on FP64 comparisons; the mixed
// form uses it because its FP64 pipe is idle while its integer pipe is busy.
__device__ __forceinline__ double min_image_cmp(double d, double L)
{
    const double hL = 0.5 * L;
    double s = 0.0;
    if (d > hL) s = -L;
    else if (d < -hL) s = L;
    return __dadd_rn(d, s);
}

template <int SIM, bool MEAS>
__device__ __forceinline__ void pair32(const ForceArgs& fa, const double4& pi, const double4& pj,
                                       bool valid, PairOut<float>& o)
{
    o.dx = __double2float_rn(min_image_cmp(__dsub_rn(pi.x, pj.x), fa.xl[0]));
    o.dy = __double2float_rn(min_image_cmp(__dsub_rn(pi.y, pj.y), fa.xl[1]));
    o.dz = __double2float_rn(min_image_cmp(__dsub_rn(pi.z, pj.z), fa.xl[2]));
    phys32<SIM, MEAS>(fa, pi.w, pj.w, valid, o);
}

// ---- one ion pair without branches ------------------------------------------
// The screened-Coulomb terms of phys64 / phys32 for a pair that sel says the
// screen selected; computed unconditionally (a placeholder r^2 = 1 for pairs
// that do not interact) and masked, so that several pairs' chains can be
// interleaved by the compiler.

// d = x_i - x_j in the minimum image.  The screen rounds (x_j - x_i)/L to
// the image integer k, so the reference's d - L (d > L/2) or d + L
// (d < -L/2) is d + k L, one FMA, when k is exact (fa.img_k, see the host
// setup); otherwise the conditional corrections themselves.
// IMGK: the caller has checked fa.img_k (the exact comparisons are then not
// compiled in).
template <bool IMGK = false>
__device__ __forceinline__ double image_k(const ForceArgs& fa, double d, float k, int c)
{
    if (IMGK) return __fma_rn((double)k, fa.xl[c], d);
    return fa.img_k ? __fma_rn((double)k, fa.xl[c], d) : min_image(d, fa.xl[c], fa.hlb[c]);
}

// The FP32 screen's r^2 when the tile's image is folded into the target
// (th as in disp_tile_x2; hi parts only, so the screening radius is the
// widened one).
__device__ __forceinline__ float2 screen_r2_tile_x2(const float2 (&th)[3], const float* __restrict__ t, int g,
                                                    int off)
{
    float2 d[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
        d[c] = __fadd2_rn(*reinterpret_cast<const float2*>(t + c * 2 * SHADOW_TILE + 8 * g + off), th[c]);
    float2 r2 = __fmul2_rn(d[2], d[2]);
    r2 = __ffma2_rn(d[1], d[1], r2);
    return __ffma2_rn(d[0], d[0], r2);
}

template <int PREC, bool MEAS, bool RANGE = true>
__device__ __forceinline__ void ion_terms_nb(const ForceArgs& fa, double dx, double dy, double dz, bool sel,
                                             PairOut<std::conditional_t<PREC == PREC_FP64, double, float>>& o);

// ion_pair_nb when the tile's image k is folded into the target: pit =
// x_i + k L (per axis), so d = pit - x_j is the pair's minimum image for
// every pair inside r_c.
template <int PREC, bool MEAS>
__device__ __forceinline__ void ion_pair_tile(const ForceArgs& fa, const double4& pit, const double4& pj, bool sel,
                                              PairOut<std::conditional_t<PREC == PREC_FP64, double, float>>& o)
{
    // only the exact-image kernels take the tile image, and those run only on
    // boxes with fa.exp_ok
    ion_terms_nb<PREC, MEAS, false>(fa, __dsub_rn(pit.x, pj.x), __dsub_rn(pit.y, pj.y), __dsub_rn(pit.z, pj.z),
                                    sel, o);
}

template <int PREC, bool MEAS, bool IMGK = false>
__device__ __forceinline__ void ion_pair_nb(const ForceArgs& fa, const double4& pi, const double4& pj, bool sel,
                                            const float (&k)[3],
                                            PairOut<std::conditional_t<PREC == PREC_FP64, double, float>>& o)
{
    const double dx = image_k<IMGK>(fa, __dsub_rn(pi.x, pj.x), k[0], 0);
    const double dy = image_k<IMGK>(fa, __dsub_rn(pi.y, pj.y), k[1], 1);
    const double dz = image_k<IMGK>(fa, __dsub_rn(pi.z, pj.z), k[2], 2);
    ion_terms_nb<PREC, MEAS, !IMGK>(fa, dx, dy, dz, sel, o);       // IMGK kernels run with fa.exp_ok
}

// The pair terms of ion_pair_nb from the minimum-image displacement.
template <int PREC, bool MEAS, bool RANGE>
__device__ __forceinline__ void ion_terms_nb(const ForceArgs& fa, double dx, double dy, double dz, bool sel,
                                             PairOut<std::conditional_t<PREC == PREC_FP64, double, float>>& o)
{
    if constexpr (PREC == PREC_FP64) {
        o.dx = dx;
        o.dy = dy;
        o.dz = dz;
        const double r2 = o.dx * o.dx + o.dy * o.dy + o.dz * o.dz;
        const bool hit = sel && r2 <= fa.rc2;
        const double r2s = hit ? r2 : 1.0;
        const double rinv = rsqrt_nr64(r2s);
        const double r = r2s * rinv;
        const double mr = fa.xmuc * r;
        const double er = exp_neg_f64<RANGE>(mr) * rinv;
        const double fs = (1.0 + mr) * er * (rinv * rinv);
        o.fs = hit ? fs : 0.0;
        o.u = (MEAS && hit) ? er - fa.evcut : 0.0;
        o.w = (MEAS && hit) ? fs * r2 : 0.0;
        o.hit = hit;
    } else {
        o.dx = __double2float_rn(dx);
        o.dy = __double2float_rn(dy);
        o.dz = __double2float_rn(dz);
        const float r2 = fmaf(o.dx, o.dx, fmaf(o.dy, o.dy, o.dz * o.dz));
        const bool hit = sel && r2 <= fa.rc2f;
        const float r2s = hit ? r2 : 1.0f;
        const float rinv = rsqrt_f32(r2s);
        const float r = r2s * rinv;
        const float mr = fa.xmucf * r;
        const float er = exp_neg_f32(mr) * rinv;
        const float fs = (1.0f + mr) * er * (rinv * rinv);
        o.fs = hit ? fs : 0.f;
        o.u = (MEAS && hit) ? er - fa.evcutf : 0.f;
        o.w = (MEAS && hit) ? fs * r2 : 0.f;
        o.hit = hit;
    }
}

// The mixed form's ion pair from screen_d_x2's displacement dj = x_j - x_i
// and r^2 (hit: the pair is selected and inside r_c), branch-free as
// ion_pair_nb.
template <bool MEAS>
__device__ __forceinline__ void ion_pair_f32(const ForceArgs& fa, float r2, bool hit, float djx, float djy,
                                             float djz, PairOut<float>& o)
{
    o.dx = -djx;
    o.dy = -djy;
    o.dz = -djz;
    const float r2s = hit ? r2 : 1.0f;
    const float rinv = rsqrtf(r2s);                    // hardware estimate, no Newton step
    const float r = r2s * rinv;
    const float mr = fa.xmucf * r;
    const float er = exp_neg_f32_xu(mr) * rinv;
    const float fs = (1.0f + mr) * er * (rinv * rinv);
    o.fs = hit ? fs : 0.f;
    o.u = (MEAS && hit) ? er - fa.evcutf : 0.f;
    o.w = (MEAS && hit) ? fs * r2 : 0.f;
    o.hit = hit;
}

// ion_pair_f32's terms for two pairs at once (the FP32 arithmetic paired):
// r2 their r^2, msk 1 for a pair that interacts and 0 otherwise.  Returns fs
// (0 for a masked pair) and, when measuring, u and w.  e^{-mu r} is the
// hardware base-2 exponential of the rounded product y = -mu r log2(e): the
// rounding of y changes the result by at most |y| 2^-24 ln 2 relative, below
// the instruction's own error (about 2 ulp) for the pairs that carry the
// force (mu r of a few), and about 6e-7 at the cutoff mu r = 10, where the
// term is weighted by e^-10; fs = q (1 + mu r) with q = e^{-mu r} / r^3.
// A masked pair takes r^2 = 1e36 instead of a multiply by the mask: then
// q = e^{-mu r} 1e-54 rounds to exactly 0 in FP32 for any mu >= 0 (1/r and
// 1/r^2 stay normal numbers, mu r finite), so fs = 0 (one FP32x2 multiply
// fewer per two pairs: mixed step 1.000 -> 0.983 ms).
template <bool MEAS>
__device__ __forceinline__ void ion_terms_x2(const ForceArgs& fa, float2 r2, float2 msk, float2& fs, float2& u,
                                             float2& w)
{
    const float L2E = 1.44269502162933349609375f;           // float(log2 e)
    const float FAR = 1e36f;
    const float2 r2s = make_float2(msk.x != 0.f ? r2.x : FAR, msk.y != 0.f ? r2.y : FAR);
    const float2 rinv = make_float2(rsqrtf(r2s.x), rsqrtf(r2s.y));
    const float2 mr = __fmul2_rn(make_float2(fa.xmucf, fa.xmucf), __fmul2_rn(r2s, rinv));
    const float2 y = __fmul2_rn(mr, make_float2(-L2E, -L2E));
    const float2 er = __fmul2_rn(make_float2(ex2_approx(y.x), ex2_approx(y.y)), rinv);
    const float2 q = __fmul2_rn(er, __fmul2_rn(rinv, rinv));
    fs = __ffma2_rn(mr, q, q);
    if constexpr (MEAS) {
        u = __fmul2_rn(__fadd2_rn(er, make_float2(-fa.evcutf, -fa.evcutf)), msk);
        w = __fmul2_rn(fs, r2);
    }
}

// The nucleon terms for two pairs in the mixed form (int_nn.f:208-229), the
// FP32 arithmetic paired; r2 their r^2, msk 1 for a pair that takes the term
// and 0 otherwise.  Adds to fs (and u, w when measuring).
//   nuclear: e = exp(-r^2 / (2 Lambda)), B = bb + cc (like pair) or bb - cc,
//            fn = (2 aa e + B) e / Lambda, u = (aa e + B) e, w = fn r^2
//   p-p Coulomb: fc = vc (1 + mu r) e^{-mu r} / r^3, u = vc e^{-mu r}/r - evcut
//            (evcut includes vc for nucleons), w = fc r^2
// Both exponentials are the hardware base-2 exponential of the rounded
// product y = -t log2(e), as in ion_terms_x2: the rounding of y changes the
// result by at most |y| 2^-24 ln 2 relative, about the instruction's own
// error (2 ulp) where the terms carry the force (nuclear r^2 / 2 Lambda and
// Coulomb mu r of a few) and below 1e-6 where they are weighted by e^-10 or
// less; 1/r is the hardware reciprocal-root estimate.
__device__ __forceinline__ float2 exp_neg_x2(float2 t)
{
    const float L2E = 1.44269502162933349609375f;           // float(log2 e)
    const float2 y = __fmul2_rn(t, make_float2(-L2E, -L2E));
    return make_float2(ex2_approx(y.x), ex2_approx(y.y));
}

template <bool MEAS>
__device__ __forceinline__ void nuclear_terms_x2(const ForceArgs& fa, float2 r2, float2 msk, float2 B, float2& fs,
                                                 float2& u, float2& w)
{
    const float2 e = exp_neg_x2(__fmul2_rn(r2, make_float2(fa.xp2if, fa.xp2if)));
    const float2 em = __fmul2_rn(e, msk);
    const float2 fn = __fmul2_rn(make_float2(fa.xpif, fa.xpif),
                                 __fmul2_rn(__ffma2_rn(make_float2(fa.aa2f, fa.aa2f), e, B), em));
    fs = __fadd2_rn(fs, fn);
    if constexpr (MEAS) {
        u = __ffma2_rn(__ffma2_rn(make_float2(fa.aaf, fa.aaf), e, B), em, u);
        w = __ffma2_rn(fn, r2, w);
    }
}

// MASKED = false: every pair of the call takes the term (msk is ignored and
// no pair may have r^2 = 0).
template <bool MEAS, bool MASKED = true>
__device__ __forceinline__ void coulomb_terms_x2(const ForceArgs& fa, float2 r2, float2 msk, float2& fs, float2& u,
                                                 float2& w)
{
    // a masked pair takes r^2 = 1e36 (as in ion_terms_x2): q rounds to 0
    const float FAR = 1e36f;
    const float2 r2s = MASKED ? make_float2(msk.x != 0.f ? r2.x : FAR, msk.y != 0.f ? r2.y : FAR) : r2;
    const float2 rinv = make_float2(rsqrtf(r2s.x), rsqrtf(r2s.y));
    const float2 mr = __fmul2_rn(make_float2(fa.xmucf, fa.xmucf), __fmul2_rn(r2s, rinv));
    const float2 er = __fmul2_rn(__fmul2_rn(exp_neg_x2(mr), rinv), make_float2(fa.vcf, fa.vcf));
    // fc = (1 + mu r) q with q = er / r^2
    const float2 rr = __fmul2_rn(rinv, rinv);
    const float2 q = __fmul2_rn(er, rr);
    const float2 fc = __ffma2_rn(mr, q, q);
    fs = __fadd2_rn(fs, fc);
    if constexpr (MEAS) {
        const float2 ue = __fadd2_rn(er, make_float2(-fa.evcutf, -fa.evcutf));
        u = MASKED ? __ffma2_rn(ue, msk, u) : __fadd2_rn(u, ue);
        w = __ffma2_rn(fc, r2, w);
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

// Plain sum of a few pair terms (one group of sources) before they enter the
// compensated per-target sum of the mixed form.
template <int PREC, bool MEAS>
struct GroupSum {
    using R = std::conditional_t<PREC == PREC_FP64, double, float>;
    R f[3];
    R s[MEAS ? NSCAL : 1];
    __device__ __forceinline__ void zero()
    {
        f[0] = f[1] = f[2] = (R)0;
#pragma unroll
        for (int k = 0; k < (MEAS ? NSCAL : 1); ++k) s[k] = (R)0;
    }
    __device__ __forceinline__ void add(const PairOut<R>& o, R weight)
    {
        const R fs = o.fs * weight;
        const R fx = fs * o.dx, fy = fs * o.dy, fz = fs * o.dz;
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
};

template <bool MEAS>
struct TargetAcc<PREC_MIXED, MEAS> {
    cf32 f[3];
    cf32 s[MEAS ? NSCAL : 1];
    // FP64 sums of the group sums that add_group2 takes (the hi/lo pair paths):
    // one conversion and one FP64 add per component on pipes the FP32 pair
    // arithmetic leaves idle, instead of seven FP32 operations of a two-sum
    double fd[3];
    double sd[MEAS ? NSCAL : 1];
    __device__ __forceinline__ void zero()
    {
        f[0] = f[1] = f[2] = cf32();
        fd[0] = fd[1] = fd[2] = 0.0;
#pragma unroll
        for (int k = 0; k < (MEAS ? NSCAL : 1); ++k) {
            s[k] = cf32();
            sd[k] = 0.0;
        }
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
    // a group's plain FP32 sum enters the compensated sums as one term
    __device__ __forceinline__ void add_group(const GroupSum<PREC_MIXED, MEAS>& g)
    {
        f[0].add(g.f[0]);
        f[1].add(g.f[1]);
        f[2].add(g.f[2]);
        if constexpr (MEAS) {
#pragma unroll
            for (int k = 0; k < NSCAL; ++k) s[k].add(g.s[k]);
        }
    }
    // a group's plain FP32 sum into the FP64 sums (exact conversion, one
    // FP64 rounding per group)
    __device__ __forceinline__ void add_group2(const GroupSum<PREC_MIXED, MEAS>& g)
    {
#pragma unroll
        for (int c = 0; c < 3; ++c) fd[c] += (double)g.f[c];
        if constexpr (MEAS) {
#pragma unroll
            for (int k = 0; k < NSCAL; ++k) sd[k] += (double)g.s[k];
        }
    }
    // only the force part of a group's sum (the measuring sums kept elsewhere)
    __device__ __forceinline__ void add_group2_force(const GroupSum<PREC_MIXED, MEAS>& g)
    {
#pragma unroll
        for (int c = 0; c < 3; ++c) fd[c] += (double)g.f[c];
    }
    __device__ __forceinline__ double force(int k) const { return f[k].value() + fd[k]; }
    __device__ __forceinline__ double scal(int k) const
    {
        if constexpr (MEAS) return s[k].value() + sd[k];
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

// Shared memory of k_force_rows: 2 stages of FTILE double4 and one shadow tile,
// 2 mbarriers and the block-reduction scratch.
constexpr int FORCE_SMEM = 2 * FTILE * (int)sizeof(double4) + 2 * SHADOW_HI_FLOATS * (int)sizeof(float) + 16 +
                           32 * NSCAL * (int)sizeof(double);

template <int SIM, int PREC, bool MEAS>
__global__ void __launch_bounds__(FBLOCK)
k_force_rows(const double4* __restrict__ pos, const float* __restrict__ posf,
             const int* __restrict__ perm, const double* __restrict__ aii, ForceArgs fa,
             double* __restrict__ a_out, double* __restrict__ part, unsigned* __restrict__ err)
{
    extern __shared__ __align__(128) unsigned char smem[];
    double4* tile = reinterpret_cast<double4*>(smem);
    float* tilef = reinterpret_cast<float*>(smem + 2 * FTILE * sizeof(double4));
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 2 * FTILE * sizeof(double4) + 2 * SHADOW_HI_FLOATS * sizeof(float));
    double* red = reinterpret_cast<double*>(smem + 2 * FTILE * sizeof(double4) + 2 * SHADOW_HI_FLOATS * sizeof(float) + 16);

    const int n = fa.n;
    const int i = blockIdx.x * FBLOCK + threadIdx.x;
    const bool active = i < n;
    const double4 pi = active ? pos[i] : make_double4(0.0, 0.0, 0.0, 0.0);
    const ScreenI si = load_screen_i(posf, active ? i : 0);
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
        const unsigned bytesf = (unsigned)SHADOW_HI_FLOATS * (unsigned)sizeof(float);
        uint64_t* b = &bar[t & 1];
        mbar_arrive_expect_tx(b, bytes + bytesf);
        bulk_g2s(tile + (t & 1) * FTILE, pos + j0, bytes, b);
        bulk_g2s(tilef + (t & 1) * SHADOW_HI_FLOATS, posf + (size_t)t * SHADOW_FLOATS, bytesf, b);
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
        const float* tlf = tilef + st * SHADOW_HI_FLOATS;
        if (active) {
#pragma unroll 2
            for (int jj = 0; jj < cnt; ++jj) {
                if ((j0 + jj) != i &&
                    screen_r2_1(fa, si, tlf, jj) <= screen_lim<SIM>(fa, si.w, tlf[shadow_off(jj, 3)])) {
                    const double4 pj = tl[jj];
                    pair_eval<SIM, PREC, MEAS>(fa, pi, pj, true, o);
                    if (o.hit) acc.add(o, SIM == SIM_MIX ? (real_t<PREC>)pj.w : (real_t<PREC>)1);
                }
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
