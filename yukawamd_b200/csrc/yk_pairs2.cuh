// yk_pairs2.cuh -- the half-pair kernels with two targets per thread.
//
// k_force_pairs2 is k_force_pairs (yk_pairs.cuh) with the target block
// doubled: a job's targets are the 2 x 128 slots of blocks R and R + 1
// (R even), and warp w holds slots 64w .. 64w + 63 of the pair, two per lane
// (64w + l and 64w + 32 + l, so a warp's targets are 64 consecutive slots of
// the Hilbert order and its box stays compact).  Every source value a lane
// reads from shared memory, every reduce-scatter of reactions and every row
// write then serves two pairs instead of one: the lane adds its two targets'
// reactions on a source before the warp reduction.
//
//   job (R, C0, C1, s) : tiles C0 <= C < C1 (C >= R) against blocks R, R + 1;
//                        writes Si slot s of both rows.
//   unit rows          : the reactions of both blocks on tile C go into the Sj
//                        row of unit (R, C); the row of unit (R + 1, C) is
//                        flagged zero (PairJobs::Sjf), so k_combine sums the
//                        same rows in the same order whatever the target
//                        block size.
//   pair (i, j)        : counts iff slot j > slot i, which only tiles R and
//                        R + 1 need to test.
//
// Three paths: ions in the FP64 form when the screen's image integers are
// exact (fa.img_k; the exact comparisons are not compiled in), ions in the
// mixed form with the hi/lo FP32 displacement (fa.lo), and nucleons in the
// mixed form with the hi/lo displacement and the flagged exact image near
// L/2 (fa.hilo).  The arithmetic per pair is that of pair_group,
// pair_group_lo and pair_group_nn_lo; only the reaction sums (two pairs per
// lane before the reduction) and the order of the target-side sums differ.
#pragma once

#include "yk_pairs.cuh"

namespace yk {

constexpr int PB2 = 2 * PB;      // target slots of a job

// Bounding box of a warp's 64 targets (two per lane).
__device__ __forceinline__ WarpBox warp_box2(const ForceArgs& fa, const double4 (&pi)[2], const bool (&act)[2],
                                             bool proton)
{
    const float inf = __int_as_float(0x7f800000);
    float lo[3], hi[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float v0 = __double2float_rn(k == 0 ? pi[0].x : k == 1 ? pi[0].y : pi[0].z);
        const float v1 = __double2float_rn(k == 0 ? pi[1].x : k == 1 ? pi[1].y : pi[1].z);
        lo[k] = fminf(act[0] ? v0 : inf, act[1] ? v1 : inf);
        hi[k] = fmaxf(act[0] ? v0 : -inf, act[1] ? v1 : -inf);
    }
    return warp_box_of(fa, lo, hi, act[0] || act[1], proton);
}

__device__ __forceinline__ float2 lds2(const float* p)
{
    return *reinterpret_cast<const float2*>(p);
}

__device__ __forceinline__ float2 dup2(float v)
{
    return make_float2(v, v);
}

// r^2 of the three FP32x2 displacement components.
__device__ __forceinline__ float2 r2_x2(const float2 (&d)[3])
{
    float2 r2 = __fmul2_rn(d[2], d[2]);
    r2 = __ffma2_rn(d[1], d[1], r2);
    return __ffma2_rn(d[0], d[0], r2);
}

// The validity bits of a group's 4 steps for one target: source jl = j0 +
// (jj ^ sw) counts if the target is active, jl is in the tile and jl > dl
// (dl = the target's slot in the job less the tile's offset from block R).
__device__ __forceinline__ unsigned valid4(int j0, int sw, int jlim, int dl, bool act)
{
    unsigned ok = 0;
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
        const int jl = j0 + (jj ^ sw);
        if (act && jl < jlim && jl > dl) ok |= 1u << jj;
    }
    return ok;
}

// pair_group_lo for two targets per lane (mixed form, ions, fa.lo).  The
// source's hi and lo parts are read once; per target the displacement is
// that of disp_tile_x2 (TILEIMG: the tile's image folded into th / tl2) or
// screen_d_x2 (each pair's own image), the terms those of ion_terms_x2.
// Measuring: the group's energy, virial and pressure-tensor sums of both
// targets, weighted by Z_i, go into the lane's FP32 tile sums ms (the job
// adds them to FP64 sums after each tile); they are sums over all pairs, so
// no per-target accumulator is needed.
template <int SIM, bool MEAS, bool CHECK, bool TILEIMG>
__device__ __forceinline__ void pair_group_lo2(const ForceArgs& fa, const ScreenI (&si)[2], const float (&nli)[2][3],
                                               const float (&th)[2][3], const float (&tl2)[2][3],
                                               const float (&wi)[2], const float* tlf, const float* tll, int j0,
                                               int jlim, const int (&dl)[2], const bool (&act)[2], int sw,
                                               TargetAcc<PREC_MIXED, MEAS> (&acc)[2], float* my_acc,
                                               float (&ms)[NSCAL])
{
    const int g = j0 >> 2;
    const int oa = 8 * g + 2 * sw, ob = 8 * g + 2 * (sw ^ 2);
    float2 xa[3], xb[3], la[3], lb[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        xa[c] = lds2(tlf + c * 2 * SHADOW_TILE + oa);
        xb[c] = lds2(tlf + c * 2 * SHADOW_TILE + ob);
        la[c] = lds2(tll + c * 2 * SHADOW_TILE + oa);
        lb[c] = lds2(tll + c * 2 * SHADOW_TILE + ob);
    }
    const float2 MAG = dup2(12582912.0f), NMAG = dup2(-12582912.0f);
    float2 da[2][3], db[2][3], ra[2], rb[2];
    unsigned m[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const float ni[3] = {si[u].nx, si[u].ny, si[u].nz};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if constexpr (TILEIMG) {
                da[u][c] = __fadd2_rn(__fadd2_rn(xa[c], dup2(th[u][c])), __fadd2_rn(la[c], dup2(tl2[u][c])));
                db[u][c] = __fadd2_rn(__fadd2_rn(xb[c], dup2(th[u][c])), __fadd2_rn(lb[c], dup2(tl2[u][c])));
            } else {
                const float2 dca = __fadd2_rn(xa[c], dup2(ni[c]));
                const float2 dcb = __fadd2_rn(xb[c], dup2(ni[c]));
                const float2 ka = __fadd2_rn(__ffma2_rn(dca, dup2(fa.invLf[c]), MAG), NMAG);
                const float2 kb = __fadd2_rn(__ffma2_rn(dcb, dup2(fa.invLf[c]), MAG), NMAG);
                float2 ea = __fadd2_rn(la[c], dup2(nli[u][c]));
                float2 eb = __fadd2_rn(lb[c], dup2(nli[u][c]));
                ea = __ffma2_rn(dup2(-fa.Ll[c]), ka, ea);
                eb = __ffma2_rn(dup2(-fa.Ll[c]), kb, eb);
                da[u][c] = __fadd2_rn(__ffma2_rn(dup2(-fa.Lh[c]), ka, dca), ea);
                db[u][c] = __fadd2_rn(__ffma2_rn(dup2(-fa.Lh[c]), kb, dcb), eb);
            }
        }
        ra[u] = r2_x2(da[u]);
        rb[u] = r2_x2(db[u]);
        m[u] = (ra[u].x <= fa.rc2f ? 1u : 0u) | (ra[u].y <= fa.rc2f ? 2u : 0u) | (rb[u].x <= fa.rc2f ? 4u : 0u) |
               (rb[u].y <= fa.rc2f ? 8u : 0u);
        if constexpr (CHECK) m[u] &= valid4(j0, sw, jlim, dl[u], act[u]);
    }
    const bool any0 = __any_sync(0xffffffffu, m[0] != 0), any1 = __any_sync(0xffffffffu, m[1] != 0);
    if (!any0 && !any1) return;
    const float* tw = tlf + 6 * SHADOW_TILE + j0;
    const float2 wja = (SIM == SIM_MIX) ? make_float2(tw[sw], tw[sw ^ 1]) : make_float2(1.f, 1.f);
    const float2 wjb = (SIM == SIM_MIX) ? make_float2(tw[sw ^ 2], tw[sw ^ 3]) : make_float2(1.f, 1.f);
    float2 ra3[3], rb3[3];
    // the terms of target u's four pairs into acc[u] and, first (u0) or not,
    // into the reactions
    auto terms = [&](int u, bool first) {
        const float2 mska = make_float2((m[u] & 1u) ? 1.f : 0.f, (m[u] & 2u) ? 1.f : 0.f);
        const float2 mskb = make_float2((m[u] & 4u) ? 1.f : 0.f, (m[u] & 8u) ? 1.f : 0.f);
        float2 fsa, ua, wa, fsb, ub, wb;
        ion_terms_x2<MEAS>(fa, ra[u], mska, fsa, ua, wa);
        ion_terms_x2<MEAS>(fa, rb[u], mskb, fsb, ub, wb);
        const float2 ga = __fmul2_rn(fsa, wja), gb = __fmul2_rn(fsb, wjb);
        GroupSum<PREC_MIXED, MEAS> gs;
        float2 fxa[3], fxb[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if constexpr (MEAS) {
                fxa[c] = __fmul2_rn(ga, da[u][c]);
                fxb[c] = __fmul2_rn(gb, db[u][c]);
                const float2 sc = __fadd2_rn(fxa[c], fxb[c]);
                gs.f[c] = -(sc.x + sc.y);
            } else {
                const float2 sc = __ffma2_rn(gb, db[u][c], __fmul2_rn(ga, da[u][c]));
                gs.f[c] = -(sc.x + sc.y);
            }
        }
        if constexpr (MEAS) {
            const float2 su = __ffma2_rn(ub, wjb, __fmul2_rn(ua, wja));
            const float2 sv = __ffma2_rn(wb, wjb, __fmul2_rn(wa, wja));
            gs.s[0] = su.x + su.y;
            gs.s[1] = sv.x + sv.y;
            const int P[6] = {0, 0, 0, 1, 1, 2}, Q[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                const float2 sp = __ffma2_rn(db[u][P[k]], fxb[Q[k]], __fmul2_rn(da[u][P[k]], fxa[Q[k]]));
                gs.s[2 + k] = sp.x + sp.y;
            }
#pragma unroll
            for (int k = 0; k < NSCAL; ++k) ms[k] = fmaf(gs.s[k], wi[u], ms[k]);
        }
        acc[u].add_group2_force(gs);
        // reaction on j: Z_i fs d (int_ion_mix.f:180), both targets' terms
        // summed in the lane
        const float2 ha = __fmul2_rn(fsa, dup2(wi[u])), hb = __fmul2_rn(fsb, dup2(wi[u]));
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if (first) {
                ra3[c] = __fmul2_rn(ha, da[u][c]);
                rb3[c] = __fmul2_rn(hb, db[u][c]);
            } else {
                ra3[c] = __ffma2_rn(ha, da[u][c], ra3[c]);
                rb3[c] = __ffma2_rn(hb, db[u][c], rb3[c]);
            }
        }
    };
    if (any0 && any1) {
        terms(0, true);
        terms(1, false);
    } else if (any0) {
        terms(0, true);          // no lane's second target has a pair in the group
    } else {
        terms(1, true);
    }
    float t[3];
    reduce_scatter4_x2(ra3, rb3, t);
    const int lane = threadIdx.x & 31;
    const int jl = j0 + sw;
    if ((lane & 7) == 0 && (!CHECK || jl < jlim)) {
        // a warp visits each group of a tile once: the row entry's only write
        my_acc[3 * jl] = t[0];
        my_acc[3 * jl + 1] = t[1];
        my_acc[3 * jl + 2] = t[2];
    }
}

// pair_group_nn_lo for two targets per lane (mixed form, nucleons, fa.hilo).
// The source's hi and lo parts are read once; per target the hi/lo
// displacement with the screen's image (screen_d_flag_x2's arithmetic), and
// the pairs flagged near |d| = L/2 take the reference's conditional minimum
// image on the FP64 positions (int_nn.f:190-195; the target's own position is
// read again from pos, the source's from gsrc).  Then the HPP terms inside
// rncut and the p-p Coulomb inside rccut (int_nn.f:208-229) for each target
// set that a lane of the warp needs.
template <bool MEAS, bool CHECK>
__device__ __forceinline__ void pair_group_nn_lo2(const ForceArgs& fa, const ScreenI (&si)[2],
                                                  const float (&nli)[2][3], const double4* __restrict__ pos,
                                                  const int (&ii)[2], const float* tlf, const float* tll,
                                                  const double4* __restrict__ gsrc, int j0, int jlim,
                                                  const int (&dl)[2], const bool (&act)[2], int sw,
                                                  TargetAcc<PREC_MIXED, MEAS> (&acc)[2], float* my_acc)
{
    const int g = j0 >> 2;
    const int oa = 8 * g + 2 * sw, ob = 8 * g + 2 * (sw ^ 2);
    float2 xa[3], xb[3], la[3], lb[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        xa[c] = lds2(tlf + c * 2 * SHADOW_TILE + oa);
        xb[c] = lds2(tlf + c * 2 * SHADOW_TILE + ob);
        la[c] = lds2(tll + c * 2 * SHADOW_TILE + oa);
        lb[c] = lds2(tll + c * 2 * SHADOW_TILE + ob);
    }
    const float* tw = tlf + 6 * SHADOW_TILE + j0;
    const float wj[4] = {tw[sw], tw[sw ^ 1], tw[sw ^ 2], tw[sw ^ 3]};
    const float2 MAG = dup2(12582912.0f), NMAG = dup2(-12582912.0f);
    float2 da[2][3], db[2][3], ra[2], rb[2];
    unsigned mn[2], mc[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const float ni[3] = {si[u].nx, si[u].ny, si[u].nz};
        unsigned fa_ = 0, fb_ = 0;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float2 dca = __fadd2_rn(xa[c], dup2(ni[c]));
            const float2 dcb = __fadd2_rn(xb[c], dup2(ni[c]));
            const float2 ka = __fadd2_rn(__ffma2_rn(dca, dup2(fa.invLf[c]), MAG), NMAG);
            const float2 kb = __fadd2_rn(__ffma2_rn(dcb, dup2(fa.invLf[c]), MAG), NMAG);
            const float2 d1a = __ffma2_rn(dup2(-fa.Lh[c]), ka, dca);         // exact
            const float2 d1b = __ffma2_rn(dup2(-fa.Lh[c]), kb, dcb);
            fa_ |= (fabsf(d1a.x) >= fa.hLm[c] ? 1u : 0u) | (fabsf(d1a.y) >= fa.hLm[c] ? 2u : 0u);
            fb_ |= (fabsf(d1b.x) >= fa.hLm[c] ? 1u : 0u) | (fabsf(d1b.y) >= fa.hLm[c] ? 2u : 0u);
            float2 ea = __fadd2_rn(la[c], dup2(nli[u][c]));
            float2 eb = __fadd2_rn(lb[c], dup2(nli[u][c]));
            ea = __ffma2_rn(dup2(-fa.Ll[c]), ka, ea);
            eb = __ffma2_rn(dup2(-fa.Ll[c]), kb, eb);
            da[u][c] = __fadd2_rn(d1a, ea);
            db[u][c] = __fadd2_rn(d1b, eb);
        }
        ra[u] = r2_x2(da[u]);
        rb[u] = r2_x2(db[u]);
        const unsigned ok = CHECK ? valid4(j0, sw, jlim, dl[u], act[u]) : 0xfu;
        const unsigned fl = (fa_ | (fb_ << 2)) & ok;
        if (__any_sync(0xffffffffu, fl != 0)) {
            // d = x_j - x_i from the reference's d = x_i - x_j and its image
            const double4 pi = pos[ii[u]];
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) {
                if ((fl >> jj) & 1u) {
                    const double4 pj = gsrc[j0 + (jj ^ sw)];
                    const float ex = -__double2float_rn(min_image(__dsub_rn(pi.x, pj.x), fa.xl[0], fa.hlb[0]));
                    const float ey = -__double2float_rn(min_image(__dsub_rn(pi.y, pj.y), fa.xl[1], fa.hlb[1]));
                    const float ez = -__double2float_rn(min_image(__dsub_rn(pi.z, pj.z), fa.xl[2], fa.hlb[2]));
                    const float r2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
                    float2(&dd)[3] = jj < 2 ? da[u] : db[u];
                    float2& rr = jj < 2 ? ra[u] : rb[u];
                    if (jj & 1) {
                        dd[0].y = ex;
                        dd[1].y = ey;
                        dd[2].y = ez;
                        rr.y = r2;
                    } else {
                        dd[0].x = ex;
                        dd[1].x = ey;
                        dd[2].x = ez;
                        rr.x = r2;
                    }
                }
            }
        }
        const float r2v[4] = {ra[u].x, ra[u].y, rb[u].x, rb[u].y};
        const bool ip = si[u].w == 1.0f;
        mn[u] = 0;
        mc[u] = 0;
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            const bool in = (ok >> jj) & 1u;
            if (in && fa.nuclear_on && r2v[jj] <= fa.rn2f) mn[u] |= 1u << jj;
            if (in && fa.coulomb_on && ip && wj[jj] == 1.0f && r2v[jj] <= fa.rc2f) mc[u] |= 1u << jj;
        }
    }
    const bool any0 = __any_sync(0xffffffffu, (mn[0] | mc[0]) != 0);
    const bool any1 = __any_sync(0xffffffffu, (mn[1] | mc[1]) != 0);
    if (!any0 && !any1) return;
    float2 fxa[2][3], fxb[2][3];
    // the terms of target u's four pairs into acc[u]; its reaction products
    // (fs d, int_nn.f:230-240) into fxa[u], fxb[u]
    auto terms = [&](int u) {
        const bool any_n = __any_sync(0xffffffffu, mn[u] != 0);
        const bool any_c = __any_sync(0xffffffffu, mc[u] != 0);
        float2 fsa = make_float2(0.f, 0.f), fsb = fsa, ua = fsa, ub = fsa, wa = fsa, wb = fsa;
        if (any_n) {
            const float2 Ba = make_float2(wj[0] == si[u].w ? fa.bpcf : fa.bmcf, wj[1] == si[u].w ? fa.bpcf : fa.bmcf);
            const float2 Bb = make_float2(wj[2] == si[u].w ? fa.bpcf : fa.bmcf, wj[3] == si[u].w ? fa.bpcf : fa.bmcf);
            nuclear_terms_x2<MEAS>(fa, ra[u], make_float2((mn[u] & 1u) ? 1.f : 0.f, (mn[u] & 2u) ? 1.f : 0.f), Ba,
                                   fsa, ua, wa);
            nuclear_terms_x2<MEAS>(fa, rb[u], make_float2((mn[u] & 4u) ? 1.f : 0.f, (mn[u] & 8u) ? 1.f : 0.f), Bb,
                                   fsb, ub, wb);
        }
        if (any_c) {
            coulomb_terms_x2<MEAS>(fa, ra[u], make_float2((mc[u] & 1u) ? 1.f : 0.f, (mc[u] & 2u) ? 1.f : 0.f), fsa,
                                   ua, wa);
            coulomb_terms_x2<MEAS>(fa, rb[u], make_float2((mc[u] & 4u) ? 1.f : 0.f, (mc[u] & 8u) ? 1.f : 0.f), fsb,
                                   ub, wb);
        }
        GroupSum<PREC_MIXED, MEAS> gs;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            fxa[u][c] = __fmul2_rn(fsa, da[u][c]);
            fxb[u][c] = __fmul2_rn(fsb, db[u][c]);
            const float2 sc = __fadd2_rn(fxa[u][c], fxb[u][c]);
            gs.f[c] = -(sc.x + sc.y);
        }
        if constexpr (MEAS) {
            const float2 su = __fadd2_rn(ua, ub);
            const float2 sv = __fadd2_rn(wa, wb);
            gs.s[0] = su.x + su.y;
            gs.s[1] = sv.x + sv.y;
            const int P[6] = {0, 0, 0, 1, 1, 2}, Q[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                const float2 sp = __ffma2_rn(db[u][P[k]], fxb[u][Q[k]], __fmul2_rn(da[u][P[k]], fxa[u][Q[k]]));
                gs.s[2 + k] = sp.x + sp.y;
            }
        }
        acc[u].add_group2(gs);
    };
    // a target set without a pair in the group (for every lane) is skipped
#pragma unroll
    for (int u = 0; u < 2; ++u) {
#pragma unroll
        for (int c = 0; c < 3; ++c) fxa[u][c] = fxb[u][c] = make_float2(0.f, 0.f);
    }
    if (any0) terms(0);
    if (any1) terms(1);
    float2 ra3[3], rb3[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        ra3[c] = __fadd2_rn(fxa[0][c], fxa[1][c]);
        rb3[c] = __fadd2_rn(fxb[0][c], fxb[1][c]);
    }
    float t[3];
    reduce_scatter4_x2(ra3, rb3, t);
    const int lane = threadIdx.x & 31;
    const int jl = j0 + sw;
    if ((lane & 7) == 0 && (!CHECK || jl < jlim)) {
        my_acc[3 * jl] = t[0];
        my_acc[3 * jl + 1] = t[1];
        my_acc[3 * jl + 2] = t[2];
    }
}

// pair_group for two targets per lane (FP64 form, ions, fa.img_k).  The
// FP32 screen reads the source's hi parts once; each selected pair's FP64
// source position is read once for both targets.  TILEIMG: the tile's image
// is folded into th (screen) and pit (FP64 target); otherwise each pair takes
// the screen's image integers (ion_pair_nb with IMGK).
template <int SIM, bool MEAS, bool CHECK, bool TILEIMG>
__device__ __forceinline__ void pair_group2(const ForceArgs& fa, const double4 (&pi)[2], const ScreenI (&si)[2],
                                            const float (&th)[2][3], const double4 (&pit)[2], const double (&wi)[2],
                                            const double4* tl, const float* tlf, int j0, int jlim, const int (&dl)[2],
                                            const bool (&act)[2], int sw, TargetAcc<PREC_FP64, MEAS> (&acc)[2],
                                            double* my_acc)
{
    const int g = j0 >> 2;
    const int oa = 8 * g + 2 * sw, ob = 8 * g + 2 * (sw ^ 2);
    float2 xa[3], xb[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        xa[c] = lds2(tlf + c * 2 * SHADOW_TILE + oa);
        xb[c] = lds2(tlf + c * 2 * SHADOW_TILE + ob);
    }
    const float2 MAG = dup2(12582912.0f), NMAG = dup2(-12582912.0f);
    float2 ka[2][3], kb[2][3];
    unsigned m[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        const float ni[3] = {si[u].nx, si[u].ny, si[u].nz};
        float2 da[3], db[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            if constexpr (TILEIMG) {
                da[c] = __fadd2_rn(xa[c], dup2(th[u][c]));
                db[c] = __fadd2_rn(xb[c], dup2(th[u][c]));
            } else {
                const float2 dca = __fadd2_rn(xa[c], dup2(ni[c]));
                const float2 dcb = __fadd2_rn(xb[c], dup2(ni[c]));
                ka[u][c] = __fadd2_rn(__ffma2_rn(dca, dup2(fa.invLf[c]), MAG), NMAG);
                kb[u][c] = __fadd2_rn(__ffma2_rn(dcb, dup2(fa.invLf[c]), MAG), NMAG);
                da[c] = __ffma2_rn(dup2(-fa.Lf[c]), ka[u][c], dca);
                db[c] = __ffma2_rn(dup2(-fa.Lf[c]), kb[u][c], dcb);
            }
        }
        const float2 ra = r2_x2(da), rb = r2_x2(db);
        m[u] = (ra.x <= fa.scr_c2 ? 1u : 0u) | (ra.y <= fa.scr_c2 ? 2u : 0u) | (rb.x <= fa.scr_c2 ? 4u : 0u) |
               (rb.y <= fa.scr_c2 ? 8u : 0u);
        if constexpr (CHECK) m[u] &= valid4(j0, sw, jlim, dl[u], act[u]);
    }
    if (!__any_sync(0xffffffffu, (m[0] | m[1]) != 0)) return;
    // Both targets' pairs are evaluated branch-free and interleaved (a path
    // per target set that has pairs, as the mixed form takes, made the FP64
    // kernel 1.4x slower: three copies of the FP64 pair terms).
    double r[4][3];
    bool any = false;
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
        const double4 pjv = tl[j0 + (jj ^ sw)];
        const double zj = (SIM == SIM_MIX) ? pjv.w : 1.0;
        PairOut<double> o[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const bool sel = ((m[u] >> jj) & 1u) != 0;
            if constexpr (TILEIMG) {
                ion_pair_tile<PREC_FP64, MEAS>(fa, pit[u], pjv, sel, o[u]);
            } else {
                const float2(&kx)[3] = jj < 2 ? ka[u] : kb[u];
                const float k[3] = {(jj & 1) ? kx[0].y : kx[0].x, (jj & 1) ? kx[1].y : kx[1].x,
                                    (jj & 1) ? kx[2].y : kx[2].x};
                ion_pair_nb<PREC_FP64, MEAS, true>(fa, pi[u], pjv, sel, k, o[u]);
            }
            acc[u].add(o[u], zj);
            any |= o[u].hit;
        }
        // reaction on j: Z_i fs d (int_ion_mix.f:180), both targets summed
        const double f0 = o[0].fs * wi[0], f1 = o[1].fs * wi[1];
        r[jj][0] = __fma_rn(f1, o[1].dx, f0 * o[0].dx);
        r[jj][1] = __fma_rn(f1, o[1].dy, f0 * o[0].dy);
        r[jj][2] = __fma_rn(f1, o[1].dz, f0 * o[0].dz);
    }
    if (__any_sync(0xffffffffu, any)) {
        double t[3];
        reduce_scatter4(r, t);
        const int lane = threadIdx.x & 31;
        const int jl = j0 + sw;
        if ((lane & 7) == 0 && (!CHECK || jl < jlim)) {
            my_acc[3 * jl] = -t[0];
            my_acc[3 * jl + 1] = -t[1];
            my_acc[3 * jl + 2] = -t[2];
        }
    }
}

// Job (R, C0, C1, sg) of k_force_pairs2: blocks R, R + 1 against source tiles
// C0 <= C < C1.  The tile pipeline, the warps' hand-off of a tile (done /
// used counters, the last warp sums the rows and refills the stage) and the
// abort path are those of pairs_job.  Returns false if a tile copy timed out.
template <int SIM, int PREC, bool MEAS, bool TB>
__device__ __forceinline__ bool pairs_job2(PairSmem<row_t<PREC>>& sm, const ForceArgs& fa, const BoxView& bx, int R,
                                           int C0, int C1, int sg, double* __restrict__ sm_row,
                                           unsigned* __restrict__ err, unsigned& q)
{
    static_assert(SIM == SIM_PURE || SIM == SIM_MIX || PREC == PREC_MIXED,
                  "two targets per thread: ions, or nucleons in the mixed form");
    constexpr bool ION = SIM == SIM_PURE || SIM == SIM_MIX;
    constexpr bool LO = PREC == PREC_MIXED;
    using R_t = real_t<PREC>;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int n = bx.n;
    int s[2];
    bool act[2];
    double4 pi[2];
    ScreenI si[2];
    R_t wi[2];
    float nli[2][3];
    int ii[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
        s[u] = 64 * warp + 32 * u + lane;
        const int i = R * PB + s[u];
        act[u] = i < n;
        ii[u] = act[u] ? i : 0;
        pi[u] = act[u] ? bx.pos[i] : make_double4(0.0, 0.0, 0.0, 0.0);
        si[u] = load_screen_i(bx.posf, act[u] ? i : 0);
        wi[u] = (SIM == SIM_MIX) ? (R_t)pi[u].w : (R_t)1;
#pragma unroll
        for (int c = 0; c < 3; ++c) nli[u][c] = LO ? -bx.posf[shadow_index(act[u] ? i : 0, 4 + c)] : 0.f;
    }
    const bool all_active = (R + 2) * PB <= n;
    const int sw = ((lane >> 4) & 1) * 2 + ((lane >> 3) & 1);
    const WarpBox box = warp_box2(fa, pi, act, !ION && ((act[0] && pi[0].w == 1.0) || (act[1] && pi[1].w == 1.0)));
    TargetAcc<PREC, MEAS> acc[2];
    acc[0].zero();
    acc[1].zero();
    // mixed ions, measuring: the lane's Z_i-weighted sums of both targets,
    // FP32 within a tile (pair_group_lo2), FP64 across tiles
    float ms[NSCAL];
    double msd[NSCAL];
#pragma unroll
    for (int k = 0; k < NSCAL; ++k) {
        ms[k] = 0.f;
        msd[k] = 0.0;
    }
    const bool tb = TB && bx.tbox != nullptr;

    if (tid == 0) {
        pairs_issue(sm, bx, C0, q, LO, tb);
        if (C0 + 1 < C1) pairs_issue(sm, bx, C0 + 1, q + 1, LO, tb);
    }
    const unsigned q0 = q;
    for (int C = C0; C < C1; ++C, ++q) {
        const int st = q & 1;
        if (!mbar_wait_abortable(&sm.bar[st], (q >> 1) & 1u, err, &sm.abort)) break;
        const int jlim = min(PB, n - C * PB);
        const int dC = (C - R) * PB;
        // pair (target u, source jl) counts iff jl > dl[u]
        const int dl[2] = {s[0] - dC, s[1] - dC};
        const int jmin = max(0, 64 * warp + 1 - dC);
        const bool full = dC >= PB2 && jlim == PB && all_active;
        const double4* tl = sm.tile[st];
        const float* tlf = sm.tilef[st];
        row_t<PREC>* my_acc = sm.acc_j[st][warp];
        bool used = false;
        const bool reach = box.any && jmin < jlim && (!tb || tile_reaches<SIM>(fa, box, sm.tb[st]));
        if constexpr (!ION) {
            if (reach) {
                unsigned gm = near_groups<SIM>(fa, box, tlf, jlim, jmin);
                used = gm != 0;
                if (used) {
#pragma unroll
                    for (int k = lane; k < PB * 3; k += 32) my_acc[k] = (row_t<PREC>)0;
                    __syncwarp();
                }
                const float* tll = reinterpret_cast<const float*>(tl);
                const double4* gsrc = bx.pos + (size_t)C * PB;
                if (full) {
                    for (; gm; gm &= gm - 1)
                        pair_group_nn_lo2<MEAS, false>(fa, si, nli, bx.pos, ii, tlf, tll, gsrc, 4 * (__ffs(gm) - 1),
                                                       jlim, dl, act, sw, acc, my_acc);
                } else {
                    for (; gm; gm &= gm - 1)
                        pair_group_nn_lo2<MEAS, true>(fa, si, nli, bx.pos, ii, tlf, tll, gsrc, 4 * (__ffs(gm) - 1),
                                                      jlim, dl, act, sw, acc, my_acc);
                }
            }
        }
        if (ION && reach) {
            int kcode = -1;
            unsigned gm = near_groups_img(fa, box, tlf, jlim, jmin, kcode);
            used = gm != 0;
            if (used) {
#pragma unroll
                for (int k = lane; k < PB * 3; k += 32) my_acc[k] = (row_t<PREC>)0;
                __syncwarp();
            }
            const bool timg = box.tile_img && kcode >= 0;
            // the tile's image folded into each target (exact on the hi grid)
            float th[2][3], tl2[2][3];
            double4 pit[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const float nh[3] = {si[u].nx, si[u].ny, si[u].nz};
                double pt[3];
                const double pc[3] = {pi[u].x, pi[u].y, pi[u].z};
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const float k = timg ? img_of(kcode, c) : 0.f;
                    th[u][c] = fmaf(-k, fa.Lh[c], nh[c]);
                    tl2[u][c] = fmaf(-k, fa.Ll[c], nli[u][c]);
                    pt[c] = LO ? 0.0 : __fma_rn((double)k, fa.xl[c], pc[c]);
                }
                pit[u] = make_double4(pt[0], pt[1], pt[2], pi[u].w);
            }
            if constexpr (LO) {
                const float* tll = reinterpret_cast<const float*>(tl);
                const float wf[2] = {(float)wi[0], (float)wi[1]};
                if (timg) {
                    if (full) {
                        for (; gm; gm &= gm - 1)
                            pair_group_lo2<SIM, MEAS, false, true>(fa, si, nli, th, tl2, wf, tlf, tll,
                                                                   4 * (__ffs(gm) - 1), jlim, dl, act, sw, acc,
                                                                   my_acc, ms);
                    } else {
                        for (; gm; gm &= gm - 1)
                            pair_group_lo2<SIM, MEAS, true, true>(fa, si, nli, th, tl2, wf, tlf, tll,
                                                                  4 * (__ffs(gm) - 1), jlim, dl, act, sw, acc,
                                                                  my_acc, ms);
                    }
                } else {
                    if (full) {
                        for (; gm; gm &= gm - 1)
                            pair_group_lo2<SIM, MEAS, false, false>(fa, si, nli, th, tl2, wf, tlf, tll,
                                                                    4 * (__ffs(gm) - 1), jlim, dl, act, sw, acc,
                                                                    my_acc, ms);
                    } else {
                        for (; gm; gm &= gm - 1)
                            pair_group_lo2<SIM, MEAS, true, false>(fa, si, nli, th, tl2, wf, tlf, tll,
                                                                   4 * (__ffs(gm) - 1), jlim, dl, act, sw, acc,
                                                                   my_acc, ms);
                    }
                }
                if constexpr (MEAS) {
#pragma unroll
                    for (int k = 0; k < NSCAL; ++k) {
                        msd[k] += (double)ms[k];
                        ms[k] = 0.f;
                    }
                }
            } else {
                if (timg) {
                    if (full) {
                        for (; gm; gm &= gm - 1)
                            pair_group2<SIM, MEAS, false, true>(fa, pi, si, th, pit, wi, tl, tlf, 4 * (__ffs(gm) - 1),
                                                                jlim, dl, act, sw, acc, my_acc);
                    } else {
                        for (; gm; gm &= gm - 1)
                            pair_group2<SIM, MEAS, true, true>(fa, pi, si, th, pit, wi, tl, tlf, 4 * (__ffs(gm) - 1),
                                                               jlim, dl, act, sw, acc, my_acc);
                    }
                } else {
                    if (full) {
                        for (; gm; gm &= gm - 1)
                            pair_group2<SIM, MEAS, false, false>(fa, pi, si, th, pit, wi, tl, tlf,
                                                                 4 * (__ffs(gm) - 1), jlim, dl, act, sw, acc, my_acc);
                    } else {
                        for (; gm; gm &= gm - 1)
                            pair_group2<SIM, MEAS, true, false>(fa, pi, si, th, pit, wi, tl, tlf,
                                                                4 * (__ffs(gm) - 1), jlim, dl, act, sw, acc, my_acc);
                    }
                }
            }
        }
        if (lane == 0) sm.used[st][warp] = used ? 1 : 0;
        // this warp is done with the tile: the last warp reduces and refills
        __threadfence_block();
        __syncwarp();
        int last = 0;
        if (lane == 0) last = atomicAdd(&sm.done[st], 1) == PWARPS - 1;
        last = __shfl_sync(0xffffffffu, last, 0);
        if (last) {
            __threadfence_block();
            if (lane == 0) sm.done[st] = 0;
            unsigned um = 0;
#pragma unroll
            for (int w = 0; w < PWARPS; ++w) um |= (unsigned)sm.used[st][w] << w;
            const long long u = tri_index(C, R);
            if (um == 0) {
                if (lane == 0) bx.Sjf[u] = 0;
            } else {
                // both blocks' reactions on tile C, the used warp rows in warp
                // order, into unit (R, C)'s row
                row_t<PREC>* dj = static_cast<row_t<PREC>*>(bx.Sj) + (size_t)u * PB * 3;
#pragma unroll 4
                for (int k = lane; k < 3 * PB; k += 32) {
                    double v = 0.0;
#pragma unroll
                    for (int w = 0; w < PWARPS; ++w)
                        if ((um >> w) & 1u) v += sm.acc_j[st][w][k];
                    dj[k] = (row_t<PREC>)v;
                }
                if (lane == 0) bx.Sjf[u] = 1;
            }
            // unit (R + 1, C) has no row of its own
            if (lane == 0 && C > R && R + 1 < bx.M) bx.Sjf[tri_index(C, R + 1)] = 0;
            __syncwarp();
            if (lane == 0 && C + 2 < C1) pairs_issue(sm, bx, C + 2, q + 2, LO, tb);
        }
    }
    q = q0 + (unsigned)(C1 - C0);
    if (__syncthreads_or(sm.abort)) return false;
    // target-side partials of job (R, sg): warps 0, 1 hold block R, warps 2, 3
    // block R + 1
    const int Rb = R + (warp >> 1);
    if (Rb < bx.M) {
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            double* di = bx.Si + (((size_t)Rb * bx.nseg_max + sg) * PB + (s[u] & (PB - 1))) * 3;
            di[0] = acc[u].force(0);
            di[1] = acc[u].force(1);
            di[2] = acc[u].force(2);
        }
    }
    if constexpr (MEAS) {
        double S[NSCAL];
#pragma unroll
        for (int k = 0; k < NSCAL; ++k) {
            if constexpr (LO && ION) S[k] = msd[k];           // already weighted by Z_i
            else S[k] = (act[0] ? acc[0].scal(k) * (double)wi[0] : 0.0) +
                        (act[1] ? acc[1].scal(k) * (double)wi[1] : 0.0);
        }
        block_sum_store<NSCAL>(S, sm.red, sm_row);
        __syncthreads();
    }
    return true;
}

// Resident CTAs per SM of k_force_pairs2 (registers: the per-target state
// is doubled).
template <int PREC, bool MEAS>
constexpr int pairs2_ctas_per_sm()
{
    return 4;
}

// Two targets per thread (yk_tuning.targets_per_thread = 2): jobs over block
// pairs (R, R + 1); PREC_FP64 on fa.img_k boxes, PREC_MIXED on fa.lo boxes.
// pj.Sjf is required.
template <int SIM, int PREC, bool MEAS>
__global__ void __launch_bounds__(PB, (pairs2_ctas_per_sm<PREC, MEAS>()))
k_force_pairs2(const double4* __restrict__ pos, const float* __restrict__ posf, PairJobs pj,
               int* __restrict__ job_counter, ForceArgs fa, double* __restrict__ Si,
               row_t<PREC>* __restrict__ Sj, double* __restrict__ Sm, unsigned* __restrict__ err)
{
    __shared__ __align__(128) PairSmem<row_t<PREC>> sm;
    pairs_smem_init(sm);
    BoxView bx;
    bx.pos = pos;
    bx.posf = posf;
    bx.Si = Si;
    bx.Sj = Sj;
    bx.tbox = pj.tbox;
    bx.Sjf = pj.Sjf;
    bx.n = fa.n;
    bx.M = pj.M;
    bx.nseg_max = pj.nseg_max;
    unsigned q = 0;
    for (;;) {
        if (threadIdx.x == 0) sm.s_job = atomicAdd(job_counter, 1);
        __syncthreads();
        const int job = sm.s_job;
        if (job >= pj.njobs) break;
        const int4 js = pj.jobs[job];
        constexpr bool TB = pairs_tile_boxes<SIM, PREC, PREC == PREC_MIXED>();
        if (!pairs_job2<SIM, PREC, MEAS, TB>(sm, fa, bx, js.x, js.y, js.z, js.w, Sm + (size_t)job * NSCAL, err, q))
            return;
    }
}

}  // namespace yk
