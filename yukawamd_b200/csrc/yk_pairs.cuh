// yk_pairs.cuh -- half-pair force kernel (Newton's third law) and its combine.
//
// The reference evaluates each unique pair once and scatters the reaction
// onto the source particle (fi += fcx; fj(:,j) -= fcx, int_ion_pure.f:160-161).
// k_force_pairs does the same on tiles of PB = 128 slots:
//
//   unit (R, C), C >= R : target block R (one slot per thread, position and
//                         sums in registers) against source tile C (one 1-D
//                         TMA bulk copy into shared memory, double-buffered).
//                         On the diagonal unit only pairs j > i count.
//   job  (R, C0, C1, s) : units C0 <= C < C1 of row R, writing Si slot s of
//                         the row; persistent CTAs pull jobs from an atomic
//                         counter in the order of the job table (long jobs
//                         first, shrinking towards the end: the engine's
//                         build_pair_jobs).
//
// Reaction sums: each warp sweeps the whole tile in groups of 4 sources.  In
// step jj of a group, lane L takes source jj ^ sw(L), sw(L) = 2*bit4(L) +
// bit3(L), so its reaction on the group's source sw(L) ends in register slot
// 0, and the slots that a halving exchange sends are the same for every lane
// (slots 2,3 over xor 16, then slot 1 over xor 8): the warp sums the 32
// lanes' reactions on the 4 sources with that reduce-scatter plus a 3-level
// butterfly (18 shuffles of 3-vector components per group instead of 4 x 15,
// no selects; FP64 in the FP64 form, FP32 in the mixed form), and lanes
// 0/8/16/24 write the four sums into the warp's own row in shared memory.
// The 4 warp rows are added in a fixed order at the end of the tile by the
// warp that finishes it last, so no atomics and no per-tile block barrier.
// A warp first skips the 4-source groups that cannot reach the bounding box
// of its targets (near_groups); the others are screened per pair on the FP32
// shadow positions, two sources per packed FP32x2 instruction, and only groups
// with a candidate take the pair terms (pair_group; pair_group_lo for the
// mixed form's ions).
//
// Outputs are partial sums in scratch (nothing is accumulated atomically):
//   Si[R][s][PB][3]       target-side sums of job (R, ., ., s)
//   Sj[tri(C,R)][PB][3]   source-side sums of unit (R, C), tri(C,R) = C(C+1)/2+R
//   Sm[job][8]            measurement sums of the job (U, W, P tensor)
// k_combine adds, for every slot, its Si and Sj entries in a fixed order
// (two interleaved groups, then the group sums), applies the reference's
// scaling and scatters to the caller's particle order.  Results are
// therefore bit-reproducible, independent of which CTA ran which job.
#pragma once

#include "yk_force.cuh"

namespace yk {

constexpr int PB = 128;           // slots per block / tile (= threads per CTA)
constexpr int PWARPS = PB / 32;

// Type of the per-warp reaction rows: a row entry is one reduce-scatter
// result, FP64 in the FP64 form and FP32 in the mixed form, so either type
// holds it exactly.
template <int PREC>
using row_t = std::conditional_t<PREC == PREC_FP64, double, float>;

struct PairJobs {
    const int4* jobs;             // (R, C0, C1, slot) per job, costliest first:
                                  // target block R, source tiles C0 <= C < C1,
                                  // Si slot of row R that the job writes
    const int* row_slots;         // Si slots written per row R
    int njobs;
    int M;                        // tiles
    int nseg_max;                 // Si slots per row in the layout (max of row_slots)
    // optional (null: every warp screens every tile, every Sj row is written):
    const float* tbox;            // per tile: centre[3], pad, half-width[3], pad (k_tile_boxes)
    unsigned char* Sjf;           // per unit tri(C,R): 1 if its Sj row was written,
                                  // 0 if the row is zero and was not written
};

// Bounding box of each 128-slot tile on the FP32 shadow hi parts (the
// coordinates near_groups screens), with the warp box's rounding margin:
// one CTA of PB threads per tile.
static __global__ void __launch_bounds__(PB)
k_tile_boxes(const float* __restrict__ posf, int n, ForceArgs fa, float* __restrict__ tbox)
{
    __shared__ float red[PWARPS][6];
    const int C = blockIdx.x, j = threadIdx.x, lane = j & 31, warp = j >> 5;
    const float inf = __int_as_float(0x7f800000);
    const bool on = C * PB + j < n;
    const float* t = posf + (size_t)C * SHADOW_FLOATS;
    float lo[3], hi[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float v = t[shadow_off(j, k)];
        float a = on ? v : inf, b = on ? v : -inf;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a = fminf(a, __shfl_xor_sync(0xffffffffu, a, o));
            b = fmaxf(b, __shfl_xor_sync(0xffffffffu, b, o));
        }
        lo[k] = a;
        hi[k] = b;
    }
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            red[warp][k] = lo[k];
            red[warp][3 + k] = hi[k];
        }
    __syncthreads();
    if (j < 3) {
        float a = red[0][j], b = red[0][3 + j];
#pragma unroll
        for (int w = 1; w < PWARPS; ++w) {
            a = fminf(a, red[w][j]);
            b = fmaxf(b, red[w][3 + j]);
        }
        const float mu = fmaf(3.814697265625e-6f, fa.Lf[j], (float)(2.0 * SHADOW_Q));
        tbox[8 * C + j] = 0.5f * (a + b);
        tbox[8 * C + 4 + j] = fmaf(0.5f, b - a, mu);
    } else if (j == 3 || j == 7) {
        tbox[8 * C + j] = 0.f;
    }
}

__host__ __device__ __forceinline__ long long tri_index(int C, int R)
{
    return (long long)C * (C + 1) / 2 + R;
}

template <int PREC>
__device__ __forceinline__ double to_f64(real_t<PREC> v)
{
    return (double)v;
}

// FP32 form of reduce_scatter4 below with the adds paired into FP32x2
// instructions (the same sums in the same order); ra holds slots 0 and 1,
// rb slots 2 and 3.
__device__ __forceinline__ void reduce_scatter4_x2(const float2 (&ra)[3], const float2 (&rb)[3], float (&t)[3])
{
    float2 a[3];
#pragma unroll
    for (int c = 0; c < 3; ++c)
        a[c] = __fadd2_rn(ra[c], make_float2(__shfl_xor_sync(0xffffffffu, rb[c].x, 16),
                                             __shfl_xor_sync(0xffffffffu, rb[c].y, 16)));
    float2 t01 = __fadd2_rn(make_float2(a[0].x, a[1].x),
                            make_float2(__shfl_xor_sync(0xffffffffu, a[0].y, 8),
                                        __shfl_xor_sync(0xffffffffu, a[1].y, 8)));
    float t2 = a[2].x + __shfl_xor_sync(0xffffffffu, a[2].y, 8);
#pragma unroll
    for (int m = 4; m > 0; m >>= 1) {
        t01 = __fadd2_rn(t01, make_float2(__shfl_xor_sync(0xffffffffu, t01.x, m),
                                          __shfl_xor_sync(0xffffffffu, t01.y, m)));
        t2 += __shfl_xor_sync(0xffffffffu, t2, m);
    }
    t[0] = t01.x;
    t[1] = t01.y;
    t[2] = t2;
}

__device__ __forceinline__ void reduce_scatter4(float (&r)[4][3], float (&t)[3])
{
    float2 ra[3], rb[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        ra[c] = make_float2(r[0][c], r[1][c]);
        rb[c] = make_float2(r[2][c], r[3][c]);
    }
    reduce_scatter4_x2(ra, rb, t);
}

// Reduce-scatter of four 3-vectors held in lane-swizzled slots (slot q of
// lane L belongs to source q ^ sw(L)).  On return t[] holds the warp-wide sum
// for source sw(L).  T is double for the FP64 form and float for the mixed
// form (whose reaction terms are FP32 products).
template <typename T>
__device__ __forceinline__ void reduce_scatter4(T (&r)[4][3], T (&t)[3])
{
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const T a0 = r[0][c] + __shfl_xor_sync(0xffffffffu, r[2][c], 16);
        const T a1 = r[1][c] + __shfl_xor_sync(0xffffffffu, r[3][c], 16);
        t[c] = a0 + __shfl_xor_sync(0xffffffffu, a1, 8);
    }
#pragma unroll
    for (int m = 4; m > 0; m >>= 1)
#pragma unroll
        for (int c = 0; c < 3; ++c) t[c] += __shfl_xor_sync(0xffffffffu, t[c], m);
}

// One group of 4 sources j0..j0+3 for the calling lane's target, taken in
// the lane's swizzled order: step jj handles source j0 + (jj ^ sw).  The
// screen runs in the same order from the paired shadow layout (steps 0, 1
// are the ordered pair at offset 2 sw of the group's blocks, steps 2, 3 the
// one at 2 (sw ^ 2)), so each step's image integers are plain registers.
// CHECK: the tile is partial, diagonal, or the CTA has inactive targets, so
// every pair needs the validity test.
// TILEIMG (ions): the tile's reachable sources share one image, folded into
// th (the screen's target hi parts) and pit (the FP64 target position), so no
// pair takes its own image.
template <int SIM, int PREC, bool MEAS, bool CHECK, bool IMGK = false, bool TILEIMG = false>
__device__ __forceinline__ void pair_group(const ForceArgs& fa, const double4& pi, const ScreenI& si,
                                           real_t<PREC> wi, const double4* tl, const float* tlf,
                                           int j0, int jlim, bool diag, bool active, int tid,
                                           int sw, TargetAcc<PREC, MEAS>& acc, row_t<PREC>* my_acc,
                                           const float2 (&th)[3] = {}, const double4& pit = double4{})
{
    using R_t = real_t<PREC>;
    const int g = j0 >> 2;
    float2 ka[3], kb[3];
    float2 ra, rb;
    if constexpr (TILEIMG) {
        ra = screen_r2_tile_x2(th, tlf, g, 2 * sw);
        rb = screen_r2_tile_x2(th, tlf, g, 2 * (sw ^ 2));
    } else {
        ra = screen_r2k_x2(fa, si, tlf, g, 2 * sw, ka);
        rb = screen_r2k_x2(fa, si, tlf, g, 2 * (sw ^ 2), kb);
    }
    const float* tw = tlf + 6 * SHADOW_TILE + j0;
    unsigned m = (ra.x <= screen_lim<SIM>(fa, si.w, tw[sw]) ? 1u : 0u) |
                 (ra.y <= screen_lim<SIM>(fa, si.w, tw[sw ^ 1]) ? 2u : 0u) |
                 (rb.x <= screen_lim<SIM>(fa, si.w, tw[sw ^ 2]) ? 4u : 0u) |
                 (rb.y <= screen_lim<SIM>(fa, si.w, tw[sw ^ 3]) ? 8u : 0u);
    if constexpr (CHECK) {
        unsigned ok = 0;
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            const int jl = j0 + (jj ^ sw);
            if (active && jl < jlim && (!diag || jl > tid)) ok |= 1u << jj;
        }
        m &= ok;
    }
    if (!__any_sync(0xffffffffu, m != 0)) return;
    R_t r[4][3];
    GroupSum<PREC, MEAS> gs;             // the mixed form adds the group, then compensates
    gs.zero();
    bool any = false;
    if constexpr (SIM == SIM_PURE || SIM == SIM_MIX) {
        // Ions: the 4 pairs are evaluated without branches, so that their
        // independent instruction chains interleave; a pair the screen did
        // not select, or outside r_c, gets zero terms.
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            const double4 pjv = tl[j0 + (jj ^ sw)];
            PairOut<R_t> o;
            if constexpr (TILEIMG) {
                ion_pair_tile<PREC, MEAS>(fa, pit, pjv, ((m >> jj) & 1u) != 0, o);
            } else {
                const float k[3] = {jj == 0 ? ka[0].x : jj == 1 ? ka[0].y : jj == 2 ? kb[0].x : kb[0].y,
                                    jj == 0 ? ka[1].x : jj == 1 ? ka[1].y : jj == 2 ? kb[1].x : kb[1].y,
                                    jj == 0 ? ka[2].x : jj == 1 ? ka[2].y : jj == 2 ? kb[2].x : kb[2].y};
                ion_pair_nb<PREC, MEAS, IMGK>(fa, pi, pjv, ((m >> jj) & 1u) != 0, k, o);
            }
            if constexpr (PREC == PREC_FP64) acc.add(o, SIM == SIM_MIX ? (R_t)pjv.w : (R_t)1);
            else gs.add(o, SIM == SIM_MIX ? (R_t)pjv.w : (R_t)1);
            const R_t fsj = o.fs * wi;               // 0 unless the pair interacts
            r[jj][0] = fsj * o.dx;
            r[jj][1] = fsj * o.dy;
            r[jj][2] = fsj * o.dz;
            any |= o.hit;
        }
    } else {
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            r[jj][0] = r[jj][1] = r[jj][2] = (R_t)0;
            if ((m >> jj) & 1u) {
                const double4 pjv = tl[j0 + (jj ^ sw)];
                PairOut<R_t> o;
                pair_eval<SIM, PREC, MEAS>(fa, pi, pjv, true, o);
                if (o.hit) {
                    if constexpr (PREC == PREC_FP64) acc.add(o, (R_t)1);
                    else gs.add(o, (R_t)1);
                    const R_t fsj = o.fs * wi;
                    r[jj][0] = fsj * o.dx;
                    r[jj][1] = fsj * o.dy;
                    r[jj][2] = fsj * o.dz;
                    any = true;
                }
            }
        }
    }
    if constexpr (PREC == PREC_MIXED) acc.add_group(gs);
    if (__any_sync(0xffffffffu, any)) {
        // reaction on j: Z_i fs d (int_ion_mix.f:180); slot jj of lane L
        // belongs to source jj ^ sw(L), as reduce_scatter4 expects
        R_t t[3];
        reduce_scatter4(r, t);
        const int lane = threadIdx.x & 31;
        const int jl = j0 + sw;
        if ((lane & 7) == 0 && (!CHECK || jl < jlim)) {
            // a warp visits each group of a tile once, so this is the row
            // entry's only write (rows start at zero for skipped groups)
            my_acc[3 * jl] = -t[0];
            my_acc[3 * jl + 1] = -t[1];
            my_acc[3 * jl + 2] = -t[2];
        }
    }
}

// pair_group for ions in the mixed form when the box allows the FP32
// displacement (fa.lo): the screen computes the final displacement and r^2
// (screen_d_x2), so its mask is the cutoff test itself and the pair terms
// need no FP64 source tile.  tll is the tile's lo part, nli the target's
// negated lo parts.  TILEIMG: the tile's reachable sources share one image,
// folded into th / tl2 (disp_tile_x2), so no pair takes its own image.
template <int SIM, bool MEAS, bool CHECK, bool TILEIMG = false>
__device__ __forceinline__ void pair_group_lo(const ForceArgs& fa, const ScreenI& si, const float (&nli)[3],
                                              const float2 (&th)[3], const float2 (&tl2)[3],
                                              float wi, const float* tlf, const float* tll, int j0, int jlim,
                                              bool diag, bool active, int tid, int sw,
                                              TargetAcc<PREC_MIXED, MEAS>& acc, float* my_acc)
{
    const int g = j0 >> 2;
    float2 da[3], db[3];
    float2 ra, rb;
    if constexpr (TILEIMG) {
        ra = disp_tile_x2(th, tl2, tlf, tll, g, 2 * sw, da);
        rb = disp_tile_x2(th, tl2, tlf, tll, g, 2 * (sw ^ 2), db);
    } else {
        ra = screen_d_x2(fa, si, nli, tlf, tll, g, 2 * sw, da);
        rb = screen_d_x2(fa, si, nli, tlf, tll, g, 2 * (sw ^ 2), db);
    }
    unsigned m = (ra.x <= fa.rc2f ? 1u : 0u) | (ra.y <= fa.rc2f ? 2u : 0u) | (rb.x <= fa.rc2f ? 4u : 0u) |
                 (rb.y <= fa.rc2f ? 8u : 0u);
    if constexpr (CHECK) {
        unsigned ok = 0;
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            const int jl = j0 + (jj ^ sw);
            if (active && jl < jlim && (!diag || jl > tid)) ok |= 1u << jj;
        }
        m &= ok;
    }
    if (!__any_sync(0xffffffffu, m != 0)) return;
    // The four pairs in two FP32x2 halves: a = steps 0, 1 and b = steps 2, 3
    // (the screen's ra, da and rb, db).  d = x_j - x_i, so the target's terms
    // carry a minus sign: F_i += fs Z_j (x_i - x_j) = -fs Z_j d
    // (int_ion_mix.f:179), and the reaction on j is fs Z_i d (:180).
    const float* tw = tlf + 6 * SHADOW_TILE + j0;
    const float2 mska = make_float2((m & 1u) ? 1.f : 0.f, (m & 2u) ? 1.f : 0.f);
    const float2 mskb = make_float2((m & 4u) ? 1.f : 0.f, (m & 8u) ? 1.f : 0.f);
    float2 fsa, ua, wa, fsb, ub, wb;
    ion_terms_x2<MEAS>(fa, ra, mska, fsa, ua, wa);
    ion_terms_x2<MEAS>(fa, rb, mskb, fsb, ub, wb);
    const float2 wja = (SIM == SIM_MIX) ? make_float2(tw[sw], tw[sw ^ 1]) : make_float2(1.f, 1.f);
    const float2 wjb = (SIM == SIM_MIX) ? make_float2(tw[sw ^ 2], tw[sw ^ 3]) : make_float2(1.f, 1.f);
    const float2 ga = __fmul2_rn(fsa, wja), gb = __fmul2_rn(fsb, wjb);
    GroupSum<PREC_MIXED, MEAS> gs;
    float2 fxa[3], fxb[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        if constexpr (MEAS) {
            // the products are kept for the pressure tensor
            fxa[c] = __fmul2_rn(ga, da[c]);
            fxb[c] = __fmul2_rn(gb, db[c]);
            const float2 sc = __fadd2_rn(fxa[c], fxb[c]);
            gs.f[c] = -(sc.x + sc.y);
        } else {
            const float2 sc = __ffma2_rn(gb, db[c], __fmul2_rn(ga, da[c]));
            gs.f[c] = -(sc.x + sc.y);
        }
    }
    if constexpr (MEAS) {
        const float2 su = __ffma2_rn(ub, wjb, __fmul2_rn(ua, wja));
        const float2 sv = __ffma2_rn(wb, wjb, __fmul2_rn(wa, wja));
        gs.s[0] = su.x + su.y;
        gs.s[1] = sv.x + sv.y;
        // pressure tensor d (x) (fs Z_j d): the two minus signs cancel
        const int P[6] = {0, 0, 0, 1, 1, 2}, Q[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const float2 sp = __ffma2_rn(db[P[k]], fxb[Q[k]], __fmul2_rn(da[P[k]], fxa[Q[k]]));
            gs.s[2 + k] = sp.x + sp.y;
        }
    }
    acc.add_group2(gs);
    const float2 wi2 = make_float2(wi, wi);
    const float2 ha = __fmul2_rn(fsa, wi2), hb = __fmul2_rn(fsb, wi2);
    float2 ra3[3], rb3[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        ra3[c] = __fmul2_rn(ha, da[c]);
        rb3[c] = __fmul2_rn(hb, db[c]);
    }
    float t[3];
    reduce_scatter4_x2(ra3, rb3, t);
    const int lane = threadIdx.x & 31;
    const int jl = j0 + sw;
    if ((lane & 7) == 0 && (!CHECK || jl < jlim)) {
        // a warp visits each group of a tile once, so this is the row
        // entry's only write (rows start at zero for skipped groups)
        my_acc[3 * jl] = t[0];
        my_acc[3 * jl + 1] = t[1];
        my_acc[3 * jl + 2] = t[2];
    }
}

// pair_group for nucleons in the mixed form (fa.hilo): the hi/lo FP32
// displacement with the screen's image integers (screen_d_flag_x2); the
// pairs that the screen flags as close to |d| = L/2 on some axis take the
// reference's conditional minimum image on the FP64 positions instead
// (int_nn.f:190-195; gsrc is the tile's FP64 slots in global memory), so every
// pair gets the reference's image.  Then the HPP terms inside rncut and the
// p-p Coulomb inside rccut (int_nn.f:208-229), two pairs per FP32x2
// instruction, a branch per term only when no lane of the warp needs it.
// MODE (warp-uniform, from the species of the warp's targets and the tile's
// sources; slots are in species-major order, so nearly every warp and tile
// holds one species):
//   NN_ANY  any species;
//   NN_NOP  no proton target (and fa.nn_short): no Coulomb term, and no flag
//           test, since a pair near |d| = L/2 is beyond the nuclear range
//           under either image;
//   NN_PP   proton targets and proton sources only, the Coulomb term on and
//           uncut (fa.coul_all): every pair is a like pair and takes the
//           Coulomb term, no species or cutoff tests (and on a full tile no
//           masks in the Coulomb terms).
constexpr int NN_ANY = 0, NN_NOP = 1, NN_PP = 2;

template <bool MEAS, bool CHECK, int MODE = NN_ANY>
__device__ __forceinline__ void pair_group_nn_lo(const ForceArgs& fa, const ScreenI& si, const float (&nli)[3],
                                                 const double4& pi, const float* tlf, const float* tll,
                                                 const double4* __restrict__ gsrc, int j0, int jlim, bool diag,
                                                 bool active, int tid, int sw, TargetAcc<PREC_MIXED, MEAS>& acc,
                                                 float* my_acc)
{
    const int g = j0 >> 2;
    float2 da[3], db[3];
    unsigned fla = 0, flb = 0;
    float2 ra, rb;
    if constexpr (MODE == NN_NOP) {
        ra = screen_d_x2(fa, si, nli, tlf, tll, g, 2 * sw, da);
        rb = screen_d_x2(fa, si, nli, tlf, tll, g, 2 * (sw ^ 2), db);
    } else {
        ra = screen_d_flag_x2(fa, si, nli, tlf, tll, g, 2 * sw, da, fla);
        rb = screen_d_flag_x2(fa, si, nli, tlf, tll, g, 2 * (sw ^ 2), db, flb);
    }
    unsigned ok = 0xfu;
    if constexpr (CHECK) {
        ok = 0;
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            const int jl = j0 + (jj ^ sw);
            if (active && jl < jlim && (!diag || jl > tid)) ok |= 1u << jj;
        }
    }
    const unsigned fl = (fla | (flb << 2)) & ok;
    if (MODE != NN_NOP && __any_sync(0xffffffffu, fl != 0)) {
        // d = x_j - x_i from the reference's d = x_i - x_j and its image
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            if ((fl >> jj) & 1u) {
                const double4 pj = gsrc[j0 + (jj ^ sw)];
                const float ex = -__double2float_rn(min_image(__dsub_rn(pi.x, pj.x), fa.xl[0], fa.hlb[0]));
                const float ey = -__double2float_rn(min_image(__dsub_rn(pi.y, pj.y), fa.xl[1], fa.hlb[1]));
                const float ez = -__double2float_rn(min_image(__dsub_rn(pi.z, pj.z), fa.xl[2], fa.hlb[2]));
                const float r2 = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
                float2(&dd)[3] = jj < 2 ? da : db;
                float2& rr = jj < 2 ? ra : rb;
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
    const float* tw = tlf + 6 * SHADOW_TILE + j0;
    float wj[4];
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) wj[jj] = MODE == NN_PP ? 1.0f : tw[jj ^ sw];
    const float r2v[4] = {ra.x, ra.y, rb.x, rb.y};
    const bool ip = MODE == NN_PP || si.w == 1.0f;
    unsigned mn = 0, mc = 0;
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
        const bool in = (ok >> jj) & 1u;
        if (in && fa.nuclear_on && r2v[jj] <= fa.rn2f) mn |= 1u << jj;
        if constexpr (MODE == NN_PP) {
            if (in) mc |= 1u << jj;
        } else if constexpr (MODE == NN_ANY) {
            if (in && fa.coulomb_on && ip && wj[jj] == 1.0f && r2v[jj] <= fa.rc2f) mc |= 1u << jj;
        }
    }
    const bool any_n = __any_sync(0xffffffffu, mn != 0);
    const bool any_c = MODE != NN_NOP && __any_sync(0xffffffffu, mc != 0);
    if (!any_n && !any_c) return;
    float2 fsa = make_float2(0.f, 0.f), fsb = fsa, ua = fsa, ub = fsa, wa = fsa, wb = fsa;
    if (any_n) {
        float2 Ba, Bb;
        if constexpr (MODE == NN_PP) {
            Ba = Bb = make_float2(fa.bpcf, fa.bpcf);
        } else {
            Ba = make_float2(wj[0] == si.w ? fa.bpcf : fa.bmcf, wj[1] == si.w ? fa.bpcf : fa.bmcf);
            Bb = make_float2(wj[2] == si.w ? fa.bpcf : fa.bmcf, wj[3] == si.w ? fa.bpcf : fa.bmcf);
        }
        nuclear_terms_x2<MEAS>(fa, ra, make_float2((mn & 1u) ? 1.f : 0.f, (mn & 2u) ? 1.f : 0.f), Ba, fsa, ua, wa);
        nuclear_terms_x2<MEAS>(fa, rb, make_float2((mn & 4u) ? 1.f : 0.f, (mn & 8u) ? 1.f : 0.f), Bb, fsb, ub, wb);
    }
    if (any_c) {
        // proton pairs of a full tile: every pair takes the term, no masks
        constexpr bool MASKED = !(MODE == NN_PP && !CHECK);
        coulomb_terms_x2<MEAS, MASKED>(fa, ra, make_float2((mc & 1u) ? 1.f : 0.f, (mc & 2u) ? 1.f : 0.f), fsa, ua,
                                       wa);
        coulomb_terms_x2<MEAS, MASKED>(fa, rb, make_float2((mc & 4u) ? 1.f : 0.f, (mc & 8u) ? 1.f : 0.f), fsb, ub,
                                       wb);
    }
    // F_i += fs (x_i - x_j) = -fs d (int_nn.f:230-240); the reaction on j is fs d
    GroupSum<PREC_MIXED, MEAS> gs;
    float2 fxa[3], fxb[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        fxa[c] = __fmul2_rn(fsa, da[c]);
        fxb[c] = __fmul2_rn(fsb, db[c]);
        const float2 sc = __fadd2_rn(fxa[c], fxb[c]);
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
            const float2 sp = __ffma2_rn(db[P[k]], fxb[Q[k]], __fmul2_rn(da[P[k]], fxa[Q[k]]));
            gs.s[2 + k] = sp.x + sp.y;
        }
    }
    acc.add_group2(gs);
    float t[3];
    reduce_scatter4_x2(fxa, fxb, t);
    const int lane = threadIdx.x & 31;
    const int jl = j0 + sw;
    if ((lane & 7) == 0 && (!CHECK || jl < jlim)) {
        my_acc[3 * jl] = t[0];
        my_acc[3 * jl + 1] = t[1];
        my_acc[3 * jl + 2] = t[2];
    }
}

// ---- which source groups can reach a warp's targets ----------------------
// The bounding box of a warp's active targets (FP32 copies), computed once per
// job; a source farther than the screening radius from the box (in the
// minimum image, with a margin that covers the rounding of the FP32 copies)
// interacts with none of the 32 targets.  near_groups() classifies a tile's
// 128 sources against the box, one source per lane at a time, and returns a
// 32-bit mask of the 4-source groups that have at least one source within
// reach; the other groups skip even the per-pair FP32 screen.
struct WarpBox {
    float lo[3], hi[3];
    float c[3], h[3];                // centre and half-width plus the rounding margin
    bool any, has_p;                 // any active target; any proton target (nucleons)
    // 2 (r_c + h) < L - 2 fm on every axis: then the one image of a tile's
    // reachable sources seen from the centre is the minimum image of every
    // pair inside r_c (near_groups_img)
    bool tile_img;
};

__device__ __forceinline__ float warp_minf(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ float warp_maxf(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// The warp's box from each lane's lower and upper corner (+inf / -inf for a
// lane without active targets).
__device__ __forceinline__ WarpBox warp_box_of(const ForceArgs& fa, const float (&lo)[3], const float (&hi)[3],
                                               bool active, bool proton)
{
    WarpBox b;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        b.lo[k] = warp_minf(lo[k]);
        b.hi[k] = warp_maxf(hi[k]);
        // margin: 2^-18 L for the FP32 arithmetic (the box, its centre and
        // the source's minimum image are each a few roundings of values below
        // L) plus 2 SHADOW_Q for the grid rounding of the shadow coordinate
        const float mu = fmaf(3.814697265625e-6f, fa.Lf[k], (float)(2.0 * SHADOW_Q));
        b.c[k] = 0.5f * (b.lo[k] + b.hi[k]);
        b.h[k] = fmaf(0.5f, b.hi[k] - b.lo[k], mu);
    }
    b.any = __any_sync(0xffffffffu, active);
    b.has_p = __any_sync(0xffffffffu, proton);
    // A pair inside r_c has |d| <= r_c < L/2 per axis in its minimum image.
    // Seen from the centre, a reachable source lies within r_c + h per axis
    // of the image k that the centre gives it, and a target within h, so the
    // pair's displacement with image k is within r_c + 2h < L - r_c per axis:
    // any other image would put the pair farther than L - r_c > r_c, so k is
    // the pair's minimum image.  Pairs outside r_c stay outside under any
    // image.  (scr_c2 is the widened screening radius; 1 fm of slack.)
    bool ok = true;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float t = 0.5f * fa.Lf[k] - b.h[k] - 1.0f;
        ok = ok && t > 0.f && t * t > fa.scr_c2;
    }
    b.tile_img = ok;
    return b;
}

// The box of a warp with one target per lane.
__device__ __forceinline__ WarpBox warp_box(const ForceArgs& fa, const double4& pi, bool active)
{
    const float inf = __int_as_float(0x7f800000);
    const double c[3] = {pi.x, pi.y, pi.z};
    float lo[3], hi[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float v = __double2float_rn(c[k]);
        lo[k] = active ? v : inf;
        hi[k] = active ? v : -inf;
    }
    return warp_box_of(fa, lo, hi, active, active && pi.w == 1.0);
}

// Lower bound of the minimum-image distance^2 from source (x, w) to the box:
// per axis, the minimum image of x - c, less the half-width.  The images of
// the box interval all have the same width, so the nearest is the one whose
// centre is nearest; a box at least L wide gives 0.
template <int SIM>
__device__ __forceinline__ bool box_reaches(const ForceArgs& fa, const WarpBox& b, const float (&x)[3], float w)
{
    const float MAGIC = 12582912.0f;
    float dist2 = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float d = x[k] - b.c[k];
        const float dm = fmaf(-fa.Lf[k], fmaf(d, fa.invLf[k], MAGIC) - MAGIC, d);
        const float m = fmaxf(fabsf(dm) - b.h[k], 0.f);
        dist2 = fmaf(m, m, dist2);
    }
    float lim;
    if constexpr (SIM == SIM_PURE || SIM == SIM_MIX) {
        lim = fa.scr_c2;
    } else {
        const bool pp = b.has_p && w == 1.0f && fa.coulomb_on;
        lim = pp ? fmaxf(fa.scr_c2, fa.scr_n2) : fa.scr_n2;
    }
    return dist2 <= lim;
}

// Whether any source of a tile can reach the warp's box: the box_reaches
// bound with the tile's box in place of the source.  Per axis the minimum-
// image distance is a metric, so a source within the tile's half-width tb[4+k]
// of its centre tb[k] is at least |mi(tb[k] - c)| - tb[4+k] from the warp
// centre: if the boxes are out of reach, so is every source of the tile.
// (Nucleons: the Coulomb radius counts if the warp has a proton target.)
template <int SIM>
__device__ __forceinline__ bool tile_reaches(const ForceArgs& fa, const WarpBox& b, const float* tb)
{
    const float MAGIC = 12582912.0f;
    float dist2 = 0.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float d = tb[k] - b.c[k];
        const float dm = fmaf(-fa.Lf[k], fmaf(d, fa.invLf[k], MAGIC) - MAGIC, d);
        const float m = fmaxf(fabsf(dm) - b.h[k] - tb[4 + k], 0.f);
        dist2 = fmaf(m, m, dist2);
    }
    float lim;
    if constexpr (SIM == SIM_PURE || SIM == SIM_MIX) {
        lim = fa.scr_c2;
    } else {
        lim = (b.has_p && fa.coulomb_on) ? fmaxf(fa.scr_c2, fa.scr_n2) : fa.scr_n2;
    }
    return dist2 <= lim;
}

// Bits 4k..4k+3 of v -> bit k (k = 0..7): which of 8 groups has a set bit.
__device__ __forceinline__ unsigned any_of_4(unsigned v)
{
    v |= v >> 1;
    v |= v >> 2;
    v &= 0x11111111u;
    v = (v | (v >> 3)) & 0x03030303u;
    v = (v | (v >> 6)) & 0x000f000fu;
    v = (v | (v >> 12)) & 0xffu;
    return v;
}

// box_reaches, also returning the image the centre gives the source: per axis
// k = rint((x - c) / L) in {-1, 0, 1}, as the low 2 bits (two's complement)
// of the magic-number sum, packed 2 bits per axis.
__device__ __forceinline__ bool box_reaches_img(const ForceArgs& fa, const WarpBox& b, const float (&x)[3],
                                                unsigned& code)
{
    const float MAGIC = 12582912.0f;
    float dist2 = 0.f;
    unsigned cd = 0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float d = x[k] - b.c[k];
        const float kb = fmaf(d, fa.invLf[k], MAGIC);
        const float dm = fmaf(-fa.Lf[k], kb - MAGIC, d);
        const float m = fmaxf(fabsf(dm) - b.h[k], 0.f);
        dist2 = fmaf(m, m, dist2);
        cd |= (__float_as_uint(kb) & 3u) << (2 * k);
    }
    code = cd;
    return dist2 <= fa.scr_c2;
}

// Image of axis c from a packed code: 0 -> 0, 1 -> +1, 3 -> -1.
__device__ __forceinline__ float img_of(int code, int c)
{
    const int b = (code >> (2 * c)) & 3;
    return b == 0 ? 0.f : (b == 1 ? 1.f : -1.f);
}

// near_groups for ions, also telling whether all reachable sources of the
// tile take the same image from the warp's centre: kcode = their packed
// image code, or -1 if they differ (or none is reachable).
__device__ __forceinline__ unsigned near_groups_img(const ForceArgs& fa, const WarpBox& b,
                                                    const float* __restrict__ tlf, int jlim, int jmin, int& kcode)
{
    const int lane = threadIdx.x & 31;
    unsigned gm = 0, c_and = 0x3fu, c_or = 0u;
#pragma unroll
    for (int blk = 0; blk < PB / 32; ++blk) {
        const int j = 32 * blk + lane;
        bool near = false;
        unsigned code = 0;
        if (b.any && j < jlim && j >= jmin) {
            const float x[3] = {tlf[shadow_off(j, 0)], tlf[shadow_off(j, 1)], tlf[shadow_off(j, 2)]};
            near = box_reaches_img(fa, b, x, code);
        }
        if (near) {
            c_and &= code;
            c_or |= code;
        }
        gm |= any_of_4(__ballot_sync(0xffffffffu, near)) << (8 * blk);
    }
    c_and = __reduce_and_sync(0xffffffffu, c_and);
    c_or = __reduce_or_sync(0xffffffffu, c_or);
    kcode = (gm != 0 && c_and == c_or) ? (int)c_or : -1;
    return gm;
}

template <int SIM>
__device__ __forceinline__ unsigned near_groups(const ForceArgs& fa, const WarpBox& b, const float* __restrict__ tlf,
                                                int jlim, int jmin)
{
    const int lane = threadIdx.x & 31;
    unsigned gm = 0;
#pragma unroll
    for (int blk = 0; blk < PB / 32; ++blk) {
        const int j = 32 * blk + lane;
        bool near = false;
        if (b.any && j < jlim && j >= jmin) {
            const float x[3] = {tlf[shadow_off(j, 0)], tlf[shadow_off(j, 1)], tlf[shadow_off(j, 2)]};
            near = box_reaches<SIM>(fa, b, x, tlf[shadow_off(j, 3)]);
        }
        gm |= any_of_4(__ballot_sync(0xffffffffu, near)) << (8 * blk);
    }
    return gm;
}

// Shared memory of the half-pair kernels (RowT: row_t of the form).
template <typename RowT>
struct PairSmem {
    double4 tile[2][PB];                  // FP64 source tiles, or the shadow lo parts (TMA)
    float tilef[2][SHADOW_HI_FLOATS];     // FP32 shadow source tiles, hi parts and w (TMA)
    alignas(16) float tb[2][8];           // the tiles' boxes (TMA, when PairJobs::tbox is set)
    RowT acc_j[2][PWARPS][PB * 3];        // per-warp reaction rows, one set per tile stage
    double red[32 * NSCAL];               // block reduction scratch
    uint64_t bar[2];                      // one mbarrier per tile stage
    int done[2];                          // warps finished with the stage's tile
    int used[2][PWARPS];                  // the warp wrote its row of the stage's tile
    int abort;                            // a tile copy timed out: every warp leaves
    int s_job;
};

// One box as a job sees it: base pointers of its slots, shadow tiles and
// scratch, and its tile geometry.
struct BoxView {
    const double4* pos;
    const float* posf;
    double* Si;
    void* Sj;                      // source-side rows, row_t of the form
    const float* tbox;             // tile boxes, or null (PairJobs::tbox)
    unsigned char* Sjf;            // Sj row flags, or null (PairJobs::Sjf)
    int n, M, nseg_max;
};

template <typename RowT>
__device__ __forceinline__ void pairs_smem_init(PairSmem<RowT>& sm)
{
    // The ion path evaluates all 4 pairs of a group and masks the terms
    // (ion_pair_nb), so it also reads the slots of a partial tile that no copy
    // filled.  Zero them once: from then on every slot holds a finite position
    // (zero, or one left by an earlier tile) and a masked pair yields 0, not NaN.
    for (int k = threadIdx.x; k < 2 * PB; k += blockDim.x) (&sm.tile[0][0])[k] = make_double4(0.0, 0.0, 0.0, 0.0);
    for (int k = threadIdx.x; k < 2 * SHADOW_HI_FLOATS; k += blockDim.x) (&sm.tilef[0][0])[k] = 0.f;
    if (threadIdx.x == 0) {
        mbar_init(&sm.bar[0], 1);
        mbar_init(&sm.bar[1], 1);
        fence_mbar_init();
        sm.done[0] = sm.done[1] = 0;
        sm.abort = 0;
    }
    __syncthreads();
}

static_assert(SHADOW_LO_FLOATS * sizeof(float) <= PB * sizeof(double4), "lo parts must fit a tile stage");

// Load source tile C of box bx into stage qq & 1 (one thread): the shadow hi
// parts, the FP64 positions or (lo) the shadow lo parts, and (tb) the tile's
// box.
template <typename RowT>
__device__ __forceinline__ void pairs_issue(PairSmem<RowT>& sm, const BoxView& bx, int C, unsigned qq, bool lo,
                                            bool tb)
{
    const int j0 = C * PB;
    const int cnt = min(PB, bx.n - j0);
    const unsigned bytes = lo ? (unsigned)SHADOW_LO_FLOATS * (unsigned)sizeof(float)
                              : (unsigned)cnt * (unsigned)sizeof(double4);
    const unsigned bytesf = (unsigned)SHADOW_HI_FLOATS * (unsigned)sizeof(float);
    const float* src = bx.posf + (size_t)C * SHADOW_FLOATS;
    uint64_t* b = &sm.bar[qq & 1];
    const unsigned bytesb = (tb && bx.tbox) ? 8u * (unsigned)sizeof(float) : 0u;
    mbar_arrive_expect_tx(b, bytes + bytesf + bytesb);
    if (lo) bulk_g2s(&sm.tile[qq & 1][0], src + SHADOW_HI_FLOATS, bytes, b);
    else bulk_g2s(&sm.tile[qq & 1][0], bx.pos + j0, bytes, b);
    bulk_g2s(&sm.tilef[qq & 1][0], src, bytesf, b);
    if (bytesb) bulk_g2s(&sm.tb[qq & 1][0], bx.tbox + 8 * (size_t)C, bytesb, b);
}

// Job (R, sg) of box bx: target block R against source tiles
// C = R + sg*seg ... (at most seg of them).  q counts the tiles this CTA has
// consumed (stage and mbarrier parity).  Writes Si / Sj rows of the box and,
// when measuring, the job's 8 sums to sm_row.  Returns false if a tile copy
// timed out (the CTA must then leave).
//
// The warps do not meet at a block barrier between tiles.  A warp that has
// finished tile C counts itself in done[stage]; the last of the four sums the
// four warps' reaction rows of the tile into the unit's Sj row (in warp
// order, so the result does not depend on which warp came last) and then
// issues the copy of tile C+2 into the freed stage.  A warp starts tile C+2
// only after that copy has landed, so it never overwrites rows that are
// still being summed.  Warps may thus run up to one tile apart, which absorbs
// the uneven work of the four target groups.
// LOMODE: whether the mixed ion path takes its displacement from the shadow's
// hi/lo parts (pair_group_lo): 0 never, 1 always (the caller has checked
// fa.lo; the FP64-tile path is then not compiled in, which frees its
// registers), 2 as fa.lo says (boxes of a batch differ).
template <int SIM, int PREC, bool MEAS, int LOMODE = 2, bool IMGK = false, bool TB = false>
__device__ __forceinline__ bool pairs_job(PairSmem<row_t<PREC>>& sm, const ForceArgs& fa, const BoxView& bx, int R,
                                          int C0, int C1, int sg, double* __restrict__ sm_row,
                                          unsigned* __restrict__ err, unsigned& q)
{
    using R_t = real_t<PREC>;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int n = bx.n;
    const int i = R * PB + tid;
    // a unit shared by 2^lg jobs (source_split): this one takes sources
    // [w0, w1) of every tile (multiples of 32)
    const int lg = (sg >> 24) & 15, part = (sg >> 20) & 15;
    sg &= 0xFFFFF;
    const int w0 = (part * PB) >> lg, w1 = ((part + 1) * PB) >> lg;
    const bool active = i < n;
    const double4 pi = active ? bx.pos[i] : make_double4(0.0, 0.0, 0.0, 0.0);
    const ScreenI si = load_screen_i(bx.posf, active ? i : 0);
    const R_t wi = (SIM == SIM_MIX) ? (R_t)pi.w : (R_t)1;   // Z_i of the reaction
    const bool all_active = (R + 1) * PB <= n;
    const int sw = ((lane >> 4) & 1) * 2 + ((lane >> 3) & 1);
    const WarpBox box = warp_box(fa, pi, active);
    // nucleons: every active target of the warp is a proton
    const bool all_p = SIM == SIM_NUCLEON && box.has_p && __all_sync(0xffffffffu, !active || pi.w == 1.0);
    TargetAcc<PREC, MEAS> acc;
    acc.zero();
    // the mixed form on a box that allows it: FP32 displacements from the
    // shadow's hi/lo parts, no FP64 source tiles (ions: fa.lo; nucleons:
    // fa.hilo, with the FP64 positions read from global memory for the rare
    // pairs near |d| = L/2)
    const bool lo = (PREC == PREC_MIXED) &&
                    (LOMODE == 1 || (LOMODE == 2 && (SIM == SIM_NUCLEON ? fa.hilo != 0 : fa.lo != 0)));
    float nli[3] = {0.f, 0.f, 0.f};
    if (lo) {
#pragma unroll
        for (int c = 0; c < 3; ++c) nli[c] = -bx.posf[shadow_index(active ? i : 0, 4 + c)];
    }
    const bool tb = TB && bx.tbox != nullptr;

    // both stages are free: every warp has passed the block barrier that
    // handed out this job
    if (tid == 0) {
        pairs_issue(sm, bx, C0, q, lo, tb);
        if (C0 + 1 < C1) pairs_issue(sm, bx, C0 + 1, q + 1, lo, tb);
    }
    const unsigned q0 = q;
    for (int C = C0; C < C1; ++C, ++q) {
        const int st = q & 1;
        if (!mbar_wait_abortable(&sm.bar[st], (q >> 1) & 1u, err, &sm.abort)) break;
        const int jlim = min(min(PB, n - C * PB), w1);
        const bool diag = (C == R);
        const double4* tl = sm.tile[st];
        const float* tlf = sm.tilef[st];
        row_t<PREC>* my_acc = sm.acc_j[st][warp];
        // The warp's row is used (zeroed, then written group by group) only
        // if some group of the tile is near its targets; otherwise it is
        // marked unused.  TB: a tile whose box is out of reach of the warp's
        // box is skipped before the per-source screen.
        bool used = false;
        auto open_row = [&](unsigned gm) {
            used = gm != 0;
            if (used) {
#pragma unroll
                for (int k = lane; k < PB * 3; k += 32) my_acc[k] = 0.0;
                __syncwarp();
            }
        };
        const bool reach = box.any && (!tb || tile_reaches<SIM>(fa, box, sm.tb[st]));
        if (reach) {
            // on the diagonal tile only sources after the warp's first target count
            const int jmin = max(diag ? 32 * warp + 1 : 0, w0);
            const bool full = !diag && jlim == PB && all_active && w0 == 0;
            if (lo) {
                if constexpr (PREC == PREC_MIXED && SIM == SIM_NUCLEON) {
                    unsigned gm = near_groups<SIM>(fa, box, tlf, jlim, jmin);
                    open_row(gm);
                    const float* tll = reinterpret_cast<const float*>(tl);
                    const double4* gsrc = bx.pos + (size_t)C * PB;
                    // the species mode of this warp on this tile (pair_group_nn_lo)
                    int mode = NN_ANY;
                    if (!box.has_p && fa.nn_short) {
                        mode = NN_NOP;
                    } else if (all_p && gm && fa.coul_all && fa.coulomb_on) {
                        bool any_n = false;
#pragma unroll
                        for (int blk = 0; blk < PB / 32; ++blk) {
                            const int j = 32 * blk + lane;
                            any_n |= j >= jmin && j < jlim && tlf[shadow_off(j, 3)] != 1.0f;
                        }
                        if (!__any_sync(0xffffffffu, any_n)) mode = NN_PP;
                    }
                    auto run = [&](auto mode_c) {
                        constexpr int MD = decltype(mode_c)::value;
                        if (full) {
                            for (; gm; gm &= gm - 1)
                                pair_group_nn_lo<MEAS, false, MD>(fa, si, nli, pi, tlf, tll, gsrc, 4 * (__ffs(gm) - 1),
                                                                  jlim, diag, active, tid, sw, acc, my_acc);
                        } else {
                            for (; gm; gm &= gm - 1)
                                pair_group_nn_lo<MEAS, true, MD>(fa, si, nli, pi, tlf, tll, gsrc, 4 * (__ffs(gm) - 1),
                                                                 jlim, diag, active, tid, sw, acc, my_acc);
                        }
                    };
                    if (mode == NN_PP) run(std::integral_constant<int, NN_PP>());
                    else if (mode == NN_NOP) run(std::integral_constant<int, NN_NOP>());
                    else run(std::integral_constant<int, NN_ANY>());
                }
                if constexpr (PREC == PREC_MIXED && (SIM == SIM_PURE || SIM == SIM_MIX)) {
                    int kcode = -1;
                    unsigned gm = near_groups_img(fa, box, tlf, jlim, jmin, kcode);
                    open_row(gm);
                    const float* tll = reinterpret_cast<const float*>(tl);
                    if (box.tile_img && kcode >= 0) {
                        // one image for the whole tile: fold it into the target
                        float2 th[3], tl2[3];
                        const float nh[3] = {si.nx, si.ny, si.nz};
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            const float k = img_of(kcode, c);
                            const float h = fmaf(-k, fa.Lh[c], nh[c]);       // exact
                            const float l = fmaf(-k, fa.Ll[c], nli[c]);
                            th[c] = make_float2(h, h);
                            tl2[c] = make_float2(l, l);
                        }
                        if (full) {
                            for (; gm; gm &= gm - 1)
                                pair_group_lo<SIM, MEAS, false, true>(fa, si, nli, th, tl2, wi, tlf, tll,
                                                                      4 * (__ffs(gm) - 1), jlim, diag, active, tid,
                                                                      sw, acc, my_acc);
                        } else {
                            for (; gm; gm &= gm - 1)
                                pair_group_lo<SIM, MEAS, true, true>(fa, si, nli, th, tl2, wi, tlf, tll,
                                                                     4 * (__ffs(gm) - 1), jlim, diag, active, tid,
                                                                     sw, acc, my_acc);
                        }
                    } else {
                        const float2 z[3] = {};
                        if (full) {
                            for (; gm; gm &= gm - 1)
                                pair_group_lo<SIM, MEAS, false>(fa, si, nli, z, z, wi, tlf, tll, 4 * (__ffs(gm) - 1),
                                                                jlim, diag, active, tid, sw, acc, my_acc);
                        } else {
                            for (; gm; gm &= gm - 1)
                                pair_group_lo<SIM, MEAS, true>(fa, si, nli, z, z, wi, tlf, tll, 4 * (__ffs(gm) - 1),
                                                               jlim, diag, active, tid, sw, acc, my_acc);
                        }
                    }
                }
            } else if (IMGK && (SIM == SIM_PURE || SIM == SIM_MIX)) {
                // ions whose screen image integers are exact: the tile image
                // when the tile has one, else each pair's own
                if constexpr (IMGK && (SIM == SIM_PURE || SIM == SIM_MIX)) {
                    int kcode = -1;
                    unsigned gm = near_groups_img(fa, box, tlf, jlim, jmin, kcode);
                    open_row(gm);
                    if (box.tile_img && kcode >= 0) {
                        float2 th[3];
                        const float nh[3] = {si.nx, si.ny, si.nz};
                        const double pc[3] = {pi.x, pi.y, pi.z};
                        double pt[3];
#pragma unroll
                        for (int c = 0; c < 3; ++c) {
                            const float k = img_of(kcode, c);
                            const float h = fmaf(-k, fa.Lh[c], nh[c]);       // exact
                            th[c] = make_float2(h, h);
                            pt[c] = __fma_rn((double)k, fa.xl[c], pc[c]);
                        }
                        const double4 pit = make_double4(pt[0], pt[1], pt[2], pi.w);
                        if (full) {
                            for (; gm; gm &= gm - 1)
                                pair_group<SIM, PREC, MEAS, false, true, true>(fa, pi, si, wi, tl, tlf,
                                                                               4 * (__ffs(gm) - 1), jlim, diag, active,
                                                                               tid, sw, acc, my_acc, th, pit);
                        } else {
                            for (; gm; gm &= gm - 1)
                                pair_group<SIM, PREC, MEAS, true, true, true>(fa, pi, si, wi, tl, tlf,
                                                                              4 * (__ffs(gm) - 1), jlim, diag, active,
                                                                              tid, sw, acc, my_acc, th, pit);
                        }
                    } else if (full) {
                        for (; gm; gm &= gm - 1)
                            pair_group<SIM, PREC, MEAS, false, true>(fa, pi, si, wi, tl, tlf, 4 * (__ffs(gm) - 1), jlim,
                                                                     diag, active, tid, sw, acc, my_acc);
                    } else {
                        for (; gm; gm &= gm - 1)
                            pair_group<SIM, PREC, MEAS, true, true>(fa, pi, si, wi, tl, tlf, 4 * (__ffs(gm) - 1), jlim,
                                                                    diag, active, tid, sw, acc, my_acc);
                    }
                }
            } else {
                unsigned gm = near_groups<SIM>(fa, box, tlf, jlim, jmin);
                open_row(gm);
                if (full) {
                    for (; gm; gm &= gm - 1)
                        pair_group<SIM, PREC, MEAS, false, IMGK>(fa, pi, si, wi, tl, tlf, 4 * (__ffs(gm) - 1), jlim,
                                                                 diag, active, tid, sw, acc, my_acc);
                } else {
                    for (; gm; gm &= gm - 1)
                        pair_group<SIM, PREC, MEAS, true, IMGK>(fa, pi, si, wi, tl, tlf, 4 * (__ffs(gm) - 1), jlim,
                                                                diag, active, tid, sw, acc, my_acc);
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
            if (um == 0 && bx.Sjf && w0 == 0 && w1 == PB) {
                // no warp had a pair: the unit's row is zero; k_combine skips it
                if (lane == 0) bx.Sjf[u] = 0;
            } else {
                // the unit's source-side row: the used warp rows in warp order
                // (an unused row is zero), FP64 in the FP64 form, FP32 (one
                // rounding of the FP32 rows summed in FP64) in the mixed form;
                // only this job's window (the other parts of a split unit
                // write the rest)
                row_t<PREC>* dj = static_cast<row_t<PREC>*>(bx.Sj) + (size_t)u * PB * 3;
#pragma unroll 4
                for (int k = 3 * w0 + lane; k < 3 * w1; k += 32) {
                    double v = 0.0;
#pragma unroll
                    for (int w = 0; w < PWARPS; ++w)
                        if ((um >> w) & 1u) v += sm.acc_j[st][w][k];
                    dj[k] = (row_t<PREC>)v;
                }
                if (lane == 0 && bx.Sjf) bx.Sjf[u] = 1;
            }
            __syncwarp();
            if (lane == 0 && C + 2 < C1) pairs_issue(sm, bx, C + 2, q + 2, lo, tb);
        }
    }
    q = q0 + (unsigned)(C1 - C0);
    if (__syncthreads_or(sm.abort)) return false;
    // target-side partial of job (R, s)
    double* di = bx.Si + (((size_t)R * bx.nseg_max + sg) * PB + tid) * 3;
    di[0] = acc.force(0);
    di[1] = acc.force(1);
    di[2] = acc.force(2);
    if constexpr (MEAS) {
        double S[NSCAL];
#pragma unroll
        for (int k = 0; k < NSCAL; ++k) S[k] = active ? acc.scal(k) * (double)wi : 0.0;
        block_sum_store<NSCAL>(S, sm.red, sm_row);
        __syncthreads();
    }
    return true;
}

// Resident CTAs per SM: 5 (96 registers); the mixed kernel that always takes
// the hi/lo displacement needs fewer registers and FP32 rows, so 6 fit.  The
// force-only nucleon form runs 7 (72 registers, no spills): the extra CTAs
// give the SM warps to issue from while a CTA's warps wait for each other at
// the end of a job (2 % faster on the 51,200-nucleon box; the ion forms were
// 2 % slower at 7).
template <int SIM, int PREC, bool LO, bool MEAS = false>
constexpr int pairs_ctas_per_sm()
{
    return (PREC == PREC_MIXED && LO) ? ((SIM == SIM_NUCLEON && !MEAS) ? 7 : 6) : 5;
}

// Whether a kernel variant tests each tile's box against each warp's box
// (PairJobs::tbox) before screening its sources: the mixed hi/lo ion kernels,
// whose per-group cost is low enough that the per-tile screen of far tiles
// matters (9 % fewer instructions on the 55,296-ion mixture).  The FP64 and
// nucleon kernels were slower with the test (register pressure).
template <int SIM, int PREC, bool LO>
constexpr bool pairs_tile_boxes()
{
    return PREC == PREC_MIXED && LO && SIM != SIM_NUCLEON;
}

// LO: the mixed ion kernel for boxes with fa.lo (pair_group_lo); IMGK: a
// kernel for ion boxes with fa.img_k (the screen's image integers replace the
// exact minimum-image comparisons, which are then not compiled in).
template <int SIM, int PREC, bool MEAS, bool LO = false, bool IMGK = false>
__global__ void __launch_bounds__(PB, (pairs_ctas_per_sm<SIM, PREC, LO, MEAS>()))
k_force_pairs(const double4* __restrict__ pos, const float* __restrict__ posf, PairJobs pj,
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
        constexpr bool TB = pairs_tile_boxes<SIM, PREC, LO>();
        if (!pairs_job<SIM, PREC, MEAS, LO ? 1 : 0, IMGK, TB>(sm, fa, bx, js.x, js.y, js.z, js.w,
                                                              Sm + (size_t)job * NSCAL, err, q))
            return;
    }
}

// Per slot: sum its target-side and source-side partials in a fixed order,
// scale (int_ion_pure.f:227-231 / int_ion_mix.f:201,273-277 / int_nn.f:318-322)
// and store into the caller's order.  One CTA per target block R (the
// heaviest blocks, with the most units, first); thread t of each of the
// COMB_GROUPS groups owns double t of the block's 128 x 3 partial rows (slot
// t / 3, component t % 3), so a warp reads 256 contiguous bytes per row.
// Group g sums the rows g, g + COMB_GROUPS, ...; the group sums are added
// in group order.  The summation order is fixed, so results are
// bit-reproducible run to run.
constexpr int COMB_GROUPS = 2;
constexpr int COMB_THREADS = COMB_GROUPS * PB * 3;

// Dynamic shared memory of k_combine for M tiles with unit flags: the flags of
// the longest row (M bytes, padded to 4) and the list of its written rows.
__host__ __device__ inline size_t comb_smem_bytes(int M)
{
    return (size_t)((M + 3) / 4) * 4 + sizeof(int) * (size_t)M;
}

template <int SIM, int PREC>
__global__ void __launch_bounds__(COMB_THREADS)
k_combine(const double* __restrict__ Si, const row_t<PREC>* __restrict__ Sj, PairJobs pj,
          const int* __restrict__ perm, const double* __restrict__ zii,
          const double* __restrict__ aii, ForceArgs fa, double* __restrict__ a_out)
{
    __shared__ double part[COMB_GROUPS][PB * 3];
    __shared__ int nz_count;
    // with pj.Sjf: row R's unit flags (R + 1 bytes, padded to 4) and then the
    // list of its written rows in ascending order (comb_smem_bytes)
    extern __shared__ int comb_dyn[];
    const int R = pj.M - 1 - (int)blockIdx.x;
    const int g = threadIdx.x / (PB * 3), t = threadIdx.x % (PB * 3);
    constexpr size_t ROW = (size_t)PB * 3;
    double F = 0.0;
    const double* si = Si + (size_t)R * pj.nseg_max * ROW + t;
    const int nseg = pj.row_slots[R];
#pragma unroll 4
    for (int s = g; s < nseg; s += COMB_GROUPS) F += si[(size_t)s * ROW];
    const row_t<PREC>* sj = Sj + (size_t)tri_index(R, 0) * ROW + t;
    if (pj.Sjf) {
        // rows flagged zero were not written (k_force_pairs); skipping them
        // leaves every sum as it was.  The flags are staged in shared memory,
        // one warp lists the written rows in ascending order, and the groups
        // take every COMB_GROUPS-th entry of the list: the row loads of the
        // unrolled loop carry no condition and issue together.
        unsigned char* sfl = reinterpret_cast<unsigned char*>(comb_dyn);
        int* nzl = comb_dyn + (R + 4) / 4;
        const unsigned char* fl = pj.Sjf + tri_index(R, 0);
        for (int r = threadIdx.x; r <= R; r += blockDim.x) sfl[r] = fl[r];
        __syncthreads();
        if (threadIdx.x < 32) {
            const int lane = threadIdx.x;
            int cnt = 0;
            for (int b = 0; b <= R; b += 32) {
                const bool on = b + lane <= R && sfl[b + lane] != 0;
                const unsigned m = __ballot_sync(0xffffffffu, on);
                if (on) nzl[cnt + __popc(m & ((1u << lane) - 1u))] = b + lane;
                cnt += __popc(m);
            }
            if (lane == 0) nz_count = cnt;
        }
        __syncthreads();
        const int cnt = nz_count;
#pragma unroll 8
        for (int q = g; q < cnt; q += COMB_GROUPS) F += (double)sj[(size_t)nzl[q] * ROW];
    } else {
#pragma unroll 4
        for (int R2 = g; R2 <= R; R2 += COMB_GROUPS) F += (double)sj[(size_t)R2 * ROW];
    }
    part[g][t] = F;
    __syncthreads();
    const int l = threadIdx.x;
    const int p = R * PB + l;
    if (l < PB && p < fa.n) {
        double Fv[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            double v = part[0][3 * l + c];
#pragma unroll
            for (int q = 1; q < COMB_GROUPS; ++q) v += part[q][3 * l + c];
            Fv[c] = v;
        }
        const int orig = perm[p];
        // only the mixture folds by Z_i; pure-ion and nucleon callers may pass zii = NULL
        store_accel<SIM>(fa, orig, SIM == SIM_MIX ? zii[orig] : 0.0, aii, Fv, a_out);
    }
}

}  // namespace yk
