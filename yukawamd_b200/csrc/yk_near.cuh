// yk_near.cuh -- half-pair force kernel over per-warp near-source lists.
//
// Same jobs, tiles, scratch and combine as k_force_pairs (yk_pairs.cuh): a
// CTA of PB = 128 threads owns target block R, one slot per thread, and
// streams source tiles C >= R through shared memory (1-D TMA bulk copies,
// double-buffered).  What differs is the work inside a tile.  Per tile, each
// warp
//
//   1. classifies the tile's 128 sources against the bounding box of its 32
//      targets (FP32, with a margin that covers the rounding of the FP32
//      copies): a source farther than the screening radius from the box
//      cannot interact with any of the warp's targets and is dropped; for a
//      kept source it finds, per axis, the one periodic image shift
//      s in {-L, 0, +L} that the reference's conditional minimum image
//      (int_ion_pure.f:147-152: d - L if d > L/2, d + L if d < -L/2) applies
//      to every pair of this warp with this source, or marks the source
//      "ambiguous" when the box straddles a decision boundary;
//   2. writes the kept sources, compacted, into its own list in shared
//      memory: the FP64 position moved by the image, x_j - s, or the raw
//      position for an ambiguous source;
//   3. walks the list in groups of 4 with the lane-swizzled reduce-scatter of
//      k_force_pairs: d = x_i - (x_j - s) in FP64 (the exact per-pair
//      minimum image for ambiguous entries), then the pair terms of the FP64
//      or mixed form, the target sum in registers and the reaction sums of
//      the 4 sources added to the entries' per-warp accumulators;
//   4. after a block barrier, thread j sums source j's per-warp reaction
//      sums in warp order into the unit's Sj row.
//
// The per-pair FP32 screen and the per-pair minimum-image tests of
// k_force_pairs disappear: the far sources never enter the list and the
// image is chosen once per (warp, source).  x_i - (x_j - s) differs from the
// reference's (x_i - x_j) + s by one rounding of x_j - s (at most half an
// ulp of L), far inside the FP64 form's 1e-12 tolerance.  All sums still run
// in a fixed order, so results are bit-reproducible.
#pragma once

#include "yk_pairs.cuh"

namespace yk {

constexpr int NEAR_AMB = 0x100;     // list entry flag: take the exact per-pair minimum image

struct NearSmem {
    double4 tile[2][PB];                  // FP64 source tiles (TMA)
    double4 spos[PWARPS][PB];             // per warp: kept sources, image-shifted
    double sacc[PWARPS][PB][3];           // per warp: reaction sums per list entry
    unsigned short sent[PWARPS][PB];      // per warp: list entry -> source index | NEAR_AMB
    signed char pos_of[PWARPS][PB];       // per warp: source index -> list entry, -1 if dropped
    double red[32 * NSCAL];               // block reduction scratch
    uint64_t bar[2];
    int s_job;
};

// Classify source pj against the warp box.  Returns true if some target of
// the box may be within the screening radius; sets the per-axis image shift
// (in units of L) and amb if any axis straddles +-L/2.
template <int SIM>
__device__ __forceinline__ bool near_classify(const ForceArgs& fa, const WarpBox& b, const double4& pj,
                                              int (&shift)[3], bool& amb)
{
    const double c[3] = {pj.x, pj.y, pj.z};
    float dist2 = 0.f;
    amb = false;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float L = fa.Lf[k], hL = 0.5f * fa.Lf[k];
        const float mu = 3.814697265625e-6f * L;                 // 2^-18 L
        const float xj = __double2float_rn(c[k]);
        const float lo = (b.lo[k] - xj) - mu;                    // range of x_i - x_j over the box
        const float hi = (b.hi[k] - xj) + mu;
        int s = 0;
        bool a = false;
        if (lo > hL) s = -1;
        else if (hi < -hL) s = 1;
        else if (!(lo >= -hL && hi <= hL)) a = true;
        shift[k] = s;
        amb |= a;
        const float lo2 = fmaf((float)s, L, lo), hi2 = fmaf((float)s, L, hi);
        const float m = a ? 0.f : fmaxf(0.f, fmaxf(lo2, -hi2));
        dist2 = fmaf(m, m, dist2);
    }
    float lim;
    if constexpr (SIM == SIM_PURE || SIM == SIM_MIX) {
        lim = fa.scr_c2;
    } else {
        const bool pp = b.has_p && pj.w == 1.0 && fa.coulomb_on;
        lim = pp ? fmaxf(fa.scr_c2, fa.scr_n2) : fa.scr_n2;
    }
    return dist2 <= lim;
}

template <int SIM, int PREC, bool MEAS>
__device__ __forceinline__ bool near_job(NearSmem& sm, const ForceArgs& fa, const BoxView& bx, int R, int C0, int C1,
                                         int sg,
                                         double* __restrict__ sm_row, unsigned* __restrict__ err, unsigned& q)
{
    using R_t = real_t<PREC>;
    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int n = bx.n;

    const int i = R * PB + tid;
    const bool active = i < n;
    const double4 pi = active ? bx.pos[i] : make_double4(0.0, 0.0, 0.0, 0.0);
    const R_t wi = (SIM == SIM_MIX) ? (R_t)pi.w : (R_t)1;   // Z_i of the reaction
    const WarpBox box = warp_box(fa, pi, active);
    const unsigned lt_mask = (1u << lane) - 1u;
    const int sw = ((lane >> 4) & 1) * 2 + ((lane >> 3) & 1);
    TargetAcc<PREC, MEAS> acc;
    acc.zero();

    if (tid == 0) {
        const int j0 = C0 * PB;
        const unsigned bytes = (unsigned)min(PB, n - j0) * (unsigned)sizeof(double4);
        mbar_arrive_expect_tx(&sm.bar[q & 1], bytes);
        bulk_g2s(&sm.tile[q & 1][0], bx.pos + j0, bytes, &sm.bar[q & 1]);
        if (C0 + 1 < C1) {
            const int j1 = (C0 + 1) * PB;
            const unsigned b1 = (unsigned)min(PB, n - j1) * (unsigned)sizeof(double4);
            mbar_arrive_expect_tx(&sm.bar[(q + 1) & 1], b1);
            bulk_g2s(&sm.tile[(q + 1) & 1][0], bx.pos + j1, b1, &sm.bar[(q + 1) & 1]);
        }
    }
    for (int C = C0; C < C1; ++C, ++q) {
        const int st = q & 1;
        const bool ok = mbar_wait_bounded(&sm.bar[st], (q >> 1) & 1u, err);
        if (__syncthreads_or(!ok)) {
            if (tid == 0 && C + 1 < C1) mbar_wait_bounded(&sm.bar[st ^ 1], ((q + 1) >> 1) & 1u, err);
            return false;
        }
        const int jlim = min(PB, n - C * PB);
        const bool diag = (C == R);
        const double4* tl = sm.tile[st];
        double4* spos = sm.spos[warp];
        double(*sacc)[3] = sm.sacc[warp];
        unsigned short* sent = sm.sent[warp];
        signed char* pos_of = sm.pos_of[warp];

        // 1-2: classify the tile's sources and build this warp's list
        int K = 0;
#pragma unroll 1
        for (int b = 0; b < PB / 32; ++b) {
            const int j = 32 * b + lane;
            const bool cand = box.any && j < jlim && (!diag || j > 32 * warp);
            double4 pj = make_double4(0.0, 0.0, 0.0, 0.0);
            int shift[3] = {0, 0, 0};
            bool amb = false, keep = false;
            if (cand) {
                pj = tl[j];
                keep = near_classify<SIM>(fa, box, pj, shift, amb);
            }
            const unsigned km = __ballot_sync(0xffffffffu, keep);
            if (keep) {
                const int e = K + __popc(km & lt_mask);
                if (!amb) {
                    // d + s L = x_i - (x_j - s L)
                    pj.x = __dsub_rn(pj.x, (double)shift[0] * fa.xl[0]);
                    pj.y = __dsub_rn(pj.y, (double)shift[1] * fa.xl[1]);
                    pj.z = __dsub_rn(pj.z, (double)shift[2] * fa.xl[2]);
                }
                spos[e] = pj;
                sent[e] = (unsigned short)(j | (amb ? NEAR_AMB : 0));
                sacc[e][0] = sacc[e][1] = sacc[e][2] = 0.0;
                pos_of[j] = (signed char)e;
            } else {
                pos_of[j] = -1;
            }
            K += __popc(km);
        }
        __syncwarp();

        // 3: the list in groups of 4 sources
#pragma unroll 1
        for (int g0 = 0; g0 < K; g0 += 4) {
            double r[4][3];
            bool any = false;
#pragma unroll
            for (int jj = 0; jj < 4; ++jj) {
                const int e = g0 + (jj ^ sw);
                r[jj][0] = r[jj][1] = r[jj][2] = 0.0;
                if (e < K) {
                    const double4 pj = spos[e];
                    const int ent = sent[e];
                    const bool valid = active && (!diag || (ent & 0xff) > tid);
                    double dx = __dsub_rn(pi.x, pj.x), dy = __dsub_rn(pi.y, pj.y), dz = __dsub_rn(pi.z, pj.z);
                    if (ent & NEAR_AMB) {
                        dx = min_image(dx, fa.xl[0], fa.hlb[0]);
                        dy = min_image(dy, fa.xl[1], fa.hlb[1]);
                        dz = min_image(dz, fa.xl[2], fa.hlb[2]);
                    }
                    PairOut<R_t> o;
                    if constexpr (PREC == PREC_FP64) {
                        o.dx = dx;
                        o.dy = dy;
                        o.dz = dz;
                        phys64<SIM, MEAS>(fa, pi.w, pj.w, valid, o);
                    } else {
                        o.dx = __double2float_rn(dx);
                        o.dy = __double2float_rn(dy);
                        o.dz = __double2float_rn(dz);
                        phys32<SIM, MEAS>(fa, pi.w, pj.w, valid, o);
                    }
                    if (o.hit) {
                        acc.add(o, SIM == SIM_MIX ? (R_t)pj.w : (R_t)1);
                        // reaction on j: Z_i fs d (int_ion_mix.f:180)
                        const R_t fsj = o.fs * wi;
                        r[jj][0] = to_f64<PREC>(fsj * o.dx);
                        r[jj][1] = to_f64<PREC>(fsj * o.dy);
                        r[jj][2] = to_f64<PREC>(fsj * o.dz);
                        any = true;
                    }
                }
            }
            if (__any_sync(0xffffffffu, any)) {
                double t[3];
                reduce_scatter4(r, t);
                const int e = g0 + sw;
                if ((lane & 7) == 0 && e < K) {
                    sacc[e][0] -= t[0];
                    sacc[e][1] -= t[1];
                    sacc[e][2] -= t[2];
                }
            }
        }
        __syncthreads();                  // tile done: stage st reusable, all lists complete
        if (tid == 0 && C + 2 < C1) {
            const int j2 = (C + 2) * PB;
            const unsigned b2 = (unsigned)min(PB, n - j2) * (unsigned)sizeof(double4);
            mbar_arrive_expect_tx(&sm.bar[st], b2);
            bulk_g2s(&sm.tile[st][0], bx.pos + j2, b2, &sm.bar[st]);
        }
        // 4: source-side partial of unit (R, C), the warps' sums in warp order
        double v[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int w = 0; w < PWARPS; ++w) {
            const int e = sm.pos_of[w][tid];
            if (e >= 0) {
                v[0] += sm.sacc[w][e][0];
                v[1] += sm.sacc[w][e][1];
                v[2] += sm.sacc[w][e][2];
            }
        }
        row_t<PREC>* dj = static_cast<row_t<PREC>*>(bx.Sj) + ((size_t)tri_index(C, R) * PB + tid) * 3;
        dj[0] = (row_t<PREC>)v[0];
        dj[1] = (row_t<PREC>)v[1];
        dj[2] = (row_t<PREC>)v[2];
    }
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

template <int SIM, int PREC, bool MEAS>
__global__ void __launch_bounds__(PB, 5)
k_force_near(const double4* __restrict__ pos, PairJobs pj, int* __restrict__ job_counter, ForceArgs fa,
             double* __restrict__ Si, row_t<PREC>* __restrict__ Sj, double* __restrict__ Sm,
             unsigned* __restrict__ err)
{
    __shared__ __align__(128) NearSmem sm;
    if (threadIdx.x == 0) {
        mbar_init(&sm.bar[0], 1);
        mbar_init(&sm.bar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();
    BoxView bx;
    bx.pos = pos;
    bx.posf = nullptr;
    bx.Si = Si;
    bx.Sj = Sj;
    bx.tbox = nullptr;
    bx.Sjf = nullptr;
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
        if (!near_job<SIM, PREC, MEAS>(sm, fa, bx, js.x, js.y, js.z, js.w, Sm + (size_t)job * NSCAL, err, q))
            return;
    }
}

}  // namespace yk
