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
//   job  (R, s)         : units C = R + s*seg ... of one row; persistent CTAs
//                         pull jobs from an atomic counter (costliest first).
//
// Reaction sums: the 4 warps of a CTA sweep the tile in 4 phases, warp w
// taking the 32-slot chunk (w + phase) mod 4, so every source slot is touched
// by one warp at a time.  For each source j that any lane hits, the warp sums
// the 32 reactions with a shuffle butterfly (in FP64 for both forms) and lane
// 0 adds it to the tile's shared accumulator; phases are separated by CTA
// barriers, so each accumulator sees its warps in a fixed order.
//
// Outputs are partial sums in scratch (nothing is accumulated atomically):
//   Si[R][s][PB][3]       target-side sums of job (R, s)
//   Sj[tri(C,R)][PB][3]   source-side sums of unit (R, C), tri(C,R) = C(C+1)/2+R
//   Sm[job][8]            measurement sums of the job (U, W, P tensor)
// k_combine adds, for every slot, its Si entries then its Sj entries in a
// fixed order, applies the reference's scaling and scatters to the caller's
// particle order.  Results are therefore bit-reproducible, independent of
// which CTA ran which job.
#pragma once

#include "yk_force.cuh"

namespace yk {

constexpr int PB = 128;           // slots per block / tile (= threads per CTA)
constexpr int PWARPS = PB / 32;

struct PairJobs {
    const int2* jobs;             // (R, s) per job, costliest first
    int njobs;
    int M;                        // tiles
    int seg;                      // source tiles per job
    int nseg_max;                 // ceil(M / seg): Si slots per row
};

__host__ __device__ __forceinline__ long long tri_index(int C, int R)
{
    return (long long)C * (C + 1) / 2 + R;
}

template <int PREC>
__device__ __forceinline__ double to_f64(real_t<PREC> v)
{
    return (double)v;
}

template <int SIM, int PREC, bool MEAS>
__global__ void __launch_bounds__(PB, 4)
k_force_pairs(const double4* __restrict__ pos, PairJobs pj, int* __restrict__ job_counter,
              ForceArgs fa, double* __restrict__ Si, double* __restrict__ Sj,
              double* __restrict__ Sm, unsigned* __restrict__ err)
{
    __shared__ __align__(128) double4 tile[2][PB];
    __shared__ double acc_j[PB * 3];
    __shared__ double red[32 * NSCAL];
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int s_job;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int n = fa.n;
    using R_t = real_t<PREC>;

    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    __syncthreads();

    unsigned q = 0;               // tiles this CTA has consumed (stage / parity)
    auto issue = [&](int C, unsigned qq) {
        const int j0 = C * PB;
        const int cnt = min(PB, n - j0);
        const unsigned bytes = (unsigned)cnt * (unsigned)sizeof(double4);
        uint64_t* b = &bar[qq & 1];
        mbar_arrive_expect_tx(b, bytes);
        bulk_g2s(&tile[qq & 1][0], pos + j0, bytes, b);
    };

    for (;;) {
        if (tid == 0) s_job = atomicAdd(job_counter, 1);
        __syncthreads();
        const int job = s_job;
        if (job >= pj.njobs) break;
        const int2 js = pj.jobs[job];
        const int R = js.x, sg = js.y;
        const int C0 = R + sg * pj.seg;
        const int C1 = min(C0 + pj.seg, pj.M);
        const int i = R * PB + tid;
        const bool active = i < n;
        const double4 pi = active ? pos[i] : make_double4(0.0, 0.0, 0.0, 0.0);
        const R_t wi = (SIM == SIM_MIX) ? (R_t)pi.w : (R_t)1;   // Z_i of the reaction
        TargetAcc<PREC, MEAS> acc;
        acc.zero();
        PairOut<R_t> o;

        if (tid == 0) {
            issue(C0, q);
            if (C0 + 1 < C1) issue(C0 + 1, q + 1);
        }
        for (int C = C0; C < C1; ++C, ++q) {
            const int st = q & 1;
            acc_j[3 * tid] = 0.0;
            acc_j[3 * tid + 1] = 0.0;
            acc_j[3 * tid + 2] = 0.0;
            const bool ok = mbar_wait_bounded(&bar[st], (q >> 1) & 1u, err);
            if (__syncthreads_or(!ok)) {
                if (tid == 0 && C + 1 < C1) mbar_wait_bounded(&bar[st ^ 1], ((q + 1) >> 1) & 1u, err);
                return;
            }
            const int jlim = min(PB, n - C * PB);
            const bool diag = (C == R);
            const double4* tl = tile[st];
#pragma unroll 1
            for (int ph = 0; ph < PWARPS; ++ph) {
                const int jb = ((warp + ph) & (PWARPS - 1)) * 32;
                const int je = min(jb + 32, jlim);
                for (int jl = jb; jl < je; ++jl) {
                    const double4 pjv = tl[jl];
                    const bool valid = active && (!diag || jl > tid);
                    pair_eval<SIM, PREC, MEAS>(fa, pi, pjv, valid, o);
                    if (o.hit) acc.add(o, SIM == SIM_MIX ? (R_t)pjv.w : (R_t)1);
                    if (__any_sync(0xffffffffu, o.hit)) {
                        // reaction on j: sum over the warp of Z_i fs d (int_ion_mix.f:180)
                        double rx = 0.0, ry = 0.0, rz = 0.0;
                        if (o.hit) {
                            const R_t fsj = o.fs * wi;
                            rx = to_f64<PREC>(fsj * o.dx);
                            ry = to_f64<PREC>(fsj * o.dy);
                            rz = to_f64<PREC>(fsj * o.dz);
                        }
#pragma unroll
                        for (int m = 16; m > 0; m >>= 1) {
                            rx += __shfl_xor_sync(0xffffffffu, rx, m);
                            ry += __shfl_xor_sync(0xffffffffu, ry, m);
                            rz += __shfl_xor_sync(0xffffffffu, rz, m);
                        }
                        if (lane == 0) {
                            acc_j[3 * jl] -= rx;
                            acc_j[3 * jl + 1] -= ry;
                            acc_j[3 * jl + 2] -= rz;
                        }
                    }
                }
                __syncthreads();
            }
            // source-side partial of unit (R, C)
            double* dj = Sj + ((size_t)tri_index(C, R) * PB + tid) * 3;
            dj[0] = acc_j[3 * tid];
            dj[1] = acc_j[3 * tid + 1];
            dj[2] = acc_j[3 * tid + 2];
            __syncthreads();                  // stage st and acc_j are free again
            if (tid == 0 && C + 2 < C1) issue(C + 2, q + 2);
        }
        // target-side partial of job (R, s)
        double* di = Si + (((size_t)R * pj.nseg_max + sg) * PB + tid) * 3;
        di[0] = acc.force(0);
        di[1] = acc.force(1);
        di[2] = acc.force(2);
        if constexpr (MEAS) {
            double S[NSCAL];
#pragma unroll
            for (int k = 0; k < NSCAL; ++k) S[k] = active ? acc.scal(k) * (double)wi : 0.0;
            block_sum_store<NSCAL>(S, red, Sm + (size_t)job * NSCAL);
            __syncthreads();
        }
    }
}

// Per slot: sum its target-side and source-side partials in a fixed order,
// scale (int_ion_pure.f:227-231 / int_ion_mix.f:201,273-277 / int_nn.f:318-322)
// and store into the caller's order.
template <int SIM>
__global__ void __launch_bounds__(256)
k_combine(const double* __restrict__ Si, const double* __restrict__ Sj, PairJobs pj,
          const int* __restrict__ perm, const double* __restrict__ zii,
          const double* __restrict__ aii, ForceArgs fa, double* __restrict__ a_out)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= fa.n) return;
    const int R = p / PB, l = p % PB;
    const int nseg = (pj.M - R + pj.seg - 1) / pj.seg;
    double F[3] = {0.0, 0.0, 0.0};
    const double* si = Si + ((size_t)R * pj.nseg_max * PB + l) * 3;
    for (int s = 0; s < nseg; ++s) {
        const double* e = si + (size_t)s * PB * 3;
        F[0] += e[0];
        F[1] += e[1];
        F[2] += e[2];
    }
    const double* sj = Sj + ((size_t)tri_index(R, 0) * PB + l) * 3;
    for (int R2 = 0; R2 <= R; ++R2) {
        const double* e = sj + (size_t)R2 * PB * 3;
        F[0] += e[0];
        F[1] += e[1];
        F[2] += e[2];
    }
    const int orig = perm[p];
    store_accel<SIM>(fa, orig, zii[orig], aii, F, a_out);
}

}  // namespace yk
