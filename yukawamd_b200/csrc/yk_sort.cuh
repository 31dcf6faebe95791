// yk_sort.cuh -- Morton (Z-order) ordering of the particles.
//
// The force kernels walk particles in "slot" order.  Sorting the slots along
// a 3-D Morton curve (10 bits per axis) makes each warp's 32 targets and each
// 128-slot source tile spatially compact, so for most (warp, source) pairs
// either every lane or no lane is inside the cutoff sphere and the
// expensive branch of the pair loop is skipped by whole warps.  The ordering
// never changes a result beyond summation order; it is refreshed every
// `sort_every` steps because particles drift.  The stable radix sort (CUB)
// keeps the permutation a deterministic function of the positions.
#pragma once

#include "yk_force.cuh"

namespace yk {

__device__ __forceinline__ unsigned spread10(unsigned v)
{
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// keys[i] = Morton code of particle i's cell on a 1024^3 grid over the box.
static __global__ void k_morton(const double* __restrict__ x, int n, double sx, double sy, double sz,
                         unsigned* __restrict__ keys, int* __restrict__ idx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int cx = min(max((int)(x[3 * i] * sx), 0), 1023);
    const int cy = min(max((int)(x[3 * i + 1] * sy), 0), 1023);
    const int cz = min(max((int)(x[3 * i + 2] * sz), 0), 1023);
    keys[i] = spread10(cx) | (spread10(cy) << 1) | (spread10(cz) << 2);
    idx[i] = i;
}

// Slot s holds particle perm[s]; iperm is the inverse; pos is repacked.
static __global__ void k_apply_perm(const int* __restrict__ perm, int* __restrict__ iperm,
                             const double* __restrict__ x, const double* __restrict__ zii,
                             double4* __restrict__ pos, float* __restrict__ posf, int n,
                             int pack_w)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int o = perm[s];
    iperm[o] = s;
    const double4 p = make_double4(x[3 * o], x[3 * o + 1], x[3 * o + 2], pack_w ? zii[o] : 0.0);
    pos[s] = p;
    posf[shadow_index(s, 0)] = (float)p.x;
    posf[shadow_index(s, 1)] = (float)p.y;
    posf[shadow_index(s, 2)] = (float)p.z;
    posf[shadow_index(s, 3)] = (float)p.w;
}

}  // namespace yk
