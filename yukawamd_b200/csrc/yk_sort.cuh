// yk_sort.cuh -- space-filling-curve ordering of the particles.
//
// The force kernels walk particles in "slot" order.  Sorting the slots along
// a 3-D Hilbert curve (10 bits per axis) makes each warp's 32 targets and each
// 128-slot source tile spatially compact, so for most (warp, source) pairs
// either every lane or no lane is inside the cutoff sphere and the
// expensive branch of the pair loop is skipped by whole warps.  The Hilbert
// curve has no long jumps (consecutive cells are face neighbours), so runs of
// 32 particles are rounder than on a Morton (Z-order) curve: on the
// 55,296-ion mixture the mean extent of a warp's targets drops from about
// 133 x 112 x 84 fm to 87 x 86 x 86 fm, and 10 % fewer (warp, 4-source)
// groups reach the pair terms.  The ordering
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

// Hilbert index of cell (x0, x1, x2) on a 2^10 grid per axis, by Skilling's
// method (J. Skilling, "Programming the Hilbert curve", AIP Conf. Proc. 707,
// 381 (2004)): turn the axes into the transposed index (undo the excess
// rotations and reflections level by level, then Gray-encode), and
// interleave the bits with axis 0 most significant in each triple.
__device__ __forceinline__ unsigned hilbert10(unsigned x0, unsigned x1, unsigned x2)
{
    unsigned X[3] = {x0, x1, x2};
#pragma unroll
    for (unsigned Q = 1u << 9; Q > 1; Q >>= 1) {
        const unsigned P = Q - 1;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            if (X[i] & Q) {
                X[0] ^= P;                                  // invert the low bits
            } else {
                const unsigned t = (X[0] ^ X[i]) & P;       // exchange the low bits
                X[0] ^= t;
                X[i] ^= t;
            }
        }
    }
    X[1] ^= X[0];
    X[2] ^= X[1];
    unsigned t = 0;
#pragma unroll
    for (unsigned Q = 1u << 9; Q > 1; Q >>= 1)
        if (X[2] & Q) t ^= Q - 1;
    X[0] ^= t;
    X[1] ^= t;
    X[2] ^= t;
    return (spread10(X[0]) << 2) | (spread10(X[1]) << 1) | spread10(X[2]);
}

// keys[i] = Hilbert index of particle i's cell on a 1024^3 grid over the box.
// With species (nucleons: 1 = proton, 0 = neutron), bit 30 puts the protons
// first: warps then hold one species, so the p-p Coulomb term, which reaches
// every proton pair, runs on whole warps instead of the ~40 % of lanes that
// are protons in a mixed warp.
static __global__ void k_morton(const double* __restrict__ x, int n, double sx, double sy, double sz,
                         unsigned* __restrict__ keys, int* __restrict__ idx,
                         const double* __restrict__ species = nullptr)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int cx = min(max((int)(x[3 * i] * sx), 0), 1023);
    const int cy = min(max((int)(x[3 * i + 1] * sy), 0), 1023);
    const int cz = min(max((int)(x[3 * i + 2] * sz), 0), 1023);
    keys[i] = hilbert10(cx, cy, cz) | ((species && species[i] != 1.0) ? (1u << 30) : 0u);
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
    store_shadow(posf, s, p.x, p.y, p.z, (float)p.w);
}

}  // namespace yk
