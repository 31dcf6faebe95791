// yk_common.cuh -- device helpers shared by the engine's kernels (sm_100a).
//
//  * 1-D TMA bulk copies global -> shared (cp.async.bulk) completed on an
//    mbarrier, with bounded waits that report a timeout instead of hanging.
//    No multicast form is used anywhere in this engine.
//  * warp / block reductions of double partial sums in a fixed order, so
//    every result is bit-reproducible run to run.
//  * compensated FP32 accumulation (Knuth two-sum) for the mixed form.
//  * an FP32 exp(-t) built from Cody-Waite reduction and a polynomial for
//    2^f on [-1/2, 1/2] (relative-error least-squares fit with Lawson
//    reweighting on Chebyshev nodes; tests/test_numerics.py checks the
//    polynomial's error bound and a float32 restatement of the function).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace yk {

// Bits of the device error word.
constexpr unsigned ERR_TIMEOUT = 1u << 0;   // a bounded mbarrier wait gave up
constexpr unsigned ERR_BOUNDS  = 1u << 1;   // an index check failed (debug builds)

// Iteration bound of every spin on an mbarrier.  One try_wait suspends the
// thread for a hardware time slice; a j-tile lands in a few microseconds, so
// the bound is only ever reached if a copy never completes.
constexpr long long SPIN_LIMIT = 1ll << 22;

__device__ __forceinline__ unsigned smem_u32(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// 1-D bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned)
// from this GPU's global memory into this CTA's shared memory.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of *bar with at most `limit` polls.  Returns
// false (and sets ERR_TIMEOUT in *err) if the phase never completed.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, unsigned* err,
                                                  long long limit = SPIN_LIMIT)
{
    for (long long it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    atomicOr(err, ERR_TIMEOUT);
    return false;
}

// As mbar_wait_bounded, for the warps of a CTA that do not meet at a block
// barrier between waits: a waiter also gives up as soon as another thread has
// raised *abort, and one that times out raises it.
__device__ __forceinline__ bool mbar_wait_abortable(uint64_t* bar, unsigned parity, unsigned* err,
                                                    volatile int* abort, long long limit = SPIN_LIMIT)
{
    for (long long it = 0; it < limit; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 63) == 63 && *abort) return false;
    }
    atomicOr(err, ERR_TIMEOUT);
    *abort = 1;
    return false;
}

// ---- reductions ----------------------------------------------------------

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum K values over the block in a fixed order; the result lands in out[k]
// (global) from thread 0.  scratch: shared double[32*K].
template <int K>
__device__ __forceinline__ void block_sum_store(double (&v)[K], double* scratch, double* out)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < K; ++k) {
        double s = warp_sum(v[k]);
        if (lane == 0) scratch[warp * K + k] = s;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double s = lane < nwarps ? scratch[lane * K + k] : 0.0;
            s = warp_sum(s);
            if (lane == 0) out[k] = s;
        }
    }
}

// ---- compensated FP32 sums ---------------------------------------------

// Knuth two-sum: s + c carries the running sum; the rounding error of every
// addition is captured exactly in c (6 flops, no branch).
struct cf32 {
    float s, c;
    __device__ __forceinline__ cf32() : s(0.f), c(0.f) {}
    __device__ __forceinline__ void add(float x)
    {
        float t = __fadd_rn(s, x);
        float bp = __fsub_rn(t, s);
        float e = __fadd_rn(__fsub_rn(s, __fsub_rn(t, bp)), __fsub_rn(x, bp));
        s = t;
        c = __fadd_rn(c, e);
    }
    __device__ __forceinline__ double value() const { return (double)s + (double)c; }
};

// Kahan sum for sums of one sign (energies, virial): 4 flops.
struct kf32 {
    float s, c;
    __device__ __forceinline__ kf32() : s(0.f), c(0.f) {}
    __device__ __forceinline__ void add(float x)
    {
        float y = __fsub_rn(x, c);
        float t = __fadd_rn(s, y);
        c = __fsub_rn(__fsub_rn(t, s), y);
        s = t;
    }
    __device__ __forceinline__ double value() const { return (double)s - (double)c; }
};

// ---- FP32 exp(-t), t >= 0 ---------------------------------------------
// e^{-t} = 2^{y}, y = -t log2(e) = k + f, |f| <= 1/2.  y is formed with the
// product's rounding error recovered by an FMA (Cody-Waite style), so f is
// accurate to ~1e-9 absolute; 2^f comes from a degree-6 polynomial fitted
// on [-1/2, 1/2] (2e-9 relative in exact arithmetic, 1e-7 = 1.7 ulp with
// FP32 Horner rounding); 2^k is applied through the exponent bits.  k is
// rounded with the 1.5*2^23 add (round to nearest even, as rintf) and read
// back as an integer from the sum's low mantissa bits, so the function uses
// only FMA-pipe and integer instructions (no conversion or rounding unit).
// Valid for t < 2.9e6; results below 2^-126 flush to zero.
__device__ __forceinline__ float exp_neg_f32(float t)
{
    const float L2E_HI = 1.44269502162933349609375f;      // float(log2 e)
    const float L2E_LO = 1.925963033500011079e-8f;       // log2 e - L2E_HI
    const float MAGIC = 12582912.0f;                      // 1.5 * 2^23
    float yh = -t * L2E_HI;
    float yl = fmaf(-t, L2E_HI, -yh);                    // exact error of -t*L2E_HI
    yl = fmaf(-t, L2E_LO, yl);
    const float kb = __fadd_rn(yh, MAGIC);               // k in the low mantissa bits
    const float k = __fsub_rn(kb, MAGIC);
    float f = (yh - k) + yl;                             // yh - k is exact
    // 2^f = sum c_m f^m, c_m fitted to 2^f on [-0.5, 0.5]
    float p = 1.5353360504377633e-4f;
    p = fmaf(p, f, 1.3398875016719103e-3f);
    p = fmaf(p, f, 9.6184369176626205e-3f);
    p = fmaf(p, f, 5.5503323674201965e-2f);
    p = fmaf(p, f, 2.4022647738456726e-1f);
    p = fmaf(p, f, 6.9314718246459961e-1f);
    p = fmaf(p, f, 1.0f);
    const int ki = __float_as_int(kb) - 0x4B400000;
    float r = __int_as_float(__float_as_int(p) + (ki << 23));
    return (k < -125.f) ? 0.f : r;
}

// ---- FP32 exp(-t), t >= 0, on the hardware base-2 exponential ----------
// e^{-t} = 2^{yh} 2^{yl} with yh = fl(-t log2 e) and yl the rest of the
// exact product (the FMA-recovered rounding error of yh plus -t times the
// low part of log2 e); 2^{yl} = 1 + yl ln 2 to first order (|yl| < 2^-24
// |yh|, so the dropped term is below 1e-13 for t < 90).  2^{yh} is the
// ex2.approx.ftz.f32 instruction of the transcendental unit.  Used where that
// unit has spare issue slots; the result is within the instruction's error
// (about 2 ulp) of e^{-t}; results below 2^-126 flush to zero.
__device__ __forceinline__ float ex2_approx(float y)
{
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(y));
    return r;
}

__device__ __forceinline__ float exp_neg_f32_xu(float t)
{
    const float L2E_HI = 1.44269502162933349609375f;      // float(log2 e)
    const float L2E_LO_LN2 = 1.3349758e-8f;              // (log2 e - L2E_HI) ln 2
    const float LN2 = 0.693147180559945309f;
    const float yh = -t * L2E_HI;
    const float e1 = fmaf(-t, L2E_HI, -yh);              // exact error of -t*L2E_HI
    const float c = fmaf(e1, LN2, -t * L2E_LO_LN2);      // yl ln 2
    const float r = ex2_approx(yh);
    return fmaf(r, c, r);
}

// ---- FP32x2: two values per instruction ----------------------------------
// x - y, correctly rounded: an FMA whose product y * (-1) is exact.
__device__ __forceinline__ float2 sub2(float2 x, float2 y)
{
    return __ffma2_rn(y, make_float2(-1.f, -1.f), x);
}

// Two compensated sums (cf32::add) advanced together.
__device__ __forceinline__ void cf32_add2(cf32& a, cf32& b, float2 x)
{
    const float2 s = make_float2(a.s, b.s);
    const float2 t = __fadd2_rn(s, x);
    const float2 bp = sub2(t, s);
    const float2 e = __fadd2_rn(sub2(s, sub2(t, bp)), sub2(x, bp));
    const float2 c = __fadd2_rn(make_float2(a.c, b.c), e);
    a.s = t.x;
    b.s = t.y;
    a.c = c.x;
    b.c = c.y;
}

// ---- FP64 exp(-t), t >= 0 -----------------------------------------------
// Table-driven method of P. T. P. Tang ("Table-driven implementation of the
// exponential function in IEEE floating-point arithmetic", ACM TOMS 15,
// 144-157, 1989): -t = (64 m + j) ln2/64 + r with |r| <= ln2/128, so
// e^{-t} = 2^m 2^{j/64} e^r.  N = 64 m + j = rint(-t 64/ln2) comes from the
// 1.5*2^52 add (its low word is N); r from two FMAs with ln2/64 split into a
// double and its remainder; e^r - 1 from its Taylor polynomial to r^5
// (truncation < 4e-17 relative); 2^{j/64} from a table of correctly rounded
// doubles; 2^m through the exponent bits.  Error <= 3 ulp for t in [0, 700]
// (tests/test_numerics.py restates it); results for t > 700 flush to zero.
static __device__ const double g_exp2_64[64] = {
    1.0, 1.0108892860517005, 1.0218971486541166, 1.0330248790212284,
    1.0442737824274138, 1.0556451783605572, 1.0671404006768237, 1.0787607977571199,
    1.0905077326652577, 1.102382583307841, 1.1143867425958924, 1.1265216186082418,
    1.1387886347566916, 1.1511892299529827, 1.1637248587775775, 1.1763969916502812,
    1.189207115002721, 1.202156731452703, 1.215247359980469, 1.22848053610687,
    1.241857812073484, 1.255380757024691, 1.2690509571917332, 1.2828700160787783,
    1.2968395546510096, 1.3109612115247644, 1.3252366431597413, 1.339667524053303,
    1.3542555469368927, 1.3690024229745905, 1.383909881963832, 1.3989796725383112,
    1.4142135623730951, 1.42961333839197, 1.4451808069770467, 1.460917794180647,
    1.4768261459394993, 1.4929077282912648, 1.5091644275934228, 1.5255981507445384,
    1.5422108254079407, 1.559004400237837, 1.5759808451078865, 1.593142151342267,
    1.6104903319492543, 1.6280274218573478, 1.645755478153965, 1.6636765803267364,
    1.681792830507429, 1.7001063537185235, 1.718619298122478, 1.7373338352737062,
    1.7562521603732995, 1.7753764925265212, 1.7947090750031072, 1.8142521755003989,
    1.8340080864093424, 1.8539791250833855, 1.8741676341103, 1.8945759815869656,
    1.9152065613971474, 1.9360617934922943, 1.9571441241754002, 1.978456026387951,
};

__device__ __forceinline__ double exp_neg_f64(double t)
{
    const double MAG = 6755399441055744.0;                // 1.5 * 2^52
    const double INV = 92.33248261689366;                 // 64 / ln 2
    const double L1 = 0.010830424696249145;               // ln2/64, rounded
    const double L2 = 3.623510646634843e-19;              // ln2/64 - L1
    const double kd = __fma_rn(-t, INV, MAG);
    const double nf = __dsub_rn(kd, MAG);
    const double r = __fma_rn(-nf, L2, __fma_rn(-nf, L1, -t));
    double q = 1.0 / 120.0;
    q = __fma_rn(q, r, 1.0 / 24.0);
    q = __fma_rn(q, r, 1.0 / 6.0);
    q = __fma_rn(q, r, 0.5);
    q = __fma_rn(q, r, 1.0);
    const double p = __dmul_rn(q, r);                     // e^r - 1
    const int ni = __double2loint(kd);
    const double tj = __ldg(&g_exp2_64[ni & 63]);
    const double res = __fma_rn(tj, p, tj);
    const int hi = __double2hiint(res) + ((ni >> 6) << 20);
    return t > 700.0 ? 0.0 : __hiloint2double(hi, __double2loint(res));
}

// FP64 1/sqrt(x) for x > 0 inside the FP32 normal range (a pair's r^2, or 1
// for a masked pair): Newton's iteration y <- y (3/2 - (x/2) y^2) from the FP32
// hardware estimate.  Each step squares the relative error (about 2^-22 ->
// 2^-43 -> below the FP64 rounding), so two steps leave the rounding errors
// of the steps themselves, a few ulp.
__device__ __forceinline__ double rsqrt_nr64(double x)
{
    double y = (double)rsqrtf(__double2float_rn(x));
    const double h = 0.5 * x;
    y = __dmul_rn(y, __fma_rn(-__dmul_rn(h, y), y, 1.5));
    y = __dmul_rn(y, __fma_rn(-__dmul_rn(h, y), y, 1.5));
    return y;
}

// FP32 1/sqrt(x): hardware estimate plus one Newton step.
__device__ __forceinline__ float rsqrt_f32(float x)
{
    float y = rsqrtf(x);
    float h = __fmul_rn(0.5f * x, y);
    return __fmul_rn(y, fmaf(-h, y, 1.5f));
}

// Minimum image of a displacement d in [-L, L] exactly as the reference's
// pair of conditional corrections (int_ion_pure.f:149-150): d - L if d > L/2,
// d + L if d < -L/2.  The comparisons run on the bit patterns (valid because
// L/2 > 0 and d is finite), which keeps them off the FP64 pipe.
__device__ __forceinline__ double min_image(double d, double L, long long hl_bits)
{
    const long long b = __double_as_longlong(d);
    double s = 0.0;
    if (b > hl_bits) s = -L;
    else if ((b ^ (long long)0x8000000000000000ull) > hl_bits) s = L;
    return __dadd_rn(d, s);
}

}  // namespace yk
