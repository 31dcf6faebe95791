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
// 144-157, 1989), with 256 table entries: -t = (256 m + j) ln2/256 + r with
// |r| <= ln2/512, so e^{-t} = 2^m 2^{j/256} e^r.  N = 256 m + j =
// rint(-t 256/ln2) comes from the 1.5*2^52 add (its low word is N); r from two
// FMAs with ln2/256 split into a double and its remainder; e^r - 1 from its
// Taylor polynomial to r^4 (truncation < 4e-17 relative); 2^{j/256} from a
// table of correctly rounded doubles; 2^m through the exponent bits.  Error
// <= 3 ulp for t in [0, 700] (tests/test_numerics.py restates it); results for
// t > 700 flush to zero.  (A 64-entry table needs the r^5 term: one FP64 FMA
// more per pair, 0.5 % of the FP64 ion force call.)
// RANGE = false leaves the t > 700 test out: the caller guarantees t <= 700.
static __device__ const double g_exp2_256[256] = {
    1.0, 1.0027112750502025, 1.0054299011128027, 1.0081558981184175,
    1.0108892860517005, 1.0136300849514894, 1.016378314910953, 1.019133996077738,
    1.0218971486541166, 1.0246677928971357, 1.0274459491187637, 1.030231637686041,
    1.0330248790212284, 1.0358256936019572, 1.0386341019613787, 1.041450124688316,
    1.0442737824274138, 1.0471050958792898, 1.0499440858006872, 1.0527907730046264,
    1.0556451783605572, 1.0585073227945128, 1.061377227289262, 1.0642549128844645,
    1.0671404006768237, 1.0700337118202419, 1.0729348675259756, 1.075843889062791,
    1.0787607977571199, 1.0816856149932152, 1.0846183622133092, 1.0875590609177697,
    1.0905077326652577, 1.0934643990728858, 1.0964290818163769, 1.099401802630222,
    1.102382583307841, 1.1053714457017412, 1.1083684117236787, 1.1113735033448175,
    1.1143867425958924, 1.1174081515673693, 1.1204377524096067, 1.12347556733302,
    1.1265216186082418, 1.129575928566288, 1.1326385195987192, 1.1357094141578055,
    1.1387886347566916, 1.1418762039695616, 1.1449721444318042, 1.148076478840179,
    1.1511892299529827, 1.154310420590216, 1.1574400736337511, 1.1605782120274988,
    1.1637248587775775, 1.1668800369524817, 1.1700437696832502, 1.1732160801636373,
    1.1763969916502812, 1.1795865274628758, 1.182784710984341, 1.1859915656609938,
    1.189207115002721, 1.1924313825831512, 1.1956643920398273, 1.1989061670743806,
    1.202156731452703, 1.2054161090051239, 1.2086843236265816, 1.2119613992768012,
    1.215247359980469, 1.2185422298274085, 1.2218460329727576, 1.2251587936371455,
    1.22848053610687, 1.2318112847340759, 1.2351510639369334, 1.2384998981998165,
    1.241857812073484, 1.245224830175258, 1.2486009771892048, 1.2519862778663162,
    1.255380757024691, 1.2587844395497165, 1.2621973503942507, 1.2656195145788063,
    1.2690509571917332, 1.2724917033894028, 1.275941778396392, 1.2794012075056693,
    1.2828700160787783, 1.2863482295460256, 1.2898358734066657, 1.2933329732290895,
    1.2968395546510096, 1.3003556433796506, 1.3038812651919358, 1.3074164459346773,
    1.3109612115247644, 1.3145155879493546, 1.318079601266064, 1.3216532776031575,
    1.3252366431597413, 1.3288297242059544, 1.3324325470831615, 1.3360451382041458,
    1.339667524053303, 1.3432997311868353, 1.3469417862329458, 1.3505937158920345,
    1.3542555469368927, 1.3579273062129011, 1.3616090206382248, 1.365300717204012,
    1.3690024229745905, 1.3727141650876684, 1.3764359707545302, 1.380167867260238,
    1.383909881963832, 1.387662042298529, 1.3914243757719262, 1.3951969099662003,
    1.3989796725383112, 1.4027726912202048, 1.4065759938190154, 1.4103896082172707,
    1.4142135623730951, 1.4180478843204152, 1.4218926021691656, 1.4257477441054942,
    1.42961333839197, 1.433489413367789, 1.4373759974489824, 1.4412731191286257,
    1.4451808069770467, 1.449099089642035, 1.4530279958490526, 1.4569675544014438,
    1.460917794180647, 1.4648787441464057, 1.4688504333369818, 1.4728328908693675,
    1.4768261459394993, 1.4808302278224719, 1.4848451658727524, 1.488870989524397,
    1.4929077282912648, 1.4969554117672355, 1.5010140696264256, 1.5050837316234065,
    1.5091644275934228, 1.5132561874526098, 1.5173590411982147, 1.5214730189088146,
    1.5255981507445384, 1.529734466947287, 1.533881997840956, 1.5380407738316568,
    1.5422108254079407, 1.5463921831410214, 1.550584877685, 1.5547889397770887,
    1.559004400237837, 1.5632312899713576, 1.567469639965553, 1.5717194812923414,
    1.5759808451078865, 1.5802537626528246, 1.5845382652524937, 1.588834384317164,
    1.593142151342267, 1.597461597908627, 1.6017927556826934, 1.606135656416771,
    1.6104903319492543, 1.6148568142048607, 1.6192351351948637, 1.6236253270173289,
    1.6280274218573478, 1.632441451987275, 1.6368674497669644, 1.6413054476440063,
    1.645755478153965, 1.6502175739206177, 1.6546917676561943, 1.6591780921616162,
    1.6636765803267364, 1.6681872651305825, 1.6727101796415966, 1.6772453570178785,
    1.681792830507429, 1.6863526334483934, 1.6909247992693053, 1.6955093614893326,
    1.7001063537185235, 1.7047158096580513, 1.709337763100463, 1.713972247929926,
    1.718619298122478, 1.723278947746274, 1.7279512309618377, 1.732636182022311,
    1.7373338352737062, 1.7420442251551564, 1.746767386199169, 1.7515033530318782,
    1.7562521603732995, 1.761013843037584, 1.7657884359332727, 1.7705759740635547,
    1.7753764925265212, 1.7801900265154245, 1.785016611318935, 1.789856282321401,
    1.7947090750031072, 1.7995750249405351, 1.804454167806624, 1.809346539371032,
    1.8142521755003989, 1.8191711121586085, 1.8241033854070534, 1.8290490314048973,
    1.8340080864093424, 1.8389805867758937, 1.843966568958626, 1.8489660695104508,
    1.8539791250833855, 1.8590057724288205, 1.864046048397789, 1.8690999899412386,
    1.8741676341103, 1.8792490180565602, 1.8843441790323345, 1.8894531543909392,
    1.8945759815869656, 1.8997126981765553, 1.9048633418176741, 1.9100279502703899,
    1.9152065613971474, 1.9203992131630474, 1.925605943636125, 1.930826790987627,
    1.9360617934922943, 1.9413109895286405, 1.9465744175792332, 1.9518521162309783,
    1.9571441241754002, 1.9624504802089273, 1.9677712232331759, 1.9731063922552343,
    1.978456026387951, 1.9838201648502194, 1.9891988469672663, 1.9945921121709402,
};

template <bool RANGE = true>
__device__ __forceinline__ double exp_neg_f64(double t)
{
    const double MAG = 6755399441055744.0;                // 1.5 * 2^52
    const double INV = 369.3299304675746;                 // 256 / ln 2
    const double L1 = 0.0027076061740622863;              // ln2/256, rounded
    const double L2 = 9.058776616587108e-20;              // ln2/256 - L1
    const double kd = __fma_rn(-t, INV, MAG);
    const double nf = __dsub_rn(kd, MAG);
    const double r = __fma_rn(-nf, L2, __fma_rn(-nf, L1, -t));
    double q = 1.0 / 24.0;
    q = __fma_rn(q, r, 1.0 / 6.0);
    q = __fma_rn(q, r, 0.5);
    q = __fma_rn(q, r, 1.0);
    const double p = __dmul_rn(q, r);                     // e^r - 1
    const int ni = __double2loint(kd);
    const double tj = __ldg(&g_exp2_256[ni & 255]);
    const double res = __fma_rn(tj, p, tj);
    const int hi = __double2hiint(res) + ((ni >> 8) << 20);
    if constexpr (!RANGE) return __hiloint2double(hi, __double2loint(res));
    return t > 700.0 ? 0.0 : __hiloint2double(hi, __double2loint(res));
}

// FP64 1/sqrt(x) for x > 0 inside the FP32 normal range (a pair's r^2, or 1
// for a masked pair): one second-order correction of the FP32 hardware
// estimate y.  With e = 1 - x y^2 (one FMA, exact but for the rounding of
// x y), 1/sqrt(x) = y (1 - e)^(-1/2) = y (1 + e/2 + 3e^2/8 + 5e^3/16 + ...);
// |e| is about 2^-21, so the dropped terms are below 2^-63 relative and the
// result is within about 1 ulp: five FP64 instructions at a dependency depth
// of four, against seven at depth six for two Newton steps.
__device__ __forceinline__ double rsqrt_nr64(double x)
{
    const double y = (double)rsqrtf(__double2float_rn(x));
    const double e = __fma_rn(-__dmul_rn(x, y), y, 1.0);
    return __fma_rn(__dmul_rn(y, e), __fma_rn(e, 0.375, 0.5), y);
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
