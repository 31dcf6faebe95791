// yk_engine.cu -- the C-ABI of include/yukawa_engine.h.
//
// One yk_ctx per simulation box.  Device state stays resident between calls:
// x, v, vold, a in the caller's (Fortran) layout and order, zii, aii, the
// Morton-ordered double4 positions the force kernels stream, the permutation
// between the two orders, scratch partial sums and the md_globals scalars.
// Every call runs on the context's own stream; calls that return results to
// the host synchronise that stream once at the end.
#include <cuda_runtime.h>

#include <algorithm>
#include <numeric>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <queue>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "../../include/yukawa_engine.h"
#include "yk_force.cuh"
#include "yk_internal.h"
#include "yk_pairs.cuh"
#include "yk_pairs2.cuh"
#include "yk_gofr.cuh"
#include "yk_near.cuh"
#include "yk_sort.cuh"
#include "yk_thermo.cuh"
#include "yk_verlet.cuh"

using namespace yk;

static std::atomic<unsigned long long> g_launches{0};
static thread_local std::string g_err_noctx;

#define YK_VERSION_STR "yukawamd_b200 0.2.0 (sm_100a)"

// FMA-throughput probe: PROBE_CHAINS independent dependent chains per thread.
constexpr int PROBE_CHAINS = 8;
template <typename T>
__global__ void __launch_bounds__(256) k_fma_probe(T* out, int iters, T a, T b)
{
    T x[PROBE_CHAINS];
#pragma unroll
    for (int q = 0; q < PROBE_CHAINS; ++q) x[q] = (T)(threadIdx.x + q);
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int q = 0; q < PROBE_CHAINS; ++q) x[q] = fma(x[q], a, b);
    }
    T s = 0;
#pragma unroll
    for (int q = 0; q < PROBE_CHAINS; ++q) s += x[q];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

// yk_set_state: flag a NaN or Inf among cnt staged values ...
__global__ void k_check_finite(const double* __restrict__ p, size_t cnt, unsigned* __restrict__ flag)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool bad = i < cnt && !isfinite(p[i]);
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}

// ... and move them into the state only if none was flagged.
__global__ void k_commit_state(const double* __restrict__ src, double* __restrict__ dst, size_t cnt,
                               const unsigned* __restrict__ flag)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < cnt && *flag == 0) dst[i] = src[i];
}

// Failure path of the bounded waits (yk_wait_selftest): one CTA of 128
// threads waits on an mbarrier that no copy is ever issued against, so its
// phase 0 never completes.  Warps 0-1 wait as the pair kernels' warps do
// (mbar_wait_abortable: the first to give up raises the abort flag, the
// others then leave), warps 2-3 as the row kernel does (mbar_wait_bounded).
// Every wait ends after at most `spins` polls and sets ERR_TIMEOUT in *err;
// nothing is in flight when the CTA exits.  out[0] counts the threads that
// gave up (all 128 when the path works).
__global__ void __launch_bounds__(128) k_wait_selftest(long long spins, unsigned* __restrict__ err,
                                                       int* __restrict__ out)
{
    __shared__ uint64_t bar;
    __shared__ int abort_flag;
    __shared__ int gave_up;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
        abort_flag = 0;
        gave_up = 0;
    }
    __syncthreads();
    const bool ok = threadIdx.x < 64 ? mbar_wait_abortable(&bar, 0u, err, &abort_flag, spins)
                                     : mbar_wait_bounded(&bar, 0u, err, spins);
    if (!ok) atomicAdd(&gave_up, 1);
    __syncthreads();
    if (threadIdx.x == 0) out[0] = gave_up;
}

// Largest scratch the half-pair kernel may take before auto mode falls back
// to the scratch-free row kernel.
constexpr size_t PAIR_SCRATCH_BUDGET = size_t(8) << 30;
// Longest job of the half-pair kernels (tiles) when the caller leaves it to
// the engine.  Measured on a B200 (force call, guided job sizes, caps 4..64):
// FP64 is best at 8 from N = 4,096 to 131,072; the mixed form at 4 for N =
// 16,384 to 55,296 and 8 at 131,072 (within 1.5 % of 4).
constexpr int DEFAULT_SEG_FP64 = 8;
constexpr int DEFAULT_SEG_MIXED = 4;
constexpr int DEFAULT_SEG = DEFAULT_SEG_FP64;
// Steps between Hilbert re-orderings.  Particles drift away from their
// warp's neighbours between sorts, the warp boxes grow and more source
// groups pass the screen, so the force call slows down step by step after a
// sort.  Measured on a B200 over 200 steps from states warmed for 300 steps
// (step time, sort included, cadences 1..50): 4 is best or within 1 % of
// best on the 55,296-ion mixture and on 51,200 nucleons, FP64 and mixed;
// against 50 it takes 12 % off the mixed ion step (1.161 -> 1.024 ms), 20 %
// off the mixed nucleon step (1.129 -> 0.904 ms), 5.5 % and 12 % off their
// FP64 steps.  A sort costs about 0.07 ms at these sizes.
constexpr int DEFAULT_SORT_EVERY = 4;
constexpr int DEFAULT_GRAPH_STEPS = 50;
constexpr int MAX_GRAPHS = 8;

struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    int K = 0, me = 0, phase = 0, series = 0, kernels = 0;
    unsigned long long stamp = 0;
};

struct yk_ctx {
    yk_params p;
    int n = 0;
    int dev = 0;
    cudaStream_t stream = nullptr;
    // state in the caller's order and layout
    double *x = nullptr, *v = nullptr, *vold = nullptr, *a = nullptr;
    double *zii = nullptr, *aii = nullptr;
    // Morton order
    double4* pos = nullptr;
    float* posf = nullptr;           // FP32 shadow of pos, tiled SoA (shadow_index)
    int *perm = nullptr, *iperm = nullptr;
    unsigned *keys0 = nullptr, *keys1 = nullptr;
    int* idx0 = nullptr;
    void* cub_tmp = nullptr;
    size_t cub_bytes = 0;
    // reductions and outputs
    double *fpart = nullptr, *kpart = nullptr;
    double *vpart = nullptr, *vsums = nullptr;   // ttot / tnorm / cancel_vcom sums
    double* a_vtot = nullptr;                   // accelerations of yk_vtot (discarded)
    double* stage = nullptr;                    // yk_set_state: x, v, vold, a as copied in, before the check
    unsigned* nonfinite = nullptr;              // yk_set_state: set by k_check_finite
    unsigned long long* gofr = nullptr;         // yk_gofr_counts histogram
    int gofr_cap = 0;
    DevScalars* ds = nullptr;
    unsigned* err = nullptr;
    double* series = nullptr;
    int series_cap = 0;
    int* series_idx = nullptr;
    DevScalars* h_ds = nullptr;
    unsigned* h_err = nullptr;
    // half-pair kernel
    double *Si = nullptr, *Sm = nullptr;
    void* Sj = nullptr;                 // source-side rows: double (FP64 form) or float (mixed form)
    float* tbox = nullptr;              // tile boxes (k_tile_boxes), 8 floats per tile
    unsigned char* Sjf = nullptr;       // per unit: its Sj row was written
    int4* jobs = nullptr;
    int* row_slots = nullptr;
    int* job_counter = nullptr;
    PairJobs pj{};
    // argument blocks and tunables
    ForceArgs fa{};
    StepArgs sa{};
    FinishArgs fz_base{};
    int nfb = 0, nvb = 0;
    int kernel = 2;                 // 1 rows, 2 pairs, 3 near lists (resolved, never 0)
    int kernel_req = 0;             // as requested (0 = auto)
    int seg = DEFAULT_SEG;
    int split = 1;                  // CTAs per unit of the half-pair kernel (yk_tuning.source_split)
    int tpt_req = 0;                // targets per thread as requested (yk_tuning.targets_per_thread; 0 auto)
    int pj_tt = 1;                  // targets per thread the job table was built for (pair_tt)
    bool seg_auto = true;           // pair_seg not set by the caller: the precision's default
    int sort_every = DEFAULT_SORT_EVERY;
    int graph_steps = DEFAULT_GRAPH_STEPS;
    long long step_count = 0;       // integrator steps since create
    double time = 0.0;
    bool pos_dirty = true;          // positions changed on the host: repack
    bool need_sort = true;
    // timers
    bool perf_on = false;
    size_t flush_bytes = 0;
    unsigned char* flush_buf = nullptr;
    std::vector<cudaEvent_t> ev_pool;
    int ev_used = 0;
    yk_perf perf{};
    // asynchronous state snapshots (checkpoint / save_config)
    double* snap = nullptr;          // 9n doubles: x, v, a
    cudaStream_t snap_stream = nullptr;
    cudaEvent_t snap_taken = nullptr, snap_done = nullptr;
    bool snap_pending = false;
    // cached K-step graphs
    std::vector<GraphEntry> graphs;
    unsigned long long graph_clock = 0;
    std::string errmsg;
};

static int fail(yk_ctx* c, int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c)
        c->errmsg = buf;
    else
        g_err_noctx = buf;
    return code;
}

#define CK(ctx, call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail((ctx), YK_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));  \
    } while (0)

// ---------------------------------------------------------------------------
// parameters -> kernel argument blocks

static double ev_cut(const yk_params& p, double scale)
{
    // int_ion_pure.f:125-130 (scale 1), int_nn.f:177-182 (scale vc)
    const double* xl = p.xl;
    if (p.rccut <= std::sqrt(xl[0] * xl[0] + xl[1] * xl[1] + xl[2] * xl[2]) / 2.0)
        return scale * std::exp(-(p.xmuc * p.rccut)) / p.rccut;
    return 0.0;
}

static void setup_args(yk_ctx* c)
{
    const yk_params& p = c->p;
    ForceArgs& f = c->fa;
    f = ForceArgs{};
    for (int k = 0; k < 3; ++k) {
        f.xl[k] = p.xl[k];
        const double hl = 0.5 * p.xl[k];
        std::memcpy(&f.hlb[k], &hl, sizeof hl);
    }
    f.rc2 = p.rccut * p.rccut;
    f.rn2 = p.rncut * p.rncut;
    f.xmuc = p.xmuc;
    f.vc = p.vc;
    f.evcut = (p.sim_type == YK_SIM_NUCLEON) ? ev_cut(p, p.vc) : ev_cut(p, 1.0);
    f.xpi = 1. / p.xpacket;
    f.xp2i = 1. / (2. * p.xpacket);
    f.aa = p.aa;
    f.aa2 = 2. * p.aa;
    f.bpc = p.bb + p.cc;
    f.bmc = p.bb - p.cc;
    if (p.sim_type == YK_SIM_PURE_ION)
        f.coef = p.frp * p.zi * p.zi * p.vc;
    else if (p.sim_type == YK_SIM_ION_MIXTURE)
        f.coef = p.frp * p.vc;
    else
        f.coef = 1.0;
    f.xmass = p.xmass;
    f.ai_xmass = p.ai * p.xmass;
    f.rc2f = (float)f.rc2;
    f.rn2f = (float)f.rn2;
    f.xmucf = (float)f.xmuc;
    f.evcutf = (float)f.evcut;
    f.vcf = (float)f.vc;
    f.xpif = (float)f.xpi;
    f.xp2if = (float)f.xp2i;
    f.aaf = (float)f.aa;
    f.aa2f = (float)f.aa2;
    f.bpcf = (float)f.bpc;
    f.bmcf = (float)f.bmc;
    // FP32 screen: widen each radius by 2^-19 L (16 ulp of the FP32 box
    // coordinates; the FP32 arithmetic of the shadow displacement is off by at
    // most ~5 ulp) plus 4 SHADOW_Q (the hi parts are on the SHADOW_Q grid, so
    // a displacement taken from them is off by up to SHADOW_Q per axis), and
    // the squares by a relative 2^-20 (three FP32 roundings of r^2 are 2e-7).
    {
        const double Lmax = std::max(p.xl[0], std::max(p.xl[1], p.xl[2]));
        const double delta = Lmax * std::ldexp(1.0, -19) + 4.0 * SHADOW_Q;
        const double grow = 1.0 + std::ldexp(1.0, -20);
        auto widen2 = [&](double r) {
            const double rs = (r + delta) * grow;
            const double r2 = rs * rs * grow;
            return r2 > 3.0e38 ? INFINITY : (float)r2;
        };
        for (int k = 0; k < 3; ++k) {
            f.Lf[k] = (float)p.xl[k];
            f.invLf[k] = (float)(1.0 / p.xl[k]);
            const double h = shadow_hi(p.xl[k]);
            f.Lh[k] = (float)h;
            f.Ll[k] = (float)(p.xl[k] - h);
        }
        f.scr_c2 = (p.sim_type == YK_SIM_NUCLEON && !p.coulomb_on) ? -1.0f : widen2(p.rccut);
        f.scr_n2 = (p.sim_type == YK_SIM_NUCLEON && p.nuclear_on) ? widen2(p.rncut) : -1.0f;
        // If every screened pair is closer than L/2 by a clear margin, the
        // image integers of the FP32 screen equal the reference's minimum-image
        // decision for every pair that interacts (a wrong image would put the
        // pair beyond L/2, outside every cutoff), and the pair kernel may use
        // them instead of the exact comparisons.
        const double Lmin = std::min(p.xl[0], std::min(p.xl[1], p.xl[2]));
        const double rscr = std::sqrt(std::max((double)f.scr_c2, (double)f.scr_n2));
        f.img_k = (std::isfinite(rscr) && rscr + std::ldexp(Lmax, -14) + 4.0 * SHADOW_Q < 0.5 * Lmin) ? 1 : 0;
        // The hi/lo displacement is exact up to its last rounding while every
        // coordinate and box length is below SHADOW_EXACT; a margin of 2 leaves
        // room for coordinates up to 2 L.
        f.lo = (f.img_k && 2.0 * Lmax < SHADOW_EXACT) ? 1 : 0;
        f.exp_ok = (std::isfinite(p.rccut) && p.xmuc >= 0.0 && p.xmuc * std::max(p.rccut, 1.0) <= 690.0) ? 1 : 0;
        f.hilo = (2.0 * Lmax < SHADOW_EXACT) ? 1 : 0;
        f.nn_short = (f.scr_n2 < 0.0f ||
                      std::sqrt((double)f.scr_n2) + std::ldexp(1.0, -5) < 0.5 * Lmin) ? 1 : 0;
        for (int k = 0; k < 3; ++k) {
            // the hi-part displacement is exact and within 2^-8 fm of the
            // reference's FP64 one, so |d| < L/2 - 2^-7 leaves the image
            // decision unambiguous
            const double t = 0.5 * p.xl[k] - std::ldexp(1.0, -7);
            float tf = (float)t;
            if ((double)tf > t) tf = std::nextafter(tf, 0.0f);
            f.hLm[k] = t > 0.0 ? tf : 0.0f;
        }
        f.hLmin = std::min(f.hLm[0], std::min(f.hLm[1], f.hLm[2]));
        f.coul_all = std::isinf(f.rc2f) ? 1 : 0;
    }
    f.n = c->n;
    f.nuclear_on = p.nuclear_on;
    f.coulomb_on = p.coulomb_on;
    f.mix_compat = (p.mix_mode == YK_MIX_COMPAT);

    StepArgs& s = c->sa;
    s = StepArgs{};
    for (int k = 0; k < 3; ++k) s.xl[k] = p.xl[k];
    s.dt = p.dt;
    s.afac = (p.integrator == YK_VV1) ? (0.5 * p.dt) * p.dt : 0.5 * (p.dt * p.dt);
    s.halfdt = 0.5 * p.dt;
    s.bfield = p.bfield;
    s.lorentz_c = (p.integrator == YK_VV3) ? (double)3.218404e-20f : 3.218404e-20;
    s.n = c->n;
    s.pack_w = (p.sim_type == YK_SIM_ION_MIXTURE || p.sim_type == YK_SIM_NUCLEON) ? 1 : 0;

    FinishArgs& z = c->fz_base;
    z = FinishArgs{};
    z.n = c->n;
    z.coef = f.coef;
    z.rho = p.rho;
    z.kT = p.kT;
    z.xmass = p.xmass;
    z.vol = p.xl[0] * p.xl[1] * p.xl[2];
    z.f_n = (double)(float)c->n;
    z.f_3n = (double)(3.0f * (float)c->n);

    c->nfb = (c->n + FBLOCK - 1) / FBLOCK;
    c->nvb = (c->n + VBLOCK - 1) / VBLOCK;
}

namespace yk {
void make_args(const yk_params& p, int n, ForceArgs* fa, StepArgs* sa, FinishArgs* fz)
{
    yk_ctx tmp;
    tmp.p = p;
    tmp.n = n;
    setup_args(&tmp);
    *fa = tmp.fa;
    *sa = tmp.sa;
    *fz = tmp.fz_base;
}

void count_launches(int k) { g_launches += k; }
}  // namespace yk

static void drop_graphs(yk_ctx* c)
{
    for (auto& g : c->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    c->graphs.clear();
}

// Scratch bytes of the half-pair kernel for n particles and segment length.
// Jobs of the half-pair kernel for M tiles, in dispatch order (costliest
// first), by guided self-scheduling: each job takes
//     d = clamp(W / (2 P), 1, smax)
// tiles from the start of the row with the most tiles left, W being the work
// not yet handed out and P the number of resident CTAs.  The bulk of the work
// goes out in long jobs (few target-side partials to write and combine, few
// job prologues), and the sizes shrink towards the end so that the persistent
// CTAs finish together.  row_slots[R] counts the Si slots of row R.
static void build_pair_jobs(int M, int smax, int P, std::vector<int4>& jobs, std::vector<int>& row_slots)
{
    jobs.clear();
    row_slots.assign(M, 0);
    std::vector<int> done(M, 0);
    long long W = (long long)M * (M + 1) / 2;
    std::priority_queue<std::pair<int, int>> rows;          // (tiles left, -R): longest row, then lowest R
    for (int R = 0; R < M; ++R) rows.push(std::make_pair(M - R, -R));
    while (!rows.empty()) {
        const int left = rows.top().first, R = -rows.top().second;
        rows.pop();
        const long long want = W / (2LL * std::max(P, 1));
        const int d = (int)std::min<long long>(left, std::min<long long>(smax, std::max<long long>(1, want)));
        const int C0 = R + done[R];
        jobs.push_back(make_int4(R, C0, C0 + d, row_slots[R]++));
        done[R] += d;
        W -= d;
        if (left > d) rows.push(std::make_pair(left - d, -R));
    }
}

// Jobs of the half-pair kernel when `split` CTAs share every unit: each unit
// (R, C) becomes `split` one-tile jobs, job `part` taking sources
// [part 128/split, (part+1) 128/split) of tile C and writing its own Si slot
// of row R.  The slot field carries the window: bits 0-19 the Si slot, 20-23
// the part, 24-27 log2(split).  Longest rows first.
static void build_split_jobs(int M, int split, std::vector<int4>& jobs, std::vector<int>& row_slots)
{
    jobs.clear();
    row_slots.assign(M, 0);
    int lg = 0;
    while ((1 << lg) < split) ++lg;
    for (int R = 0; R < M; ++R)
        for (int C = R; C < M; ++C)
            for (int part = 0; part < split; ++part)
                jobs.push_back(make_int4(R, C, C + 1, row_slots[R]++ | (part << 20) | (lg << 24)));
}

// Jobs of k_force_pairs2 (two targets per thread) for M tiles: a job
// (R, C0, C1, s), R even, takes source tiles C0 <= C < C1 (C >= R) against
// blocks R and R + 1 and writes Si slot s of both rows.  The same guided
// self-scheduling as build_pair_jobs over the block pairs, a tile of a pair
// counting one CTA tile step; row_slots of both rows count the pair's jobs.
static void build_pair_jobs2(int M, int smax, int P, std::vector<int4>& jobs, std::vector<int>& row_slots)
{
    jobs.clear();
    row_slots.assign(M, 0);
    const int np = (M + 1) / 2;
    std::vector<int> done(np, 0), cnt(np, 0);
    long long W = 0;
    std::priority_queue<std::pair<int, int>> rows;          // (tiles left, -pair)
    for (int p = 0; p < np; ++p) {
        W += M - 2 * p;
        rows.push(std::make_pair(M - 2 * p, -p));
    }
    while (!rows.empty()) {
        const int left = rows.top().first, p = -rows.top().second;
        rows.pop();
        const long long want = W / (2LL * std::max(P, 1));
        const int d = (int)std::min<long long>(left, std::min<long long>(smax, std::max<long long>(1, want)));
        const int R = 2 * p, C0 = R + done[p];
        jobs.push_back(make_int4(R, C0, C0 + d, cnt[p]++));
        done[p] += d;
        W -= d;
        if (left > d) rows.push(std::make_pair(left - d, -p));
    }
    for (int p = 0; p < np; ++p) {
        row_slots[2 * p] = cnt[p];
        if (2 * p + 1 < M) row_slots[2 * p + 1] = cnt[p];
    }
}

// Targets per thread of the half-pair kernel for the context as it stands:
// 2 (k_force_pairs2) for ion boxes on the paths that kernel has (FP64 with
// exact screen images, mixed with the hi/lo displacement) when requested,
// else 1.  Automatic (0): 2 for mixed-form ion boxes of TPT2_AUTO_MIN_N
// particles or more.  Measured on a B200 (force call, CUDA events): the
// 55,296-ion mixture mixed 1.050 -> 1.004 ms with two targets (jobs of up
// to 8 tiles), FP64 2.21 -> 2.46 ms (four CTAs per SM instead of five, and
// the larger warp boxes evaluate more masked pairs); the 4,096-ion OCP mixed
// 0.046 -> 0.048 ms (too few jobs); the 51,200-nucleon box mixed 1.15 ->
// 1.40 ms (its one-target kernel runs 7 CTAs per SM, and 64-nucleon warp
// boxes are large against the 11.5 fm nuclear cutoff), so nucleons take two
// targets only when asked (the tuner tries it).
constexpr int TPT2_AUTO_MIN_N = 16384;
constexpr int DEFAULT_SEG_MIXED_TT2 = 8;

static int pair_tt(const yk_ctx* c)
{
    if (c->split > 1 || c->kernel_req == 3) return 1;
    const bool mixed = c->p.precision == YK_PREC_MIXED;
    if (c->p.sim_type == YK_SIM_NUCLEON) {
        // nucleons: the mixed form on the hi/lo displacement only
        return (c->tpt_req == 2 && mixed && c->fa.hilo) ? 2 : 1;
    }
    if (c->p.sim_type != YK_SIM_PURE_ION && c->p.sim_type != YK_SIM_ION_MIXTURE) return 1;
    const int want = c->tpt_req != 0 ? c->tpt_req : ((mixed && c->n >= TPT2_AUTO_MIN_N) ? 2 : 1);
    if (want != 2) return 1;
    return (mixed ? c->fa.lo : (c->fa.img_k && c->fa.exp_ok)) ? 2 : 1;
}

static int auto_pair_seg(const yk_ctx* c)
{
    if (c->p.precision == YK_PREC_MIXED) return pair_tt(c) == 2 ? DEFAULT_SEG_MIXED_TT2 : DEFAULT_SEG_MIXED;
    return DEFAULT_SEG_FP64;
}

// Resident CTAs of the half-pair kernels on a device (6 per SM), for the job
// builder's job lengths.
static int pair_ctas(int dev)
{
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return 6 * sms;
}

// Bytes of one source-side (Sj) value: the row type of the form.
static size_t sj_elem_bytes(int precision)
{
    return precision == YK_PREC_MIXED ? sizeof(float) : sizeof(double);
}

static size_t pair_scratch_bytes(int n, int seg, int dev, int precision)
{
    const int M = (n + PB - 1) / PB;
    const size_t sj_bytes = sj_elem_bytes(precision) * ((size_t)M * (M + 1) / 2) * PB * 3;
    if (sj_bytes > PAIR_SCRATCH_BUDGET) return sj_bytes;       // too large anyway: skip the job list
    std::vector<int4> jobs;
    std::vector<int> slots;
    build_pair_jobs(M, seg, pair_ctas(dev), jobs, slots);
    const size_t nseg = M > 0 ? (size_t)*std::max_element(slots.begin(), slots.end()) : 0;
    return sj_bytes + sizeof(double) * ((size_t)M * nseg * PB * 3 + jobs.size() * NSCAL) +
           sizeof(int4) * jobs.size() + sizeof(int) * (size_t)M + sizeof(float) * 8 * (size_t)M +
           (size_t)M * (M + 1) / 2;
}

static void free_pairs(yk_ctx* c)
{
    cudaFree(c->Si);
    cudaFree(c->Sj);
    cudaFree(c->Sm);
    cudaFree(c->jobs);
    c->Si = c->Sm = nullptr;
    c->Sj = nullptr;
    c->jobs = nullptr;
    cudaFree(c->row_slots);
    c->row_slots = nullptr;
    cudaFree(c->tbox);
    c->tbox = nullptr;
    cudaFree(c->Sjf);
    c->Sjf = nullptr;
    c->pj = PairJobs{};
}

// Build the job table of the half-pair kernel (build_pair_jobs) and its
// scratch.  Unused Sj / Si slots are never read.
static int setup_pairs(yk_ctx* c)
{
    free_pairs(c);
    const int M = (c->n + PB - 1) / PB;
    if (c->seg_auto) c->seg = auto_pair_seg(c);
    std::vector<int4> jobs;
    std::vector<int> slots;
    // the near-list kernel reads whole tiles: no split for it
    c->pj_tt = pair_tt(c);
    if (c->split > 1 && c->kernel_req != 3) build_split_jobs(M, c->split, jobs, slots);
    else if (c->pj_tt == 2) build_pair_jobs2(M, c->seg, pair_ctas(c->dev) * 4 / 6, jobs, slots);
    else build_pair_jobs(M, c->seg, pair_ctas(c->dev), jobs, slots);
    const int nseg = M > 0 ? *std::max_element(slots.begin(), slots.end()) : 0;
    const size_t units = (size_t)M * (M + 1) / 2;
    CK(c, cudaMalloc(&c->Sj, sj_elem_bytes(c->p.precision) * units * PB * 3));
    CK(c, cudaMalloc((void**)&c->Si, sizeof(double) * (size_t)M * nseg * PB * 3));
    CK(c, cudaMalloc((void**)&c->Sm, sizeof(double) * jobs.size() * NSCAL));
    CK(c, cudaMalloc((void**)&c->jobs, sizeof(int4) * jobs.size()));
    CK(c, cudaMalloc((void**)&c->row_slots, sizeof(int) * (size_t)std::max(M, 1)));
    CK(c, cudaMalloc((void**)&c->tbox, sizeof(float) * 8 * (size_t)std::max(M, 1)));
    CK(c, cudaMalloc((void**)&c->Sjf, std::max<size_t>(units, 1)));
    CK(c, cudaMemcpy(c->jobs, jobs.data(), sizeof(int4) * jobs.size(), cudaMemcpyHostToDevice));
    CK(c, cudaMemcpy(c->row_slots, slots.data(), sizeof(int) * slots.size(), cudaMemcpyHostToDevice));
    c->pj.jobs = c->jobs;
    c->pj.row_slots = c->row_slots;
    c->pj.njobs = (int)jobs.size();
    c->pj.M = M;
    c->pj.nseg_max = nseg;
    c->pj.tbox = c->tbox;
    c->pj.Sjf = c->Sjf;
    return YK_OK;
}

// A new box can change whether k_force_pairs2 applies (fa.img_k, fa.lo):
// rebuild the job table when it does.
static int refresh_pair_tt(yk_ctx* c)
{
    if (c->kernel == 2 && pair_tt(c) != c->pj_tt) {
        CK(c, cudaSetDevice(c->dev));
        CK(c, cudaStreamSynchronize(c->stream));
        return setup_pairs(c);
    }
    return YK_OK;
}

static int resolve_kernel(yk_ctx* c)
{
    int k = c->kernel_req;
    // Automatic choice: the per-pair-screened half-pair kernel while its
    // scratch fits, else the row kernel.  (The near-list kernel, 3, is an
    // autotuner candidate: with nucleons in species-major slot order it is
    // 1.35x slower than kernel 2 on the 51,200-nucleon box, and on the
    // 55,296-ion mixture 1.5x slower.)
    if (k == 0) k = (pair_scratch_bytes(c->n, c->seg, c->dev, c->p.precision) <= PAIR_SCRATCH_BUDGET) ? 2 : 1;
    if (k == 2 || k == 3) {
        int rc = setup_pairs(c);
        if (rc) return rc;
    } else {
        free_pairs(c);
    }
    c->kernel = k;
    return YK_OK;
}

// ---------------------------------------------------------------------------
// launch helpers (all on c->stream; they only enqueue)

static cudaEvent_t next_event(yk_ctx* c)
{
    if (c->ev_used == (int)c->ev_pool.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        c->ev_pool.push_back(e);
    }
    return c->ev_pool[c->ev_used++];
}

// Morton sort (full) or repack with the current order (sort = false).
static int enqueue_order(yk_ctx* c, bool sort)
{
    const int n = c->n, nb = c->nvb;
    cudaStream_t st = c->stream;
    int k = 0;
    if (sort) {
        if (c->sort_every < 0) {
            // fixed identity order
            k_morton<<<nb, VBLOCK, 0, st>>>(c->x, n, 0.0, 0.0, 0.0, c->keys0, c->perm);
        } else {
            const bool nuc = c->p.sim_type == YK_SIM_NUCLEON;
            k_morton<<<nb, VBLOCK, 0, st>>>(c->x, n, 1024.0 / c->p.xl[0], 1024.0 / c->p.xl[1],
                                            1024.0 / c->p.xl[2], c->keys0, c->idx0, nuc ? c->zii : nullptr);
            size_t bytes = c->cub_bytes;
            cub::DeviceRadixSort::SortPairs(c->cub_tmp, bytes, c->keys0, c->keys1, c->idx0, c->perm, n,
                                            0, nuc ? 31 : 30, st);
        }
        ++k;
        c->need_sort = false;
    }
    k_apply_perm<<<nb, VBLOCK, 0, st>>>(c->perm, c->iperm, c->x, c->zii, c->pos, c->posf, n,
                                        c->sa.pack_w);
    c->pos_dirty = false;
    return k + 1;
}

// The mixed kernels have a variant that always takes the hi/lo shadow
// displacement (k_force_pairs<..., true>), for boxes that allow it: fa.lo
// for ions, fa.hilo for nucleons.
template <int SIM, int PREC>
static bool lo_path(const ForceArgs& fa)
{
    return PREC == PREC_MIXED && (SIM == SIM_NUCLEON ? fa.hilo != 0 : fa.lo != 0);
}

// Persistent grid of a PB-thread kernel on device dev (the current device):
// resident CTAs per SM times the SM count.  Cached per (kernel, device); the
// entries are atomics, so two first calls at once only repeat the query.
constexpr int GRID_CACHE_DEVICES = 64;

template <auto KERNEL>
static int persistent_grid(int dev)
{
    static std::atomic<int> cache[GRID_CACHE_DEVICES];
    const bool cached = dev >= 0 && dev < GRID_CACHE_DEVICES;
    int g = cached ? cache[dev].load(std::memory_order_relaxed) : 0;
    if (g == 0) {
        int per_sm = 0, sms = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, KERNEL, PB, 0);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        g = std::max(1, per_sm) * std::max(1, sms);
        if (cached) cache[dev].store(g, std::memory_order_relaxed);
    }
    return g;
}

template <int SIM, int PREC, bool MEAS>
static int launch_force_t(yk_ctx* c)
{
    if (c->kernel == 1) {
        k_force_rows<SIM, PREC, MEAS><<<c->nfb, FBLOCK, FORCE_SMEM, c->stream>>>(
            c->pos, c->posf, c->perm, c->aii, c->fa, c->a, c->fpart, c->err);
        return 1;
    }
    cudaMemsetAsync(c->job_counter, 0, sizeof(int), c->stream);
    PairJobs pj = c->pj;
    row_t<PREC>* Sj = static_cast<row_t<PREC>*>(c->Sj);
    const int njobs = c->pj.njobs;
    int k = 2;
    if (c->kernel == 3) {
        // the near-list kernel writes every Sj row and takes no tile boxes
        pj.tbox = nullptr;
        pj.Sjf = nullptr;
        const int grid = persistent_grid<k_force_near<SIM, PREC, MEAS>>(c->dev);
        k_force_near<SIM, PREC, MEAS><<<std::min(grid, njobs), PB, 0, c->stream>>>(
            c->pos, pj, c->job_counter, c->fa, c->Si, Sj, c->Sm, c->err);
    } else if (c->pj_tt == 2) {
        // two targets per thread: ion boxes with fa.lo (mixed) or fa.img_k and fa.exp_ok (FP64), nucleon boxes with
        // fa.hilo (mixed) only (pair_tt)
        if constexpr (SIM != SIM_NUCLEON || PREC == PREC_MIXED) {
            if (pairs_tile_boxes<SIM, PREC, PREC == PREC_MIXED>()) {
                k_tile_boxes<<<c->pj.M, PB, 0, c->stream>>>(c->posf, c->n, c->fa, c->tbox);
                ++k;
            } else {
                pj.tbox = nullptr;
            }
            const int grid = persistent_grid<k_force_pairs2<SIM, PREC, MEAS>>(c->dev);
            k_force_pairs2<SIM, PREC, MEAS><<<std::min(grid, njobs), PB, 0, c->stream>>>(
                c->pos, c->posf, pj, c->job_counter, c->fa, c->Si, Sj, c->Sm, c->err);
        }
    } else {
        if (lo_path<SIM, PREC>(c->fa) && pairs_tile_boxes<SIM, PREC, true>()) {
            k_tile_boxes<<<c->pj.M, PB, 0, c->stream>>>(c->posf, c->n, c->fa, c->tbox);
            ++k;
        } else {
            pj.tbox = nullptr;
        }
        if (lo_path<SIM, PREC>(c->fa)) {
            if constexpr (PREC == PREC_MIXED) {
                const int grid = persistent_grid<k_force_pairs<SIM, PREC, MEAS, true>>(c->dev);
                k_force_pairs<SIM, PREC, MEAS, true><<<std::min(grid, njobs), PB, 0, c->stream>>>(
                    c->pos, c->posf, pj, c->job_counter, c->fa, c->Si, Sj, c->Sm, c->err);
            }
        } else if (SIM != SIM_NUCLEON && c->fa.img_k && c->fa.exp_ok) {
            if constexpr (SIM != SIM_NUCLEON) {
                const int grid = persistent_grid<k_force_pairs<SIM, PREC, MEAS, false, true>>(c->dev);
                k_force_pairs<SIM, PREC, MEAS, false, true><<<std::min(grid, njobs), PB, 0, c->stream>>>(
                    c->pos, c->posf, pj, c->job_counter, c->fa, c->Si, Sj, c->Sm, c->err);
            }
        } else {
            const int grid = persistent_grid<k_force_pairs<SIM, PREC, MEAS>>(c->dev);
            k_force_pairs<SIM, PREC, MEAS><<<std::min(grid, njobs), PB, 0, c->stream>>>(
                c->pos, c->posf, pj, c->job_counter, c->fa, c->Si, Sj, c->Sm, c->err);
        }
    }
    // dynamic shared memory: the unit flags of one row and the list of its
    // written rows (comb_smem_bytes); above 40 KB (M > 8,000 tiles, only on an
    // explicit half-pair request past the scratch budget) it needs the opt-in
    const size_t fl_bytes = pj.Sjf ? comb_smem_bytes(c->pj.M) : 0;
    if (fl_bytes > (size_t)40 << 10)
        cudaFuncSetAttribute(k_combine<SIM, PREC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fl_bytes);
    k_combine<SIM, PREC><<<c->pj.M, COMB_THREADS, fl_bytes, c->stream>>>(c->Si, Sj, pj, c->perm, c->zii, c->aii,
                                                                         c->fa, c->a);
    return k;
}

template <int SIM>
static int launch_force_s(yk_ctx* c, bool meas)
{
    if (c->p.precision == YK_PREC_MIXED)
        return meas ? launch_force_t<SIM, PREC_MIXED, true>(c) : launch_force_t<SIM, PREC_MIXED, false>(c);
    return meas ? launch_force_t<SIM, PREC_FP64, true>(c) : launch_force_t<SIM, PREC_FP64, false>(c);
}

static int enqueue_force_body(yk_ctx* c, bool meas)
{
    switch (c->p.sim_type) {
    case YK_SIM_PURE_ION: return launch_force_s<SIM_PURE>(c, meas);
    case YK_SIM_ION_MIXTURE: return launch_force_s<SIM_MIX>(c, meas);
    case YK_SIM_NUCLEON: return launch_force_s<SIM_NUCLEON>(c, meas);
    default:  // 'B-field': a = 0 (int_control.f:80-81)
        cudaMemsetAsync(c->a, 0, sizeof(double) * 3 * (size_t)(c->n + 3), c->stream);
        return 0;
    }
}

// Returns the number of kernels enqueued.  Under yk_perf_enable the force
// call is bracketed by an event pair (events are consumed in pairs).
static int enqueue_force(yk_ctx* c, bool meas, bool timed = false)
{
    if (!timed) return enqueue_force_body(c, meas);
    cudaEventRecord(next_event(c), c->stream);
    int k = enqueue_force_body(c, meas);
    cudaEventRecord(next_event(c), c->stream);
    return k;
}

static int enqueue_finish(yk_ctx* c, bool meas, int kin_mode, bool series)
{
    FinishArgs z = c->fz_base;
    const bool has_force = c->p.sim_type != YK_SIM_BFIELD;
    z.force_mode = has_force ? 1 : 0;
    z.do_meas = meas ? 1 : 0;
    if (c->kernel >= 2) {
        z.nfp = (has_force && meas) ? c->pj.njobs : 0;
        z.half = 1.0;                   // each unique pair counted once
    } else {
        z.nfp = (has_force && meas) ? c->nfb : 0;
        z.half = 0.5;                   // each pair counted from both sides
    }
    z.kin_mode = kin_mode;
    z.nkp = (kin_mode == 2) ? c->nvb : 0;
    k_finish<<<1, 256, 0, c->stream>>>(c->kernel >= 2 ? c->Sm : c->fpart, c->kpart, z, c->a, c->ds,
                                       series ? c->series : nullptr, c->series_idx);
    return 1;
}

// One integrator step; returns kernels enqueued.  resort: refresh the
// Morton order before the step.
static int enqueue_newton(yk_ctx* c, bool meas, bool series, bool resort, bool timed = false)
{
    int k = 0;
    // A repack of positions set on the host is not needed here: the drift
    // moves them and k_pack_slots packs the moved ones.
    if (resort || c->need_sort) k += enqueue_order(c, true);
    const int nb = c->nvb;
    const int nb3 = (int)((3LL * c->n + VBLOCK - 1) / VBLOCK);   // element-wise drifts
    cudaStream_t st = c->stream;
    const StepArgs& s = c->sa;
    switch (c->p.integrator) {
    case YK_VV1:
        k_drift_vv1<<<nb3, VBLOCK, 0, st>>>(c->x, c->v, c->a, s);
        break;
    case YK_VV3:
        k_drift_vv3<<<nb, VBLOCK, 0, st>>>(c->x, c->v, c->a, c->zii, c->aii, s);
        break;
    default:
        k_drift_vv2<<<nb3, VBLOCK, 0, st>>>(c->x, c->v, c->vold, c->a, s);
        break;
    }
    k_pack_slots<<<nb, VBLOCK, 0, st>>>(c->perm, c->x, c->zii, c->pos, c->posf, c->n, s.pack_w);
    c->pos_dirty = false;
    k += 2;
    k += enqueue_force(c, meas, timed);
    int kin_mode;
    switch (c->p.integrator) {
    case YK_VV1:
        k_post_vv1<<<nb, VBLOCK, 0, st>>>(c->v, c->a, c->aii, c->kpart, s);
        kin_mode = 2;
        break;
    case YK_VV3:
        k_post_vv3<<<nb, VBLOCK, 0, st>>>(c->v, c->a, c->zii, c->aii, c->kpart, s);
        kin_mode = 2;
        break;
    default: {
        const bool bf = c->p.bfield != 0.0;
        if (meas) {
            if (bf) k_post_vv2<true, true><<<nb, VBLOCK, 0, st>>>(c->v, c->vold, c->a, c->zii, c->aii, c->kpart, s);
            else k_post_vv2<true, false><<<nb, VBLOCK, 0, st>>>(c->v, c->vold, c->a, c->zii, c->aii, c->kpart, s);
        } else {
            if (bf) k_post_vv2<false, true><<<nb, VBLOCK, 0, st>>>(c->v, c->vold, c->a, c->zii, c->aii, c->kpart, s);
            else k_post_vv2<false, false><<<nb, VBLOCK, 0, st>>>(c->v, c->vold, c->a, c->zii, c->aii, c->kpart, s);
        }
        kin_mode = meas ? 2 : 1;
    }
    }
    ++k;
    k += enqueue_finish(c, meas, kin_mode, series);
    return k;
}

static bool sort_due(const yk_ctx* c, long long step)
{
    return c->sort_every > 0 && step % c->sort_every == 0;
}

// Copy scalars and the error word back and wait for the stream.
static int sync_and_check(yk_ctx* c)
{
    CK(c, cudaMemcpyAsync(c->h_ds, c->ds, sizeof(DevScalars), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaMemcpyAsync(c->h_err, c->err, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    CK(c, cudaGetLastError());
    if (*c->h_err) {
        unsigned e = *c->h_err;
        cudaMemsetAsync(c->err, 0, sizeof(unsigned), c->stream);
        cudaStreamSynchronize(c->stream);
        if (e & ERR_TIMEOUT)
            return fail(c, YK_ERR_TIMEOUT, "a device-side wait timed out (error word 0x%x)", e);
        return fail(c, YK_ERR_CUDA, "device error word 0x%x", e);
    }
    return YK_OK;
}

static void fill_scalars(const yk_ctx* c, yk_scalars* out)
{
    if (!out) return;
    const DevScalars& s = *c->h_ds;
    out->ev = s.ev;
    out->vir = s.vir;
    out->px = s.px;
    out->ek = s.ek;
    for (int k = 0; k < 9; ++k) out->pp[k] = s.pp[k];
    out->time = c->time;
}

static bool all_finite(const double* p, size_t cnt)
{
    for (size_t i = 0; i < cnt; ++i)
        if (!std::isfinite(p[i])) return false;
    return true;
}

static int check_params(const yk_params* p)
{
    if (p->sim_type < YK_SIM_NUCLEON || p->sim_type > YK_SIM_BFIELD)
        return fail(nullptr, YK_ERR_ARG, "sim_type %d is not one of 1..4", p->sim_type);
    if (p->precision != YK_PREC_FP64 && p->precision != YK_PREC_MIXED)
        return fail(nullptr, YK_ERR_ARG, "precision %d is not 0 or 1", p->precision);
    if (p->integrator < YK_VV1 || p->integrator > YK_VV3)
        return fail(nullptr, YK_ERR_ARG, "integrator %d is not 1..3", p->integrator);
    if (!(p->dt > 0.0) || !std::isfinite(p->dt)) return fail(nullptr, YK_ERR_ARG, "dt must be > 0");
    for (int k = 0; k < 3; ++k)
        if (!(p->xl[k] > 0.0) || !std::isfinite(p->xl[k]))
            return fail(nullptr, YK_ERR_ARG, "box edge xl(%d) must be > 0", k + 1);
    if (p->sim_type == YK_SIM_PURE_ION && !(p->ai > 0.0))
        return fail(nullptr, YK_ERR_ARG, "pure-ion runs need ai > 0");
    if (!(p->xmass > 0.0)) return fail(nullptr, YK_ERR_ARG, "xmass must be > 0");
    if (p->sim_type == YK_SIM_NUCLEON && p->nuclear_on && !(p->xpacket > 0.0))
        return fail(nullptr, YK_ERR_ARG, "xpacket must be > 0");
    return YK_OK;
}

static int finish_run(yk_ctx* c, int nsteps, bool want_series, yk_scalars* series)
{
    if (want_series) {
        std::vector<double> h(13 * (size_t)nsteps);
        CK(c, cudaMemcpy(h.data(), c->series, sizeof(double) * h.size(), cudaMemcpyDeviceToHost));
        for (int s = 0; s < nsteps; ++s) {
            const double* o = &h[13 * (size_t)s];
            c->time = c->time + c->p.dt;
            series[s].ev = o[0];
            series[s].vir = o[1];
            series[s].px = o[2];
            series[s].ek = o[3];
            for (int q = 0; q < 9; ++q) series[s].pp[q] = o[4 + q];
            series[s].time = c->time;
        }
    } else {
        for (int s = 0; s < nsteps; ++s) c->time = c->time + c->p.dt;
    }
    return YK_OK;
}

// Graph of K steps starting at a step count divisible by sort_every (so the
// sort falls on local step 0) with measuring phase `phase` (local step l,
// 1-based, measures when (phase + l) % me == 0).
static GraphEntry* get_graph(yk_ctx* c, int K, int me, int phase, bool series, int* rc)
{
    *rc = YK_OK;
    for (auto& g : c->graphs)
        if (g.K == K && g.me == me && g.phase == phase && g.series == (series ? 1 : 0)) {
            g.stamp = ++c->graph_clock;
            return &g;
        }
    if ((int)c->graphs.size() >= MAX_GRAPHS) {
        auto it = std::min_element(c->graphs.begin(), c->graphs.end(),
                                   [](const GraphEntry& u, const GraphEntry& w) { return u.stamp < w.stamp; });
        cudaGraphExecDestroy(it->exec);
        c->graphs.erase(it);
    }
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        *rc = fail(c, YK_ERR_CUDA, "graph capture begin: %s", cudaGetErrorString(e));
        return nullptr;
    }
    int kernels = 0;
    for (int l = 1; l <= K; ++l) {
        const bool meas = me > 0 && (phase + l) % me == 0;
        const bool resort = c->sort_every > 0 && (l - 1) % c->sort_every == 0;
        kernels += enqueue_newton(c, meas, series, resort);
    }
    e = cudaStreamEndCapture(c->stream, &g);
    if (e != cudaSuccess) {
        *rc = fail(c, YK_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
        return nullptr;
    }
    GraphEntry ent;
    e = cudaGraphInstantiate(&ent.exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        *rc = fail(c, YK_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
        return nullptr;
    }
    ent.K = K;
    ent.me = me;
    ent.phase = phase;
    ent.series = series ? 1 : 0;
    ent.kernels = kernels;
    ent.stamp = ++c->graph_clock;
    c->graphs.push_back(ent);
    return &c->graphs.back();
}

// ---------------------------------------------------------------------------
// C-ABI

extern "C" {

const char* yk_version(void) { return YK_VERSION_STR; }

static long long copy_jobs(const std::vector<int4>& list, const std::vector<int>& slots, int* jobs,
                           long long max_jobs, int* row_slots);

long long yk_pair_jobs(int m, int cap, int ctas, int* jobs, long long max_jobs, int* row_slots)
{
    if (m < 1 || cap < 1 || ctas < 1 || max_jobs < 0 || (jobs == nullptr && max_jobs > 0))
        return -(long long)YK_ERR_ARG;
    std::vector<int4> list;
    std::vector<int> slots;
    build_pair_jobs(m, cap, ctas, list, slots);
    return copy_jobs(list, slots, jobs, max_jobs, row_slots);
}

long long yk_pair_jobs2(int m, int cap, int ctas, int* jobs, long long max_jobs, int* row_slots)
{
    if (m < 1 || cap < 1 || ctas < 1 || max_jobs < 0 || (jobs == nullptr && max_jobs > 0))
        return -(long long)YK_ERR_ARG;
    std::vector<int4> list;
    std::vector<int> slots;
    build_pair_jobs2(m, cap, ctas, list, slots);
    return copy_jobs(list, slots, jobs, max_jobs, row_slots);
}

static long long copy_jobs(const std::vector<int4>& list, const std::vector<int>& slots, int* jobs,
                           long long max_jobs, int* row_slots)
{
    const long long k = std::min<long long>(max_jobs, (long long)list.size());
    for (long long j = 0; j < k; ++j) {
        jobs[4 * j] = list[j].x;
        jobs[4 * j + 1] = list[j].y;
        jobs[4 * j + 2] = list[j].z;
        jobs[4 * j + 3] = list[j].w;
    }
    if (row_slots) std::copy(slots.begin(), slots.end(), row_slots);
    return (long long)list.size();
}

unsigned long long yk_kernel_launch_count(void) { return g_launches.load(); }

int yk_params_default(yk_params* p)
{
    if (!p) return YK_ERR_ARG;
    std::memset(p, 0, sizeof *p);
    p->sim_type = YK_SIM_PURE_ION;
    p->precision = YK_PREC_FP64;
    p->integrator = YK_VV2;
    p->mix_mode = YK_MIX_COMPAT;
    p->coulomb_on = 1;
    p->nuclear_on = 0;
    p->rccut = 1.0e50;                  // md_globals.f:120
    p->vc = (1.0 / 137.036) * 197.327;  // ALPHA*HBARC, md_globals.f:122
    p->frp = 1.0;
    p->xmass = 931.00;
    p->xpacket = 1.25;                  // md_globals.f:127-130
    p->aa = 110.0;
    p->bb = -26.0;
    p->cc = 24.0;
    return YK_OK;
}

const char* yk_last_error(const yk_ctx* ctx)
{
    return ctx ? ctx->errmsg.c_str() : g_err_noctx.c_str();
}

int yk_destroy(yk_ctx* c)
{
    if (!c) return fail(nullptr, YK_ERR_ARG, "ctx is NULL");
    cudaSetDevice(c->dev);
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->snap_stream) cudaStreamSynchronize(c->snap_stream);
    drop_graphs(c);
    free_pairs(c);
    void* bufs[] = {c->x, c->v, c->vold, c->a, c->zii, c->aii, c->pos, c->posf, c->perm, c->iperm,
                    c->keys0, c->keys1, c->idx0, c->cub_tmp, c->fpart, c->kpart, c->vpart, c->vsums,
                    c->ds, c->err,
                    c->series, c->series_idx, c->job_counter, c->flush_buf, c->snap, c->a_vtot, c->gofr,
                    c->stage, c->nonfinite};
    for (void* b : bufs) cudaFree(b);
    if (c->snap_taken) cudaEventDestroy(c->snap_taken);
    if (c->snap_done) cudaEventDestroy(c->snap_done);
    if (c->snap_stream) cudaStreamDestroy(c->snap_stream);
    cudaFreeHost(c->h_ds);
    cudaFreeHost(c->h_err);
    for (cudaEvent_t e : c->ev_pool) cudaEventDestroy(e);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return YK_OK;
}

int yk_create(const yk_params* p, int n, const double* x, const double* v, const double* zii,
              const double* aii, yk_ctx** out)
{
    if (!out) return fail(nullptr, YK_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!p || !x) return fail(nullptr, YK_ERR_ARG, "params and x are required");
    if (n < 1) return fail(nullptr, YK_ERR_ARG, "n must be >= 1 (got %d)", n);
    if (n > (1 << 26)) return fail(nullptr, YK_ERR_ARG, "n = %d exceeds 2^26", n);
    int rc = check_params(p);
    if (rc) return rc;
    if ((p->sim_type == YK_SIM_ION_MIXTURE || p->sim_type == YK_SIM_NUCLEON) && !zii)
        return fail(nullptr, YK_ERR_ARG, "this sim_type needs zii");
    if (p->sim_type == YK_SIM_ION_MIXTURE && !aii)
        return fail(nullptr, YK_ERR_ARG, "ion-mixture runs need aii");
    if (!all_finite(x, 3 * (size_t)n) || (v && !all_finite(v, 3 * (size_t)n)) ||
        (zii && !all_finite(zii, n)) || (aii && !all_finite(aii, n)))
        return fail(nullptr, YK_ERR_NONFINITE, "NaN or Inf in an input array");
    if (aii)
        for (int i = 0; i < n; ++i)
            if (!(aii[i] > 0.0)) return fail(nullptr, YK_ERR_ARG, "aii(%d) must be > 0", i);

    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1)
        return fail(nullptr, YK_ERR_CUDA, "no CUDA device available");
    if (p->device < 0 || p->device >= ndev)
        return fail(nullptr, YK_ERR_ARG, "device %d out of range (have %d)", p->device, ndev);

    yk_ctx* c = new yk_ctx();
    c->p = *p;
    c->n = n;
    c->dev = p->device;
    c->time = p->time;
    if (cudaSetDevice(c->dev) != cudaSuccess) {
        delete c;
        return fail(nullptr, YK_ERR_CUDA, "cudaSetDevice(%d) failed", p->device);
    }
    setup_args(c);
    c->seg = auto_pair_seg(c);

    // HBM admission: refuse up front rather than fail half-way.
    size_t cub_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, (unsigned*)nullptr, (unsigned*)nullptr,
                                    (int*)nullptr, (int*)nullptr, n, 0, 31);
    size_t bytes = sizeof(double) * (3 * (size_t)n * 3 + 3 * (size_t)(n + 3) + 2 * (size_t)n) +
                   (sizeof(double4) + sizeof(float) * SHADOW_FLOATS / SHADOW_TILE) * ((size_t)n + SHADOW_TILE) + sizeof(int) * 5 * (size_t)n + cub_bytes +
                   sizeof(double) * (size_t)(8 * c->nfb + NKIN * c->nvb) + 4096;
    const size_t pair_bytes = pair_scratch_bytes(n, c->seg, c->dev, p->precision);
    const bool pairs_fit = pair_bytes <= PAIR_SCRATCH_BUDGET;
    if (pairs_fit) bytes += pair_bytes;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        delete c;
        return fail(nullptr, YK_ERR_CUDA, "cudaMemGetInfo failed");
    }
    if (bytes + (64u << 20) > free_b) {
        delete c;
        return fail(nullptr, YK_ERR_NOMEM, "needs %zu bytes, %zu free", bytes, free_b);
    }

#define ALLOC(ptr, cnt)                                                                 \
    do {                                                                                \
        if (cudaMalloc((void**)&(ptr), sizeof(*(ptr)) * (size_t)(cnt)) != cudaSuccess) { \
            yk_destroy(c);                                                              \
            return fail(nullptr, YK_ERR_NOMEM, "cudaMalloc of " #ptr " failed");        \
        }                                                                               \
    } while (0)
    ALLOC(c->x, 3 * (size_t)n);
    ALLOC(c->v, 3 * (size_t)n);
    ALLOC(c->vold, 3 * (size_t)n);
    ALLOC(c->a, 3 * (size_t)(n + 3));
    ALLOC(c->zii, n);
    ALLOC(c->aii, n);
    ALLOC(c->pos, n);
    ALLOC(c->posf, (size_t)SHADOW_FLOATS * ((n + SHADOW_TILE - 1) / SHADOW_TILE));
    ALLOC(c->perm, n);
    ALLOC(c->iperm, n);
    ALLOC(c->keys0, n);
    ALLOC(c->keys1, n);
    ALLOC(c->idx0, n);
    ALLOC(c->fpart, 8 * (size_t)c->nfb);
    ALLOC(c->kpart, NKIN * (size_t)c->nvb);
    ALLOC(c->vpart, NVSUM * (size_t)c->nvb);
    ALLOC(c->vsums, 8);
    ALLOC(c->ds, 1);
    ALLOC(c->err, 1);
    ALLOC(c->series_idx, 1);
    ALLOC(c->job_counter, 1);
#undef ALLOC
    c->cub_bytes = cub_bytes;
    if (cudaMalloc(&c->cub_tmp, std::max<size_t>(cub_bytes, 16)) != cudaSuccess) {
        yk_destroy(c);
        return fail(nullptr, YK_ERR_NOMEM, "sort scratch");
    }
    if (cudaMallocHost((void**)&c->h_ds, sizeof(DevScalars)) != cudaSuccess ||
        cudaMallocHost((void**)&c->h_err, sizeof(unsigned)) != cudaSuccess) {
        yk_destroy(c);
        return fail(nullptr, YK_ERR_NOMEM, "pinned host staging failed");
    }
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        yk_destroy(c);
        return fail(nullptr, YK_ERR_CUDA, "stream creation failed");
    }
    if ((rc = resolve_kernel(c)) != YK_OK) {
        std::string m = c->errmsg;
        yk_destroy(c);
        return fail(nullptr, rc, "%s", m.c_str());
    }
    cudaStream_t st = c->stream;
    std::vector<double> fill(n);
    cudaMemcpyAsync(c->x, x, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st);
    if (v) cudaMemcpyAsync(c->v, v, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st);
    else cudaMemsetAsync(c->v, 0, sizeof(double) * 3 * n, st);
    cudaMemsetAsync(c->vold, 0, sizeof(double) * 3 * n, st);
    cudaMemsetAsync(c->a, 0, sizeof(double) * 3 * (n + 3), st);
    if (zii) {
        cudaMemcpyAsync(c->zii, zii, sizeof(double) * n, cudaMemcpyHostToDevice, st);
    } else {
        for (int i = 0; i < n; ++i) fill[i] = p->zi;
        cudaMemcpyAsync(c->zii, fill.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st);
        cudaStreamSynchronize(st);
    }
    if (aii) {
        cudaMemcpyAsync(c->aii, aii, sizeof(double) * n, cudaMemcpyHostToDevice, st);
    } else {
        for (int i = 0; i < n; ++i) fill[i] = p->ai > 0.0 ? p->ai : 1.0;
        cudaMemcpyAsync(c->aii, fill.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st);
    }
    cudaMemsetAsync(c->posf, 0, sizeof(float) * SHADOW_FLOATS * ((n + SHADOW_TILE - 1) / SHADOW_TILE), st);
    cudaMemsetAsync(c->ds, 0, sizeof(DevScalars), st);
    cudaMemsetAsync(c->err, 0, sizeof(unsigned), st);
    cudaMemsetAsync(c->series_idx, 0, sizeof(int), st);
    c->need_sort = true;
    g_launches += enqueue_order(c, true);
    if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
        yk_destroy(c);
        return fail(nullptr, YK_ERR_CUDA, "initial upload failed");
    }
    *out = c;
    return YK_OK;
}

int yk_get_tuning(yk_ctx* c, yk_tuning* out)
{
    if (!c || !out) return fail(c, YK_ERR_ARG, "ctx and out are required");
    out->force_kernel = c->kernel;          // the resolved kernel (1 rows, 2 pairs, 3 near lists)
    out->pair_seg = c->seg;
    out->sort_every = c->sort_every;
    out->graph_steps = c->graph_steps;
    out->source_split = c->kernel == 2 ? c->split : 1;
    out->targets_per_thread = c->kernel == 2 ? c->pj_tt : 1;
    return YK_OK;
}

int yk_set_tuning(yk_ctx* c, const yk_tuning* t)
{
    if (!c || !t) return fail(c, YK_ERR_ARG, "ctx and tuning are required");
    if (t->force_kernel < 0 || t->force_kernel > 3) return fail(c, YK_ERR_ARG, "force_kernel must be 0..3");
    if (t->pair_seg < 0 || t->graph_steps < 0 || t->sort_every < -1)
        return fail(c, YK_ERR_ARG, "bad tuning values");
    if (t->source_split != 0 && t->source_split != 1 && t->source_split != 2 && t->source_split != 4)
        return fail(c, YK_ERR_ARG, "source_split must be 0, 1, 2 or 4");
    if (t->targets_per_thread < 0 || t->targets_per_thread > 2)
        return fail(c, YK_ERR_ARG, "targets_per_thread must be 0, 1 or 2");
    c->split = t->source_split > 1 ? t->source_split : 1;
    c->tpt_req = t->targets_per_thread;
    CK(c, cudaSetDevice(c->dev));
    CK(c, cudaStreamSynchronize(c->stream));
    drop_graphs(c);
    c->kernel_req = t->force_kernel;
    c->seg_auto = t->pair_seg <= 0;
    c->seg = t->pair_seg > 0 ? t->pair_seg : auto_pair_seg(c);
    const int old_sort = c->sort_every;
    c->sort_every = t->sort_every == 0 ? DEFAULT_SORT_EVERY : t->sort_every;
    c->graph_steps = t->graph_steps > 0 ? t->graph_steps : DEFAULT_GRAPH_STEPS;
    if (old_sort != c->sort_every) c->need_sort = true;
    int rc = resolve_kernel(c);
    if (rc) return rc;
    return YK_OK;
}

int yk_accel(yk_ctx* c, int do_meas, double* a_out, yk_scalars* out)
{
    if (!c) return fail(nullptr, YK_ERR_ARG, "ctx is NULL");
    CK(c, cudaSetDevice(c->dev));
    const bool meas = do_meas != 0;
    int k = 0;
    if (c->need_sort || c->pos_dirty) k += enqueue_order(c, c->need_sort);
    k += enqueue_force(c, meas);
    k += enqueue_finish(c, meas, 0, false);
    g_launches += k;
    if (a_out)
        CK(c, cudaMemcpyAsync(a_out, c->a, sizeof(double) * 3 * (size_t)(c->n + 3),
                              cudaMemcpyDeviceToHost, c->stream));
    int rc = sync_and_check(c);
    if (rc) return rc;
    fill_scalars(c, out);
    return YK_OK;
}

int yk_vtot(yk_ctx* c, double* ev, double* px)
{
    if (!c || !ev || !px) return fail(c, YK_ERR_ARG, "ctx, ev and px are required");
    CK(c, cudaSetDevice(c->dev));
    if (!c->a_vtot) CK(c, cudaMalloc(&c->a_vtot, sizeof(double) * 3 * (size_t)(c->n + 3)));
    // a measuring force call whose accelerations go to a side buffer, so the
    // state's a (which the next step's drift reads) is left as it was
    int k = 0;
    if (c->need_sort || c->pos_dirty) k += enqueue_order(c, c->need_sort);
    std::swap(c->a, c->a_vtot);
    k += enqueue_force(c, true);
    k += enqueue_finish(c, true, 0, false);
    std::swap(c->a, c->a_vtot);
    g_launches += k;
    int rc = sync_and_check(c);
    if (rc) return rc;
    yk_scalars s;
    fill_scalars(c, &s);
    *ev = s.ev;
    *px = s.px;
    return YK_OK;
}

int yk_gofr_counts(yk_ctx* c, int nbin, double* counts)
{
    if (!c || !counts) return fail(c, YK_ERR_ARG, "ctx and counts are required");
    if (nbin < 1 || nbin > GOFR_MAX_BINS) return fail(c, YK_ERR_ARG, "nbin must be 1..%d (got %d)", GOFR_MAX_BINS, nbin);
    CK(c, cudaSetDevice(c->dev));
    if (c->gofr_cap < nbin) {
        if (c->gofr) CK(c, cudaFree(c->gofr));
        c->gofr = nullptr;
        c->gofr_cap = 0;
        CK(c, cudaMalloc((void**)&c->gofr, sizeof(unsigned long long) * (size_t)nbin));
        c->gofr_cap = nbin;
    }
    int k = 0;
    if (c->need_sort || c->pos_dirty) k += enqueue_order(c, c->need_sort);
    GofrArgs g{};
    const double xlmin = std::min(c->p.xl[0], std::min(c->p.xl[1], c->p.xl[2]));
    for (int d = 0; d < 3; ++d) g.xl[d] = c->p.xl[d];
    const float f4 = (2.0f * (float)nbin) / std::sqrt(3.0f);     // REAL*4 in g.f:56
    g.fac2 = (double)f4 / xlmin;
    g.tiny = (double)1.e-15f;
    g.nbin = nbin;
    g.n = c->n;
    g.M = (c->n + GOFR_BLOCK - 1) / GOFR_BLOCK;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->dev);
    const long long units = (long long)g.M * (g.M + 1) / 2;
    const int grid = (int)std::min<long long>(units, 8LL * sms);
    const size_t smem = GOFR_BLOCK * sizeof(double4) + sizeof(unsigned) * (size_t)nbin;
    CK(c, cudaFuncSetAttribute(k_gofr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    CK(c, cudaMemsetAsync(c->gofr, 0, sizeof(unsigned long long) * (size_t)nbin, c->stream));
    k_gofr<<<grid, GOFR_BLOCK, smem, c->stream>>>(c->pos, g, c->gofr);
    g_launches += k + 1;
    std::vector<unsigned long long> h(nbin);
    CK(c, cudaMemcpyAsync(h.data(), c->gofr, sizeof(unsigned long long) * (size_t)nbin, cudaMemcpyDeviceToHost,
                          c->stream));
    int rc = sync_and_check(c);
    if (rc) return rc;
    for (int b = 0; b < nbin; ++b) counts[b] += (double)h[b];
    return YK_OK;
}

int yk_newton(yk_ctx* c, int do_meas, yk_scalars* out)
{
    if (!c) return fail(nullptr, YK_ERR_ARG, "ctx is NULL");
    CK(c, cudaSetDevice(c->dev));
    int k = enqueue_newton(c, do_meas != 0, false, sort_due(c, c->step_count));
    g_launches += k;
    int rc = sync_and_check(c);
    if (rc) return rc;
    c->step_count += 1;
    c->time = c->time + c->p.dt;            // vel_verlet_2.f:114
    fill_scalars(c, out);
    return YK_OK;
}

int yk_run(yk_ctx* c, int nsteps, int meas_every, yk_scalars* series)
{
    if (!c) return fail(nullptr, YK_ERR_ARG, "ctx is NULL");
    if (nsteps < 0 || meas_every < 0) return fail(c, YK_ERR_ARG, "nsteps and meas_every must be >= 0");
    if (nsteps == 0) return YK_OK;
    CK(c, cudaSetDevice(c->dev));
    const bool want_series = series != nullptr;
    if (want_series && c->series_cap < nsteps) {
        drop_graphs(c);
        cudaFree(c->series);
        c->series = nullptr;
        c->series_cap = 0;
        CK(c, cudaMalloc((void**)&c->series, sizeof(double) * 13 * (size_t)nsteps));
        c->series_cap = nsteps;
    }
    CK(c, cudaMemsetAsync(c->series_idx, 0, sizeof(int), c->stream));
    const int me = meas_every;
    auto meas_at = [&](int s) { return me > 0 && s % me == 0; };
    int k = 0;
    if (c->perf_on) {
        // Timed path: step by step, an event pair around every step (after
        // its L2 flush, so the flush lies between timed steps) and one
        // around every force call inside it.
        c->ev_used = 0;
        std::vector<int> step_ev;
        step_ev.reserve(2 * (size_t)nsteps);
        for (int s = 1; s <= nsteps; ++s) {
            if (c->flush_bytes)
                CK(c, cudaMemsetAsync(c->flush_buf, s & 0xff, c->flush_bytes, c->stream));
            step_ev.push_back(c->ev_used);
            CK(c, cudaEventRecord(next_event(c), c->stream));
            k += enqueue_newton(c, meas_at(s), want_series, sort_due(c, c->step_count), true);
            c->step_count += 1;
            step_ev.push_back(c->ev_used);
            CK(c, cudaEventRecord(next_event(c), c->stream));
        }
        g_launches += k;
        int rc = sync_and_check(c);
        if (rc) return rc;
        float ms = 0.f;
        for (int s = 0; s < nsteps; ++s) {
            const int a = step_ev[2 * s], b = step_ev[2 * s + 1];
            CK(c, cudaEventElapsedTime(&ms, c->ev_pool[a], c->ev_pool[b]));
            c->perf.run_ms += ms;
            // the force calls' event pairs lie between the step's own two
            for (int q = a + 1; q + 1 < b; q += 2) {
                CK(c, cudaEventElapsedTime(&ms, c->ev_pool[q], c->ev_pool[q + 1]));
                c->perf.force_ms += ms;
                c->perf.force_calls += 1;
            }
        }
        c->perf.steps += nsteps;
        return finish_run(c, nsteps, want_series, series);
    }
    // Eager steps until the step count is aligned with the sort cadence,
    // then graphs of K steps, then the rest.  K is a multiple of sort_every
    // and, when that keeps the graph within 4 graph_steps, of meas_every
    // too, so that every graph of the run starts at the same measuring
    // phase and one captured graph serves them all.
    int s = 1;
    int unit = c->sort_every > 0 ? c->sort_every : 1;
    if (me > 0) {
        const long long l = (long long)unit / std::gcd(unit, me) * me;
        if (l <= 4LL * std::max(c->graph_steps, unit)) unit = (int)l;
    }
    const int K = c->sort_every > 0 || me > 0 ? unit * std::max(1, c->graph_steps / unit) : c->graph_steps;
    while (s <= nsteps && c->sort_every > 0 && c->step_count % c->sort_every != 0) {
        k += enqueue_newton(c, meas_at(s), want_series, sort_due(c, c->step_count));
        c->step_count += 1;
        ++s;
    }
    if (c->pos_dirty || c->need_sort) k += enqueue_order(c, c->need_sort);
    while (s + K - 1 <= nsteps) {
        int rc = YK_OK;
        GraphEntry* g = get_graph(c, K, me, me > 0 ? (s - 1) % me : 0, want_series, &rc);
        if (!g) return rc;
        CK(c, cudaGraphLaunch(g->exec, c->stream));
        k += g->kernels;
        c->step_count += K;
        s += K;
    }
    for (; s <= nsteps; ++s) {
        k += enqueue_newton(c, meas_at(s), want_series, sort_due(c, c->step_count));
        c->step_count += 1;
    }
    g_launches += k;
    int rc = sync_and_check(c);
    if (rc) return rc;
    return finish_run(c, nsteps, want_series, series);
}

int yk_get_state(yk_ctx* c, double* x, double* v, double* vold, double* a)
{
    if (!c) return fail(nullptr, YK_ERR_ARG, "ctx is NULL");
    CK(c, cudaSetDevice(c->dev));
    const size_t b = sizeof(double) * 3 * (size_t)c->n;
    if (x) CK(c, cudaMemcpyAsync(x, c->x, b, cudaMemcpyDeviceToHost, c->stream));
    if (v) CK(c, cudaMemcpyAsync(v, c->v, b, cudaMemcpyDeviceToHost, c->stream));
    if (vold) CK(c, cudaMemcpyAsync(vold, c->vold, b, cudaMemcpyDeviceToHost, c->stream));
    if (a) CK(c, cudaMemcpyAsync(a, c->a, b, cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    return YK_OK;
}

int yk_snapshot_wait(yk_ctx* c)
{
    if (!c) return fail(nullptr, YK_ERR_ARG, "ctx is NULL");
    if (!c->snap_pending) return YK_OK;
    CK(c, cudaSetDevice(c->dev));
    c->snap_pending = false;
    CK(c, cudaEventSynchronize(c->snap_done));
    return YK_OK;
}

int yk_snapshot_begin(yk_ctx* c, double* x, double* v, double* a)
{
    if (!c) return fail(nullptr, YK_ERR_ARG, "ctx is NULL");
    CK(c, cudaSetDevice(c->dev));
    int rc = yk_snapshot_wait(c);           // one snapshot in flight at a time
    if (rc) return rc;
    if (!c->snap) {
        CK(c, cudaMalloc(&c->snap, sizeof(double) * 9 * (size_t)c->n));
        CK(c, cudaStreamCreateWithFlags(&c->snap_stream, cudaStreamNonBlocking));
        CK(c, cudaEventCreateWithFlags(&c->snap_taken, cudaEventDisableTiming));
        CK(c, cudaEventCreateWithFlags(&c->snap_done, cudaEventDisableTiming));
    }
    const size_t cnt = 3 * (size_t)c->n, b = sizeof(double) * cnt;
    double* host[3] = {x, v, a};
    const double* src[3] = {c->x, c->v, c->a};
    // device-to-device on the engine's stream: ordered after every step already
    // enqueued, and the next step may overwrite x, v, a as soon as it is done
    for (int k = 0; k < 3; ++k)
        if (host[k]) CK(c, cudaMemcpyAsync(c->snap + k * cnt, src[k], b, cudaMemcpyDeviceToDevice, c->stream));
    CK(c, cudaEventRecord(c->snap_taken, c->stream));
    // device-to-host on the side stream, overlapping the following steps
    CK(c, cudaStreamWaitEvent(c->snap_stream, c->snap_taken, 0));
    for (int k = 0; k < 3; ++k)
        if (host[k]) CK(c, cudaMemcpyAsync(host[k], c->snap + k * cnt, b, cudaMemcpyDeviceToHost, c->snap_stream));
    CK(c, cudaEventRecord(c->snap_done, c->snap_stream));
    c->snap_pending = true;
    return YK_OK;
}

int yk_set_state(yk_ctx* c, const double* x, const double* v, const double* vold, const double* a)
{
    if (!c) return fail(nullptr, YK_ERR_ARG, "ctx is NULL");
    CK(c, cudaSetDevice(c->dev));
    const size_t cnt = 3 * (size_t)c->n;
    const size_t b = sizeof(double) * cnt;
    if (!c->stage) {
        CK(c, cudaMalloc((void**)&c->stage, 4 * b));
        CK(c, cudaMalloc((void**)&c->nonfinite, sizeof(unsigned)));
    }
    // The arrays are copied into a staging buffer and checked for NaN / Inf
    // on the device; only if all are finite does k_commit_state move them
    // into the state, so a rejected call leaves the state as it was.
    const double* src[4] = {x, v, vold, a};
    double* dst[4] = {c->x, c->v, c->vold, c->a};
    CK(c, cudaMemsetAsync(c->nonfinite, 0, sizeof(unsigned), c->stream));
    int k = 0;
    for (int q = 0; q < 4; ++q) {
        if (!src[q]) continue;
        CK(c, cudaMemcpyAsync(c->stage + q * cnt, src[q], b, cudaMemcpyHostToDevice, c->stream));
        k_check_finite<<<(int)((cnt + 255) / 256), 256, 0, c->stream>>>(c->stage + q * cnt, cnt, c->nonfinite);
        ++k;
    }
    for (int q = 0; q < 4; ++q) {
        if (!src[q]) continue;
        k_commit_state<<<(int)((cnt + 255) / 256), 256, 0, c->stream>>>(c->stage + q * cnt, dst[q], cnt,
                                                                         c->nonfinite);
        ++k;
    }
    unsigned bad = 0;
    CK(c, cudaMemcpyAsync(c->h_err, c->nonfinite, sizeof(unsigned), cudaMemcpyDeviceToHost, c->stream));
    CK(c, cudaStreamSynchronize(c->stream));
    bad = *c->h_err;
    *c->h_err = 0;
    g_launches += k;
    if (bad) return fail(c, YK_ERR_NONFINITE, "NaN or Inf in a state array");
    // new positions keep the current slot order (the next scheduled sort
    // refreshes it); the packed copies are rebuilt by the next call that
    // reads them (a force call) or moves the positions first (a step)
    if (x) c->pos_dirty = true;
    return YK_OK;
}

int yk_set_box(yk_ctx* c, const double xl[3])
{
    if (!c || !xl) return fail(c, YK_ERR_ARG, "ctx and xl are required");
    for (int k = 0; k < 3; ++k)
        if (!(xl[k] > 0.0) || !std::isfinite(xl[k])) return fail(c, YK_ERR_ARG, "xl must be > 0");
    bool same = true;
    for (int k = 0; k < 3; ++k) same = same && c->p.xl[k] == xl[k];
    if (same) return YK_OK;
    for (int k = 0; k < 3; ++k) c->p.xl[k] = xl[k];
    setup_args(c);
    drop_graphs(c);
    return refresh_pair_tt(c);
}

// ---- gen_utils.f / strain.f on the device ---------------------------------

static_assert(TBLOCK == VBLOCK, "k_vsums runs on the Verlet block count nvb");

static int enqueue_vsums(yk_ctx* c)
{
    k_vsums<<<c->nvb, TBLOCK, 0, c->stream>>>(c->v, c->aii, c->n, c->vpart);
    k_vreduce<<<1, TBLOCK, 0, c->stream>>>(c->vpart, c->nvb, c->vsums);
    return 2;
}

static int enqueue_tnorm(yk_ctx* c)
{
    int k = enqueue_vsums(c);
    k_vscale<<<(3 * c->n + 255) / 256, 256, 0, c->stream>>>(c->v, c->n, c->vsums, c->p.xmass,
                                                           (double)(float)c->n, c->p.kT);
    return k + 1;
}

int yk_ttot(yk_ctx* c, double* eka)
{
    if (!c || !eka) return fail(c, YK_ERR_ARG, "ctx and eka are required");
    CK(c, cudaSetDevice(c->dev));
    g_launches += enqueue_vsums(c);
    double h[NVSUM];
    CK(c, cudaMemcpyAsync(h, c->vsums, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    int rc = sync_and_check(c);
    if (rc) return rc;
    *eka = (0.5 * c->p.xmass * h[4]) / (double)(float)c->n;     // gen_utils.f:52
    return YK_OK;
}

int yk_tnorm(yk_ctx* c)
{
    if (!c) return fail(nullptr, YK_ERR_ARG, "ctx is NULL");
    if (!(c->p.kT > 0.0)) return fail(c, YK_ERR_ARG, "tnorm needs kT > 0");
    CK(c, cudaSetDevice(c->dev));
    g_launches += enqueue_tnorm(c);
    return sync_and_check(c);
}

int yk_cancel_vcom(yk_ctx* c)
{
    if (!c) return fail(nullptr, YK_ERR_ARG, "ctx is NULL");
    if (!(c->p.kT > 0.0)) return fail(c, YK_ERR_ARG, "cancel_vcom ends with tnorm, which needs kT > 0");
    CK(c, cudaSetDevice(c->dev));
    int k = enqueue_vsums(c);
    k_vshift<<<(3 * c->n + 255) / 256, 256, 0, c->stream>>>(c->v, c->n, c->vsums);
    k += 1 + enqueue_tnorm(c);
    g_launches += k;
    return sync_and_check(c);
}

int yk_strain(yk_ctx* c, const double deps[3], const double xl0[3], double xl_out[3])
{
    if (!c || !deps || !xl0) return fail(c, YK_ERR_ARG, "ctx, deps and xl0 are required");
    CK(c, cudaSetDevice(c->dev));
    // strain.f:31-69: new edge lengths (volume-preserving normal strain)
    const double XNOSTRAIN = 1000.0, dt = c->p.dt;
    double xl[3] = {c->p.xl[0], c->p.xl[1], c->p.xl[2]};
    const int sel = (deps[0] != XNOSTRAIN ? 1 : 0) + (deps[1] != XNOSTRAIN ? 2 : 0) + (deps[2] != XNOSTRAIN ? 4 : 0);
    switch (sel) {
    case 0: break;
    case 1:
        xl[0] = xl[0] + deps[0] * dt * xl0[0];
        xl[1] = xl0[1] * std::sqrt(xl0[0] / xl[0]);
        xl[2] = xl0[2] * std::sqrt(xl0[0] / xl[0]);
        break;
    case 2:
        xl[1] = xl[1] + deps[1] * dt * xl0[1];
        xl[0] = xl0[0] * std::sqrt(xl0[1] / xl[1]);
        xl[2] = xl0[2] * std::sqrt(xl0[1] / xl[1]);
        break;
    case 3:
        xl[0] = xl[0] + deps[0] * dt * xl0[0];
        xl[1] = xl[1] + deps[1] * dt * xl0[1];
        xl[2] = xl0[2] * (xl0[0] / xl[0]) * (xl0[1] / xl[1]);
        break;
    case 4:
        xl[2] = xl[2] + deps[2] * dt * xl0[2];
        xl[0] = xl0[0] * std::sqrt(xl0[2] / xl[2]);
        xl[1] = xl0[1] * std::sqrt(xl0[2] / xl[2]);
        break;
    case 5:
        xl[0] = xl[0] + deps[0] * dt * xl0[0];
        xl[2] = xl[2] + deps[2] * dt * xl0[2];
        xl[1] = xl0[1] * (xl0[0] / xl[0]) * (xl0[2] / xl[2]);
        break;
    case 6:
        xl[1] = xl[1] + deps[1] * dt * xl0[1];
        xl[2] = xl[2] + deps[2] * dt * xl0[2];
        xl[0] = xl0[0] * (xl0[1] / xl[1]) * (xl0[2] / xl[2]);
        break;
    default:
        xl[0] = xl[0] + deps[0] * dt * xl0[0];
        xl[1] = xl[1] + deps[1] * dt * xl0[1];
        xl[2] = xl[2] + deps[2] * dt * xl0[2];
        break;
    }
    for (int k = 0; k < 3; ++k)
        if (!(xl[k] > 0.0) || !std::isfinite(xl[k])) return fail(c, YK_ERR_ARG, "strain made xl(%d) <= 0", k + 1);
    // strain.f:73-79 (the re-wrap) runs even without strain
    k_strain_wrap<<<(3 * c->n + 255) / 256, 256, 0, c->stream>>>(c->x, c->n, xl[0], xl[1], xl[2]);
    g_launches += 1;
    if (sel != 0) {
        for (int k = 0; k < 3; ++k) c->p.xl[k] = xl[k];
        setup_args(c);
        drop_graphs(c);
        const int rc = refresh_pair_tt(c);
        if (rc) return rc;
    }
    c->pos_dirty = true;
    if (xl_out)
        for (int k = 0; k < 3; ++k) xl_out[k] = xl[k];
    return sync_and_check(c);
}

int yk_perf_enable(yk_ctx* c, int enable, size_t flush_bytes)
{
    if (!c) return fail(nullptr, YK_ERR_ARG, "ctx is NULL");
    CK(c, cudaSetDevice(c->dev));
    c->perf_on = enable != 0;
    c->perf = yk_perf{};
    if (flush_bytes != c->flush_bytes) {
        cudaFree(c->flush_buf);
        c->flush_buf = nullptr;
        c->flush_bytes = 0;
        if (flush_bytes) {
            CK(c, cudaMalloc((void**)&c->flush_buf, flush_bytes));
            c->flush_bytes = flush_bytes;
        }
    }
    return YK_OK;
}

int yk_perf_read(yk_ctx* c, yk_perf* out)
{
    if (!c || !out) return fail(c, YK_ERR_ARG, "ctx and out are required");
    *out = c->perf;
    return YK_OK;
}

int yk_peak_probe(int device, int kind, double* tflops)
{
    if (!tflops || (kind != 0 && kind != 1)) return fail(nullptr, YK_ERR_ARG, "bad peak probe arguments");
    if (cudaSetDevice(device) != cudaSuccess) return fail(nullptr, YK_ERR_CUDA, "cudaSetDevice failed");
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int blocks = sms * 8, threads = 256, iters = 1 << 13;
    void* out = nullptr;
    if (cudaMalloc(&out, sizeof(double) * blocks * threads) != cudaSuccess)
        return fail(nullptr, YK_ERR_NOMEM, "probe buffer");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 7; ++rep) {
        cudaEventRecord(e0);
        if (kind == 0) k_fma_probe<double><<<blocks, threads>>>((double*)out, iters, 0.9999999, 1e-7);
        else k_fma_probe<float><<<blocks, threads>>>((float*)out, iters, 0.9999999f, 1e-7f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep >= 2 && ms < best) best = ms;
    }
    g_launches += 7;
    cudaError_t e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess) return fail(nullptr, YK_ERR_CUDA, "probe: %s", cudaGetErrorString(e));
    const double fmas = (double)blocks * threads * iters * PROBE_CHAINS;
    *tflops = 2.0 * fmas / (best * 1e-3) / 1e12;
    return YK_OK;
}

int yk_wait_selftest(yk_ctx* c, long long spins, int* gave_up)
{
    if (!c) return fail(nullptr, YK_ERR_ARG, "ctx is NULL");
    if (spins < 1 || spins > SPIN_LIMIT)
        return fail(c, YK_ERR_ARG, "spins must be in [1, %lld] (got %lld)", SPIN_LIMIT, spins);
    CK(c, cudaSetDevice(c->dev));
    // the count goes through the packed-scalar scratch of k_finish, which the
    // next force call rewrites
    int* dcount = reinterpret_cast<int*>(c->ds);
    k_wait_selftest<<<1, 128, 0, c->stream>>>(spins, c->err, dcount);
    g_launches += 1;
    int h = -1;
    CK(c, cudaMemcpyAsync(&h, dcount, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    const int rc = sync_and_check(c);
    if (gave_up) *gave_up = h;
    return rc;
}

int yk_host_register(void* ptr, size_t bytes)
{
    if (!ptr || !bytes) return fail(nullptr, YK_ERR_ARG, "bad host buffer");
    cudaError_t e = cudaHostRegister(ptr, bytes, cudaHostRegisterDefault);
    if (e != cudaSuccess) return fail(nullptr, YK_ERR_CUDA, "cudaHostRegister: %s", cudaGetErrorString(e));
    return YK_OK;
}

int yk_host_unregister(void* ptr)
{
    if (!ptr) return fail(nullptr, YK_ERR_ARG, "bad host buffer");
    cudaError_t e = cudaHostUnregister(ptr);
    if (e != cudaSuccess) return fail(nullptr, YK_ERR_CUDA, "cudaHostUnregister: %s", cudaGetErrorString(e));
    return YK_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Force call without device allocation (yk_accel_noalloc).
//
// Some callers cannot allocate device memory at the moment they need forces:
// applications that hand every byte of device memory to their own pool
// allocator at start-up and forbid allocations behind its back, and callers
// that cannot afford the device-wide synchronisation that cudaFree (and at
// times cudaMalloc) imposes on every other stream of the GPU.  For them this
// entry point evaluates one force call on caller-owned device arrays and keeps
// all of its working memory -- packed positions, their FP32 shadow, the slot
// order, the job table and the partial sums of the half-pair kernel -- in the
// file-scope array below.  The call itself waits for its stream and copies
// the scalars to the host before it returns.
// The array is created when the library's device code is loaded and stays
// on every GPU that loaded it until the process exits.  It caps n at
// NOALLOC_MAX_N; larger calls are rejected.  All calls share the array: two
// calls that overlap on the GPU (different streams, or different host
// threads on one device) race and corrupt each other's results.

constexpr int NOALLOC_MAX_N = 4096;
constexpr int NOALLOC_SEG = 4;
constexpr size_t NOALLOC_BYTES = size_t(4) << 20;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

// Device address of g_noalloc_scratch per device, looked up on the first call
// on that device (with the device current).
constexpr int NOALLOC_MAX_DEVICES = 64;
static void* g_noalloc_addr[NOALLOC_MAX_DEVICES];
static std::mutex g_noalloc_mutex;

__global__ void k_noalloc_prepare(int* perm, int n, int4* jobs, int* row_slots, int M, int seg)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) perm[s] = s;                      // slots in the caller's order
    if (s == 0) {
        int k = 0;
        for (int R = 0; R < M; ++R) {
            int q = 0;
            for (; q * seg < M - R; ++q) jobs[k++] = make_int4(R, R + q * seg, min(R + (q + 1) * seg, M), q);
            row_slots[R] = q;
        }
    }
}

// Byte layout of the scratch for n particles (256-byte aligned pieces).
struct NoallocLayout {
    size_t pos, posf, perm, iperm, Si, Sj, Sm, jobs, row_slots, ds, counter, err, total;
    int M, nseg, njobs;
};

static NoallocLayout noalloc_layout(int n)
{
    NoallocLayout L{};
    L.M = (n + PB - 1) / PB;
    L.nseg = (L.M + NOALLOC_SEG - 1) / NOALLOC_SEG;
    L.njobs = 0;
    for (int R = 0; R < L.M; ++R) L.njobs += (L.M - R + NOALLOC_SEG - 1) / NOALLOC_SEG;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t at = off;
        off += (bytes + 255) & ~size_t(255);
        return at;
    };
    L.pos = take(sizeof(double4) * (size_t)n);
    L.posf = take(sizeof(float) * SHADOW_FLOATS * (size_t)L.M);
    L.perm = take(sizeof(int) * (size_t)n);
    L.iperm = take(sizeof(int) * (size_t)n);
    L.Si = take(sizeof(double) * 3 * PB * (size_t)L.M * L.nseg);
    L.Sj = take(sizeof(double) * 3 * PB * ((size_t)L.M * (L.M + 1) / 2));
    L.Sm = take(sizeof(double) * NSCAL * (size_t)L.njobs);
    L.jobs = take(sizeof(int4) * (size_t)L.njobs);
    L.row_slots = take(sizeof(int) * (size_t)L.M);
    L.ds = take(sizeof(DevScalars));
    L.counter = take(sizeof(int));
    L.err = take(sizeof(unsigned));
    L.total = off;
    return L;
}

template <int SIM, int PREC, bool MEAS>
static void noalloc_force(int dev, cudaStream_t st, const double4* pos, const float* posf, PairJobs pj,
                          int* counter, const ForceArgs& fa, double* Si, void* Sj_v, double* Sm, unsigned* err,
                          const int* perm, const double* zii, const double* aii, double* a)
{
    row_t<PREC>* Sj = static_cast<row_t<PREC>*>(Sj_v);
    if (lo_path<SIM, PREC>(fa)) {
        if constexpr (PREC == PREC_MIXED) {
            const int grid = persistent_grid<k_force_pairs<SIM, PREC, MEAS, true>>(dev);
            k_force_pairs<SIM, PREC, MEAS, true><<<std::min(grid, pj.njobs), PB, 0, st>>>(pos, posf, pj, counter,
                                                                                   fa, Si, Sj, Sm, err);
        }
    } else {
        const int grid = persistent_grid<k_force_pairs<SIM, PREC, MEAS>>(dev);
        k_force_pairs<SIM, PREC, MEAS><<<std::min(grid, pj.njobs), PB, 0, st>>>(pos, posf, pj, counter, fa, Si,
                                                                                Sj, Sm, err);
    }
    k_combine<SIM, PREC><<<pj.M, COMB_THREADS, 0, st>>>(Si, Sj, pj, perm, zii, aii, fa, a);
}

template <int SIM>
static void noalloc_force_s(bool mixed, bool meas, int dev, cudaStream_t st, const double4* pos,
                            const float* posf, PairJobs pj, int* counter, const ForceArgs& fa, double* Si,
                            void* Sj, double* Sm, unsigned* err, const int* perm, const double* zii,
                            const double* aii, double* a)
{
    if (mixed) {
        if (meas) noalloc_force<SIM, PREC_MIXED, true>(dev, st, pos, posf, pj, counter, fa, Si, Sj, Sm, err, perm, zii, aii, a);
        else noalloc_force<SIM, PREC_MIXED, false>(dev, st, pos, posf, pj, counter, fa, Si, Sj, Sm, err, perm, zii, aii, a);
    } else {
        if (meas) noalloc_force<SIM, PREC_FP64, true>(dev, st, pos, posf, pj, counter, fa, Si, Sj, Sm, err, perm, zii, aii, a);
        else noalloc_force<SIM, PREC_FP64, false>(dev, st, pos, posf, pj, counter, fa, Si, Sj, Sm, err, perm, zii, aii, a);
    }
}

extern "C" int yk_accel_noalloc(const yk_params* p, int n, const double* x_dev, const double* zii_dev,
                                const double* aii_dev, int do_meas, double* a_dev, yk_scalars* out,
                                void* stream)
{
    if (!p || !x_dev || !a_dev) return fail(nullptr, YK_ERR_ARG, "params, x and a are required");
    if (n < 1) return fail(nullptr, YK_ERR_ARG, "n must be >= 1 (got %d)", n);
    if (n > NOALLOC_MAX_N)
        return fail(nullptr, YK_ERR_ARG,
                    "yk_accel_noalloc handles at most n = %d particles (got %d); use yk_create/yk_accel",
                    NOALLOC_MAX_N, n);
    int rc = check_params(p);
    if (rc) return rc;
    if ((p->sim_type == YK_SIM_ION_MIXTURE || p->sim_type == YK_SIM_NUCLEON) && !zii_dev)
        return fail(nullptr, YK_ERR_ARG, "this sim_type needs zii");
    if (p->sim_type == YK_SIM_ION_MIXTURE && !aii_dev)
        return fail(nullptr, YK_ERR_ARG, "ion-mixture runs need aii");
    const NoallocLayout L = noalloc_layout(n);
    if (L.total > NOALLOC_BYTES)
        return fail(nullptr, YK_ERR_ARG, "n = %d needs %zu scratch bytes, more than the %zu available", n,
                    L.total, NOALLOC_BYTES);

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(nullptr, YK_ERR_CUDA, "cudaGetDevice failed");
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(nullptr, YK_ERR_ARG, "device %d not supported", dev);
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc_addr[dev]) {
            // first call on this device: device-side address of the array
            cudaError_t e = cudaGetSymbolAddress(&g_noalloc_addr[dev], g_noalloc_scratch);
            if (e != cudaSuccess) {
                g_noalloc_addr[dev] = nullptr;
                return fail(nullptr, YK_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            }
        }
        base = g_noalloc_addr[dev];
    }
    unsigned char* b = static_cast<unsigned char*>(base);
    double4* pos = reinterpret_cast<double4*>(b + L.pos);
    float* posf = reinterpret_cast<float*>(b + L.posf);
    int* perm = reinterpret_cast<int*>(b + L.perm);
    int* iperm = reinterpret_cast<int*>(b + L.iperm);
    double* Si = reinterpret_cast<double*>(b + L.Si);
    void* Sj = b + L.Sj;
    double* Sm = reinterpret_cast<double*>(b + L.Sm);
    int4* jobs = reinterpret_cast<int4*>(b + L.jobs);
    int* row_slots = reinterpret_cast<int*>(b + L.row_slots);
    DevScalars* ds = reinterpret_cast<DevScalars*>(b + L.ds);
    int* counter = reinterpret_cast<int*>(b + L.counter);
    unsigned* err = reinterpret_cast<unsigned*>(b + L.err);

    // argument blocks from the same builder the engine uses (no allocation)
    yk_ctx tmp;
    tmp.p = *p;
    tmp.n = n;
    setup_args(&tmp);
    const ForceArgs& fa = tmp.fa;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const bool meas = do_meas != 0;

    // clear what must start at zero: shadow padding, scalars, counter, error word
    CK(nullptr, cudaMemsetAsync(posf, 0, sizeof(float) * SHADOW_FLOATS * (size_t)L.M, st));
    CK(nullptr, cudaMemsetAsync(ds, 0, sizeof(DevScalars), st));
    CK(nullptr, cudaMemsetAsync(counter, 0, sizeof(int), st));
    CK(nullptr, cudaMemsetAsync(err, 0, sizeof(unsigned), st));
    k_noalloc_prepare<<<(n + 255) / 256, 256, 0, st>>>(perm, n, jobs, row_slots, L.M, NOALLOC_SEG);
    k_apply_perm<<<(n + VBLOCK - 1) / VBLOCK, VBLOCK, 0, st>>>(perm, iperm, x_dev, zii_dev, pos, posf, n,
                                                              tmp.sa.pack_w);
    int k = 2;
    PairJobs pj{};
    pj.jobs = jobs;
    pj.njobs = L.njobs;
    pj.M = L.M;
    pj.row_slots = row_slots;
    pj.nseg_max = L.nseg;
    const bool mixed = p->precision == YK_PREC_MIXED;
    switch (p->sim_type) {
    case YK_SIM_PURE_ION:
        noalloc_force_s<SIM_PURE>(mixed, meas, dev, st, pos, posf, pj, counter, fa, Si, Sj, Sm, err, perm, zii_dev,
                                  aii_dev, a_dev);
        k += 2;
        break;
    case YK_SIM_ION_MIXTURE:
        noalloc_force_s<SIM_MIX>(mixed, meas, dev, st, pos, posf, pj, counter, fa, Si, Sj, Sm, err, perm, zii_dev,
                                 aii_dev, a_dev);
        k += 2;
        break;
    case YK_SIM_NUCLEON:
        noalloc_force_s<SIM_NUCLEON>(mixed, meas, dev, st, pos, posf, pj, counter, fa, Si, Sj, Sm, err, perm,
                                     zii_dev, aii_dev, a_dev);
        k += 2;
        break;
    default:  // 'B-field': a = 0
        CK(nullptr, cudaMemsetAsync(a_dev, 0, sizeof(double) * 3 * (size_t)(n + 3), st));
        break;
    }
    FinishArgs z = tmp.fz_base;
    const bool has_force = p->sim_type != YK_SIM_BFIELD;
    z.force_mode = has_force ? 1 : 0;
    z.do_meas = meas ? 1 : 0;
    z.nfp = (has_force && meas) ? L.njobs : 0;
    z.half = 1.0;
    z.kin_mode = 0;
    z.nkp = 0;
    k_finish<<<1, 256, 0, st>>>(Sm, nullptr, z, a_dev, ds, nullptr, nullptr);
    ++k;
    g_launches += k;

    DevScalars h{};
    unsigned herr = 0;
    CK(nullptr, cudaMemcpyAsync(&h, ds, sizeof h, cudaMemcpyDeviceToHost, st));
    CK(nullptr, cudaMemcpyAsync(&herr, err, sizeof herr, cudaMemcpyDeviceToHost, st));
    CK(nullptr, cudaStreamSynchronize(st));
    CK(nullptr, cudaGetLastError());
    if (herr) return fail(nullptr, (herr & ERR_TIMEOUT) ? YK_ERR_TIMEOUT : YK_ERR_CUDA,
                          "device error word 0x%x", herr);
    if (out) {
        out->ev = h.ev;
        out->vir = h.vir;
        out->px = h.px;
        out->ek = h.ek;
        for (int q = 0; q < 9; ++q) out->pp[q] = h.pp[q];
        out->time = p->time;
    }
    return YK_OK;
}
