// yk_batch.cu -- batches of independent boxes (yk_batch_* in the C-ABI).
//
// Layout.  Boxes are concatenated.  In the caller's order, box r owns
// particles [P_r, P_r + n_r) of x, v, vold, zii, aii and the block
// [A_r, A_r + 3(n_r+3)) of a (its own a(3,0:n+2)).  In slot order (Morton
// within each box) box r owns slots [S_r, S_r + 128 T_r): every box starts on
// a 128-slot tile, so a tile never mixes boxes and per-box tile indices are
// the single-box ones shifted by S_r / 128.  Unused slots at the end of a
// box's last tile are never active.
//
// One descriptor per box (RepDesc) holds its kernel argument blocks and
// offsets.  The force kernel pulls jobs (box, R, s, local job) from one
// queue, costliest first, loads the box's ForceArgs into shared memory and
// runs the same job body as the single-box kernel (pairs_job).  Every job
// writes only its own box's scratch rows, so a box's results are the same
// whatever other boxes share the batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <mutex>
#include <vector>

#include <cub/device/device_radix_sort.cuh>

#include "yk_internal.h"
#include "yk_pairs.cuh"
#include "yk_sort.cuh"

using namespace yk;

namespace {

constexpr int BATCH_SEG = 8;
constexpr int BATCH_GRAPH_STEPS = 50;
constexpr int BATCH_MAX_GRAPHS = 8;

struct RepDesc {
    ForceArgs fa;
    StepArgs sa;
    FinishArgs fz;
    int P;              // first particle (caller order)
    int S;              // first slot (multiple of 128)
    int T;              // tiles
    int nseg;           // Si rows per target block
    long long Sj_off;   // doubles
    long long Si_off;   // doubles
    long long A;        // first double of the box's a(3,0:n+2)
    int sm_off;         // first Sm row
    int njobs;
    int seg;            // source tiles per job
    int kb0, nkb;       // integrator blocks (and kinetic partial rows)
    double raw_scale;   // factor on the packed raw sums: 1/zi^2 for pure-ion
                        // boxes (run as mixtures, their sums carry Z_i Z_j)
};

// ---- kernels ---------------------------------------------------------------

// Key = (box, [species,] Hilbert index): boxes stay contiguous; in nucleon
// batches the protons of each box come first (as k_morton).
__global__ void k_b_morton(const double* __restrict__ x, const int* __restrict__ rep_of,
                           const RepDesc* __restrict__ rd, int ntot, unsigned long long* __restrict__ keys,
                           int* __restrict__ idx, const double* __restrict__ species)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ntot) return;
    const int r = rep_of[i];
    const double* L = rd[r].sa.xl;
    const int cx = min(max((int)(x[3 * i] * (1024.0 / L[0])), 0), 1023);
    const int cy = min(max((int)(x[3 * i + 1] * (1024.0 / L[1])), 0), 1023);
    const int cz = min(max((int)(x[3 * i + 2] * (1024.0 / L[2])), 0), 1023);
    const unsigned m = hilbert10(cx, cy, cz);
    keys[i] = species ? (((unsigned long long)r << 31) | ((species[i] != 1.0 ? 1ull : 0ull) << 30) | m)
                      : (((unsigned long long)r << 30) | m);
    idx[i] = i;
}

// Sorted position k of particle o -> slot S_r + (k - P_r) of its box.
__global__ void k_b_place(const int* __restrict__ idx_sorted, const int* __restrict__ rep_of,
                          const RepDesc* __restrict__ rd, const double* __restrict__ x,
                          const double* __restrict__ zii, double4* __restrict__ pos, float* __restrict__ posf,
                          int* __restrict__ perm, int* __restrict__ iperm, int ntot)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ntot) return;
    const int o = idx_sorted[k];
    const int r = rep_of[o];
    const int slot = rd[r].S + (k - rd[r].P);
    perm[slot] = o;
    iperm[o] = slot;
    const double xn[3] = {x[3 * o], x[3 * o + 1], x[3 * o + 2]};
    store_pos(pos, posf, slot, xn, zii[o]);
}

// Repack slots with the current order (after a host-side state change).
__global__ void k_b_repack(const int* __restrict__ iperm, const double* __restrict__ x,
                           const double* __restrict__ zii, double4* __restrict__ pos, float* __restrict__ posf,
                           int ntot)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= ntot) return;
    const double xn[3] = {x[3 * o], x[3 * o + 1], x[3 * o + 2]};
    store_pos(pos, posf, iperm[o], xn, zii[o]);
}

// vel_verlet_2.f:33-54 for every box (block table: box, block within box).
__global__ void __launch_bounds__(VBLOCK)
k_b_drift(const int2* __restrict__ vb, const RepDesc* __restrict__ rd, double* __restrict__ x,
          double* __restrict__ v, double* __restrict__ vold, const double* __restrict__ a,
          const double* __restrict__ zii, const int* __restrict__ iperm, double4* __restrict__ pos,
          float* __restrict__ posf)
{
    const int2 t = vb[blockIdx.x];
    const RepDesc* d = rd + t.x;
    const int local = t.y * VBLOCK + threadIdx.x;
    const StepArgs s = d->sa;
    if (local >= s.n) return;
    const int gi = d->P + local;
    const double* ar = a + d->A;
    double xn[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int e = 3 * gi + k;
        const double vi = v[e], ai = ar[3 * local + k];
        xn[k] = drift1(x[e], vi, ai, s, k);
        x[e] = xn[k];
        vold[e] = vi;
        v[e] = __dadd_rn(vi, __dmul_rn(s.dt, ai));
    }
    store_pos(pos, posf, iperm[gi], xn, zii[gi]);
}

// vel_verlet_2.f:75-95 for every box; kinetic partials per block.
template <bool KIN>
__global__ void __launch_bounds__(VBLOCK)
k_b_post(const int2* __restrict__ vb, const RepDesc* __restrict__ rd, double* __restrict__ v,
         const double* __restrict__ vold, const double* __restrict__ a, const double* __restrict__ aii,
         double* __restrict__ kpart)
{
    __shared__ double red[32 * NKIN];
    const int2 t = vb[blockIdx.x];
    const RepDesc* d = rd + t.x;
    const int local = t.y * VBLOCK + threadIdx.x;
    const double dt = d->sa.dt;
    double tk[NKIN] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (local < d->sa.n) {
        const int gi = d->P + local;
        const double* ar = a + d->A;
        double vv[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double vp = __dadd_rn(vold[3 * gi + k], __dmul_rn(dt, ar[3 * local + k]));
            vv[k] = __dmul_rn(0.5, __dadd_rn(v[3 * gi + k], vp));
            v[3 * gi + k] = vv[k];
        }
        kin_sums<KIN>(tk, aii[gi], vv[0], vv[1], vv[2]);
    }
    if constexpr (KIN) block_sum_store<NKIN>(tk, red, kpart + (size_t)blockIdx.x * NKIN);
}

template <int SIM, int PREC, bool MEAS, bool LO = false>
__global__ void __launch_bounds__(PB, (pairs_ctas_per_sm<PREC, LO>()))
k_force_pairs_batch(const double4* __restrict__ pos, const float* __restrict__ posf,
                    const int4* __restrict__ jobs, int njobs, int* __restrict__ counter,
                    const RepDesc* __restrict__ rd, double* __restrict__ Si, double* __restrict__ Sj,
                    double* __restrict__ Sm, unsigned* __restrict__ err)
{
    __shared__ __align__(128) PairSmem<row_t<PREC>> sm;
    __shared__ __align__(16) ForceArgs sfa;
    __shared__ int4 sjob;
    pairs_smem_init(sm);
    unsigned q = 0;
    for (;;) {
        if (threadIdx.x == 0) {
            const int j = atomicAdd(counter, 1);
            sjob = j < njobs ? jobs[j] : make_int4(-1, 0, 0, 0);
        }
        __syncthreads();
        const int4 jb = sjob;
        if (jb.x < 0) break;
        const RepDesc* d = rd + jb.x;
        for (int w = threadIdx.x; w < (int)(sizeof(ForceArgs) / 4); w += blockDim.x)
            reinterpret_cast<int*>(&sfa)[w] = reinterpret_cast<const int*>(&d->fa)[w];
        __syncthreads();
        BoxView bx;
        bx.pos = pos + d->S;
        bx.posf = posf + (size_t)(d->S / SHADOW_TILE) * SHADOW_FLOATS;
        bx.Si = Si + d->Si_off;
        bx.Sj = Sj + d->Sj_off;
        bx.n = sfa.n;
        bx.M = d->T;
        bx.nseg_max = d->nseg;
        const int C0 = jb.y + jb.z * d->seg;
        if (!pairs_job<SIM, PREC, MEAS, LO ? 1 : 2>(sm, sfa, bx, jb.y, C0, min(C0 + d->seg, bx.M), jb.z,
                                                    Sm + (size_t)(d->sm_off + jb.w) * NSCAL, err, q))
            return;
    }
}

template <int SIM>
__global__ void __launch_bounds__(256)
k_b_combine(const int* __restrict__ tile_rep, const RepDesc* __restrict__ rd, const double* __restrict__ Si,
            const double* __restrict__ Sj, const int* __restrict__ perm, const double* __restrict__ zii,
            const double* __restrict__ aii, double* __restrict__ a, int total_slots)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= total_slots) return;
    const RepDesc* d = rd + tile_rep[p >> 7];
    const int pl = p - d->S;
    if (pl >= d->fa.n) return;
    const int R = pl / PB, l = pl % PB;
    const int nseg = (d->T - R + d->seg - 1) / d->seg;
    double F[3] = {0.0, 0.0, 0.0};
    const double* si = Si + d->Si_off + ((size_t)R * d->nseg * PB + l) * 3;
    for (int s = 0; s < nseg; ++s) {
        const double* e = si + (size_t)s * PB * 3;
        F[0] += e[0];
        F[1] += e[1];
        F[2] += e[2];
    }
    const double* sj = Sj + d->Sj_off + ((size_t)tri_index(R, 0) * PB + l) * 3;
    for (int R2 = 0; R2 <= R; ++R2) {
        const double* e = sj + (size_t)R2 * PB * 3;
        F[0] += e[0];
        F[1] += e[1];
        F[2] += e[2];
    }
    const int orig = perm[p];
    store_accel<SIM>(d->fa, orig - d->P, zii[orig], aii + d->P, F, a + d->A);
}

// One block per box.  kin_mode / meas as in k_finish; the series slot of box r
// at the current step is series[(*series_idx) * nrep + r].
__global__ void __launch_bounds__(256)
k_b_finish(const RepDesc* __restrict__ rd, const double* __restrict__ Sm, const double* __restrict__ kpart,
           double* __restrict__ a, DevScalars* __restrict__ ds, double* __restrict__ series,
           const int* __restrict__ series_idx, int nrep, int meas, int kin_mode)
{
    const int r = blockIdx.x;
    const RepDesc* d = rd + r;
    FinishArgs z = d->fz;
    z.force_mode = 1;
    z.do_meas = meas;
    z.nfp = meas ? d->njobs : 0;
    z.half = d->raw_scale;
    z.kin_mode = kin_mode;
    z.nkp = kin_mode == 2 ? d->nkb : 0;
    double* slot = series ? series + ((size_t)(*series_idx) * nrep + r) * 13 : nullptr;
    finish_body(Sm + (size_t)d->sm_off * NSCAL, kpart + (size_t)d->kb0 * NKIN, z, a + d->A, ds + r, slot);
}

__global__ void k_b_series_next(int* series_idx) { *series_idx += 1; }

}  // namespace

// ---------------------------------------------------------------------------

struct GraphB {
    cudaGraphExec_t exec = nullptr;
    int K = 0, me = 0, phase = 0, series = 0, kernels = 0;
    unsigned long long stamp = 0;
};

struct yk_batch {
    int nrep = 0, ntot = 0, stot = 0, ntiles = 0, nvb = 0;
    int dev = 0;
    int sim = 0, prec = 0;          // SIM_MIX or SIM_NUCLEON; PREC_*
    cudaStream_t stream = nullptr;
    std::vector<int> n, P, S;
    std::vector<long long> A;
    std::vector<double> time, dt;
    double *x = nullptr, *v = nullptr, *vold = nullptr, *a = nullptr, *zii = nullptr, *aii = nullptr;
    int* rep_of = nullptr;
    double4* pos = nullptr;
    float* posf = nullptr;
    int *perm = nullptr, *iperm = nullptr;
    unsigned long long *keys0 = nullptr, *keys1 = nullptr;
    int *idx0 = nullptr, *idx1 = nullptr;
    void* cub_tmp = nullptr;
    size_t cub_bytes = 0;
    int key_bits = 31;
    RepDesc* rd = nullptr;
    int4* jobs = nullptr;
    int njobs = 0;
    int* counter = nullptr;
    int* tile_rep = nullptr;
    int2* vblocks = nullptr;
    double *Si = nullptr, *Sj = nullptr, *Sm = nullptr, *kpart = nullptr;
    DevScalars* ds = nullptr;
    unsigned* err = nullptr;
    double* series = nullptr;
    int series_cap = 0;
    int* series_idx = nullptr;
    int force_grid = 0, force_grid_lo = 0;
    bool all_lo = false;            // every box allows the mixed ion hi/lo displacement (fa.lo)
    int seg = BATCH_SEG, graph_steps = BATCH_GRAPH_STEPS;
    std::vector<RepDesc> hrd;       // host copy of the descriptors
    bool need_sort = true, pos_dirty = false;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::vector<GraphB> graphs;
    unsigned long long graph_clock = 0;
    std::string errmsg;
};

static thread_local std::string g_batch_err;

static int bfail(yk_batch* b, int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (b) b->errmsg = buf;
    else g_batch_err = buf;
    return code;
}

#define BCK(b, call)                                                                           \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return bfail((b), YK_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));  \
    } while (0)

static int enqueue_sort(yk_batch* b)
{
    const int nb = (b->ntot + 255) / 256;
    cudaStream_t st = b->stream;
    k_b_morton<<<nb, 256, 0, st>>>(b->x, b->rep_of, b->rd, b->ntot, b->keys0, b->idx0,
                                   b->sim == SIM_NUCLEON ? b->zii : nullptr);
    size_t bytes = b->cub_bytes;
    cub::DeviceRadixSort::SortPairs(b->cub_tmp, bytes, b->keys0, b->keys1, b->idx0, b->idx1, b->ntot, 0,
                                    b->key_bits, st);
    k_b_place<<<nb, 256, 0, st>>>(b->idx1, b->rep_of, b->rd, b->x, b->zii, b->pos, b->posf, b->perm, b->iperm,
                                  b->ntot);
    b->need_sort = false;
    b->pos_dirty = false;
    return 2;
}

template <int SIM, int PREC, bool MEAS>
static int launch_force_b(yk_batch* b)
{
    if (b->force_grid == 0) {
        int per_sm = 0, per_sm_lo = 0, sms = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_force_pairs_batch<SIM, PREC, MEAS>, PB, 0);
        if constexpr (PREC == PREC_MIXED && SIM != SIM_NUCLEON)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_lo, k_force_pairs_batch<SIM, PREC, MEAS, true>,
                                                          PB, 0);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->dev);
        b->force_grid = std::max(1, per_sm) * std::max(1, sms);
        b->force_grid_lo = std::max(1, per_sm_lo) * std::max(1, sms);
    }
    cudaMemsetAsync(b->counter, 0, sizeof(int), b->stream);
    bool launched = false;
    if constexpr (PREC == PREC_MIXED && SIM != SIM_NUCLEON) {
        if (b->all_lo) {
            k_force_pairs_batch<SIM, PREC, MEAS, true><<<std::min(b->force_grid_lo, b->njobs), PB, 0, b->stream>>>(
                b->pos, b->posf, b->jobs, b->njobs, b->counter, b->rd, b->Si, b->Sj, b->Sm, b->err);
            launched = true;
        }
    }
    if (!launched)
        k_force_pairs_batch<SIM, PREC, MEAS><<<std::min(b->force_grid, b->njobs), PB, 0, b->stream>>>(
            b->pos, b->posf, b->jobs, b->njobs, b->counter, b->rd, b->Si, b->Sj, b->Sm, b->err);
    k_b_combine<SIM><<<(b->stot + 255) / 256, 256, 0, b->stream>>>(b->tile_rep, b->rd, b->Si, b->Sj, b->perm,
                                                                   b->zii, b->aii, b->a, b->stot);
    return 2;
}

template <int SIM>
static int launch_force_bs(yk_batch* b, bool meas)
{
    if (b->prec == PREC_MIXED)
        return meas ? launch_force_b<SIM, PREC_MIXED, true>(b) : launch_force_b<SIM, PREC_MIXED, false>(b);
    return meas ? launch_force_b<SIM, PREC_FP64, true>(b) : launch_force_b<SIM, PREC_FP64, false>(b);
}

static int enqueue_force_b(yk_batch* b, bool meas)
{
    return b->sim == SIM_NUCLEON ? launch_force_bs<SIM_NUCLEON>(b, meas) : launch_force_bs<SIM_MIX>(b, meas);
}

static int enqueue_step_b(yk_batch* b, bool meas, bool series, bool resort)
{
    int k = 0;
    cudaStream_t st = b->stream;
    if (resort || b->need_sort) k += enqueue_sort(b);
    else if (b->pos_dirty) {
        k_b_repack<<<(b->ntot + 255) / 256, 256, 0, st>>>(b->iperm, b->x, b->zii, b->pos, b->posf, b->ntot);
        b->pos_dirty = false;
        ++k;
    }
    k_b_drift<<<b->nvb, VBLOCK, 0, st>>>(b->vblocks, b->rd, b->x, b->v, b->vold, b->a, b->zii, b->iperm, b->pos,
                                        b->posf);
    ++k;
    k += enqueue_force_b(b, meas);
    if (meas) k_b_post<true><<<b->nvb, VBLOCK, 0, st>>>(b->vblocks, b->rd, b->v, b->vold, b->a, b->aii, b->kpart);
    else k_b_post<false><<<b->nvb, VBLOCK, 0, st>>>(b->vblocks, b->rd, b->v, b->vold, b->a, b->aii, b->kpart);
    ++k;
    k_b_finish<<<b->nrep, 256, 0, st>>>(b->rd, b->Sm, b->kpart, b->a, b->ds, series ? b->series : nullptr,
                                        b->series_idx, b->nrep, meas ? 1 : 0, meas ? 2 : 1);
    ++k;
    if (series) {
        k_b_series_next<<<1, 1, 0, st>>>(b->series_idx);
        ++k;
    }
    return k;
}

static int sync_check_b(yk_batch* b)
{
    unsigned herr = 0;
    BCK(b, cudaMemcpyAsync(&herr, b->err, sizeof herr, cudaMemcpyDeviceToHost, b->stream));
    BCK(b, cudaStreamSynchronize(b->stream));
    BCK(b, cudaGetLastError());
    if (herr) {
        cudaMemsetAsync(b->err, 0, sizeof(unsigned), b->stream);
        cudaStreamSynchronize(b->stream);
        return bfail(b, (herr & ERR_TIMEOUT) ? YK_ERR_TIMEOUT : YK_ERR_CUDA, "device error word 0x%x", herr);
    }
    return YK_OK;
}

static void drop_graphs_b(yk_batch* b)
{
    for (auto& g : b->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    b->graphs.clear();
}

static GraphB* graph_b(yk_batch* b, int K, int me, int phase, bool series, int* rc)
{
    *rc = YK_OK;
    for (auto& g : b->graphs)
        if (g.K == K && g.me == me && g.phase == phase && g.series == (series ? 1 : 0)) {
            g.stamp = ++b->graph_clock;
            return &g;
        }
    if ((int)b->graphs.size() >= BATCH_MAX_GRAPHS) {
        auto it = std::min_element(b->graphs.begin(), b->graphs.end(),
                                   [](const GraphB& u, const GraphB& w) { return u.stamp < w.stamp; });
        cudaGraphExecDestroy(it->exec);
        b->graphs.erase(it);
    }
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        *rc = bfail(b, YK_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
        return nullptr;
    }
    int kernels = 0;
    for (int l = 1; l <= K; ++l) kernels += enqueue_step_b(b, me > 0 && (phase + l) % me == 0, series, l == 1);
    e = cudaStreamEndCapture(b->stream, &g);
    if (e != cudaSuccess) {
        *rc = bfail(b, YK_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
        return nullptr;
    }
    GraphB ent;
    e = cudaGraphInstantiate(&ent.exec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) {
        *rc = bfail(b, YK_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
        return nullptr;
    }
    ent.K = K;
    ent.me = me;
    ent.phase = phase;
    ent.series = series ? 1 : 0;
    ent.kernels = kernels;
    ent.stamp = ++b->graph_clock;
    b->graphs.push_back(ent);
    return &b->graphs.back();
}

extern "C" {

const char* yk_batch_last_error(const yk_batch* b) { return b ? b->errmsg.c_str() : g_batch_err.c_str(); }

// Batches are created and destroyed often (the serving loop rebuilds a group
// whenever its membership changes), so their device arrays come from the
// device's stream-ordered memory pool, which keeps up to POOL_KEEP bytes of
// freed memory cached between batches: a rebuild then costs no cudaMalloc /
// cudaFree round trips to the driver.
constexpr uint64_t POOL_KEEP = 8ull << 30;

static void pool_setup(int dev)
{
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lk(mu);
    if (std::find(done.begin(), done.end(), dev) != done.end()) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = POOL_KEEP;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    done.push_back(dev);
}

// Bytes the pool holds cached but unused (free for the next batch).
static size_t pool_cached(int dev)
{
    cudaMemPool_t pool;
    uint64_t reserved = 0, used = 0;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) return 0;
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
    return reserved > used ? (size_t)(reserved - used) : 0;
}

// Job table and target-side scratch layout for segment length seg: a job is
// (box, target block R, segment s) over at most seg source tiles; jobs run
// costliest first.  Fills the descriptors' seg, nseg, Si_off, sm_off, njobs.
static void layout_jobs(yk_batch* b, int seg, std::vector<int4>& sorted, long long& si_total)
{
    std::vector<int4> jobs;
    std::vector<int> jcost;
    long long si = 0;
    int smo = 0;
    for (int r = 0; r < b->nrep; ++r) {
        RepDesc& d = b->hrd[r];
        const int T = d.T;
        d.seg = seg;
        d.nseg = (T + seg - 1) / seg;
        d.Si_off = si;
        d.sm_off = smo;
        int local = 0;
        for (int R = 0; R < T; ++R)
            for (int s = 0; s * seg < T - R; ++s) {
                jobs.push_back(make_int4(r, R, s, local++));
                const int tiles = std::min(seg, T - R - s * seg);
                jcost.push_back(2 * tiles - (s == 0 ? 1 : 0));
            }
        d.njobs = local;
        si += (long long)T * d.nseg * PB * 3;
        smo += local;
    }
    std::vector<int> order(jobs.size());
    for (size_t k = 0; k < order.size(); ++k) order[k] = (int)k;
    std::stable_sort(order.begin(), order.end(), [&](int u, int w) { return jcost[u] > jcost[w]; });
    sorted.resize(jobs.size());
    for (size_t k = 0; k < order.size(); ++k) sorted[k] = jobs[order[k]];
    b->njobs = (int)sorted.size();
    b->seg = seg;
    si_total = si;
}

int yk_batch_get_tuning(yk_batch* b, yk_tuning* out)
{
    if (!b || !out) return bfail(b, YK_ERR_ARG, "batch and out are required");
    out->force_kernel = 2;
    out->pair_seg = b->seg;
    out->sort_every = b->graph_steps;       // the batch re-sorts at the start of every graph
    out->graph_steps = b->graph_steps;
    return YK_OK;
}

int yk_batch_set_tuning(yk_batch* b, const yk_tuning* t)
{
    if (!b || !t) return bfail(b, YK_ERR_ARG, "batch and tuning are required");
    if (t->force_kernel != 0 && t->force_kernel != 2)
        return bfail(b, YK_ERR_UNSUPPORTED, "a batch runs the half-pair kernel (force_kernel 0 or 2)");
    if (t->pair_seg < 0 || t->graph_steps < 0) return bfail(b, YK_ERR_ARG, "bad tuning values");
    BCK(b, cudaSetDevice(b->dev));
    BCK(b, cudaStreamSynchronize(b->stream));
    drop_graphs_b(b);
    b->graph_steps = t->graph_steps > 0 ? t->graph_steps : BATCH_GRAPH_STEPS;
    const int seg = t->pair_seg > 0 ? t->pair_seg : BATCH_SEG;
    if (seg == b->seg) return YK_OK;
    std::vector<int4> sorted;
    long long si = 0;
    layout_jobs(b, seg, sorted, si);
    cudaFreeAsync(b->Si, b->stream);
    cudaFreeAsync(b->Sm, b->stream);
    cudaFreeAsync(b->jobs, b->stream);
    b->Si = b->Sm = nullptr;
    b->jobs = nullptr;
    if (cudaMallocAsync((void**)&b->Si, sizeof(double) * (size_t)std::max<long long>(si, 1), b->stream) != cudaSuccess ||
        cudaMallocAsync((void**)&b->Sm, sizeof(double) * 8 * (size_t)std::max(b->njobs, 1), b->stream) != cudaSuccess ||
        cudaMallocAsync((void**)&b->jobs, sizeof(int4) * (size_t)std::max(b->njobs, 1), b->stream) != cudaSuccess)
        return bfail(b, YK_ERR_NOMEM, "re-allocating the job scratch for pair_seg %d failed", seg);
    BCK(b, cudaMemcpyAsync(b->rd, b->hrd.data(), sizeof(RepDesc) * b->nrep, cudaMemcpyHostToDevice, b->stream));
    BCK(b, cudaMemcpyAsync(b->jobs, sorted.data(), sizeof(int4) * sorted.size(), cudaMemcpyHostToDevice,
                           b->stream));
    return sync_check_b(b);
}

int yk_batch_destroy(yk_batch* b)
{
    if (!b) return bfail(nullptr, YK_ERR_ARG, "batch is NULL");
    cudaSetDevice(b->dev);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graphs_b(b);
    void* bufs[] = {b->x,     b->v,     b->vold,  b->a,      b->zii,     b->aii,     b->rep_of, b->pos,
                    b->posf,  b->perm,  b->iperm, b->keys0,  b->keys1,   b->idx0,    b->idx1,   b->cub_tmp,
                    b->rd,    b->jobs,  b->counter, b->tile_rep, b->vblocks, b->Si, b->Sj,   b->Sm,
                    b->kpart, b->ds,    b->err,   b->series, b->series_idx};
    if (b->stream) {
        for (void* p : bufs)
            if (p) cudaFreeAsync(p, b->stream);            // back to the pool
        cudaStreamSynchronize(b->stream);
    }
    if (b->e0) cudaEventDestroy(b->e0);
    if (b->e1) cudaEventDestroy(b->e1);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return YK_OK;
}

int yk_batch_create(int nrep, const yk_params* params, const int* n, const double* const* x,
                    const double* const* v, const double* const* zii, const double* const* aii, int device,
                    yk_batch** out)
{
    if (!out) return bfail(nullptr, YK_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (nrep < 1 || !params || !n || !x) return bfail(nullptr, YK_ERR_ARG, "nrep, params, n and x are required");
    const bool nuc = params[0].sim_type == YK_SIM_NUCLEON;
    const int prec = params[0].precision;
    long long ntot = 0, stot = 0;
    for (int r = 0; r < nrep; ++r) {
        const yk_params& p = params[r];
        if (n[r] < 1) return bfail(nullptr, YK_ERR_ARG, "box %d: n must be >= 1", r);
        if (!x[r]) return bfail(nullptr, YK_ERR_ARG, "box %d: x is NULL", r);
        if (p.sim_type == YK_SIM_BFIELD || (p.sim_type == YK_SIM_NUCLEON) != nuc)
            return bfail(nullptr, YK_ERR_ARG, "box %d: a batch holds either ion boxes or nucleon boxes", r);
        if (p.precision != prec) return bfail(nullptr, YK_ERR_ARG, "box %d: one precision per batch", r);
        if (p.integrator != YK_VV2 || p.bfield != 0.0)
            return bfail(nullptr, YK_ERR_ARG, "box %d: batches run vel_verlet_2 without B field", r);
        if (!(p.dt > 0.0) || !(p.xl[0] > 0.0) || !(p.xl[1] > 0.0) || !(p.xl[2] > 0.0) || !(p.xmass > 0.0))
            return bfail(nullptr, YK_ERR_ARG, "box %d: dt, xl and xmass must be > 0", r);
        if ((p.sim_type != YK_SIM_PURE_ION) && (!zii || !zii[r]))
            return bfail(nullptr, YK_ERR_ARG, "box %d: zii required", r);
        if (p.sim_type == YK_SIM_ION_MIXTURE && (!aii || !aii[r]))
            return bfail(nullptr, YK_ERR_ARG, "box %d: aii required", r);
        if (p.sim_type == YK_SIM_PURE_ION && !(p.ai > 0.0))
            return bfail(nullptr, YK_ERR_ARG, "box %d: pure-ion boxes need ai > 0", r);
        for (long long e = 0; e < 3LL * n[r]; ++e)
            if (!std::isfinite(x[r][e]) || (v && v[r] && !std::isfinite(v[r][e])))
                return bfail(nullptr, YK_ERR_NONFINITE, "box %d: NaN or Inf in x or v", r);
        ntot += n[r];
        stot += (long long)PB * ((n[r] + PB - 1) / PB);
    }
    if (ntot > (1LL << 28) || stot > (1LL << 30)) return bfail(nullptr, YK_ERR_ARG, "batch too large");
    if (cudaSetDevice(device) != cudaSuccess) return bfail(nullptr, YK_ERR_CUDA, "cudaSetDevice(%d) failed", device);

    yk_batch* b = new yk_batch();
    b->nrep = nrep;
    b->ntot = (int)ntot;
    b->stot = (int)stot;
    b->ntiles = (int)(stot / PB);
    b->dev = device;
    b->sim = nuc ? SIM_NUCLEON : SIM_MIX;
    b->prec = prec == YK_PREC_MIXED ? PREC_MIXED : PREC_FP64;
    b->n.assign(n, n + nrep);
    b->P.resize(nrep);
    b->S.resize(nrep);
    b->A.resize(nrep);
    b->time.resize(nrep);
    b->dt.resize(nrep);

    // host-side layout, descriptors, job table, block tables
    b->hrd.resize(nrep);
    std::vector<RepDesc>& rd = b->hrd;
    std::vector<int> tile_rep;
    std::vector<int2> vblocks;
    long long P = 0, S = 0, A = 0, sj = 0, si = 0;
    for (int r = 0; r < nrep; ++r) {
        yk_params p = params[r];
        RepDesc& d = rd[r];
        d.raw_scale = 1.0;
        if (p.sim_type == YK_SIM_PURE_ION) {
            // run through the mixture kernels (Z_i = zi); keep the pure-ion
            // scaling of the scalars, int_ion_pure.f:233-242
            ForceArgs fa_pure;
            StepArgs sa_pure;
            make_args(p, n[r], &fa_pure, &sa_pure, &d.fz);
            d.raw_scale = 1.0 / (p.zi * p.zi);
            p.sim_type = YK_SIM_ION_MIXTURE;
            p.mix_mode = YK_MIX_FIXED;
            FinishArgs fz_mix;
            make_args(p, n[r], &d.fa, &d.sa, &fz_mix);
        } else {
            make_args(p, n[r], &d.fa, &d.sa, &d.fz);
        }
        d.sa.pack_w = 1;
        const int T = (n[r] + PB - 1) / PB;
        d.P = (int)P;
        d.S = (int)S;
        d.T = T;
        d.Sj_off = sj;
        d.A = A;
        const int nb = (n[r] + VBLOCK - 1) / VBLOCK;
        d.kb0 = (int)vblocks.size();
        d.nkb = nb;
        for (int q = 0; q < nb; ++q) vblocks.push_back(make_int2(r, q));
        for (int t = 0; t < T; ++t) tile_rep.push_back(r);
        b->P[r] = (int)P;
        b->S[r] = (int)S;
        b->A[r] = A;
        b->time[r] = params[r].time;
        b->dt[r] = params[r].dt;
        P += n[r];
        S += (long long)T * PB;
        A += 3LL * (n[r] + 3);
        sj += (long long)T * (T + 1) / 2 * PB * 3;
    }
    std::vector<int4> sorted;
    layout_jobs(b, BATCH_SEG, sorted, si);
    b->nvb = (int)vblocks.size();
    b->all_lo = !nuc;
    for (int r = 0; r < nrep; ++r) b->all_lo = b->all_lo && rd[r].fa.lo != 0;
    int bits = 1;
    while ((1 << bits) < nrep) ++bits;
    b->key_bits = (nuc ? 31 : 30) + bits;

    // admission: refuse up front when the device cannot hold the batch
    size_t cub_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, cub_bytes, (unsigned long long*)nullptr,
                                    (unsigned long long*)nullptr, (int*)nullptr, (int*)nullptr, (int)ntot, 0,
                                    b->key_bits);
    const size_t need = sizeof(double) * (size_t)(9 * ntot + A + 2 * ntot + sj + si + 8LL * b->njobs +
                                                  (long long)NKIN * b->nvb) +
                        sizeof(double4) * stot + sizeof(float) * (SHADOW_FLOATS / SHADOW_TILE) * stot + sizeof(int) * (3 * ntot + 2 * stot) +
                        sizeof(unsigned long long) * 2 * ntot + cub_bytes + sizeof(RepDesc) * nrep +
                        sizeof(int4) * b->njobs + (64u << 20);
    size_t free_b = 0, total_b = 0;
    pool_setup(device);
    cudaMemGetInfo(&free_b, &total_b);
    free_b += pool_cached(device);
    if (need > free_b) {
        delete b;
        return bfail(nullptr, YK_ERR_NOMEM, "batch needs %zu bytes, %zu free", need, free_b);
    }

    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
        yk_batch_destroy(b);
        return bfail(nullptr, YK_ERR_CUDA, "stream creation failed");
    }
#define BALLOC(ptr, cnt)                                                                    \
    do {                                                                                    \
        if (cudaMallocAsync((void**)&(ptr), sizeof(*(ptr)) * (size_t)std::max<long long>((cnt), 1), b->stream) != \
            cudaSuccess) {                                                                  \
            yk_batch_destroy(b);                                                            \
            return bfail(nullptr, YK_ERR_NOMEM, "device allocation of " #ptr " failed");    \
        }                                                                                   \
    } while (0)
    BALLOC(b->x, 3 * ntot);
    BALLOC(b->v, 3 * ntot);
    BALLOC(b->vold, 3 * ntot);
    BALLOC(b->a, A);
    BALLOC(b->zii, ntot);
    BALLOC(b->aii, ntot);
    BALLOC(b->rep_of, ntot);
    BALLOC(b->pos, stot);
    BALLOC(b->posf, (size_t)SHADOW_FLOATS / SHADOW_TILE * stot);      // stot is a multiple of SHADOW_TILE
    BALLOC(b->perm, stot);
    BALLOC(b->iperm, ntot);
    BALLOC(b->keys0, ntot);
    BALLOC(b->keys1, ntot);
    BALLOC(b->idx0, ntot);
    BALLOC(b->idx1, ntot);
    BALLOC(b->rd, nrep);
    BALLOC(b->jobs, b->njobs);
    BALLOC(b->counter, 1);
    BALLOC(b->tile_rep, b->ntiles);
    BALLOC(b->vblocks, b->nvb);
    BALLOC(b->Si, si);
    BALLOC(b->Sj, sj);
    BALLOC(b->Sm, 8LL * b->njobs);
    BALLOC(b->kpart, (long long)NKIN * b->nvb);
    BALLOC(b->ds, nrep);
    BALLOC(b->err, 1);
    BALLOC(b->series_idx, 1);
#undef BALLOC
    b->cub_bytes = cub_bytes;
    if (cudaMallocAsync(&b->cub_tmp, std::max<size_t>(cub_bytes, 16), b->stream) != cudaSuccess ||
        cudaEventCreate(&b->e0) != cudaSuccess || cudaEventCreate(&b->e1) != cudaSuccess) {
        yk_batch_destroy(b);
        return bfail(nullptr, YK_ERR_NOMEM, "batch set-up failed");
    }

    std::vector<double> hx(3 * ntot), hv(3 * ntot, 0.0), hz(ntot), ha(ntot);
    std::vector<int> hrep(ntot);
    for (int r = 0; r < nrep; ++r) {
        const long long o = b->P[r];
        std::memcpy(&hx[3 * o], x[r], sizeof(double) * 3 * n[r]);
        if (v && v[r]) std::memcpy(&hv[3 * o], v[r], sizeof(double) * 3 * n[r]);
        for (int i = 0; i < n[r]; ++i) {
            hz[o + i] = (zii && zii[r]) ? zii[r][i] : params[r].zi;
            ha[o + i] = (aii && aii[r]) ? aii[r][i] : (params[r].ai > 0.0 ? params[r].ai : 1.0);
            hrep[o + i] = r;
        }
    }
    cudaStream_t st = b->stream;
    cudaMemcpyAsync(b->x, hx.data(), sizeof(double) * hx.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(b->v, hv.data(), sizeof(double) * hv.size(), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(b->vold, 0, sizeof(double) * 3 * ntot, st);
    cudaMemsetAsync(b->a, 0, sizeof(double) * A, st);
    cudaMemcpyAsync(b->zii, hz.data(), sizeof(double) * ntot, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(b->aii, ha.data(), sizeof(double) * ntot, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(b->rep_of, hrep.data(), sizeof(int) * ntot, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(b->pos, 0, sizeof(double4) * stot, st);
    cudaMemsetAsync(b->posf, 0, sizeof(float) * SHADOW_FLOATS / SHADOW_TILE * stot, st);
    cudaMemsetAsync(b->perm, 0xff, sizeof(int) * stot, st);
    cudaMemcpyAsync(b->rd, rd.data(), sizeof(RepDesc) * nrep, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(b->jobs, sorted.data(), sizeof(int4) * sorted.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(b->tile_rep, tile_rep.data(), sizeof(int) * tile_rep.size(), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(b->vblocks, vblocks.data(), sizeof(int2) * vblocks.size(), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(b->ds, 0, sizeof(DevScalars) * nrep, st);
    cudaMemsetAsync(b->err, 0, sizeof(unsigned), st);
    cudaMemsetAsync(b->series_idx, 0, sizeof(int), st);
    count_launches(enqueue_sort(b));
    if (cudaStreamSynchronize(st) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
        yk_batch_destroy(b);
        return bfail(nullptr, YK_ERR_CUDA, "batch upload failed");
    }
    *out = b;
    return YK_OK;
}

int yk_batch_accel(yk_batch* b, int do_meas, yk_scalars* out)
{
    if (!b) return bfail(nullptr, YK_ERR_ARG, "batch is NULL");
    BCK(b, cudaSetDevice(b->dev));
    const bool meas = do_meas != 0;
    int k = 0;
    if (b->need_sort) k += enqueue_sort(b);
    k += enqueue_force_b(b, meas);
    k_b_finish<<<b->nrep, 256, 0, b->stream>>>(b->rd, b->Sm, b->kpart, b->a, b->ds, nullptr, b->series_idx,
                                               b->nrep, meas ? 1 : 0, 0);
    ++k;
    count_launches(k);
    std::vector<DevScalars> h(b->nrep);
    BCK(b, cudaMemcpyAsync(h.data(), b->ds, sizeof(DevScalars) * b->nrep, cudaMemcpyDeviceToHost, b->stream));
    int rc = sync_check_b(b);
    if (rc) return rc;
    if (out)
        for (int r = 0; r < b->nrep; ++r) {
            out[r].ev = h[r].ev;
            out[r].vir = h[r].vir;
            out[r].px = h[r].px;
            out[r].ek = h[r].ek;
            for (int q = 0; q < 9; ++q) out[r].pp[q] = h[r].pp[q];
            out[r].time = b->time[r];
        }
    return YK_OK;
}

int yk_batch_run(yk_batch* b, int nsteps, int meas_every, yk_scalars* series, double* ms)
{
    if (!b) return bfail(nullptr, YK_ERR_ARG, "batch is NULL");
    if (nsteps < 0 || meas_every < 0) return bfail(b, YK_ERR_ARG, "nsteps and meas_every must be >= 0");
    if (ms) *ms = 0.0;
    if (nsteps == 0) return YK_OK;
    BCK(b, cudaSetDevice(b->dev));
    const bool want = series != nullptr;
    if (want && b->series_cap < nsteps) {
        drop_graphs_b(b);
        cudaFreeAsync(b->series, b->stream);
        b->series = nullptr;
        b->series_cap = 0;
        BCK(b, cudaMallocAsync((void**)&b->series, sizeof(double) * 13 * (size_t)nsteps * b->nrep, b->stream));
        b->series_cap = nsteps;
    }
    cudaStream_t st = b->stream;
    BCK(b, cudaMemsetAsync(b->series_idx, 0, sizeof(int), st));
    BCK(b, cudaEventRecord(b->e0, st));
    const int me = meas_every;
    const int K = b->graph_steps;
    int k = 0, s = 1;
    if (b->pos_dirty || b->need_sort) k += enqueue_sort(b);
    while (s + K - 1 <= nsteps) {
        int rc = YK_OK;
        GraphB* g = graph_b(b, K, me, me > 0 ? (s - 1) % me : 0, want, &rc);
        if (!g) return rc;
        BCK(b, cudaGraphLaunch(g->exec, st));
        k += g->kernels;
        s += K;
    }
    for (; s <= nsteps; ++s) k += enqueue_step_b(b, me > 0 && s % me == 0, want, false);
    BCK(b, cudaEventRecord(b->e1, st));
    count_launches(k);
    int rc = sync_check_b(b);
    if (rc) return rc;
    if (ms) {
        float f = 0.f;
        cudaEventElapsedTime(&f, b->e0, b->e1);
        *ms = f;
    }
    if (want) {
        std::vector<double> h(13 * (size_t)nsteps * b->nrep);
        BCK(b, cudaMemcpy(h.data(), b->series, sizeof(double) * h.size(), cudaMemcpyDeviceToHost));
        for (int q = 0; q < nsteps; ++q)
            for (int r = 0; r < b->nrep; ++r) {
                const double* o = &h[13 * ((size_t)q * b->nrep + r)];
                yk_scalars& y = series[(size_t)q * b->nrep + r];
                b->time[r] = b->time[r] + b->dt[r];
                y.ev = o[0];
                y.vir = o[1];
                y.px = o[2];
                y.ek = o[3];
                for (int c = 0; c < 9; ++c) y.pp[c] = o[4 + c];
                y.time = b->time[r];
            }
    } else {
        for (int q = 0; q < nsteps; ++q)
            for (int r = 0; r < b->nrep; ++r) b->time[r] = b->time[r] + b->dt[r];
    }
    return YK_OK;
}

int yk_batch_get_state(yk_batch* b, int rep, double* x, double* v, double* vold, double* a)
{
    if (!b) return bfail(nullptr, YK_ERR_ARG, "batch is NULL");
    if (rep < 0 || rep >= b->nrep) return bfail(b, YK_ERR_ARG, "box %d out of range", rep);
    BCK(b, cudaSetDevice(b->dev));
    const size_t off = 3 * (size_t)b->P[rep], bytes = sizeof(double) * 3 * (size_t)b->n[rep];
    cudaStream_t st = b->stream;
    if (x) BCK(b, cudaMemcpyAsync(x, b->x + off, bytes, cudaMemcpyDeviceToHost, st));
    if (v) BCK(b, cudaMemcpyAsync(v, b->v + off, bytes, cudaMemcpyDeviceToHost, st));
    if (vold) BCK(b, cudaMemcpyAsync(vold, b->vold + off, bytes, cudaMemcpyDeviceToHost, st));
    if (a) BCK(b, cudaMemcpyAsync(a, b->a + b->A[rep], sizeof(double) * 3 * (size_t)(b->n[rep] + 3),
                                  cudaMemcpyDeviceToHost, st));
    BCK(b, cudaStreamSynchronize(st));
    return YK_OK;
}

int yk_batch_set_state(yk_batch* b, int rep, const double* x, const double* v, const double* vold,
                       const double* a)
{
    if (!b) return bfail(nullptr, YK_ERR_ARG, "batch is NULL");
    if (rep < 0 || rep >= b->nrep) return bfail(b, YK_ERR_ARG, "box %d out of range", rep);
    const size_t cnt = 3 * (size_t)b->n[rep];
    for (size_t e = 0; e < cnt; ++e)
        if ((x && !std::isfinite(x[e])) || (v && !std::isfinite(v[e])) || (vold && !std::isfinite(vold[e])))
            return bfail(b, YK_ERR_NONFINITE, "box %d: NaN or Inf in a state array", rep);
    BCK(b, cudaSetDevice(b->dev));
    const size_t off = 3 * (size_t)b->P[rep], bytes = sizeof(double) * cnt;
    cudaStream_t st = b->stream;
    if (x) BCK(b, cudaMemcpyAsync(b->x + off, x, bytes, cudaMemcpyHostToDevice, st));
    if (v) BCK(b, cudaMemcpyAsync(b->v + off, v, bytes, cudaMemcpyHostToDevice, st));
    if (vold) BCK(b, cudaMemcpyAsync(b->vold + off, vold, bytes, cudaMemcpyHostToDevice, st));
    if (a) BCK(b, cudaMemcpyAsync(b->a + b->A[rep], a, sizeof(double) * 3 * (size_t)(b->n[rep] + 3),
                                  cudaMemcpyHostToDevice, st));
    if (x) b->pos_dirty = true;
    BCK(b, cudaStreamSynchronize(st));
    return YK_OK;
}

}  // extern "C"
