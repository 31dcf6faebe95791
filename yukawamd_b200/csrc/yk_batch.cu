// yk_batch.cu -- batches of independent boxes (yk_batch_* in the C-ABI).
//
// A batch has a fixed number of slots (boxes it can hold at once) and fixed
// capacities for particles, tiles and half-pair scratch.  yk_batch_create
// makes a batch whose capacities are exactly its boxes; yk_batch_create_slots
// makes an empty one that the serving loop fills and drains with
// yk_batch_admit / yk_batch_retire between runs, without moving or copying
// the boxes that stay.
//
// Layout.  Box r (in slot r) owns particle units [P_r, P_r + n_r + 3) of the
// caller-order arrays x, v, vold, zii, aii (n_r particles plus three unused
// units, so that its a(3,0:n+2) is a[3 P_r, 3 (P_r + n_r + 3)) ), and tiles
// [S_r / 128, S_r / 128 + T_r) of the slot-order arrays pos, posf, perm:
// every box starts on a 128-slot tile, so a tile never mixes boxes and
// per-box tile indices are the single-box ones shifted by S_r / 128.  Both
// ranges come from first-fit allocators and stay put while the box is held.
// The half-pair scratch (Sj, Si, Sm), the job table and the integrator block
// table only live through one force call or step; they are laid out afresh,
// packed, over the boxes held whenever the set of boxes changes.
//
// Launch shapes depend only on the capacities (kernels skip empty slots and
// unused table entries; the job count is read from device memory), so the
// CUDA graphs of yk_batch_run stay valid across admissions and retirements.
//
// Every box has a step budget (left[r]): each step's kernels skip a box whose
// budget is spent, and k_b_finish counts it down, so a box admitted for s
// steps takes exactly s steps even when a K-step graph runs past them.
//
// Each box is ordered on its own (a segmented radix sort over the boxes'
// particle ranges, keys as the single-box engine's), its work items write
// only its own scratch rows, and the reductions run in a fixed order, so a
// box's results are the same bits whatever other boxes share the batch and
// whenever they come and go (admissions happen between graphs, where every
// box is re-sorted anyway).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <cub/device/device_segmented_radix_sort.cuh>

#include "yk_internal.h"
#include "yk_pairs.cuh"
#include "yk_sort.cuh"

using namespace yk;

namespace {

constexpr int BATCH_SEG = 8;
constexpr int BATCH_GRAPH_STEPS = 50;
// Steps between the boxes' re-orderings inside a graph (each graph starts
// with one): the single-box engine's cadence, for the same reason (the warp
// boxes grow as particles move away from their sorted neighbours).
constexpr int BATCH_SORT_EVERY = 4;
constexpr int SORT_AT_GRAPH_START_ONLY = INT_MAX;
constexpr int BATCH_MAX_GRAPHS = 8;
constexpr int UNLIMITED = INT_MAX;   // step budget of the boxes of yk_batch_create

struct RepDesc {
    ForceArgs fa;
    StepArgs sa;
    FinishArgs fz;
    int active;         // the slot holds a box
    int P;              // first particle unit (caller order)
    int S;              // first slot (multiple of 128)
    int T;              // tiles
    int nseg;           // Si rows per target block
    long long Sj_off;   // values (row_t of the batch's form)
    long long Si_off;   // doubles
    long long A;        // first double of the box's a(3,0:n+2) = 3 P
    int sm_off;         // first Sm row
    int njobs;
    int seg;            // source tiles per job
    int kb0, nkb;       // integrator blocks (and kinetic partial rows)
    double raw_scale;   // factor on the packed raw sums: 1/zi^2 for pure-ion
                        // boxes (run as mixtures, their sums carry Z_i Z_j)
};

// ---- kernels ---------------------------------------------------------------

// Sort keys of the particles of the boxes in sel (all boxes if sel is NULL):
// the single-box engine's Hilbert keys (k_morton), protons first in nucleon
// boxes.
__global__ void k_b_morton(const double* __restrict__ x, const int* __restrict__ rep_of,
                           const RepDesc* __restrict__ rd, const int* __restrict__ sel, int ucap,
                           unsigned* __restrict__ keys, int* __restrict__ idx, const double* __restrict__ species)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ucap) return;
    const int r = rep_of[i];
    if (r < 0 || (sel && !sel[r])) return;
    const double* L = rd[r].sa.xl;
    const int cx = min(max((int)(x[3 * i] * (1024.0 / L[0])), 0), 1023);
    const int cy = min(max((int)(x[3 * i + 1] * (1024.0 / L[1])), 0), 1023);
    const int cz = min(max((int)(x[3 * i + 2] * (1024.0 / L[2])), 0), 1023);
    keys[i] = hilbert10(cx, cy, cz) | ((species && species[i] != 1.0) ? (1u << 30) : 0u);
    idx[i] = i;
}

// Sorted position k (inside its box's particle range) -> slot S_r + (k - P_r).
__global__ void k_b_place(const int* __restrict__ idx_sorted, const int* __restrict__ rep_of,
                          const RepDesc* __restrict__ rd, const int* __restrict__ sel, const double* __restrict__ x,
                          const double* __restrict__ zii, double4* __restrict__ pos, float* __restrict__ posf,
                          int* __restrict__ perm, int* __restrict__ iperm, int ucap)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ucap) return;
    const int r = rep_of[k];
    if (r < 0 || (sel && !sel[r])) return;
    const int o = idx_sorted[k];
    const int slot = rd[r].S + (k - rd[r].P);
    perm[slot] = o;
    iperm[o] = slot;
    const double xn[3] = {x[3 * o], x[3 * o + 1], x[3 * o + 2]};
    store_pos(pos, posf, slot, xn, zii[o]);
}

// Repack slots with the current order (after a host-side state change).
__global__ void k_b_repack(const int* __restrict__ iperm, const int* __restrict__ rep_of,
                           const double* __restrict__ x, const double* __restrict__ zii, double4* __restrict__ pos,
                           float* __restrict__ posf, int ucap)
{
    const int o = blockIdx.x * blockDim.x + threadIdx.x;
    if (o >= ucap || rep_of[o] < 0) return;
    const double xn[3] = {x[3 * o], x[3 * o + 1], x[3 * o + 2]};
    store_pos(pos, posf, iperm[o], xn, zii[o]);
}

// vel_verlet_2.f:33-54 for every box, one thread per element (component
// e % 3 of the box's particle e / 3), in the caller's order: three CTAs per
// entry of the block table (box, block within box; entries of box -1 are
// unused), each over a contiguous third of the block's 3 VBLOCK elements, so
// every warp access is 256 contiguous bytes and the three loads of a thread
// are independent.  The slot-ordered copies follow in k_b_pack.
__global__ void __launch_bounds__(VBLOCK)
k_b_drift(const int2* __restrict__ vb, const RepDesc* __restrict__ rd, const int* __restrict__ left,
          double* __restrict__ x, double* __restrict__ v, double* __restrict__ vold, const double* __restrict__ a)
{
    const int2 t = vb[blockIdx.x / 3];
    if (t.x < 0 || left[t.x] <= 0) return;
    const RepDesc* d = rd + t.x;
    const int le = 3 * VBLOCK * t.y + (int)(blockIdx.x % 3) * VBLOCK + threadIdx.x;   // element in the box
    const StepArgs& s = d->sa;
    if (le >= 3 * s.n) return;
    const size_t e = 3 * (size_t)d->P + le;
    const double xi = x[e], vi = v[e], ai = a[d->A + le];
    x[e] = drift1(xi, vi, ai, s, le % 3);
    vold[e] = vi;
    v[e] = __dadd_rn(vi, __dmul_rn(s.dt, ai));
}

// The slot-ordered FP64 positions and FP32 shadow of every box that steps, a
// thread per slot: the position is gathered through perm and the slot's
// words are written in slot order (a warp writes contiguous runs), instead of
// being scattered through the permutation by the drift kernel.
__global__ void __launch_bounds__(256)
k_b_pack(const int* __restrict__ tile_rep, const RepDesc* __restrict__ rd, const int* __restrict__ left,
         const int* __restrict__ perm, const double* __restrict__ x, const double* __restrict__ zii,
         double4* __restrict__ pos, float* __restrict__ posf, int total_slots)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= total_slots) return;
    const int r = tile_rep[p >> 7];
    if (r < 0 || left[r] <= 0) return;
    if (p - rd[r].S >= rd[r].fa.n) return;
    const int o = perm[p];
    const double xn[3] = {x[3 * o], x[3 * o + 1], x[3 * o + 2]};
    store_pos(pos, posf, p, xn, zii[o]);
}

// vel_verlet_2.f:75-95 for every box; kinetic partials per block.
template <bool KIN>
__global__ void __launch_bounds__(VBLOCK)
k_b_post(const int2* __restrict__ vb, const RepDesc* __restrict__ rd, const int* __restrict__ left,
         double* __restrict__ v, const double* __restrict__ vold, const double* __restrict__ a,
         const double* __restrict__ aii, double* __restrict__ kpart)
{
    __shared__ double red[32 * NKIN];
    const int2 t = vb[blockIdx.x];
    if (t.x < 0 || left[t.x] <= 0) return;
    const RepDesc* d = rd + t.x;
    const int local = t.y * VBLOCK + threadIdx.x;
    const double dt = d->sa.dt;
    double tk[NKIN] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (local < d->sa.n) {
        const int gi = d->P + local;
        const double* ar = a + d->A;
        double vv[3], vo[3], aa[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            vv[k] = v[3 * gi + k];
            vo[k] = vold[3 * gi + k];
            aa[k] = ar[3 * local + k];
        }
        const double am = aii[gi];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const double vp = __dadd_rn(vo[k], __dmul_rn(dt, aa[k]));
            vv[k] = __dmul_rn(0.5, __dadd_rn(vv[k], vp));
            v[3 * gi + k] = vv[k];
        }
        kin_sums<KIN>(tk, am, vv[0], vv[1], vv[2]);
    }
    if constexpr (KIN) block_sum_store<NKIN>(tk, red, kpart + (size_t)blockIdx.x * NKIN);
}

// The persistent force kernel over the work items of jobs[0 .. *njobs); the
// items of boxes whose step budget is spent are passed over.
template <int SIM, int PREC, bool MEAS, bool LO = false>
// (6 CTAs per SM for the mixed hi/lo form: at 7, the box descriptors spill)
__global__ void __launch_bounds__(PB, (pairs_ctas_per_sm<SIM_MIX, PREC, LO>()))
k_force_pairs_batch(const double4* __restrict__ pos, const float* __restrict__ posf,
                    const int4* __restrict__ jobs, const int* __restrict__ njobs_p, int* __restrict__ counter,
                    const RepDesc* __restrict__ rd, const int* __restrict__ left, double* __restrict__ Si,
                    row_t<PREC>* __restrict__ Sj, double* __restrict__ Sm, unsigned* __restrict__ err)
{
    __shared__ __align__(128) PairSmem<row_t<PREC>> sm;
    __shared__ __align__(16) ForceArgs sfa;
    __shared__ int4 sjob;
    pairs_smem_init(sm);
    const int njobs = *njobs_p;
    unsigned q = 0;
    for (;;) {
        if (threadIdx.x == 0) {
            int4 jb;
            do {
                const int j = atomicAdd(counter, 1);
                jb = j < njobs ? jobs[j] : make_int4(-1, 0, 0, 0);
            } while (jb.x >= 0 && left[jb.x] <= 0);
            sjob = jb;
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
        bx.tbox = nullptr;
        bx.Sjf = nullptr;
        bx.n = sfa.n;
        bx.M = d->T;
        bx.nseg_max = d->nseg;
        const int C0 = jb.y + jb.z * d->seg;
        if (!pairs_job<SIM, PREC, MEAS, LO ? 1 : 2>(sm, sfa, bx, jb.y, C0, min(C0 + d->seg, bx.M), jb.z,
                                                    Sm + (size_t)(d->sm_off + jb.w) * NSCAL, err, q))
            return;
    }
}

// Per slot of the boxes in sel (all if NULL) whose budget is not spent: the
// fixed-order sum of its partials, the reference's scaling, and the store to
// the caller's order (as k_combine).  tile_rep: box of every tile, -1 unused.
template <int SIM, int PREC>
__global__ void __launch_bounds__(256)
k_b_combine(const int* __restrict__ tile_rep, const RepDesc* __restrict__ rd, const int* __restrict__ sel,
            const int* __restrict__ left, const double* __restrict__ Si, const row_t<PREC>* __restrict__ Sj,
            const int* __restrict__ perm, const double* __restrict__ zii, const double* __restrict__ aii,
            double* __restrict__ a, int total_slots)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= total_slots) return;
    const int r = tile_rep[p >> 7];
    if (r < 0 || (sel && !sel[r]) || left[r] <= 0) return;
    const RepDesc* d = rd + r;
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
    const row_t<PREC>* sj = Sj + d->Sj_off + ((size_t)tri_index(R, 0) * PB + l) * 3;
    for (int R2 = 0; R2 <= R; ++R2) {
        const row_t<PREC>* e = sj + (size_t)R2 * PB * 3;
        F[0] += e[0];
        F[1] += e[1];
        F[2] += e[2];
    }
    const int orig = perm[p];
    store_accel<SIM>(d->fa, orig - d->P, zii[orig], aii + d->P, F, a + d->A);
}

// One block per slot.  kin_mode / meas as in k_finish; the series entry of
// box r at the current step is series[(*series_idx) * nslots + r].  In a
// step (step = 1) the box's budget is counted down.
__global__ void __launch_bounds__(256)
k_b_finish(const RepDesc* __restrict__ rd, const int* __restrict__ sel, int* __restrict__ left,
           const double* __restrict__ Sm, const double* __restrict__ kpart, double* __restrict__ a,
           DevScalars* __restrict__ ds, double* __restrict__ series, const int* __restrict__ series_idx,
           int nslots, int meas, int kin_mode, int step)
{
    const int r = blockIdx.x;
    const RepDesc* d = rd + r;
    if (!d->active || (sel && !sel[r])) return;
    const int lr = left[r];
    if (lr <= 0) return;
    FinishArgs z = d->fz;
    z.force_mode = 1;
    z.do_meas = meas;
    z.nfp = meas ? d->njobs : 0;
    z.half = d->raw_scale;
    z.kin_mode = kin_mode;
    z.nkp = kin_mode == 2 ? d->nkb : 0;
    double* slot = series ? series + ((size_t)(*series_idx) * nslots + r) * 13 : nullptr;
    finish_body(Sm + (size_t)d->sm_off * NSCAL, kpart + (size_t)d->kb0 * NKIN, z, a + d->A, ds + r, slot);
    if (step && threadIdx.x == 0) left[r] = lr == UNLIMITED ? lr : lr - 1;
}

__global__ void k_b_series_next(int* series_idx) { *series_idx += 1; }

// First-fit allocator of ranges of [0, cap): free ranges by start, merged
// with their neighbours when given back.
struct RangeAlloc {
    long long cap = 0;
    std::map<long long, long long> free_;
    void init(long long c)
    {
        cap = c;
        free_.clear();
        if (c > 0) free_[0] = c;
    }
    long long take(long long len)
    {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < len) continue;
            const long long at = it->first, rest = it->second - len;
            free_.erase(it);
            if (rest > 0) free_[at + len] = rest;
            return at;
        }
        return -1;
    }
    void give(long long at, long long len)
    {
        auto nx = free_.lower_bound(at);
        if (nx != free_.end() && at + len == nx->first) {
            len += nx->second;
            nx = free_.erase(nx);
        }
        if (nx != free_.begin()) {
            auto pv = std::prev(nx);
            if (pv->first + pv->second == at) {
                pv->second += len;
                return;
            }
        }
        free_[at] = len;
    }
};

}  // namespace

// ---------------------------------------------------------------------------

struct GraphB {
    cudaGraphExec_t exec = nullptr;
    int K = 0, me = 0, phase = 0, series = 0, kernels = 0;
    unsigned long long stamp = 0;
};

struct yk_batch {
    int nslots = 0;                 // boxes the batch can hold
    int nrep = 0;                   // boxes held
    int ucap = 0, tcap = 0;         // particle units and tiles
    long long pair_cap = 0;         // half-pair units
    long long sj_cap = 0, si_cap = 0, sm_cap = 0, jobs_cap = 0;
    int cap_seg = 0;                // the shortest segment length si_cap / jobs_cap hold
    int vb_cap = 0;
    int dev = 0;
    int sim = 0, prec = 0;          // SIM_MIX or SIM_NUCLEON; PREC_*
    int prec_api = 0;
    cudaStream_t stream = nullptr;
    std::vector<char> held;
    std::vector<int> n;
    std::vector<double> time, dt;
    RangeAlloc ualloc, talloc;
    double *x = nullptr, *v = nullptr, *vold = nullptr, *a = nullptr, *zii = nullptr, *aii = nullptr;
    int* rep_of = nullptr;
    double4* pos = nullptr;
    float* posf = nullptr;
    int *perm = nullptr, *iperm = nullptr;
    unsigned *keys0 = nullptr, *keys1 = nullptr;
    int *idx0 = nullptr, *idx1 = nullptr;
    int *seg_b = nullptr, *seg_e = nullptr;          // sort segments of all held boxes
    int *segn_b = nullptr, *segn_e = nullptr;        // ... of the boxes being admitted
    void* cub_tmp = nullptr;
    size_t cub_bytes = 0;
    int key_bits = 30;
    RepDesc* rd = nullptr;
    int* left = nullptr;            // step budget per slot
    int* sel = nullptr;             // boxes being admitted
    int4* jobs = nullptr;           // work items of all held boxes
    int4* jobs_sel = nullptr;       // ... of the boxes being admitted
    int* njobs_dev = nullptr;       // [0] all, [1] admitted
    int njobs = 0, njobs_sel = 0;
    int* counter = nullptr;
    int* tile_rep = nullptr;
    int2* vblocks = nullptr;
    double *Si = nullptr, *Sm = nullptr, *kpart = nullptr;
    void* Sj = nullptr;             // source-side rows: double (FP64) or float (mixed)
    DevScalars* ds = nullptr;
    unsigned* err = nullptr;
    double* series = nullptr;
    int series_cap = 0;
    int* series_idx = nullptr;
    int force_grid = 0, force_grid_lo = 0;
    bool all_lo = false;            // every held box allows the mixed hi/lo displacement (fa.lo / fa.hilo)
    int seg = BATCH_SEG, graph_steps = BATCH_GRAPH_STEPS;
    int sort_every = BATCH_SORT_EVERY;
    int since_sort = 0;             // steps run since the last re-ordering (eager steps)
    std::vector<RepDesc> hrd;       // host copy of the descriptors
    bool pos_dirty = false;
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

// Slot order of the held boxes (sel_new: only the boxes being admitted).
static int enqueue_sort(yk_batch* b, bool sel_new)
{
    cudaStream_t st = b->stream;
    const int nb = (b->ucap + 255) / 256;
    const int* sel = sel_new ? b->sel : nullptr;
    k_b_morton<<<nb, 256, 0, st>>>(b->x, b->rep_of, b->rd, sel, b->ucap, b->keys0, b->idx0,
                                   b->sim == SIM_NUCLEON ? b->zii : nullptr);
    size_t bytes = b->cub_bytes;
    cub::DeviceSegmentedRadixSort::SortPairs(b->cub_tmp, bytes, b->keys0, b->keys1, b->idx0, b->idx1, b->ucap,
                                             b->nslots, sel_new ? b->segn_b : b->seg_b,
                                             sel_new ? b->segn_e : b->seg_e, 0, b->key_bits, st);
    k_b_place<<<nb, 256, 0, st>>>(b->idx1, b->rep_of, b->rd, sel, b->x, b->zii, b->pos, b->posf, b->perm,
                                  b->iperm, b->ucap);
    if (!sel_new) b->pos_dirty = false;
    return 3;
}

// Force call over all held boxes (sel_new = false) or over the boxes being
// admitted (their own job table; the other boxes' state is not touched).
template <int SIM, int PREC, bool MEAS>
static int launch_force_b(yk_batch* b, bool sel_new)
{
    if (b->force_grid == 0) {
        int per_sm = 0, per_sm_lo = 0, sms = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_force_pairs_batch<SIM, PREC, MEAS>, PB, 0);
        if constexpr (PREC == PREC_MIXED)
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_lo, k_force_pairs_batch<SIM, PREC, MEAS, true>,
                                                          PB, 0);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->dev);
        b->force_grid = std::max(1, per_sm) * std::max(1, sms);
        b->force_grid_lo = std::max(1, per_sm_lo) * std::max(1, sms);
    }
    const int4* jobs = sel_new ? b->jobs_sel : b->jobs;
    const int* njp = b->njobs_dev + (sel_new ? 1 : 0);
    cudaMemsetAsync(b->counter, 0, sizeof(int), b->stream);
    bool launched = false;
    if constexpr (PREC == PREC_MIXED) {
        if (b->all_lo) {
            k_force_pairs_batch<SIM, PREC, MEAS, true><<<b->force_grid_lo, PB, 0, b->stream>>>(
                b->pos, b->posf, jobs, njp, b->counter, b->rd, b->left, b->Si, static_cast<row_t<PREC>*>(b->Sj),
                b->Sm, b->err);
            launched = true;
        }
    }
    if (!launched)
        k_force_pairs_batch<SIM, PREC, MEAS><<<b->force_grid, PB, 0, b->stream>>>(
            b->pos, b->posf, jobs, njp, b->counter, b->rd, b->left, b->Si, static_cast<row_t<PREC>*>(b->Sj),
            b->Sm, b->err);
    k_b_combine<SIM, PREC><<<(b->tcap * PB + 255) / 256, 256, 0, b->stream>>>(b->tile_rep, b->rd, sel_new ? b->sel : nullptr,
                                                                 b->left, b->Si, static_cast<row_t<PREC>*>(b->Sj),
                                                                 b->perm, b->zii, b->aii,
                                                                 b->a, b->tcap * PB);
    return 2;
}

template <int SIM>
static int launch_force_bs(yk_batch* b, bool meas, bool sel_new)
{
    if (b->prec == PREC_MIXED)
        return meas ? launch_force_b<SIM, PREC_MIXED, true>(b, sel_new) : launch_force_b<SIM, PREC_MIXED, false>(b, sel_new);
    return meas ? launch_force_b<SIM, PREC_FP64, true>(b, sel_new) : launch_force_b<SIM, PREC_FP64, false>(b, sel_new);
}

static int enqueue_force_b(yk_batch* b, bool meas, bool sel_new = false)
{
    return b->sim == SIM_NUCLEON ? launch_force_bs<SIM_NUCLEON>(b, meas, sel_new)
                                 : launch_force_bs<SIM_MIX>(b, meas, sel_new);
}

static int enqueue_step_b(yk_batch* b, bool meas, bool series, bool resort)
{
    int k = 0;
    cudaStream_t st = b->stream;
    if (resort) k += enqueue_sort(b, false);
    else if (b->pos_dirty) {
        k_b_repack<<<(b->ucap + 255) / 256, 256, 0, st>>>(b->iperm, b->rep_of, b->x, b->zii, b->pos, b->posf,
                                                          b->ucap);
        b->pos_dirty = false;
        ++k;
    }
    k_b_drift<<<3 * b->vb_cap, VBLOCK, 0, st>>>(b->vblocks, b->rd, b->left, b->x, b->v, b->vold, b->a);
    k_b_pack<<<(b->tcap * PB + 255) / 256, 256, 0, st>>>(b->tile_rep, b->rd, b->left, b->perm, b->x, b->zii,
                                                          b->pos, b->posf, b->tcap * PB);
    k += 2;
    k += enqueue_force_b(b, meas);
    if (meas)
        k_b_post<true><<<b->vb_cap, VBLOCK, 0, st>>>(b->vblocks, b->rd, b->left, b->v, b->vold, b->a, b->aii,
                                                     b->kpart);
    else
        k_b_post<false><<<b->vb_cap, VBLOCK, 0, st>>>(b->vblocks, b->rd, b->left, b->v, b->vold, b->a, b->aii,
                                                      b->kpart);
    ++k;
    k_b_finish<<<b->nslots, 256, 0, st>>>(b->rd, nullptr, b->left, b->Sm, b->kpart, b->a, b->ds,
                                          series ? b->series : nullptr, b->series_idx, b->nslots, meas ? 1 : 0,
                                          meas ? 2 : 1, 1);
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
    for (int l = 1; l <= K; ++l)
        kernels += enqueue_step_b(b, me > 0 && (phase + l) % me == 0, series, (l - 1) % b->sort_every == 0);
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

// Work items of box r for segment length seg, with their costs.
static void box_jobs(int r, int T, int seg, std::vector<int4>& jobs, std::vector<int>& cost)
{
    int local = 0;
    for (int R = 0; R < T; ++R)
        for (int s = 0; s * seg < T - R; ++s) {
            jobs.push_back(make_int4(r, R, s, local++));
            const int tiles = std::min(seg, T - R - s * seg);
            cost.push_back(2 * tiles - (s == 0 ? 1 : 0));
        }
}

static void costliest_first(std::vector<int4>& jobs, const std::vector<int>& cost)
{
    std::vector<int> order(jobs.size());
    for (size_t k = 0; k < order.size(); ++k) order[k] = (int)k;
    std::stable_sort(order.begin(), order.end(), [&](int u, int w) { return cost[u] > cost[w]; });
    std::vector<int4> out(jobs.size());
    for (size_t k = 0; k < order.size(); ++k) out[k] = jobs[order[k]];
    jobs.swap(out);
}

static long long units_of(int T) { return (long long)T * (T + 1) / 2; }
static long long nseg_of(int T, int seg) { return (T + seg - 1) / seg; }

// Si rows and jobs that boxes of at most `units` half-pair units on at most
// `tiles` tiles can need with segments of `seg` tiles: a box of T tiles takes
// T ceil(T / seg) <= T^2 / seg + T <= 2 units / seg + T of each.
static long long jobs_bound(long long units, long long tiles, int seg) { return 2 * units / seg + 2 * tiles; }

// Si, Sm and the job tables sized for segment length seg.
static int alloc_job_scratch(yk_batch* b, int seg)
{
    const long long jb = jobs_bound(b->pair_cap, b->tcap, seg);
    cudaStream_t st = b->stream;
    cudaFreeAsync(b->Si, st);
    cudaFreeAsync(b->Sm, st);
    cudaFreeAsync(b->jobs, st);
    cudaFreeAsync(b->jobs_sel, st);
    b->Si = b->Sm = nullptr;
    b->jobs = b->jobs_sel = nullptr;
    b->si_cap = jb * PB * 3;
    b->jobs_cap = jb;
    b->sm_cap = NSCAL * jb;
    b->cap_seg = 0;
    if (cudaMallocAsync((void**)&b->Si, sizeof(double) * (size_t)b->si_cap, st) != cudaSuccess ||
        cudaMallocAsync((void**)&b->Sm, sizeof(double) * (size_t)b->sm_cap, st) != cudaSuccess ||
        cudaMallocAsync((void**)&b->jobs, sizeof(int4) * (size_t)jb, st) != cudaSuccess ||
        cudaMallocAsync((void**)&b->jobs_sel, sizeof(int4) * (size_t)jb, st) != cudaSuccess)
        return bfail(b, YK_ERR_NOMEM, "device allocation of the job scratch for pair_seg %d failed", seg);
    b->cap_seg = seg;
    return YK_OK;
}

// Scratch and tables of the held boxes for segment length seg (packed in
// slot order), with the capacities checked; newsel marks the boxes being
// admitted (their own job table and sort segments).  Uploads everything.
static int relayout(yk_batch* b, int seg, const std::vector<char>& newsel)
{
    long long sj = 0, si = 0;
    int smo = 0;
    std::vector<int4> jobs, jobs_sel;
    std::vector<int> cost, cost_sel;
    std::vector<int2> vblocks;
    std::vector<int> tile_rep(b->tcap, -1), seg_b(b->nslots, 0), seg_e(b->nslots, 0), segn_b(b->nslots, 0),
        segn_e(b->nslots, 0), selv(b->nslots, 0);
    bool all_lo = true;
    int held = 0;
    for (int r = 0; r < b->nslots; ++r) {
        RepDesc& d = b->hrd[r];
        if (!b->held[r]) {
            d.active = 0;
            continue;
        }
        ++held;
        d.active = 1;
        d.seg = seg;
        d.nseg = (int)nseg_of(d.T, seg);
        d.Sj_off = sj;
        d.Si_off = si;
        d.sm_off = smo;
        const size_t j0 = jobs.size();
        box_jobs(r, d.T, seg, jobs, cost);
        d.njobs = (int)(jobs.size() - j0);
        if (!newsel.empty() && newsel[r]) {
            for (size_t k = j0; k < jobs.size(); ++k) {
                jobs_sel.push_back(jobs[k]);
                cost_sel.push_back(cost[k]);
            }
            segn_b[r] = d.P;
            segn_e[r] = d.P + d.fa.n;
            selv[r] = 1;
        }
        sj += units_of(d.T) * PB * 3;
        si += (long long)d.T * d.nseg * PB * 3;
        smo += d.njobs;
        const int nb = (d.fa.n + VBLOCK - 1) / VBLOCK;
        d.kb0 = (int)vblocks.size();
        d.nkb = nb;
        for (int q = 0; q < nb; ++q) vblocks.push_back(make_int2(r, q));
        for (int t = 0; t < d.T; ++t) tile_rep[d.S / PB + t] = r;
        seg_b[r] = d.P;
        seg_e[r] = d.P + d.fa.n;
        all_lo = all_lo && (b->sim == SIM_NUCLEON ? d.fa.hilo : d.fa.lo) != 0;
    }
    if (sj > b->sj_cap || si > b->si_cap || (long long)smo * NSCAL > b->sm_cap ||
        (long long)jobs.size() > b->jobs_cap || (int)vblocks.size() > b->vb_cap)
        return bfail(b, YK_ERR_NOMEM, "the boxes need more half-pair scratch than the batch holds");
    costliest_first(jobs, cost);
    costliest_first(jobs_sel, cost_sel);
    vblocks.resize(b->vb_cap, make_int2(-1, 0));
    b->njobs = (int)jobs.size();
    b->njobs_sel = (int)jobs_sel.size();
    b->seg = seg;
    b->nrep = held;
    b->all_lo = held > 0 && all_lo;
    const int nj[2] = {b->njobs, b->njobs_sel};
    cudaStream_t st = b->stream;
    BCK(b, cudaMemcpyAsync(b->rd, b->hrd.data(), sizeof(RepDesc) * b->nslots, cudaMemcpyHostToDevice, st));
    if (!jobs.empty())
        BCK(b, cudaMemcpyAsync(b->jobs, jobs.data(), sizeof(int4) * jobs.size(), cudaMemcpyHostToDevice, st));
    if (!jobs_sel.empty())
        BCK(b, cudaMemcpyAsync(b->jobs_sel, jobs_sel.data(), sizeof(int4) * jobs_sel.size(),
                               cudaMemcpyHostToDevice, st));
    BCK(b, cudaMemcpyAsync(b->njobs_dev, nj, sizeof nj, cudaMemcpyHostToDevice, st));
    BCK(b, cudaMemcpyAsync(b->vblocks, vblocks.data(), sizeof(int2) * vblocks.size(), cudaMemcpyHostToDevice, st));
    BCK(b, cudaMemcpyAsync(b->tile_rep, tile_rep.data(), sizeof(int) * tile_rep.size(), cudaMemcpyHostToDevice,
                           st));
    BCK(b, cudaMemcpyAsync(b->seg_b, seg_b.data(), sizeof(int) * b->nslots, cudaMemcpyHostToDevice, st));
    BCK(b, cudaMemcpyAsync(b->seg_e, seg_e.data(), sizeof(int) * b->nslots, cudaMemcpyHostToDevice, st));
    BCK(b, cudaMemcpyAsync(b->segn_b, segn_b.data(), sizeof(int) * b->nslots, cudaMemcpyHostToDevice, st));
    BCK(b, cudaMemcpyAsync(b->segn_e, segn_e.data(), sizeof(int) * b->nslots, cudaMemcpyHostToDevice, st));
    BCK(b, cudaMemcpyAsync(b->sel, selv.data(), sizeof(int) * b->nslots, cudaMemcpyHostToDevice, st));
    // these host vectors die on return: wait for the copies
    BCK(b, cudaStreamSynchronize(st));
    return YK_OK;
}

// Checks of one box's arguments (the same for every way into a batch).
static int check_box(yk_batch* b, const yk_params& p, int n, const double* x, const double* v, const double* zii,
                     const double* aii, bool nuc, int prec)
{
    if (n < 1) return bfail(b, YK_ERR_ARG, "n must be >= 1");
    if (!x) return bfail(b, YK_ERR_ARG, "x is NULL");
    if (p.sim_type == YK_SIM_BFIELD || (p.sim_type == YK_SIM_NUCLEON) != nuc)
        return bfail(b, YK_ERR_ARG, "a batch holds either ion boxes or nucleon boxes");
    if (p.precision != prec) return bfail(b, YK_ERR_ARG, "one precision per batch");
    if (p.integrator != YK_VV2 || p.bfield != 0.0)
        return bfail(b, YK_ERR_ARG, "batches run vel_verlet_2 without B field");
    if (!(p.dt > 0.0) || !(p.xl[0] > 0.0) || !(p.xl[1] > 0.0) || !(p.xl[2] > 0.0) || !(p.xmass > 0.0))
        return bfail(b, YK_ERR_ARG, "dt, xl and xmass must be > 0");
    if (p.sim_type != YK_SIM_PURE_ION && !zii) return bfail(b, YK_ERR_ARG, "zii required");
    if (p.sim_type == YK_SIM_ION_MIXTURE && !aii) return bfail(b, YK_ERR_ARG, "aii required");
    if (p.sim_type == YK_SIM_PURE_ION && !(p.ai > 0.0)) return bfail(b, YK_ERR_ARG, "pure-ion boxes need ai > 0");
    for (long long e = 0; e < 3LL * n; ++e)
        if (!std::isfinite(x[e]) || (v && !std::isfinite(v[e])))
            return bfail(b, YK_ERR_NONFINITE, "NaN or Inf in x or v");
    return YK_OK;
}

// Puts boxes into free slots: particle and tile ranges, descriptors and state
// (v NULL: zero velocities), step budgets (steps NULL: unlimited).  No sort
// and no force call.  slots_out[k] receives box k's slot.  On failure no new
// box is held.
static int place_boxes(yk_batch* b, int count, const yk_params* params, const int* n, const double* const* x,
                       const double* const* v, const double* const* zii, const double* const* aii,
                       const long long* steps, int* slots_out)
{
    const bool nuc = b->sim == SIM_NUCLEON;
    for (int k = 0; k < count; ++k) {
        int rc = check_box(b, params[k], n[k], x[k], v ? v[k] : nullptr, zii ? zii[k] : nullptr,
                           aii ? aii[k] : nullptr, nuc, b->prec_api);
        if (rc) return rc;
    }
    std::vector<int> slots;
    std::vector<long long> U, Tt;
    auto undo = [&]() {
        for (size_t k = 0; k < slots.size(); ++k) {
            b->held[slots[k]] = 0;
            b->ualloc.give(U[k], n[k] + 3);
            b->talloc.give(Tt[k], (n[k] + PB - 1) / PB);
        }
    };
    for (int k = 0; k < count; ++k) {
        int r = -1;
        for (int q = 0; q < b->nslots; ++q)
            if (!b->held[q]) {
                r = q;
                break;
            }
        const int T = (n[k] + PB - 1) / PB;
        const long long u = r < 0 ? -1 : b->ualloc.take(n[k] + 3);
        const long long t = (u < 0) ? -1 : b->talloc.take(T);
        if (r < 0 || u < 0 || t < 0) {
            if (u >= 0) b->ualloc.give(u, n[k] + 3);
            undo();
            return bfail(b, YK_ERR_NOMEM, "no free slot, particle range or tile range for a box of %d", n[k]);
        }
        b->held[r] = 1;
        slots.push_back(r);
        U.push_back(u);
        Tt.push_back(t);
    }
    cudaStream_t st = b->stream;
    for (int k = 0; k < count; ++k) {
        const int r = slots[k];
        yk_params p = params[k];
        RepDesc& d = b->hrd[r];
        d = RepDesc{};
        d.raw_scale = 1.0;
        if (p.sim_type == YK_SIM_PURE_ION) {
            // run through the mixture kernels (Z_i = zi); keep the pure-ion
            // scaling of the scalars, int_ion_pure.f:233-242
            ForceArgs fa_pure;
            StepArgs sa_pure;
            make_args(p, n[k], &fa_pure, &sa_pure, &d.fz);
            d.raw_scale = 1.0 / (p.zi * p.zi);
            p.sim_type = YK_SIM_ION_MIXTURE;
            p.mix_mode = YK_MIX_FIXED;
            FinishArgs fz_mix;
            make_args(p, n[k], &d.fa, &d.sa, &fz_mix);
        } else {
            make_args(p, n[k], &d.fa, &d.sa, &d.fz);
        }
        d.sa.pack_w = 1;
        d.P = (int)U[k];
        d.S = (int)(Tt[k] * PB);
        d.T = (n[k] + PB - 1) / PB;
        d.A = 3LL * U[k];
        b->n[r] = n[k];
        b->time[r] = params[k].time;
        b->dt[r] = params[k].dt;
        const size_t nn = (size_t)n[k];
        std::vector<double> hz(nn), ha(nn);
        std::vector<int> hrep(nn + 3, r);
        hrep[nn] = hrep[nn + 1] = hrep[nn + 2] = -1;
        for (size_t i = 0; i < nn; ++i) {
            hz[i] = (zii && zii[k]) ? zii[k][i] : params[k].zi;
            ha[i] = (aii && aii[k]) ? aii[k][i] : (params[k].ai > 0.0 ? params[k].ai : 1.0);
        }
        const int lft = steps ? (int)std::min<long long>(steps[k], UNLIMITED - 1) : UNLIMITED;
        const size_t o = (size_t)U[k];
        BCK(b, cudaMemcpyAsync(b->x + 3 * o, x[k], sizeof(double) * 3 * nn, cudaMemcpyHostToDevice, st));
        if (v && v[k]) BCK(b, cudaMemcpyAsync(b->v + 3 * o, v[k], sizeof(double) * 3 * nn, cudaMemcpyHostToDevice, st));
        else BCK(b, cudaMemsetAsync(b->v + 3 * o, 0, sizeof(double) * 3 * nn, st));
        BCK(b, cudaMemsetAsync(b->vold + 3 * o, 0, sizeof(double) * 3 * nn, st));
        BCK(b, cudaMemsetAsync(b->a + 3 * o, 0, sizeof(double) * 3 * (nn + 3), st));
        BCK(b, cudaMemcpyAsync(b->zii + o, hz.data(), sizeof(double) * nn, cudaMemcpyHostToDevice, st));
        BCK(b, cudaMemcpyAsync(b->aii + o, ha.data(), sizeof(double) * nn, cudaMemcpyHostToDevice, st));
        BCK(b, cudaMemcpyAsync(b->rep_of + o, hrep.data(), sizeof(int) * (nn + 3), cudaMemcpyHostToDevice, st));
        BCK(b, cudaMemsetAsync(b->posf + (size_t)Tt[k] * SHADOW_FLOATS, 0, sizeof(float) * SHADOW_FLOATS * d.T, st));
        BCK(b, cudaMemsetAsync(b->pos + (size_t)d.S, 0, sizeof(double4) * PB * d.T, st));
        BCK(b, cudaMemsetAsync(b->perm + (size_t)d.S, 0xff, sizeof(int) * PB * d.T, st));
        BCK(b, cudaMemcpyAsync(b->left + r, &lft, sizeof(int), cudaMemcpyHostToDevice, st));
        BCK(b, cudaMemsetAsync(b->ds + r, 0, sizeof(DevScalars), st));
        BCK(b, cudaStreamSynchronize(st));              // host vectors above die here
        if (slots_out) slots_out[k] = r;
    }
    return YK_OK;
}

static void fill_out(const yk_batch* b, const DevScalars& h, int r, yk_scalars& o)
{
    o.ev = h.ev;
    o.vir = h.vir;
    o.px = h.px;
    o.ek = h.ek;
    for (int q = 0; q < 9; ++q) o.pp[q] = h.pp[q];
    o.time = b->time[r];
}

extern "C" {

const char* yk_batch_last_error(const yk_batch* b) { return b ? b->errmsg.c_str() : g_batch_err.c_str(); }

// Batches are created and destroyed often (the serving loop creates one per
// group), so their device arrays come from the device's stream-ordered memory
// pool, which keeps up to POOL_KEEP bytes of freed memory cached between
// batches.
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

int yk_batch_get_tuning(yk_batch* b, yk_tuning* out)
{
    if (!b || !out) return bfail(b, YK_ERR_ARG, "batch and out are required");
    out->force_kernel = 2;
    out->pair_seg = b->seg;
    out->sort_every = b->sort_every == SORT_AT_GRAPH_START_ONLY ? -1 : b->sort_every;
    out->graph_steps = b->graph_steps;
    out->source_split = 1;
    out->targets_per_thread = 1;
    return YK_OK;
}

int yk_batch_set_tuning(yk_batch* b, const yk_tuning* t)
{
    if (!b || !t) return bfail(b, YK_ERR_ARG, "batch and tuning are required");
    if (t->force_kernel != 0 && t->force_kernel != 2)
        return bfail(b, YK_ERR_UNSUPPORTED, "a batch runs the half-pair kernel (force_kernel 0 or 2)");
    if (t->pair_seg < 0 || t->graph_steps < 0 || t->sort_every < -1) return bfail(b, YK_ERR_ARG, "bad tuning values");
    if (t->source_split > 1) return bfail(b, YK_ERR_UNSUPPORTED, "a batch runs whole source tiles (source_split 0 or 1)");
    if (t->targets_per_thread > 1)
        return bfail(b, YK_ERR_UNSUPPORTED, "a batch runs one target per thread (targets_per_thread 0 or 1)");
    BCK(b, cudaSetDevice(b->dev));
    BCK(b, cudaStreamSynchronize(b->stream));
    drop_graphs_b(b);
    b->graph_steps = t->graph_steps > 0 ? t->graph_steps : BATCH_GRAPH_STEPS;
    // -1: only at the start of each graph
    b->sort_every = t->sort_every > 0 ? t->sort_every : t->sort_every < 0 ? SORT_AT_GRAPH_START_ONLY : BATCH_SORT_EVERY;
    const int seg = t->pair_seg > 0 ? t->pair_seg : BATCH_SEG;
    if (seg == b->seg) return YK_OK;
    if (seg < b->cap_seg) {
        // shorter segments take more Si rows and jobs
        int rc = alloc_job_scratch(b, seg);
        if (rc) return rc;
    }
    return relayout(b, seg, {});
}

int yk_batch_destroy(yk_batch* b)
{
    if (!b) return bfail(nullptr, YK_ERR_ARG, "batch is NULL");
    cudaSetDevice(b->dev);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graphs_b(b);
    void* bufs[] = {b->x,       b->v,      b->vold,    b->a,        b->zii,     b->aii,     b->rep_of,
                    b->pos,     b->posf,   b->perm,    b->iperm,    b->keys0,   b->keys1,   b->idx0,
                    b->idx1,    b->seg_b,  b->seg_e,   b->segn_b,   b->segn_e,  b->cub_tmp, b->rd,
                    b->left,    b->sel,    b->jobs,    b->jobs_sel, b->njobs_dev, b->counter, b->tile_rep,
                    b->vblocks, b->Si,     b->Sj,      b->Sm,       b->kpart,   b->ds,      b->err,
                    b->series,  b->series_idx};
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

// An empty batch with the given capacities: nslots boxes, max_units particle
// units (n + 3 per box), max_tiles tiles, max_pair_units half-pair units
// (T (T + 1) / 2 per box of T tiles).
static int create_empty(int sim, int prec_api, int nslots, long long max_units, long long max_tiles,
                        long long max_pair_units, int device, yk_batch** out)
{
    *out = nullptr;
    if (nslots < 1 || max_units < 4 || max_tiles < 1 || max_pair_units < 1)
        return bfail(nullptr, YK_ERR_ARG, "slots, particles, tiles and pair units must be >= 1");
    if (max_units > (1LL << 28) || max_tiles * PB > (1LL << 30))
        return bfail(nullptr, YK_ERR_ARG, "batch too large");
    if (cudaSetDevice(device) != cudaSuccess) return bfail(nullptr, YK_ERR_CUDA, "cudaSetDevice(%d) failed", device);
    yk_batch* b = new yk_batch();
    b->nslots = nslots;
    b->ucap = (int)max_units;
    b->tcap = (int)max_tiles;
    b->pair_cap = max_pair_units;
    b->sj_cap = max_pair_units * PB * 3;
    const long long jb = jobs_bound(max_pair_units, max_tiles, BATCH_SEG);
    b->vb_cap = (int)(max_units / VBLOCK + nslots);
    b->dev = device;
    b->sim = sim;
    b->prec_api = prec_api;
    b->prec = prec_api == YK_PREC_MIXED ? PREC_MIXED : PREC_FP64;
    b->key_bits = sim == SIM_NUCLEON ? 31 : 30;
    b->held.assign(nslots, 0);
    b->n.assign(nslots, 0);
    b->time.assign(nslots, 0.0);
    b->dt.assign(nslots, 0.0);
    b->hrd.assign(nslots, RepDesc{});
    b->ualloc.init(max_units);
    b->talloc.init(max_tiles);

    size_t cub_bytes = 0;
    cub::DeviceSegmentedRadixSort::SortPairs(nullptr, cub_bytes, (unsigned*)nullptr, (unsigned*)nullptr,
                                             (int*)nullptr, (int*)nullptr, b->ucap, nslots, (int*)nullptr,
                                             (int*)nullptr, 0, b->key_bits);
    const long long U = max_units, S = max_tiles * PB;
    const size_t sj_elem = b->prec == PREC_MIXED ? sizeof(float) : sizeof(double);
    const size_t need = sj_elem * (size_t)b->sj_cap + sizeof(double) * (size_t)(14 * U + jb * PB * 3 + NSCAL * jb +
                                                  (long long)NKIN * b->vb_cap) +
                        sizeof(double4) * S + sizeof(float) * (SHADOW_FLOATS / SHADOW_TILE) * S +
                        sizeof(int) * (4 * U + S + max_tiles) + sizeof(unsigned) * 2 * U + cub_bytes +
                        sizeof(RepDesc) * nslots + sizeof(int4) * 2 * jb + (64u << 20);
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
    BALLOC(b->x, 3 * U);
    BALLOC(b->v, 3 * U);
    BALLOC(b->vold, 3 * U);
    BALLOC(b->a, 3 * U);
    BALLOC(b->zii, U);
    BALLOC(b->aii, U);
    BALLOC(b->rep_of, U);
    BALLOC(b->pos, S);
    BALLOC(b->posf, (long long)SHADOW_FLOATS * max_tiles);
    BALLOC(b->perm, S);
    BALLOC(b->iperm, U);
    BALLOC(b->keys0, U);
    BALLOC(b->keys1, U);
    BALLOC(b->idx0, U);
    BALLOC(b->idx1, U);
    BALLOC(b->seg_b, nslots);
    BALLOC(b->seg_e, nslots);
    BALLOC(b->segn_b, nslots);
    BALLOC(b->segn_e, nslots);
    BALLOC(b->rd, nslots);
    BALLOC(b->left, nslots);
    BALLOC(b->sel, nslots);
    BALLOC(b->njobs_dev, 2);
    BALLOC(b->counter, 1);
    BALLOC(b->tile_rep, max_tiles);
    BALLOC(b->vblocks, b->vb_cap);
    if (cudaMallocAsync(&b->Sj, (b->prec == PREC_MIXED ? sizeof(float) : sizeof(double)) * (size_t)b->sj_cap,
                        b->stream) != cudaSuccess) {
        yk_batch_destroy(b);
        return bfail(nullptr, YK_ERR_NOMEM, "device allocation of Sj failed");
    }
    BALLOC(b->kpart, (long long)NKIN * b->vb_cap);
    BALLOC(b->ds, nslots);
    BALLOC(b->err, 1);
    BALLOC(b->series_idx, 1);
#undef BALLOC
    b->cub_bytes = cub_bytes;
    if (cudaMallocAsync(&b->cub_tmp, std::max<size_t>(cub_bytes, 16), b->stream) != cudaSuccess ||
        cudaEventCreate(&b->e0) != cudaSuccess || cudaEventCreate(&b->e1) != cudaSuccess ||
        alloc_job_scratch(b, BATCH_SEG) != YK_OK) {
        yk_batch_destroy(b);
        return bfail(nullptr, YK_ERR_NOMEM, "batch set-up failed");
    }
    cudaStream_t st = b->stream;
    cudaMemsetAsync(b->rep_of, 0xff, sizeof(int) * U, st);         // -1: no box
    cudaMemsetAsync(b->left, 0, sizeof(int) * nslots, st);
    cudaMemsetAsync(b->ds, 0, sizeof(DevScalars) * nslots, st);
    cudaMemsetAsync(b->err, 0, sizeof(unsigned), st);
    cudaMemsetAsync(b->series_idx, 0, sizeof(int), st);
    int rc = relayout(b, BATCH_SEG, {});
    if (rc) {
        std::string m = b->errmsg;
        yk_batch_destroy(b);
        return bfail(nullptr, rc, "%s", m.c_str());
    }
    *out = b;
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
    long long units = 0, tiles = 0, pairs = 0;
    for (int r = 0; r < nrep; ++r) {
        if (n[r] < 1) return bfail(nullptr, YK_ERR_ARG, "box %d: n must be >= 1", r);
        const int T = (n[r] + PB - 1) / PB;
        units += n[r] + 3;
        tiles += T;
        pairs += units_of(T);
    }
    if (units > (1LL << 28) || tiles * PB > (1LL << 30)) return bfail(nullptr, YK_ERR_ARG, "batch too large");
    yk_batch* b = nullptr;
    int rc = create_empty(nuc ? SIM_NUCLEON : SIM_MIX, params[0].precision, nrep, units, tiles, pairs, device, &b);
    if (rc) return rc;
    std::vector<int> slots(nrep);
    rc = place_boxes(b, nrep, params, n, x, v, zii, aii, nullptr, slots.data());
    if (rc == YK_OK) rc = relayout(b, b->seg, std::vector<char>(nrep, 1));
    if (rc) {
        std::string m = b->errmsg;
        yk_batch_destroy(b);
        return bfail(nullptr, rc, "%s", m.c_str());
    }
    count_launches(enqueue_sort(b, false));
    if (cudaStreamSynchronize(b->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess) {
        yk_batch_destroy(b);
        return bfail(nullptr, YK_ERR_CUDA, "batch upload failed");
    }
    *out = b;
    return YK_OK;
}

int yk_batch_create_slots(const yk_params* proto, int nslots, long long max_particles, long long max_pair_units,
                          int device, yk_batch** out)
{
    if (!out) return bfail(nullptr, YK_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!proto) return bfail(nullptr, YK_ERR_ARG, "proto is required");
    if (proto->sim_type == YK_SIM_BFIELD) return bfail(nullptr, YK_ERR_ARG, "a batch holds ion or nucleon boxes");
    if (nslots < 1 || max_particles < 1 || max_pair_units < 1)
        return bfail(nullptr, YK_ERR_ARG, "nslots, max_particles and max_pair_units must be >= 1");
    const long long units = max_particles + 3LL * nslots;
    const long long tiles = (max_particles + PB - 1) / PB + nslots;
    return create_empty(proto->sim_type == YK_SIM_NUCLEON ? SIM_NUCLEON : SIM_MIX, proto->precision, nslots, units,
                        tiles, max_pair_units, device, out);
}

int yk_batch_admit(yk_batch* b, const yk_params* p, int n, const double* x, const double* v, const double* zii,
                   const double* aii, long long steps, int* slot, yk_scalars* out)
{
    if (!b) return bfail(nullptr, YK_ERR_ARG, "batch is NULL");
    if (!p || !slot) return bfail(b, YK_ERR_ARG, "params and slot are required");
    if (steps < 1) return bfail(b, YK_ERR_ARG, "steps must be >= 1");
    BCK(b, cudaSetDevice(b->dev));
    BCK(b, cudaStreamSynchronize(b->stream));
    const double* xs[1] = {x};
    const double* vs[1] = {v};
    const double* zs[1] = {zii};
    const double* as[1] = {aii};
    int r = -1;
    int rc = place_boxes(b, 1, p, &n, xs, vs, zs, as, &steps, &r);
    if (rc) return rc;
    std::vector<char> newsel(b->nslots, 0);
    newsel[r] = 1;
    rc = relayout(b, b->seg, newsel);
    if (rc) {
        // does not fit the scratch: give the slot back
        const std::string m = b->errmsg;
        b->held[r] = 0;
        b->ualloc.give(b->hrd[r].P, n + 3);
        b->talloc.give(b->hrd[r].S / PB, b->hrd[r].T);
        std::vector<int> hrep(n + 3, -1);
        cudaMemcpyAsync(b->rep_of + b->hrd[r].P, hrep.data(), sizeof(int) * hrep.size(), cudaMemcpyHostToDevice,
                        b->stream);
        cudaMemsetAsync(b->left + r, 0, sizeof(int), b->stream);
        b->n[r] = 0;
        relayout(b, b->seg, {});
        return bfail(b, rc, "%s", m.c_str());
    }
    // md.F:69 for the new run only: its slot order and its initial forces
    // (a measuring force call over its own work items)
    int k = enqueue_sort(b, true);
    k += enqueue_force_b(b, true, true);
    k_b_finish<<<b->nslots, 256, 0, b->stream>>>(b->rd, b->sel, b->left, b->Sm, b->kpart, b->a, b->ds, nullptr,
                                                 b->series_idx, b->nslots, 1, 0, 0);
    ++k;
    count_launches(k);
    DevScalars h{};
    BCK(b, cudaMemcpyAsync(&h, b->ds + r, sizeof h, cudaMemcpyDeviceToHost, b->stream));
    rc = sync_check_b(b);
    if (rc) return rc;
    *slot = r;
    if (out) fill_out(b, h, r, *out);
    return YK_OK;
}

int yk_batch_retire(yk_batch* b, int slot, double* x, double* v, double* vold, double* a)
{
    if (!b) return bfail(nullptr, YK_ERR_ARG, "batch is NULL");
    if (slot < 0 || slot >= b->nslots || !b->held[slot]) return bfail(b, YK_ERR_ARG, "slot %d holds no box", slot);
    int rc = yk_batch_get_state(b, slot, x, v, vold, a);
    if (rc) return rc;
    const RepDesc d = b->hrd[slot];
    b->ualloc.give(d.P, b->n[slot] + 3);
    b->talloc.give(d.S / PB, d.T);
    b->held[slot] = 0;
    const int zero = 0;
    std::vector<int> hrep(b->n[slot] + 3, -1);
    BCK(b, cudaMemcpyAsync(b->left + slot, &zero, sizeof(int), cudaMemcpyHostToDevice, b->stream));
    BCK(b, cudaMemcpyAsync(b->rep_of + d.P, hrep.data(), sizeof(int) * hrep.size(), cudaMemcpyHostToDevice,
                           b->stream));
    b->n[slot] = 0;
    return relayout(b, b->seg, {});       // synchronises the stream before hrep dies
}

int yk_batch_steps_left(yk_batch* b, int* left)
{
    if (!b || !left) return bfail(b, YK_ERR_ARG, "batch and left are required");
    BCK(b, cudaSetDevice(b->dev));
    std::vector<int> h(b->nslots);
    BCK(b, cudaMemcpyAsync(h.data(), b->left, sizeof(int) * b->nslots, cudaMemcpyDeviceToHost, b->stream));
    BCK(b, cudaStreamSynchronize(b->stream));
    for (int r = 0; r < b->nslots; ++r) left[r] = b->held[r] ? h[r] : -1;
    return YK_OK;
}

int yk_batch_accel(yk_batch* b, int do_meas, yk_scalars* out)
{
    if (!b) return bfail(nullptr, YK_ERR_ARG, "batch is NULL");
    BCK(b, cudaSetDevice(b->dev));
    const bool meas = do_meas != 0;
    int k = 0;
    if (b->pos_dirty) {
        k += enqueue_sort(b, false);
        b->since_sort = 0;
    }
    k += enqueue_force_b(b, meas);
    k_b_finish<<<b->nslots, 256, 0, b->stream>>>(b->rd, nullptr, b->left, b->Sm, b->kpart, b->a, b->ds, nullptr,
                                                 b->series_idx, b->nslots, meas ? 1 : 0, 0, 0);
    ++k;
    count_launches(k);
    std::vector<DevScalars> h(b->nslots);
    BCK(b, cudaMemcpyAsync(h.data(), b->ds, sizeof(DevScalars) * b->nslots, cudaMemcpyDeviceToHost, b->stream));
    int rc = sync_check_b(b);
    if (rc) return rc;
    if (out)
        for (int r = 0; r < b->nslots; ++r) fill_out(b, h[r], r, out[r]);
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
        BCK(b, cudaMallocAsync((void**)&b->series, sizeof(double) * 13 * (size_t)nsteps * b->nslots, b->stream));
        b->series_cap = nsteps;
    }
    // budgets before the run: a box's clock advances only by the steps it takes
    std::vector<int> before(b->nslots);
    BCK(b, cudaMemcpyAsync(before.data(), b->left, sizeof(int) * b->nslots, cudaMemcpyDeviceToHost, b->stream));
    cudaStream_t st = b->stream;
    if (want) BCK(b, cudaMemsetAsync(b->series, 0, sizeof(double) * 13 * (size_t)nsteps * b->nslots, st));
    BCK(b, cudaMemsetAsync(b->series_idx, 0, sizeof(int), st));
    BCK(b, cudaEventRecord(b->e0, st));
    const int me = meas_every;
    const int K = b->graph_steps;
    int k = 0, s = 1;
    if (b->pos_dirty) {
        k += enqueue_sort(b, false);
        b->since_sort = 0;
    }
    while (s + K - 1 <= nsteps) {
        int rc = YK_OK;
        GraphB* g = graph_b(b, K, me, me > 0 ? (s - 1) % me : 0, want, &rc);
        if (!g) return rc;
        BCK(b, cudaGraphLaunch(g->exec, st));
        k += g->kernels;
        s += K;
        // the graph's last re-ordering was at its step 1 + se floor((K - 1) / se)
        b->since_sort = (K - 1) % b->sort_every + 1;
    }
    for (; s <= nsteps; ++s) {
        const bool resort = b->since_sort >= b->sort_every;
        k += enqueue_step_b(b, me > 0 && s % me == 0, want, resort);
        b->since_sort = resort ? 1 : b->since_sort + 1;
    }
    BCK(b, cudaEventRecord(b->e1, st));
    count_launches(k);
    int rc = sync_check_b(b);
    if (rc) return rc;
    if (ms) {
        float f = 0.f;
        cudaEventElapsedTime(&f, b->e0, b->e1);
        *ms = f;
    }
    std::vector<double> h;
    if (want) {
        h.resize(13 * (size_t)nsteps * b->nslots);
        BCK(b, cudaMemcpy(h.data(), b->series, sizeof(double) * h.size(), cudaMemcpyDeviceToHost));
    }
    for (int r = 0; r < b->nslots; ++r) {
        const int took = b->held[r] ? std::min(nsteps, before[r]) : 0;
        for (int q = 0; q < nsteps; ++q) {
            if (q < took) b->time[r] = b->time[r] + b->dt[r];
            if (!want) continue;
            yk_scalars& y = series[(size_t)q * b->nslots + r];
            const double* o = &h[13 * ((size_t)q * b->nslots + r)];
            y.ev = o[0];
            y.vir = o[1];
            y.px = o[2];
            y.ek = o[3];
            for (int c = 0; c < 9; ++c) y.pp[c] = o[4 + c];
            y.time = q < took ? b->time[r] : 0.0;
        }
    }
    return YK_OK;
}

int yk_batch_get_state(yk_batch* b, int rep, double* x, double* v, double* vold, double* a)
{
    if (!b) return bfail(nullptr, YK_ERR_ARG, "batch is NULL");
    if (rep < 0 || rep >= b->nslots || !b->held[rep]) return bfail(b, YK_ERR_ARG, "box %d out of range", rep);
    BCK(b, cudaSetDevice(b->dev));
    const RepDesc& d = b->hrd[rep];
    const size_t off = 3 * (size_t)d.P, bytes = sizeof(double) * 3 * (size_t)b->n[rep];
    cudaStream_t st = b->stream;
    if (x) BCK(b, cudaMemcpyAsync(x, b->x + off, bytes, cudaMemcpyDeviceToHost, st));
    if (v) BCK(b, cudaMemcpyAsync(v, b->v + off, bytes, cudaMemcpyDeviceToHost, st));
    if (vold) BCK(b, cudaMemcpyAsync(vold, b->vold + off, bytes, cudaMemcpyDeviceToHost, st));
    if (a) BCK(b, cudaMemcpyAsync(a, b->a + d.A, sizeof(double) * 3 * (size_t)(b->n[rep] + 3),
                                  cudaMemcpyDeviceToHost, st));
    BCK(b, cudaStreamSynchronize(st));
    return YK_OK;
}

int yk_batch_set_state(yk_batch* b, int rep, const double* x, const double* v, const double* vold,
                       const double* a)
{
    if (!b) return bfail(nullptr, YK_ERR_ARG, "batch is NULL");
    if (rep < 0 || rep >= b->nslots || !b->held[rep]) return bfail(b, YK_ERR_ARG, "box %d out of range", rep);
    const size_t cnt = 3 * (size_t)b->n[rep];
    for (size_t e = 0; e < cnt; ++e)
        if ((x && !std::isfinite(x[e])) || (v && !std::isfinite(v[e])) || (vold && !std::isfinite(vold[e])))
            return bfail(b, YK_ERR_NONFINITE, "box %d: NaN or Inf in a state array", rep);
    BCK(b, cudaSetDevice(b->dev));
    const RepDesc& d = b->hrd[rep];
    const size_t off = 3 * (size_t)d.P, bytes = sizeof(double) * cnt;
    cudaStream_t st = b->stream;
    if (x) BCK(b, cudaMemcpyAsync(b->x + off, x, bytes, cudaMemcpyHostToDevice, st));
    if (v) BCK(b, cudaMemcpyAsync(b->v + off, v, bytes, cudaMemcpyHostToDevice, st));
    if (vold) BCK(b, cudaMemcpyAsync(b->vold + off, vold, bytes, cudaMemcpyHostToDevice, st));
    if (a) BCK(b, cudaMemcpyAsync(b->a + d.A, a, sizeof(double) * 3 * (size_t)(b->n[rep] + 3),
                                  cudaMemcpyHostToDevice, st));
    if (x) b->pos_dirty = true;
    BCK(b, cudaStreamSynchronize(st));
    return YK_OK;
}

}  // extern "C"
