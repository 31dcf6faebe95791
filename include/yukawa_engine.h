/*
 * yukawa_engine.h -- C-ABI of the B200 force-and-integrate engine.
 *
 * The engine replaces the hot path of the MD 6.2.0 Fortran code (Berry and
 * Horowitz, Indiana University): the O(N^2) minimum-image pair sums of
 * int_ion_pure.f / int_ion_mix.f / int_nn.f and the velocity-Verlet updates of
 * vel_verlet_1/2/3.f.  The Fortran driver talks to those routines through two
 * argument-less entry points that read and write module globals
 * (md_globals.f:153-172):
 *
 *     subroutine accel(do_measurements)     int_control.f:52-81
 *     subroutine newton(do_measurements)    vel_verlet_2.f:18-120
 *
 * This header is the plain C surface that a thin ISO_C_BINDING shim binds in
 * their place.  Every entry point takes plain host pointers and sizes, returns
 * an int status (YK_OK = 0) and never aborts; the shim maps a non-zero status
 * to md_exit(1, yk_last_error(ctx)), which is how the Fortran code reports
 * every fatal error (md_utils.f:158-183).
 *
 * Array layouts are the Fortran ones, so the shim passes c_loc() of the module
 * arrays unchanged:
 *     x, v, vold   real(8) (3, 0:n-1)  -> double[3*n]      x0,y0,z0,x1,...
 *     a            real(8) (3, 0:n+2)  -> double[3*(n+3)]  columns n..n+2 hold
 *                                         the packed raw sums that the
 *                                         reference passes through its single
 *                                         MPI_allreduce (int_ion_pure.f:217-226)
 *     zii, aii     real(8) (0:n-1)     -> double[n]
 *     pp           real(8) (3,3)       -> double[9] column-major
 *
 * All device state (positions, velocities, old velocities, accelerations,
 * charges, masses) stays resident in HBM between calls.  Host arrays are read
 * only by yk_create / yk_set_state and written only by yk_get_state and by the
 * a_out argument of yk_accel.
 */
#ifndef YUKAWA_ENGINE_H
#define YUKAWA_ENGINE_H

#include <stddef.h>

#if defined(__GNUC__)
#define YK_API __attribute__((visibility("default")))
#else
#define YK_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define YK_OK               0
#define YK_ERR_ARG          1   /* bad argument: n < 1, NULL pointer, dt <= 0 ... */
#define YK_ERR_CUDA         2   /* a CUDA runtime call failed                    */
#define YK_ERR_NOMEM        3   /* device allocation refused / admission refused */
#define YK_ERR_STATE        4   /* call out of order (e.g. destroyed context)    */
#define YK_ERR_TIMEOUT      5   /* a bounded device-side wait gave up            */
#define YK_ERR_NONFINITE    6   /* NaN / Inf in an input array                   */
#define YK_ERR_UNSUPPORTED  7   /* option not available in this build            */

/* ---- simulation types: the cases of accel's select (int_control.f:69-87) */
#define YK_SIM_NUCLEON      1   /* 'nucleon'      -> accel_nn        */
#define YK_SIM_PURE_ION     2   /* 'pure-ion'     -> accel_ion_pure  */
#define YK_SIM_ION_MIXTURE  3   /* 'ion-mixture'  -> accel_ion_mix   */
#define YK_SIM_BFIELD       4   /* 'B-field'      -> a = 0           */

/* ---- arithmetic of the pair terms -------------------------------------- */
#define YK_PREC_FP64        0   /* all FP64: the drop-in form                    */
#define YK_PREC_MIXED       1   /* FP64 positions, velocities and Verlet update;
                                   FP32 displacement (exact differences of
                                   grid-rounded coordinates plus a correction;
                                   nucleon pairs within 2^-7 fm of |d| = L/2 on
                                   an axis take the FP64 minimum image, cast)
                                   and FP32 pair terms with compensated
                                   (two-sum) accumulation                       */

/* ---- integrators -------------------------------------------------------- */
#define YK_VV1              1   /* vel_verlet_1.f: two half kicks              */
#define YK_VV2              2   /* vel_verlet_2.f: the linked one (default)    */
#define YK_VV3              3   /* vel_verlet_3.f: Spreiter-Walter B-field     */

/* ---- ion-mixture last-particle charge factor (int_ion_mix.f:158,201) ---- */
#define YK_MIX_COMPAT       0   /* as the reference: a(:,n-1) lacks zii(n-1)   */
#define YK_MIX_FIXED        1   /* physically correct: every a(:,i) has zii(i) */

/*
 * Run parameters: the md_globals module variables that accel / newton read
 * (md_globals.f:36-140).  yk_params_default() fills the reference defaults.
 */
typedef struct yk_params {
    int    sim_type;      /* YK_SIM_*                                         */
    int    precision;     /* YK_PREC_*                                        */
    int    integrator;    /* YK_VV1 / YK_VV2 / YK_VV3                         */
    int    mix_mode;      /* YK_MIX_COMPAT / YK_MIX_FIXED                     */
    int    coulomb_on;    /* coulomb == 'screened-coulomb'  (int_nn.f:167)   */
    int    nuclear_on;    /* nuclear == 'HPP'               (int_nn.f:168)   */
    int    device;        /* CUDA device ordinal                              */
    int    reserved0;
    double xl[3];         /* box edge lengths (fm)                            */
    double rccut;         /* screened-Coulomb cutoff radius (fm), default 1e50 */
    double rncut;         /* nuclear cutoff radius (fm)                       */
    double xmuc;          /* inverse screening length 1/lambda (1/fm)         */
    double vc;            /* Coulomb coupling alpha*hbar*c (MeV fm)           */
    double frp;           /* ion form factor                                  */
    double xmass;         /* nucleon mass (MeV)                               */
    double rho;           /* particle density (1/fm^3)                        */
    double kT;            /* temperature (MeV)                                */
    double dt;            /* time step (fm/c)                                 */
    double bfield;        /* uniform B field along z (Gauss)                  */
    double zi, ai;        /* pure-ion charge and mass numbers                 */
    double aa, bb, cc;    /* HPP nuclear parameters (MeV)                     */
    double xpacket;       /* HPP Lambda (fm^2)                                */
    double time;          /* simulation clock (fm/c)                          */
} yk_params;

/*
 * Scalar outputs of accel / newton: the md_globals variables ev, vir, px, ek,
 * pp(3,3) and time.  pp is column-major like the Fortran array.
 */
typedef struct yk_scalars {
    double ev;            /* potential energy per particle (MeV)   */
    double vir;           /* virial sum                             */
    double px;            /* instantaneous pressure (MeV/fm^3)      */
    double ek;            /* kinetic energy per particle (MeV)      */
    double pp[9];         /* pressure tensor                        */
    double time;          /* simulation clock after the call        */
} yk_scalars;

typedef struct yk_ctx yk_ctx;

/* Fill *p with the reference defaults of md_globals.f:115-140
 * (vc = ALPHA*HBARC, xmass = 931, rccut = 1e50, aa/bb/cc/xpacket = HPP, ...). */
YK_API int yk_params_default(yk_params* p);

/* Create an engine for n particles and copy the initial state to the device.
 * Replaces the allocate/bcast block of input1.F:379-407 for the device side.
 * v may be NULL (zero velocities).  zii / aii may be NULL for pure-ion runs
 * (then every particle has zi / ai).  The arrays are copied, not retained. */
YK_API int yk_create(const yk_params* p, int n,
              const double* x, const double* v,
              const double* zii, const double* aii,
              yk_ctx** out);

YK_API int yk_destroy(yk_ctx* ctx);

/* Message of the last failed call on ctx (static string if ctx is NULL). */
YK_API const char* yk_last_error(const yk_ctx* ctx);

/* Force call: replaces accel(do_measurements), int_control.f:52-81.
 * Computes accelerations from the device-resident positions.  If a_out is not
 * NULL it receives a(3,0:n+2) exactly as the reference leaves it: scaled
 * accelerations in columns 0..n-1 and the raw packed sums (ev, vir, 0, pxx,
 * pxy, pxz, pyy, pyz, pzz) in columns n..n+2.  out may be NULL. */
YK_API int yk_accel(yk_ctx* ctx, int do_meas, double* a_out, yk_scalars* out);

/* One integrator step: replaces newton(do_measurements), vel_verlet_2.f:18
 * (or vel_verlet_1.f:16 / vel_verlet_3.f:20 by params.integrator).  Works on
 * the device-resident state; nothing is copied to or from host arrays. */
YK_API int yk_newton(yk_ctx* ctx, int do_meas, yk_scalars* out);

/* nsteps integrator steps back to back on the device, launched as CUDA graphs.
 * Step s (1-based) measures when meas_every > 0 and s % meas_every == 0.
 * series, if not NULL, receives nsteps yk_scalars (zeros on non-measuring
 * steps, as the reference leaves them).  One host synchronisation at the end. */
YK_API int yk_run(yk_ctx* ctx, int nsteps, int meas_every, yk_scalars* series);

/* Host <-> device state sync points (before save_config / checkpoint /
 * dump_data and around host-side tnorm / cancel_vcom / strain).  Any pointer
 * may be NULL to skip that array.  a is double[3*n] (columns 0..n-1). */
YK_API int yk_get_state(yk_ctx* ctx, double* x, double* v, double* vold, double* a);
YK_API int yk_set_state(yk_ctx* ctx, const double* x, const double* v,
                 const double* vold, const double* a);

/* Potential energy per particle and pressure without touching the state:
 * the energy-only routines vtot_ion_pure / vtot_ion_mix / vtot_nn
 * (int_ion_pure.f:28-87, int_ion_mix.f:30-94, int_nn.f:37-119), which give
 * the same ev and px as a measuring accel.  (The reference never calls them:
 * its vtot dispatch has no caller.)  Runs one measuring force call into a
 * side buffer, so the accelerations of the state stay as they are. */
YK_API int yk_vtot(yk_ctx* ctx, double* ev, double* px);

/* The pair-distance histogram of the two-particle correlation function
 * g(r): subroutine g with ig > 0 (g.f:55-66; its calls are commented out in
 * md.F:64, 154, 184).  For every unique pair of the current positions,
 * rr = pdist(i, j) (gen_utils.f:115-128) goes to bin
 * min(nbin, int(fac2 rr + 1)), fac2 = 2 float(nbin) / sqrt(3) / min(xl), with
 * the reference's arithmetic; the counts are ADDED to counts[0..nbin-1], as g
 * accumulates gg(:, ig).  nbin <= 8192.  The normalization of g with
 * ig = -1 (g.f:97-130) is host arithmetic: yukawamd_b200/gofr.py. */
YK_API int yk_gofr_counts(yk_ctx* ctx, int nbin, double* counts);

/* Asynchronous state snapshot for checkpoint and save_config
 * (md_utils.f:19-114, which write x and v, or x, v and a, through
 * rw_xvb.f:148-203).  yk_snapshot_begin copies the current x, v and a
 * (any pointer may be NULL; a is double[3*n]) into a device buffer on the
 * engine's stream, then into the caller's host buffers on a second stream,
 * and returns without waiting: the following steps run while the copy to
 * the host drains.  The host buffers hold the snapshot once
 * yk_snapshot_wait returns; they should be page-locked (yk_host_register)
 * for the copy to overlap.  A second yk_snapshot_begin first waits for the
 * one in flight.  The first call allocates the 72*n-byte device buffer. */
YK_API int yk_snapshot_begin(yk_ctx* ctx, double* x, double* v, double* a);
YK_API int yk_snapshot_wait(yk_ctx* ctx);

/* The reference driver's per-step host passes, on the device state
 * (gen_utils.f:40-110, strain.f:19-82):
 *   yk_ttot         average kinetic energy per particle -> *eka
 *   yk_tnorm        rescale velocities to eka = 1.5 kT
 *   yk_cancel_vcom  remove the centre-of-mass velocity, then tnorm
 *   yk_strain       volume-preserving normal strain of the box at rates
 *                   deps (1000 = no strain in that direction) relative to
 *                   the gage dimensions xl0, then re-wrap x > xl; the new
 *                   edge lengths go to xl_out (may be NULL). */
YK_API int yk_ttot(yk_ctx* ctx, double* eka);
YK_API int yk_tnorm(yk_ctx* ctx);
YK_API int yk_cancel_vcom(yk_ctx* ctx);
YK_API int yk_strain(yk_ctx* ctx, const double deps[3], const double xl0[3],
                     double xl_out[3]);

/* New box edge lengths (strain.f changes xl every step). */
YK_API int yk_set_box(yk_ctx* ctx, const double xl[3]);

/*
 * Batches of independent boxes.  The reference runs one box per process; the
 * engine can also advance many boxes together (ensembles, served requests):
 * one persistent force kernel pulls (box, target block, source segment)
 * work items of all boxes from one queue, the integrator kernels cover all
 * boxes per launch, and yk_batch_run captures K steps of all boxes in one
 * CUDA graph.  Each box keeps its own parameters, N, state and scalars, and
 * its results do not depend on which other boxes share the batch.
 *
 * A batch holds either ion boxes (pure-ion and ion-mixture; pure-ion boxes
 * run through the mixture kernels with every Z equal to zi) or nucleon
 * boxes, all with one precision, integrator YK_VV2 and no B field.  Per-box
 * arrays are passed as arrays of pointers: x[r] double[3 n[r]], v[r] (or
 * NULL), zii[r] / aii[r] (NULL allowed where yk_create allows it).
 */
typedef struct yk_batch yk_batch;

YK_API int yk_batch_create(int nrep, const yk_params* params, const int* n,
                           const double* const* x, const double* const* v,
                           const double* const* zii, const double* const* aii,
                           int device, yk_batch** out);
YK_API int yk_batch_destroy(yk_batch* b);
YK_API const char* yk_batch_last_error(const yk_batch* b);
/* accel(do_meas) of every box; out: nrep scalars or NULL. */
YK_API int yk_batch_accel(yk_batch* b, int do_meas, yk_scalars* out);
/* nsteps newton steps of every box; step s (1-based) measures when
 * meas_every > 0 and s % meas_every == 0.  series: nsteps*nrep scalars,
 * step-major (series[s*nrep + r]) or NULL.  ms: CUDA-event time of the
 * device work or NULL. */
YK_API int yk_batch_run(yk_batch* b, int nsteps, int meas_every,
                        yk_scalars* series, double* ms);
/* State of box rep: x, v, vold double[3 n[rep]]; a double[3(n[rep]+3)].
 * Any pointer may be NULL. */
YK_API int yk_batch_get_state(yk_batch* b, int rep, double* x, double* v,
                              double* vold, double* a);
YK_API int yk_batch_set_state(yk_batch* b, int rep, const double* x,
                              const double* v, const double* vold,
                              const double* a);

/*
 * Slots, for serving (no counterpart in the reference, which runs one box
 * per process).  yk_batch_create_slots makes an empty batch of nslots slots
 * that holds at most max_particles particles and max_pair_units half-pair
 * units (T (T + 1) / 2 per box of T = ceil(n / 128) tiles) at once; proto
 * gives the kind (ion or nucleon) and precision of every box it will hold.
 * The boxes of yk_batch_create are slots 0 .. nrep-1 of a batch that is full.
 *
 * yk_batch_admit puts one box into a free slot (*slot) with a budget of
 * `steps` newton steps, copies its x, v (NULL: zero), zii, aii in, orders it
 * and makes its initial measuring force call (md.F:69) -- over its own work
 * items only; the other boxes are neither moved nor recomputed.  out (may be
 * NULL) receives its scalars.  YK_ERR_NOMEM when no slot, particle range,
 * tile range or scratch is free (nothing changes then).
 *
 * yk_batch_run advances every held box by up to nsteps steps: a box whose
 * budget runs out stops at exactly its budget (its later series entries are
 * zero), also inside a CUDA graph.  series is nsteps * nslots long.
 *
 * yk_batch_steps_left: the remaining budget of every slot (left[nslots]; -1
 * for an empty slot).  yk_batch_retire copies the box's state out (any
 * pointer may be NULL) and frees its slot.  Call these between runs only.
 */
YK_API int yk_batch_create_slots(const yk_params* proto, int nslots,
                                 long long max_particles,
                                 long long max_pair_units, int device,
                                 yk_batch** out);
YK_API int yk_batch_admit(yk_batch* b, const yk_params* p, int n,
                          const double* x, const double* v,
                          const double* zii, const double* aii,
                          long long steps, int* slot, yk_scalars* out);
YK_API int yk_batch_retire(yk_batch* b, int slot, double* x, double* v,
                           double* vold, double* a);
YK_API int yk_batch_steps_left(yk_batch* b, int* left);

/*
 * Engine tunables (not reference parameters): which force kernel runs and
 * how its work is cut.  yk_create picks defaults; the autotuner
 * (yukawamd_b200/tune.py) measures the alternatives and sets them here.
 */
typedef struct yk_tuning {
    int force_kernel;     /* 0 auto, 1 row kernel (each pair from both sides),
                             2 half-pair kernel (Newton's third law, scratch),
                             3 half-pair kernel over per-warp near-source lists;
                             yk_get_tuning reports the kernel auto resolved to */
    int pair_seg;         /* longest job of the half-pair kernels, in source
                             tiles (jobs shrink towards the end of the job
                             list); 0 = automatic (8 FP64, 4 mixed)         */
    int sort_every;       /* steps between Hilbert re-orderings (-1 = never,
                             0 = automatic: 4)                              */
    int graph_steps;      /* steps per CUDA graph of yk_run: the graphs take
                             the most whole multiples of u that fit (at least
                             one), u = sort_every or, when it is at most
                             4 graph_steps, lcm(sort_every, meas_every)    */
    int source_split;     /* CTAs of the half-pair kernel (2, or auto when it
                             picks 2) that share one 128-target block, each
                             taking a contiguous 1/split of every source tile,
                             so split x more CTAs (threads per target) work on
                             a small box: 1, 2 or 4 (jobs of one tile then);
                             0 = 1; ignored by kernels 1 and 3.  Batches: 0/1 */
    int targets_per_thread; /* targets each thread of the half-pair kernel
                             holds: 1, or 2 (blocks of 256 targets, every
                             source read and reaction reduction shared by two
                             pairs) for ion boxes on the FP64 path with exact
                             screen images or the mixed hi/lo path (other
                             boxes take 1); 0 = automatic.  yk_get_tuning
                             reports the value in use.  Batches: 0/1        */
} yk_tuning;

YK_API int yk_get_tuning(yk_ctx* ctx, yk_tuning* out);
YK_API int yk_set_tuning(yk_ctx* ctx, const yk_tuning* t);

/* The batch's tunables: pair_seg (source tiles per job, all boxes) and
 * graph_steps (steps per CUDA graph of yk_batch_run) and sort_every (steps
 * between the boxes' Hilbert re-orderings, counted from the start of each
 * graph, which always re-sorts; 0 = automatic: 4).  force_kernel must be 0
 * or 2.  Changing pair_seg rebuilds the job table and its scratch. */
YK_API int yk_batch_get_tuning(yk_batch* b, yk_tuning* out);
YK_API int yk_batch_set_tuning(yk_batch* b, const yk_tuning* t);

/*
 * Timers, the counterpart of the reference's perf.f report (perf.f:60-178:
 * 'newton', 'accel' and 'calc_a' wall-clock timers).  With yk_perf_enable(ctx,
 * 1, flush_bytes) the following yk_run calls launch step by step (no graph)
 * with a CUDA event pair around every force kernel and around the whole run,
 * and, if flush_bytes > 0, overwrite a device buffer of that size before every
 * step so that no step starts from a warm L2.  yk_perf_read returns the sums
 * since the last enable.
 */
typedef struct yk_perf {
    double run_ms;            /* event time of the timed steps, each from
                                 the end of its L2 flush to its end       */
    double force_ms;          /* event time of the force kernels          */
    long long steps;          /* integrator steps timed                   */
    long long force_calls;    /* force kernels timed                      */
} yk_perf;

YK_API int yk_perf_enable(yk_ctx* ctx, int enable, size_t flush_bytes);
YK_API int yk_perf_read(yk_ctx* ctx, yk_perf* out);

/* Measured peak of a pipe on device `device`: kind 0 = FP64 FMA, kind 1 =
 * FP32 FMA, in TFLOP/s (2 flops per FMA), from a register-resident FMA chain
 * over the whole GPU.  Used for roofline denominators. */
YK_API int yk_peak_probe(int device, int kind, double* tflops);

/* The half-pair kernel's job table for m tiles of 128 slots, as yk_create
 * builds it: jobs of at most cap source tiles, in dispatch order, sized by
 * guided self-scheduling for ctas resident CTAs.  A job is four ints
 * (R, C0, C1, slot): target block R, source tiles C0 <= C < C1 (C0 >= R),
 * and the slot of row R's target-side partial that it writes.  Writes at
 * most max_jobs jobs to jobs (NULL: only count) and the m slot counts to
 * row_slots (NULL allowed); returns the number of jobs, or -YK_ERR_ARG.
 * Host arithmetic only (no GPU), for inspecting and testing the schedule.
 * No counterpart in the reference. */
YK_API long long yk_pair_jobs(int m, int cap, int ctas, int* jobs, long long max_jobs, int* row_slots);

/* The job table of the half-pair kernel with two targets per thread
 * (yk_tuning.targets_per_thread = 2), same arguments: a job (R, C0, C1, slot)
 * has R even and takes blocks R and R + 1 against source tiles C0 <= C < C1
 * (C0 >= R), writing that slot of both rows' target-side partials; row_slots
 * of both rows count the pair's jobs.  Host arithmetic only.  No counterpart
 * in the reference. */
YK_API long long yk_pair_jobs2(int m, int cap, int ctas, int* jobs, long long max_jobs, int* row_slots);

/*
 * Force call that allocates no device memory.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory when
 * they need forces -- applications whose own pool allocator owns all device
 * memory, and callers that cannot afford the device-wide synchronisation of
 * cudaFree / cudaMalloc on their other streams.  It computes what yk_accel
 * computes, for
 * one box given entirely by caller-owned DEVICE arrays: x_dev double[3n],
 * zii_dev / aii_dev double[n] (NULL allowed where yk_create allows NULL),
 * a_dev double[3(n+3)] (output, same layout as yk_accel's a_out).  out (host)
 * may be NULL; stream may be NULL (legacy default stream).  The call waits
 * for its stream before returning.
 *
 * Limits: n <= 4096.  Working memory is one fixed 4 MiB array in the
 * library's device code, held by every GPU that loads the library until the
 * process exits.  The first call on a device looks up that array's address;
 * make that first call before starting any stream capture.  Every call reuses
 * the same array, so calls that overlap on the GPU race: serialise them.
 */
YK_API int yk_accel_noalloc(const yk_params* p, int n,
                            const double* x_dev, const double* zii_dev,
                            const double* aii_dev, int do_meas,
                            double* a_dev, yk_scalars* out, void* stream);

/* Failure-path check of the device-side waits.  The reference has no device
 * and no error codes (a fatal error calls md_exit, md_utils.f:158-183); the
 * engine's kernels instead bound every wait on a tile copy and report
 * YK_ERR_TIMEOUT.  This launches one CTA on ctx's stream that waits, with
 * both of the kernels' wait forms limited to `spins` polls (1 .. 2^22), on a
 * barrier that no copy ever completes, so every wait gives up.  Returns
 * YK_ERR_TIMEOUT through the same error word and check as yk_accel, clears
 * it, and leaves the context usable; *gave_up (may be NULL) receives the
 * number of threads that gave up (128).  Any other return is a failure of
 * the check itself. */
YK_API int yk_wait_selftest(yk_ctx* ctx, long long spins, int* gave_up);

/* Page-lock a caller-owned host buffer so that yk_get_state / yk_set_state
 * copy it by DMA.  Optional. */
YK_API int yk_host_register(void* ptr, size_t bytes);
YK_API int yk_host_unregister(void* ptr);

/* Number of kernels this library has launched in this process (all contexts).
 * Used by benchmarks to report how much device work a measured region did. */
YK_API unsigned long long yk_kernel_launch_count(void);

/* Library version string. */
YK_API const char* yk_version(void);

#ifdef __cplusplus
}
#endif

#endif /* YUKAWA_ENGINE_H */
