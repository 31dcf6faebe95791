/*
 * yk_oracle.h -- CPU restatement of the MD 6.2.0 hot path (TEST
 * INFRASTRUCTURE ONLY).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py (its CPU-baseline leg and
 * its reference arm) may load this code, and only as the checker or as the
 * timed CPU baseline.  The engine never links or calls it.
 *
 * Parity status: the reference ships no tests, golden vectors or fixtures,
 * and its Fortran cannot be compiled here (no Fortran compiler on either
 * machine), so this restatement is NOT pinned by reference outputs ("parity
 * unpinned").  It is pinned instead by independent known-answer cases computed
 * at 50 significant digits from the same formulas (tests/golden/make_kat.py).
 *
 * Structs come from the public header so that the oracle and the engine take
 * byte-identical parameters.
 */
#ifndef YK_ORACLE_H
#define YK_ORACLE_H

#include "../include/yukawa_engine.h"

#ifdef __cplusplus
extern "C" {
#endif

/* accel(do_measurements): int_control.f:52-81 dispatching to
 * accel_nn (int_nn.f:130-345), accel_ion_pure (int_ion_pure.f:98-254),
 * accel_ion_mix (int_ion_mix.f:105-295) or the B-field case (a = 0).
 * a: double[3*(n+3)].  s: receives ev, vir, px, pp (upper triangle as the
 * reference sets it, mirrored to the lower triangle). */
int orc_accel(const yk_params* p, int n, const double* x,
              const double* zii, const double* aii,
              int do_meas, double* a, yk_scalars* s);

/* newton(do_measurements) of vel_verlet_2.f:18-120 (integrator 2), or the
 * argument-less newton of vel_verlet_1.f:16-89 / vel_verlet_3.f:20-100
 * (integrators 1 and 3; those always compute ek and pp).  x, v, vold, a are
 * updated in place; a is double[3*(n+3)].  *time += dt.  s->pp carries the
 * pressure tensor in and out like the md_globals variable pp. */
int orc_newton(const yk_params* p, int n, double* x, double* v, double* vold,
               double* a, const double* zii, const double* aii,
               int do_meas, yk_scalars* s);

/* gen_utils.f:40-110 and strain.f:19-82. */
double orc_ttot(const yk_params* p, int n, const double* v, const double* aii);
void   orc_tnorm(const yk_params* p, int n, double* v, const double* aii);
void   orc_cancel_vcom(const yk_params* p, int n, double* v, const double* aii);
/* deps: strain rates (1000 = none, md_globals.f:22); xl0: gage dimensions;
 * xl: current dimensions, updated in place; x re-wrapped. */
void   orc_strain(const yk_params* p, int n, double* x, double* xl,
                  const double* xl0, const double* deps);

/* Derived parameters of input1.F. */
double orc_rncut(double aa, double bb, double cc, double xpacket); /* :296-311 */
double orc_thomas_fermi_xmuc(double ztot, double rho, int n);    /* :266-278 */

/* g(r) pair-distance histogram of g.f:55-66, added to counts[0..nbin-1]. */
int orc_gofr_counts(const yk_params* p, int n, const double* x, int nbin, double* counts);

/* Energy-only routines (dead code in the reference; int_ion_pure.f:28-87,
 * int_ion_mix.f:30-94, int_nn.f:37-119).  Returns evavg and pressure. */
int orc_vtot(const yk_params* p, int n, const double* x, const double* zii,
             double* evavg, double* pressure);

/* Restrict the accel loops to target rows i0 <= i < i1 (timing samples
 * only; results are then partial).  orc_set_row_range(0, 0x7fffffff)
 * restores the full loop. */
void orc_set_row_range(int i0, int i1);

/* OpenMP threads used by the loops above (1 = the serial build's order). */
void orc_set_threads(int nthreads);
int  orc_max_threads(void);
/* 1 when built with long double accumulators (the "exact" variant). */
int  orc_long_double_accum(void);

#ifdef __cplusplus
}
#endif
#endif
