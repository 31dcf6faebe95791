/*
 * yk_oracle.c -- CPU restatement of the MD 6.2.0 hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA engine and the timed CPU
 * baseline.  Nothing in the engine links or calls this file.
 *
 * Parity unpinned by reference outputs (the reference has no tests and no
 * Fortran compiler exists here); pinned by the 50-digit known-answer cases
 * of tests/golden/make_kat.py.
 *
 * Each routine follows its Fortran source statement by statement: the same
 * i < j loop, the same minimum-image branches, the same left-to-right
 * evaluation order of every expression, the same OpenMP reduction structure
 * (one "omp for" over j per target particle i, followed by an "omp single"
 * fold), and the Fortran single-precision promotions float(n) and 3.0*n.  It
 * must be compiled with -ffp-contract=off (the reference is built by gfortran
 * for baseline x86-64, which has no FMA) and without -ffast-math.
 *
 * Build: oracle/Makefile -> oracle/liborc.so (double accumulators, the
 * reference's arithmetic) and oracle/liborc_ld.so (-DORC_LONG_DOUBLE: the
 * same loops with long double accumulators, used to measure how far any
 * summation order is from the exact sum).
 */
#include "yk_oracle.h"

#include <math.h>
#include <string.h>
#include <stdlib.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORC_LONG_DOUBLE
typedef long double acc_t;
#else
typedef double acc_t;
#endif

/* Fortran default-REAL promotions: float(n) and 3.0*n are REAL*4. */
static double f_float(int n) { return (double)(float)n; }
static double f_3n(int n) { return (double)(3.0f * (float)n); }

/* Target-row window of the accel loops (i runs from row_lo to row_hi).  The
 * default is the reference's full range 0..n-2; bench.py narrows it to time a
 * bounded sample of one force call on the full-size box. */
static int g_row0 = 0, g_row1 = 0x7fffffff;
static int row_lo(void) { return g_row0 > 0 ? g_row0 : 0; }
static int row_hi(int n) { return (g_row1 - 1 < n - 2) ? g_row1 - 1 : n - 2; }

void orc_set_row_range(int i0, int i1)
{
    g_row0 = i0;
    g_row1 = i1;
}

/* md_globals.f:24-28 */
static const double HBARC = 197.327;
static const double ALPHA = 1.0 / 137.036;
static const double ME = 0.510999;
static const double PI = 3.14159265358979324;

void orc_set_threads(int nthreads)
{
#ifdef _OPENMP
    omp_set_num_threads(nthreads > 0 ? nthreads : 1);
#else
    (void)nthreads;
#endif
}

int orc_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

int orc_long_double_accum(void)
{
#ifdef ORC_LONG_DOUBLE
    return 1;
#else
    return 0;
#endif
}

/* evcut: int_ion_pure.f:125-130 / int_ion_mix.f:140-145 (scale 1) and
 * int_nn.f:177-182 (scale vc). */
static double ev_cut(const yk_params* p, double scale)
{
    const double* xl = p->xl;
    if (p->rccut <= sqrt(xl[0] * xl[0] + xl[1] * xl[1] + xl[2] * xl[2]) / 2.0)
        return scale * exp(-(p->xmuc * p->rccut)) / p->rccut;
    return 0.0;
}

/* Minimum-image displacement x(:,i)-x(:,j), int_ion_pure.f:146-152. */
static inline double min_image(const double* x, int i, int j,
                               const double* xl, const double* halfl,
                               double* xx)
{
    double r2 = 0.0;
    for (int k = 0; k < 3; ++k) {
        xx[k] = x[3 * i + k] - x[3 * j + k];
        if (xx[k] > +halfl[k]) xx[k] = xx[k] - xl[k];
        if (xx[k] < -halfl[k]) xx[k] = xx[k] + xl[k];
        r2 = r2 + xx[k] * xx[k];
    }
    return r2;
}

static void pack_scalars(acc_t* fj, int n, acc_t evx, acc_t virx,
                         acc_t pxx, acc_t pxy, acc_t pxz,
                         acc_t pyy, acc_t pyz, acc_t pzz)
{
    fj[3 * n + 0] = evx;
    fj[3 * n + 1] = virx;
    fj[3 * n + 2] = 0.0;
    fj[3 * (n + 1) + 0] = pxx;
    fj[3 * (n + 1) + 1] = pxy;
    fj[3 * (n + 1) + 2] = pxz;
    fj[3 * (n + 2) + 0] = pyy;
    fj[3 * (n + 2) + 1] = pyz;
    fj[3 * (n + 2) + 2] = pzz;
}

/* Unpack a(:,n..n+2) scaled by c into ev, vir, pp (int_ion_pure.f:232-248). */
static void unpack_scalars(const double* a, int n, double c, int do_meas,
                           const yk_params* p, yk_scalars* s)
{
    if (do_meas) {
        s->ev = c * a[3 * n + 0];
        s->vir = c * a[3 * n + 1];
        s->pp[0] = c * a[3 * (n + 1) + 0];          /* pp(1,1) */
        s->pp[3] = c * a[3 * (n + 1) + 1];          /* pp(1,2) */
        s->pp[6] = c * a[3 * (n + 1) + 2];          /* pp(1,3) */
        s->pp[4] = c * a[3 * (n + 2) + 0];          /* pp(2,2) */
        s->pp[7] = c * a[3 * (n + 2) + 1];          /* pp(2,3) */
        s->pp[8] = c * a[3 * (n + 2) + 2];          /* pp(3,3) */
        s->pp[1] = s->pp[3];
        s->pp[2] = s->pp[6];
        s->pp[5] = s->pp[7];
        s->ev = s->ev / f_float(n);
        s->px = p->rho * (p->kT + s->vir / f_3n(n));
    } else {
        s->ev = 0.0;
        s->vir = 0.0;
        s->px = 0.0;
        for (int k = 0; k < 9; ++k) s->pp[k] = 0.0;
    }
}

/* accel_ion_pure, int_ion_pure.f:98-254. */
static void accel_ion_pure(const yk_params* p, int n, const double* x,
                           int do_meas, double* a, yk_scalars* s)
{
    acc_t* fj = (acc_t*)calloc((size_t)3 * (n + 3), sizeof(acc_t));
    double halfl[3], xl[3];
    for (int k = 0; k < 3; ++k) { xl[k] = p->xl[k]; halfl[k] = 0.5 * xl[k]; }
    const double rccut2 = p->rccut * p->rccut;
    const double evcut = ev_cut(p, 1.0);
    const double xmuc = p->xmuc;
    acc_t evx = 0.0, virx = 0.0;
    acc_t fi[3] = {0.0, 0.0, 0.0};
    acc_t pxx = 0.0, pxy = 0.0, pxz = 0.0, pyy = 0.0, pyz = 0.0, pzz = 0.0;

    if (do_meas) {
        #pragma omp parallel
        for (int i = row_lo(); i <= row_hi(n); ++i) {
            #pragma omp for reduction(+:evx,virx,fi[:3],pxx,pxy,pxz,pyy,pyz,pzz)
            for (int j = i + 1; j <= n - 1; ++j) {
                double xx[3];
                double r2 = min_image(x, i, j, xl, halfl, xx);
                if (r2 <= rccut2) {
                    double r = sqrt(r2);
                    double fc = exp(-(xmuc * r)) / (r * r2);
                    evx = evx + (fc * r2 - evcut);
                    fc = (1. + xmuc * r) * fc;
                    virx = virx + fc * r2;
                    double fcx[3];
                    for (int k = 0; k < 3; ++k) fcx[k] = fc * xx[k];
                    for (int k = 0; k < 3; ++k) fi[k] = fi[k] + fcx[k];
                    for (int k = 0; k < 3; ++k) fj[3 * j + k] = fj[3 * j + k] - fcx[k];
                    pxx = pxx + xx[0] * fcx[0];
                    pxy = pxy + xx[0] * fcx[1];
                    pxz = pxz + xx[0] * fcx[2];
                    pyy = pyy + xx[1] * fcx[1];
                    pyz = pyz + xx[1] * fcx[2];
                    pzz = pzz + xx[2] * fcx[2];
                }
            }
            #pragma omp single
            {
                for (int k = 0; k < 3; ++k) { fj[3 * i + k] = fj[3 * i + k] + fi[k]; fi[k] = 0.0; }
            }
        }
    } else {
        #pragma omp parallel
        for (int i = row_lo(); i <= row_hi(n); ++i) {
            #pragma omp for reduction(+:fi[:3])
            for (int j = i + 1; j <= n - 1; ++j) {
                double xx[3];
                double r2 = min_image(x, i, j, xl, halfl, xx);
                if (r2 <= rccut2) {
                    double r = sqrt(r2);
                    double fc = (1. + xmuc * r) * exp(-(xmuc * r)) / (r * r2);
                    double fcx[3];
                    for (int k = 0; k < 3; ++k) fcx[k] = fc * xx[k];
                    for (int k = 0; k < 3; ++k) fi[k] = fi[k] + fcx[k];
                    for (int k = 0; k < 3; ++k) fj[3 * j + k] = fj[3 * j + k] - fcx[k];
                }
            }
            #pragma omp single
            {
                for (int k = 0; k < 3; ++k) { fj[3 * i + k] = fj[3 * i + k] + fi[k]; fi[k] = 0.0; }
            }
        }
    }
    pack_scalars(fj, n, evx, virx, pxx, pxy, pxz, pyy, pyz, pzz);
    /* MPI_allreduce over one rank is a copy (md_comm_ser.f:83-121). */
    for (int k = 0; k < 3 * (n + 3); ++k) a[k] = (double)fj[k];
    const double c = p->frp * p->zi * p->zi * p->vc;   /* ((frp*zi)*zi)*vc */
    #pragma omp parallel for
    for (int i = 0; i <= n - 1; ++i)
        for (int k = 0; k < 3; ++k)
            a[3 * i + k] = c * a[3 * i + k] / (p->ai * p->xmass);
    unpack_scalars(a, n, c, do_meas, p, s);
    free(fj);
}

/* accel_ion_mix, int_ion_mix.f:105-295, including the last-particle charge
 * factor that the i loop (:158, :222) never applies to particle n-1 when
 * mix_mode == YK_MIX_COMPAT. */
static void accel_ion_mix(const yk_params* p, int n, const double* x,
                          const double* zii, const double* aii,
                          int do_meas, double* a, yk_scalars* s)
{
    acc_t* fj = (acc_t*)calloc((size_t)3 * (n + 3), sizeof(acc_t));
    double halfl[3], xl[3];
    for (int k = 0; k < 3; ++k) { xl[k] = p->xl[k]; halfl[k] = 0.5 * xl[k]; }
    const double rccut2 = p->rccut * p->rccut;
    const double evcut = ev_cut(p, 1.0);
    const double xmuc = p->xmuc;
    acc_t ev = 0.0, vir = 0.0;
    acc_t ppa[6] = {0, 0, 0, 0, 0, 0};   /* pp(1,1) pp(1,2) pp(1,3) pp(2,2) pp(2,3) pp(3,3) */
    acc_t evx = 0.0, virx = 0.0;
    acc_t fi[3] = {0.0, 0.0, 0.0};
    acc_t pxx = 0.0, pxy = 0.0, pxz = 0.0, pyy = 0.0, pyz = 0.0, pzz = 0.0;

    if (do_meas) {
        #pragma omp parallel
        for (int i = row_lo(); i <= row_hi(n); ++i) {
            #pragma omp for reduction(+:evx,virx,fi[:3],pxx,pxy,pxz,pyy,pyz,pzz) schedule(runtime)
            for (int j = i + 1; j <= n - 1; ++j) {
                double xx[3];
                double r2 = min_image(x, i, j, xl, halfl, xx);
                if (r2 <= rccut2) {
                    double r = sqrt(r2);
                    double fc = exp(-(xmuc * r)) / (r * r2);
                    evx = evx + zii[j] * (fc * r2 - evcut);
                    fc = (1. + xmuc * r) * fc;
                    virx = virx + zii[j] * fc * r2;
                    double fx = fc * xx[0];
                    fi[0] = fi[0] + zii[j] * fx;
                    fj[3 * j + 0] = fj[3 * j + 0] - zii[i] * fx;
                    pxx = pxx + xx[0] * (zii[j] * fx);
                    double fy = fc * xx[1];
                    fi[1] = fi[1] + zii[j] * fy;
                    fj[3 * j + 1] = fj[3 * j + 1] - zii[i] * fy;
                    pxy = pxy + xx[0] * (zii[j] * fy);
                    pyy = pyy + xx[1] * (zii[j] * fy);
                    double fz = fc * xx[2];
                    fi[2] = fi[2] + zii[j] * fz;
                    fj[3 * j + 2] = fj[3 * j + 2] - zii[i] * fz;
                    pxz = pxz + xx[0] * (zii[j] * fz);
                    pyz = pyz + xx[1] * (zii[j] * fz);
                    pzz = pzz + xx[2] * (zii[j] * fz);
                }
            }
            #pragma omp single
            {
                ev = ev + zii[i] * evx;
                vir = vir + zii[i] * virx;
                for (int k = 0; k < 3; ++k) fj[3 * i + k] = zii[i] * (fj[3 * i + k] + fi[k]);
                ppa[0] = ppa[0] + zii[i] * pxx;
                ppa[1] = ppa[1] + zii[i] * pxy;
                ppa[2] = ppa[2] + zii[i] * pxz;
                ppa[3] = ppa[3] + zii[i] * pyy;
                ppa[4] = ppa[4] + zii[i] * pyz;
                ppa[5] = ppa[5] + zii[i] * pzz;
                evx = 0.0; virx = 0.0;
                fi[0] = fi[1] = fi[2] = 0.0;
                pxx = pxy = pxz = pyy = pyz = pzz = 0.0;
            }
        }
    } else {
        #pragma omp parallel
        for (int i = row_lo(); i <= row_hi(n); ++i) {
            #pragma omp for reduction(+:fi[:3]) schedule(runtime)
            for (int j = i + 1; j <= n - 1; ++j) {
                double xx[3];
                double r2 = min_image(x, i, j, xl, halfl, xx);
                if (r2 <= rccut2) {
                    double r = sqrt(r2);
                    double fc = (1. + xmuc * r) * exp(-(xmuc * r)) / (r * r2);
                    double fx = fc * xx[0];
                    fi[0] = fi[0] + zii[j] * fx;
                    fj[3 * j + 0] = fj[3 * j + 0] - zii[i] * fx;
                    double fy = fc * xx[1];
                    fi[1] = fi[1] + zii[j] * fy;
                    fj[3 * j + 1] = fj[3 * j + 1] - zii[i] * fy;
                    double fz = fc * xx[2];
                    fi[2] = fi[2] + zii[j] * fz;
                    fj[3 * j + 2] = fj[3 * j + 2] - zii[i] * fz;
                }
            }
            #pragma omp single
            {
                for (int k = 0; k < 3; ++k) fj[3 * i + k] = zii[i] * (fj[3 * i + k] + fi[k]);
                fi[0] = fi[1] = fi[2] = 0.0;
            }
        }
    }
    if (p->mix_mode == YK_MIX_FIXED && n >= 1)
        for (int k = 0; k < 3; ++k) fj[3 * (n - 1) + k] = zii[n - 1] * fj[3 * (n - 1) + k];

    pack_scalars(fj, n, ev, vir, ppa[0], ppa[1], ppa[2], ppa[3], ppa[4], ppa[5]);
    for (int k = 0; k < 3 * (n + 3); ++k) a[k] = (double)fj[k];
    const double c = p->frp * p->vc;
    #pragma omp parallel for schedule(runtime)
    for (int i = 0; i <= n - 1; ++i)
        for (int k = 0; k < 3; ++k)
            a[3 * i + k] = c * a[3 * i + k] / (aii[i] * p->xmass);
    unpack_scalars(a, n, c, do_meas, p, s);
    free(fj);
}

/* accel_nn, int_nn.f:130-345. */
static void accel_nn(const yk_params* p, int n, const double* x,
                     const double* zii, int do_meas, double* a, yk_scalars* s)
{
    acc_t* fj = (acc_t*)calloc((size_t)3 * (n + 3), sizeof(acc_t));
    const int coulomb_on = p->coulomb_on, nuclear_on = p->nuclear_on;
    double halfl[3], xl[3];
    for (int k = 0; k < 3; ++k) { xl[k] = p->xl[k]; halfl[k] = 0.5 * xl[k]; }
    const double xpacketi = 1. / p->xpacket;
    const double xpacket2i = 1. / (2. * p->xpacket);
    const double rncut2 = p->rncut * p->rncut;
    const double rccut2 = p->rccut * p->rccut;
    const double evcut = ev_cut(p, p->vc);
    const double xmuc = p->xmuc, vc = p->vc;
    const double aa = p->aa, bb = p->bb, cc = p->cc;
    acc_t evx = 0.0, virx = 0.0;
    acc_t fi[3] = {0.0, 0.0, 0.0};
    acc_t pxx = 0.0, pxy = 0.0, pxz = 0.0, pyy = 0.0, pyz = 0.0, pzz = 0.0;

    if (do_meas) {
        #pragma omp parallel
        for (int i = row_lo(); i <= row_hi(n); ++i) {
            #pragma omp for reduction(+:evx,virx,fi[:3],pxx,pxy,pxz,pyy,pyz,pzz)
            for (int j = i + 1; j <= n - 1; ++j) {
                double fn = 0.0, fc = 0.0;
                int fzero = 1;
                double xx[3];
                double r2 = min_image(x, i, j, xl, halfl, xx);
                if (nuclear_on && r2 <= rncut2) {
                    double expfac = exp(-(r2 * xpacket2i));
                    double xbbcc = (zii[i] == zii[j]) ? bb + cc : bb - cc;
                    evx = evx + (aa * expfac + xbbcc) * expfac;
                    fn = xpacketi * (2. * aa * expfac + xbbcc) * expfac;
                    virx = virx + fn * r2;
                    fzero = 0;
                }
                if (coulomb_on && r2 <= rccut2) {
                    if (zii[i] == 1.0 && zii[j] == 1.0) {
                        double r = sqrt(r2);
                        fc = vc * exp(-(xmuc * r)) / (r * r2);
                        evx = evx + (fc * r2 - evcut);
                        fc = (1. + xmuc * r) * fc;
                        virx = virx + fc * r2;
                        fzero = 0;
                    }
                }
                if (!fzero) {
                    double fncx[3];
                    for (int k = 0; k < 3; ++k) fncx[k] = (fn + fc) * xx[k];
                    for (int k = 0; k < 3; ++k) fi[k] = fi[k] + fncx[k];
                    for (int k = 0; k < 3; ++k) fj[3 * j + k] = fj[3 * j + k] - fncx[k];
                    pxx = pxx + xx[0] * fncx[0];
                    pxy = pxy + xx[0] * fncx[1];
                    pxz = pxz + xx[0] * fncx[2];
                    pyy = pyy + xx[1] * fncx[1];
                    pyz = pyz + xx[1] * fncx[2];
                    pzz = pzz + xx[2] * fncx[2];
                }
            }
            #pragma omp single
            {
                for (int k = 0; k < 3; ++k) { fj[3 * i + k] = fj[3 * i + k] + fi[k]; fi[k] = 0.0; }
            }
        }
    } else {
        #pragma omp parallel
        for (int i = row_lo(); i <= row_hi(n); ++i) {
            #pragma omp for reduction(+:fi[:3])
            for (int j = i + 1; j <= n - 1; ++j) {
                double fn = 0.0, fc = 0.0;
                int fzero = 1;
                double xx[3];
                double r2 = min_image(x, i, j, xl, halfl, xx);
                if (nuclear_on && r2 <= rncut2) {
                    double expfac = exp(-(r2 * xpacket2i));
                    double xbbcc = (zii[i] == zii[j]) ? bb + cc : bb - cc;
                    fn = xpacketi * (2. * aa * expfac + xbbcc) * expfac;
                    fzero = 0;
                }
                if (coulomb_on && r2 <= rccut2) {
                    if (zii[i] == 1.0 && zii[j] == 1.0) {
                        double r = sqrt(r2);
                        fc = vc * (1. + xmuc * r) * exp(-(xmuc * r)) / (r * r2);
                        fzero = 0;
                    }
                }
                if (!fzero) {
                    double fncx[3];
                    for (int k = 0; k < 3; ++k) fncx[k] = (fn + fc) * xx[k];
                    for (int k = 0; k < 3; ++k) fi[k] = fi[k] + fncx[k];
                    for (int k = 0; k < 3; ++k) fj[3 * j + k] = fj[3 * j + k] - fncx[k];
                }
            }
            #pragma omp single
            {
                for (int k = 0; k < 3; ++k) { fj[3 * i + k] = fj[3 * i + k] + fi[k]; fi[k] = 0.0; }
            }
        }
    }
    pack_scalars(fj, n, evx, virx, pxx, pxy, pxz, pyy, pyz, pzz);
    for (int k = 0; k < 3 * (n + 3); ++k) a[k] = (double)fj[k];
    #pragma omp parallel for
    for (int i = 0; i <= n - 1; ++i)
        for (int k = 0; k < 3; ++k)
            a[3 * i + k] = a[3 * i + k] / p->xmass;
    unpack_scalars(a, n, 1.0, do_meas, p, s);
    free(fj);
}

int orc_accel(const yk_params* p, int n, const double* x,
              const double* zii, const double* aii,
              int do_meas, double* a, yk_scalars* s)
{
    if (!p || !x || !a || !s || n < 1) return YK_ERR_ARG;
    switch (p->sim_type) {
    case YK_SIM_NUCLEON:
        if (!zii) return YK_ERR_ARG;
        accel_nn(p, n, x, zii, do_meas, a, s);
        return YK_OK;
    case YK_SIM_PURE_ION:
        accel_ion_pure(p, n, x, do_meas, a, s);
        return YK_OK;
    case YK_SIM_ION_MIXTURE:
        if (!zii || !aii) return YK_ERR_ARG;
        accel_ion_mix(p, n, x, zii, aii, do_meas, a, s);
        return YK_OK;
    case YK_SIM_BFIELD:
        /* int_control.f:80-81: a = 0; ev, px, pp keep their previous values. */
        memset(a, 0, sizeof(double) * 3 * (size_t)(n + 3));
        return YK_OK;
    default:
        return YK_ERR_ARG;
    }
}

/* Kinetic part of the pressure tensor and ek (vel_verlet_2.f:84-106). */
static void kinetic_finish(const yk_params* p, int n, const double* v,
                           const double* aii, yk_scalars* s)
{
    acc_t vxx = 0.0, vxy = 0.0, vxz = 0.0, vyy = 0.0, vyz = 0.0, vzz = 0.0;
    #pragma omp parallel for reduction(+:vxx,vxy,vxz,vyy,vyz,vzz) schedule(runtime)
    for (int i = 0; i <= n - 1; ++i) {
        const double* vi = v + 3 * i;
        vxx = vxx + aii[i] * vi[0] * vi[0];
        vxy = vxy + aii[i] * vi[0] * vi[1];
        vxz = vxz + aii[i] * vi[0] * vi[2];
        vyy = vyy + aii[i] * vi[1] * vi[1];
        vyz = vyz + aii[i] * vi[1] * vi[2];
        vzz = vzz + aii[i] * vi[2] * vi[2];
    }
    const double xmass = p->xmass;
    s->ek = (0.5 * xmass) * (double)(vxx + vyy + vzz) / f_float(n);
    s->pp[0] = s->pp[0] + xmass * (double)vxx;
    s->pp[3] = s->pp[3] + xmass * (double)vxy;
    s->pp[6] = s->pp[6] + xmass * (double)vxz;
    s->pp[4] = s->pp[4] + xmass * (double)vyy;
    s->pp[7] = s->pp[7] + xmass * (double)vyz;
    s->pp[8] = s->pp[8] + xmass * (double)vzz;
    s->pp[1] = s->pp[3];
    s->pp[2] = s->pp[6];
    s->pp[5] = s->pp[7];
    const double vol = p->xl[0] * p->xl[1] * p->xl[2];
    for (int k = 0; k < 9; ++k) s->pp[k] = s->pp[k] / vol;
}

/* Drift with one periodic wrap (vel_verlet_2.f:33-43). */
static void drift(const yk_params* p, int n, double* x, const double* v,
                  const double* a, double afac)
{
    const double dt = p->dt;
    #pragma omp parallel for schedule(runtime)
    for (int i = 0; i <= n - 1; ++i)
        for (int k = 0; k < 3; ++k) {
            x[3 * i + k] = x[3 * i + k] + v[3 * i + k] * dt + afac * a[3 * i + k];
            if (x[3 * i + k] < 0.0) x[3 * i + k] = x[3 * i + k] + p->xl[k];
            if (x[3 * i + k] > p->xl[k]) x[3 * i + k] = x[3 * i + k] - p->xl[k];
        }
}

static int newton_vv2(const yk_params* p, int n, double* x, double* v,
                      double* vold, double* a, const double* zii,
                      const double* aii, int do_meas, yk_scalars* s)
{
    const double dt = p->dt;
    const double afac = 0.5 * (dt * dt);
    drift(p, n, x, v, a, afac);
    #pragma omp parallel for schedule(runtime)
    for (int i = 0; i <= n - 1; ++i)
        for (int k = 0; k < 3; ++k) {
            vold[3 * i + k] = v[3 * i + k];
            v[3 * i + k] = v[3 * i + k] + dt * a[3 * i + k];
        }
    int rc = orc_accel(p, n, x, zii, aii, do_meas, a, s);
    if (rc) return rc;
    if (p->bfield != 0.0) {                       /* vel_verlet_2.f:61-69 */
        #pragma omp parallel for schedule(runtime)
        for (int i = 0; i <= n - 1; ++i) {
            double omega = (3.218404e-20) * zii[i] * p->bfield / aii[i];
            a[3 * i + 0] = a[3 * i + 0] + v[3 * i + 1] * omega;
            a[3 * i + 1] = a[3 * i + 1] - v[3 * i + 0] * omega;
        }
    }
    #pragma omp parallel for schedule(runtime)
    for (int i = 0; i <= n - 1; ++i)
        for (int k = 0; k < 3; ++k) {
            double vp = vold[3 * i + k] + dt * a[3 * i + k];
            v[3 * i + k] = 0.5 * (v[3 * i + k] + vp);
        }
    if (do_meas) {
        kinetic_finish(p, n, v, aii, s);
    } else {
        s->ek = 0.0;
        for (int k = 0; k < 9; ++k) s->pp[k] = 0.0;
    }
    s->time = s->time + dt;
    return YK_OK;
}

/* vel_verlet_1.f:16-89: half kick, drift, accel, half kick; always measures
 * ek and pp. */
static int newton_vv1(const yk_params* p, int n, double* x, double* v,
                      double* a, const double* zii, const double* aii,
                      int do_meas, yk_scalars* s)
{
    const double dt = p->dt;
    const double afac = 0.5 * dt * dt;
    drift(p, n, x, v, a, afac);
    const double halfdt = 0.5 * dt;
    #pragma omp parallel for schedule(runtime)
    for (int i = 0; i <= n - 1; ++i)
        for (int k = 0; k < 3; ++k) v[3 * i + k] = v[3 * i + k] + halfdt * a[3 * i + k];
    int rc = orc_accel(p, n, x, zii, aii, do_meas, a, s);
    if (rc) return rc;
    #pragma omp parallel for schedule(runtime)
    for (int i = 0; i <= n - 1; ++i)
        for (int k = 0; k < 3; ++k) v[3 * i + k] = v[3 * i + k] + halfdt * a[3 * i + k];
    kinetic_finish(p, n, v, aii, s);
    s->time = s->time + dt;
    return YK_OK;
}

/* vel_verlet_3.f:20-100, Spreiter-Walter.  The first stage updates v(1,i)
 * before v(2,i) reads it (:259-260), as the reference does; the constant is
 * the REAL*4 literal 3.218404e-20 (:257, :276). */
static int newton_vv3(const yk_params* p, int n, double* x, double* v,
                      double* a, const double* zii, const double* aii,
                      int do_meas, yk_scalars* s)
{
    const double dt = p->dt;
    const double afac = 0.5 * (dt * dt);
    drift(p, n, x, v, a, afac);
    const double halfdt = 0.5 * dt;
    const double c = (double)3.218404e-20f;
    #pragma omp parallel for schedule(runtime)
    for (int i = 0; i <= n - 1; ++i) {
        double omega = c * zii[i] * p->bfield / aii[i];
        double omegap = halfdt * omega;
        double* vi = v + 3 * i;
        const double* ai = a + 3 * i;
        vi[0] = (1.0 - omegap * omegap) * vi[0] + 2.0 * omegap * vi[1]
              + halfdt * (ai[0] + omegap * ai[1]);
        vi[1] = (1.0 - omegap * omegap) * vi[1] - 2.0 * omegap * vi[0]
              + halfdt * (ai[1] - omegap * ai[0]);
        vi[2] = vi[2] + halfdt * ai[2];
    }
    int rc = orc_accel(p, n, x, zii, aii, do_meas, a, s);
    if (rc) return rc;
    #pragma omp parallel for schedule(runtime)
    for (int i = 0; i <= n - 1; ++i) {
        double omega = c * zii[i] * p->bfield / aii[i];
        double omegap = halfdt * omega;
        double* vi = v + 3 * i;
        const double* ai = a + 3 * i;
        vi[0] = (vi[0] + halfdt * (ai[0] + omegap * ai[1])) / (1.0 + omegap * omegap);
        vi[1] = (vi[1] + halfdt * (ai[1] - omegap * ai[0])) / (1.0 + omegap * omegap);
        vi[2] = vi[2] + halfdt * ai[2];
    }
    kinetic_finish(p, n, v, aii, s);
    s->time = s->time + dt;
    return YK_OK;
}

int orc_newton(const yk_params* p, int n, double* x, double* v, double* vold,
               double* a, const double* zii, const double* aii,
               int do_meas, yk_scalars* s)
{
    if (!p || !x || !v || !a || !s || !aii || n < 1) return YK_ERR_ARG;
    switch (p->integrator) {
    case YK_VV1: return newton_vv1(p, n, x, v, a, zii, aii, do_meas, s);
    case YK_VV2:
        if (!vold) return YK_ERR_ARG;
        return newton_vv2(p, n, x, v, vold, a, zii, aii, do_meas, s);
    case YK_VV3: return newton_vv3(p, n, x, v, a, zii, aii, do_meas, s);
    default: return YK_ERR_ARG;
    }
}

/* ttot, gen_utils.f:40-55. */
double orc_ttot(const yk_params* p, int n, const double* v, const double* aii)
{
    acc_t ekx = 0.0;
    #pragma omp parallel for reduction(+:ekx)
    for (int i = 0; i <= n - 1; ++i) {
        const double* vi = v + 3 * i;
        ekx = ekx + aii[i] * (vi[0] * vi[0] + vi[1] * vi[1] + vi[2] * vi[2]);
    }
    return (0.5 * p->xmass * (double)ekx) / f_float(n);
}

/* tnorm, gen_utils.f:64-76. */
void orc_tnorm(const yk_params* p, int n, double* v, const double* aii)
{
    double eka = orc_ttot(p, n, v, aii);
    double fac = sqrt(eka / (1.5 * p->kT));
    #pragma omp parallel for
    for (int i = 0; i <= n - 1; ++i)
        for (int k = 0; k < 3; ++k) v[3 * i + k] = v[3 * i + k] / fac;
}

/* cancel_vcom, gen_utils.f:87-110 (ends with tnorm). */
void orc_cancel_vcom(const yk_params* p, int n, double* v, const double* aii)
{
    acc_t mtot = 0.0, ptot[3] = {0.0, 0.0, 0.0};
    #pragma omp parallel for reduction(+:mtot,ptot[:3])
    for (int i = 0; i <= n - 1; ++i) {
        mtot = mtot + aii[i];
        for (int k = 0; k < 3; ++k) ptot[k] = ptot[k] + aii[i] * v[3 * i + k];
    }
    double vcom[3];
    for (int k = 0; k < 3; ++k) vcom[k] = (double)ptot[k] / (double)mtot;
    #pragma omp parallel for
    for (int i = 0; i <= n - 1; ++i)
        for (int k = 0; k < 3; ++k) v[3 * i + k] = v[3 * i + k] - vcom[k];
    orc_tnorm(p, n, v, aii);
}

/* strain, strain.f:19-82. */
void orc_strain(const yk_params* p, int n, double* x, double* xl,
                const double* xl0, const double* deps)
{
    const double XNOSTRAIN = 1000.0, dt = p->dt;
    int i0 = 0, i1 = 0, i2 = 0;
    if (deps[0] != XNOSTRAIN) i0 = 1;
    if (deps[1] != XNOSTRAIN) i1 = 2;
    if (deps[2] != XNOSTRAIN) i2 = 4;
    switch (i2 + i1 + i0) {
    case 0: break;
    case 1:
        xl[0] = xl[0] + deps[0] * dt * xl0[0];
        xl[1] = xl0[1] * sqrt(xl0[0] / xl[0]);
        xl[2] = xl0[2] * sqrt(xl0[0] / xl[0]);
        break;
    case 2:
        xl[1] = xl[1] + deps[1] * dt * xl0[1];
        xl[0] = xl0[0] * sqrt(xl0[1] / xl[1]);
        xl[2] = xl0[2] * sqrt(xl0[1] / xl[1]);
        break;
    case 3:
        xl[0] = xl[0] + deps[0] * dt * xl0[0];
        xl[1] = xl[1] + deps[1] * dt * xl0[1];
        xl[2] = xl0[2] * (xl0[0] / xl[0]) * (xl0[1] / xl[1]);
        break;
    case 4:
        xl[2] = xl[2] + deps[2] * dt * xl0[2];
        xl[0] = xl0[0] * sqrt(xl0[2] / xl[2]);
        xl[1] = xl0[1] * sqrt(xl0[2] / xl[2]);
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
    case 7:
        xl[0] = xl[0] + deps[0] * dt * xl0[0];
        xl[1] = xl[1] + deps[1] * dt * xl0[1];
        xl[2] = xl[2] + deps[2] * dt * xl0[2];
        break;
    }
    #pragma omp parallel for schedule(runtime)
    for (int i = 0; i <= n - 1; ++i)
        for (int k = 0; k < 3; ++k)
            if (x[3 * i + k] > xl[k]) x[3 * i + k] = x[3 * i + k] - xl[k];
}

/* Automatic nuclear cutoff, input1.F:296-311. */
double orc_rncut(double aa, double bb, double cc, double xpacket)
{
    double xepsilon = (sqrt(2.0 * xpacket) / (2.0 * (-bb + cc))) * 0.0001 * pow(2.0, -53);
    double rncut = sqrt(-log((-bb - cc) / (2.0 * aa)));
    double rncut0 = rncut;
    double xdeltar = 1.0;
    for (;;) {
        while (rncut * exp(-(rncut * rncut)) > xepsilon) {
            rncut0 = rncut;
            rncut = rncut + xdeltar;
        }
        if (xdeltar < 0.11) break;
        xdeltar = xdeltar / 10.0;
        rncut = rncut0;
    }
    return rncut * sqrt(2.0 * xpacket);
}

/* Thomas-Fermi inverse screening length, input1.F:260-278. */
double orc_thomas_fermi_xmuc(double ztot, double rho, int n)
{
    double rhoe = (ztot * rho) / n;
    double xkf = pow(3.0 * (PI * PI) * rhoe, 1.0 / 3.0) * HBARC;
    double ef = sqrt(xkf * xkf + ME * ME);
    double qtf = 2.0 * sqrt((ALPHA / PI) * xkf * ef);
    return qtf / HBARC;
}

/* vtot_ion_pure / vtot_ion_mix / vtot_nn: potential energy per particle and
 * pressure without forces (int_ion_pure.f:28-87, int_ion_mix.f:30-94,
 * int_nn.f:37-119).  These use the abs/min image form of the energy loops. */
int orc_vtot(const yk_params* p, int n, const double* x, const double* zii,
             double* evavg, double* pressure)
{
    if (!p || !x || !evavg || !pressure || n < 1) return YK_ERR_ARG;
    const double* xl = p->xl;
    const double rccut2 = p->rccut * p->rccut;
    acc_t t0 = 0.0, t1 = 0.0;
    if (p->sim_type == YK_SIM_PURE_ION || p->sim_type == YK_SIM_ION_MIXTURE) {
        const int mix = p->sim_type == YK_SIM_ION_MIXTURE;
        if (mix && !zii) return YK_ERR_ARG;
        const double evcut = ev_cut(p, 1.0);
        for (int i = 0; i <= n - 2; ++i) {
            acc_t x0 = 0.0, x1 = 0.0;
            for (int j = i + 1; j <= n - 1; ++j) {
                double r2 = 0.;
                for (int k = 0; k < 3; ++k) {
                    double xx = fabs(x[3 * i + k] - x[3 * j + k]);
                    xx = fmin(xx, xl[k] - xx);
                    r2 = r2 + xx * xx;
                }
                if (r2 <= rccut2) {
                    double r = sqrt(r2);
                    double evx = exp(-(p->xmuc * r)) / r;
                    double zj = mix ? zii[j] : 1.0;
                    if (mix) {
                        x0 = x0 + zj * (evx - evcut);
                        x1 = x1 + zj * (1. + p->xmuc * r) * evx;
                    } else {
                        x0 = x0 + (evx - evcut);
                        x1 = x1 + (1. + p->xmuc * r) * evx;
                    }
                }
            }
            if (mix) { t0 = t0 + zii[i] * x0; t1 = t1 + zii[i] * x1; }
            else { t0 = t0 + x0; t1 = t1 + x1; }
        }
        double c = mix ? p->frp * p->vc : p->frp * p->zi * p->zi * p->vc;
        t0 = c * t0;
        t1 = c * t1;
    } else if (p->sim_type == YK_SIM_NUCLEON) {
        if (!zii) return YK_ERR_ARG;
        const double xpacketi = 1. / p->xpacket;
        const double xpacket2i = 1. / (2.0 * p->xpacket);
        const double rncut2 = p->rncut * p->rncut;
        const double evcut = ev_cut(p, p->vc);
        for (int i = 0; i <= n - 2; ++i)
            for (int j = i + 1; j <= n - 1; ++j) {
                double r2 = 0.0;
                for (int k = 0; k < 3; ++k) {
                    double xx = fabs(x[3 * i + k] - x[3 * j + k]);
                    xx = fmin(xx, xl[k] - xx);
                    r2 = r2 + xx * xx;
                }
                if (p->nuclear_on && r2 <= rncut2) {
                    double expfac = exp(-(r2 * xpacket2i));
                    double xbbcc = (zii[i] == zii[j]) ? p->bb + p->cc : p->bb - p->cc;
                    t0 = t0 + (p->aa * expfac + xbbcc) * expfac;
                    t1 = t1 + (r2 * xpacketi) * (2. * p->aa * expfac + xbbcc) * expfac;
                }
                if (p->coulomb_on && r2 <= rccut2 && zii[i] == 1.0 && zii[j] == 1.0) {
                    double r = sqrt(r2);
                    double expfac = p->vc * exp(-(p->xmuc * r)) / r;
                    t0 = t0 + (expfac - evcut);
                    t1 = t1 + (1. + p->xmuc * r) * expfac;
                }
            }
    } else {
        *evavg = 0.0;
        *pressure = 0.0;
        return YK_OK;
    }
    *evavg = (double)t0 / f_float(n);
    *pressure = p->rho * (p->kT + (double)t1 / f_3n(n));
    return YK_OK;
}

/* The pair-distance histogram of subroutine g (g.f:55-66): for every unique
 * pair, rr = pdist(i, j) (gen_utils.f:115-128: per axis min(|d|, xl - |d|),
 * sqrt of the sum, plus the REAL*4 literal 1.e-15), bin ii = min(nbin,
 * int(fac2*rr + 1)) with fac2 = 2.*float(nbin)/sqrt(3.)/xlmin evaluated as the
 * Fortran does (REAL*4 up to the division by xlmin).  Adds 1 to counts[ii-1]. */
int orc_gofr_counts(const yk_params* p, int n, const double* x, int nbin, double* counts)
{
    if (!p || !x || !counts || n < 1 || nbin < 1) return YK_ERR_ARG;
    const double* xl = p->xl;
    const double xlmin = fmin(xl[0], fmin(xl[1], xl[2]));
    const float f4 = (2.0f * (float)nbin) / sqrtf(3.0f);
    const double fac2 = (double)f4 / xlmin;
    const double tiny = (double)1.e-15f;
    for (int i = 0; i <= n - 2; ++i)
        for (int j = i + 1; j <= n - 1; ++j) {
            double rr = 0.;
            for (int k = 0; k < 3; ++k) {
                double yy = fabs(x[3 * i + k] - x[3 * j + k]);
                yy = fmin(yy, xl[k] - yy);
                rr = rr + yy * yy;
            }
            rr = sqrt(rr) + tiny;
            int ii = (int)(fac2 * rr + 1.0);
            if (ii > nbin) ii = nbin;
            counts[ii - 1] += 1.0;
        }
    return YK_OK;
}
