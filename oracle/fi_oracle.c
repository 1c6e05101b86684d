/*
 * fi_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * A CPU, Float64 restatement of the FastIsostasy.jl laterally-variable ELVA path:
 * the right-hand side update_diagnostics! and the adaptive BS3 integrator that
 * run!/step! drive.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load this file, and only as the checker; the product library
 * (fastisostasy.jl_b200/csrc) never links, calls or falls back to it.
 *
 * Every function cites the reference file:line it restates.  Third-party
 * arithmetic absent from the reference tree is restated from its published
 * algorithm and named where used:
 *   - FFTW / CUFFT 2D transforms: an exact DFT, here a mixed-radix Stockham FFT;
 *   - OrdinaryDiffEq BS3 (OrdinaryDiffEqLowOrderRK, compat 1.2) with the default
 *     PI step-size controller, Hairer's initial-step heuristic, tstops and
 *     DiscreteCallback/FSAL semantics of OrdinaryDiffEqCore;
 *   - FastGaussQuadrature.gausslegendre(4): closed-form 4-point nodes/weights;
 *   - Interpolations.linear_interpolation: piecewise-linear on the knots.
 */
#include "fi_oracle.h"

#include <complex.h>
#undef I /* the integrator variables are named I; the imaginary unit is _Complex_I */
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double re, im; } cpx;

/* ======================================================================
 * FFT: complex mixed-radix Stockham autosort transform (natural order in
 * and out).  Stands in for FFTW's plan_fft!/plan_ifft!/plan_rfft, which the
 * reference uses at src/tools.jl:100-108 and src/convolutions.jl:229-244.
 * ====================================================================== */
typedef struct {
    int n, nf, naive;
    int fac[48];
    cpx* tw; /* tw[m] = exp(-2 pi i m / n) */
} or_fft;

static void fft_plan_init(or_fft* p, int n) {
    p->n = n;
    p->nf = 0;
    int m = n;
    while (m % 4 == 0) { p->fac[p->nf++] = 4; m /= 4; }
    while (m % 2 == 0) { p->fac[p->nf++] = 2; m /= 2; }
    for (int f = 3; f * f <= m; f += 2)
        while (m % f == 0) { p->fac[p->nf++] = f; m /= f; }
    if (m > 1) p->fac[p->nf++] = m;
    p->naive = 0;
    for (int f = 0; f < p->nf; f++) if (p->fac[f] > 64) p->naive = 1;
    p->tw = (cpx*)malloc(sizeof(cpx) * (size_t)n);
    for (int k = 0; k < n; k++) {
        long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)k / (long double)n;
        p->tw[k].re = (double)cosl(a);
        p->tw[k].im = (double)sinl(a);
    }
}

static void fft_plan_free(or_fft* p) { free(p->tw); p->tw = NULL; }

/* One transform of length n on data (contiguous), work is n scratch. */
static void fft_exec(const or_fft* p, cpx* data, cpx* work, int inverse) {
    const int n = p->n;
    if (n == 1) return;
    if (p->naive) { /* a prime factor above 64: direct DFT */
        for (int q = 0; q < n; q++) {
            double sr = 0.0, si = 0.0;
            for (int r = 0; r < n; r++) {
                cpx w = p->tw[(int)(((long long)q * r) % n)];
                if (inverse) w.im = -w.im;
                sr += data[r].re * w.re - data[r].im * w.im;
                si += data[r].re * w.im + data[r].im * w.re;
            }
            work[q].re = sr; work[q].im = si;
        }
        memcpy(data, work, sizeof(cpx) * (size_t)n);
        return;
    }
    cpx* src = data;
    cpx* dst = work;
    int Ns = 1;
    cpx v[64], y[64];
    for (int f = 0; f < p->nf; f++) {
        const int R = p->fac[f];
        const int nb = n / R;
        const int stride = n / (Ns * R);
        const int nR = n / R;
        for (int j = 0; j < nb; j++) {
            const int k = j % Ns;
            for (int r = 0; r < R; r++) v[r] = src[j + r * nb];
            for (int r = 1; r < R; r++) {
                cpx w = p->tw[(k * r * stride) % n];
                if (inverse) w.im = -w.im;
                double re = v[r].re * w.re - v[r].im * w.im;
                double im = v[r].re * w.im + v[r].im * w.re;
                v[r].re = re; v[r].im = im;
            }
            if (R == 2) {
                y[0].re = v[0].re + v[1].re; y[0].im = v[0].im + v[1].im;
                y[1].re = v[0].re - v[1].re; y[1].im = v[0].im - v[1].im;
            } else if (R == 4) {
                double ar = v[0].re + v[2].re, ai = v[0].im + v[2].im;
                double br = v[0].re - v[2].re, bi = v[0].im - v[2].im;
                double cr = v[1].re + v[3].re, ci = v[1].im + v[3].im;
                double dr = v[1].re - v[3].re, di = v[1].im - v[3].im;
                /* forward: -i * d ; inverse: +i * d */
                double er = inverse ? -di : di, ei = inverse ? dr : -dr;
                y[0].re = ar + cr; y[0].im = ai + ci;
                y[2].re = ar - cr; y[2].im = ai - ci;
                y[1].re = br + er; y[1].im = bi + ei;
                y[3].re = br - er; y[3].im = bi - ei;
            } else {
                for (int q = 0; q < R; q++) {
                    double sr = 0.0, si = 0.0;
                    for (int r = 0; r < R; r++) {
                        cpx w = p->tw[((q * r) % R) * nR];
                        if (inverse) w.im = -w.im;
                        sr += v[r].re * w.re - v[r].im * w.im;
                        si += v[r].re * w.im + v[r].im * w.re;
                    }
                    y[q].re = sr; y[q].im = si;
                }
            }
            const int idxD = (j / Ns) * Ns * R + k;
            for (int q = 0; q < R; q++) dst[idxD + q * Ns] = y[q];
        }
        cpx* t = src; src = dst; dst = t;
        Ns *= R;
    }
    if (src != data) memcpy(data, src, sizeof(cpx) * (size_t)n);
}

/* 2D transform of an nx-by-ny array (x fastest).  The inverse is normalised
 * by 1/(nx*ny) like AbstractFFTs' plan_ifft!. */
static void fft2(const or_fft* px, const or_fft* py, cpx* a, int nx, int ny, int inverse) {
    int nmax = nx > ny ? nx : ny;
#pragma omp parallel
    {
        cpx* work = (cpx*)malloc(sizeof(cpx) * (size_t)nmax);
        cpx* col = (cpx*)malloc(sizeof(cpx) * (size_t)ny);
#pragma omp for schedule(static)
        for (int j = 0; j < ny; j++) fft_exec(px, a + (size_t)j * nx, work, inverse);
#pragma omp for schedule(static)
        for (int i = 0; i < nx; i++) {
            for (int j = 0; j < ny; j++) col[j] = a[i + (size_t)j * nx];
            fft_exec(py, col, work, inverse);
            for (int j = 0; j < ny; j++) a[i + (size_t)j * nx] = col[j];
        }
        free(work);
        free(col);
    }
    if (inverse) {
        const double s = 1.0 / ((double)nx * (double)ny);
        const size_t n = (size_t)nx * ny;
#pragma omp parallel for schedule(static)
        for (size_t k = 0; k < n; k++) { a[k].re *= s; a[k].im *= s; }
    }
}

/* nextfastfft(n) = nextprod((2,3,5,7), n), src/convolutions.jl:17-19 */
int32_t or_nextfastfft(int32_t n) {
    if (n <= 1) return 1;
    for (int32_t m = n;; m++) {
        int32_t r = m;
        while (r % 2 == 0) r /= 2;
        while (r % 3 == 0) r /= 3;
        while (r % 5 == 0) r /= 5;
        while (r % 7 == 0) r /= 7;
        if (r == 1) return m;
    }
}

/* ======================================================================
 * Simulation state
 * ====================================================================== */
typedef int (*or_rhs_fn)(void* ctx, double t, double* u, double* du);

typedef struct {
    int n;
    or_rhs_fn f;
    void* ctx;
    double t0, t1, t, dt, dtpropose, dtmax, dtmin;
    double qold, q11, EEst, reltol, abstol;
    int accept_step, reeval_fsal, u_modified, initialized;
    int64_t iter, naccept, nreject, max_steps;
    double *u, *uprev, *k1, *k2, *k3, *k4, *tmp, *utilde;
    double* tstops;
    int ntstops, captstops;
    int nout, kout;
    const double* tout;
    void (*record)(void* ctx, int k, double t);
    int status;
    /* step-sequence replay / record (same semantics as the library's
       fi_set_step_replay / fi_record_steps) */
    int euler;          /* Euler with the fixed step dt_fixed (dt_min), no error control */
    double dt_fixed;
    double* replay;
    int64_t replay_n, replay_i;
    double* rec;
    int64_t rec_cap, rec_n;
} or_integ;

struct or_sim {
    fi_config cfg;
    int nx, ny, mx, my, Mx, My;
    int i1, i2, j1, j2; /* 1-based crop indices of samesize_conv */
    double dx, dy, A;
    double *x, *y;
    double rho_sw_ice;
    or_fft fx, fy, fMx, fMy;
    /* solid Earth and domain fields */
    double *D, *eta, *R, *mask, *pseudodiff, *spinv;
    int R_given, n_ch;
    double *ch_ratio, *ch_thick;
    /* Green's functions and their padded spectra */
    int n_table;
    double *rm, *GE;
    double *Ge, *Gg;
    cpx *Ge_hat, *Gg_hat;
    /* ice forcing */
    int K;
    double *t_ice, *H_tab;
    /* reference state */
    double *u_ref, *ue_ref, *dz_ss_ref, *z_b_ref, *H_ice_ref, *H_af_ref, *z_ss_ref;
    /* current state */
    double *u, *ue, *dudt, *H_ice, *H_af, *z_b, *dz_ss, *z_ss;
    double *c_ice, *c_sw, *c_sed, *c_litho, *c_mantle, *c_load, *c_full;
    int64_t count_sparse;
    /* sea level beyond the surface (src/sealevel.jl:242-332, src/barystatic_sealevel.jl) */
    double z_bsl, A_bsl, V_af, V_den, V_pov, delta_V;
    double *H_water, *mask_gr, *mask_oc;
    /* other rheologies (src/deformation.jl:29-89): ELRA relaxation time, equilibrium
       displacement and the viscous (Kelvin-function) Green's function */
    double *tau, *u_eq, *Gv;
    cpx *Gv_hat, *fftU;
    int n_osurf, n_bslh;
    double *osurf_z, *osurf_A, *bslh_t, *bslh_z;
    /* work buffers */
    double *rhs, *bxx, *byy, *bx, *bxy, *Mxx, *Myy, *Mxy, *buf;
    cpx *fftrhs, *convbuf;
    double* cropped;
    /* integrator */
    or_integ I;
    double* out_t;
    double *out_u, *out_ue, *out_dudt, *out_dz_ss;
    int64_t nf;
    double* tout_copy;
    int initialized, u_set;
    char err[256];
};

static int set_err(or_sim* s, int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(s->err, sizeof(s->err), fmt, ap);
    va_end(ap);
    return code;
}

static double* dalloc(size_t n) { return (double*)calloc(n ? n : 1, sizeof(double)); }

void or_set_threads(int32_t n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* ======================================================================
 * Finite differences, CPU edge rules (src/derivatives.jl:48-57, 66-76,
 * 114-124, 166-191).  Dx = K*dx with K == 1 (correct_distortion = false).
 * ====================================================================== */
static void dxx_(double* du, const double* u, int nx, int ny, double Dx) {
    const double s = Dx * Dx;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++) {
        const double* a = u + (size_t)j * nx;
        double* d = du + (size_t)j * nx;
        for (int i = 1; i < nx - 1; i++) d[i] = (a[i + 1] - 2 * a[i] + a[i - 1]) / s;
        d[0] = (a[2] - 2 * a[1] + a[0]) / s;
        d[nx - 1] = (a[nx - 1] - 2 * a[nx - 2] + a[nx - 3]) / s;
    }
}

static void dyy_(double* du, const double* u, int nx, int ny, double Dy) {
    const double s = Dy * Dy;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++) {
        double* d = du + (size_t)j * nx;
        if (j > 0 && j < ny - 1) {
            const double *am = u + (size_t)(j - 1) * nx, *a0 = u + (size_t)j * nx, *ap = u + (size_t)(j + 1) * nx;
            for (int i = 0; i < nx; i++) d[i] = (ap[i] - 2 * a0[i] + am[i]) / s;
        } else if (j == 0) {
            const double *a0 = u, *a1 = u + nx, *a2 = u + 2 * (size_t)nx;
            for (int i = 0; i < nx; i++) d[i] = (a2[i] - 2 * a1[i] + a0[i]) / s;
        } else {
            const double *a0 = u + (size_t)(ny - 1) * nx, *a1 = u + (size_t)(ny - 2) * nx, *a2 = u + (size_t)(ny - 3) * nx;
            for (int i = 0; i < nx; i++) d[i] = (a0[i] - 2 * a1[i] + a2[i]) / s;
        }
    }
}

static void dx_(double* du, const double* u, int nx, int ny, double Dx) {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++) {
        const double* a = u + (size_t)j * nx;
        double* d = du + (size_t)j * nx;
        for (int i = 1; i < nx - 1; i++) d[i] = (a[i + 1] - a[i - 1]) / (2 * Dx);
        d[0] = (a[1] - a[0]) / Dx;
        d[nx - 1] = (a[nx - 1] - a[nx - 2]) / Dx;
    }
}

static void dy_(double* du, const double* u, int nx, int ny, double Dy) {
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++) {
        double* d = du + (size_t)j * nx;
        if (j > 0 && j < ny - 1) {
            const double *am = u + (size_t)(j - 1) * nx, *ap = u + (size_t)(j + 1) * nx;
            for (int i = 0; i < nx; i++) d[i] = (ap[i] - am[i]) / (2 * Dy);
        } else if (j == 0) {
            for (int i = 0; i < nx; i++) d[i] = (u[nx + i] - u[i]) / Dy;
        } else {
            const double *a0 = u + (size_t)(ny - 1) * nx, *a1 = u + (size_t)(ny - 2) * nx;
            for (int i = 0; i < nx; i++) d[i] = (a0[i] - a1[i]) / Dy;
        }
    }
}

/* update_second_derivatives!(uxx, uyy, ux, uxy, u, domain), derivatives.jl:48-57 */
void or_second_derivatives(int32_t nx, int32_t ny, double Dx, double Dy, const double* u,
                           double* uxx, double* uyy, double* ux, double* uxy) {
    dxx_(uxx, u, nx, ny, Dx);
    dyy_(uyy, u, nx, ny, Dy);
    dx_(ux, u, nx, ny, Dx);
    dy_(uxy, ux, nx, ny, Dy);
}

/* ======================================================================
 * Boundary conditions: OffsetBC with CornerBC weights
 * (src/boundary_conditions.jl:144-148, 199-207, 231-243)
 * ====================================================================== */
static void corner_bc(double* X, int nx, int ny, double x_border) {
    /* W = 1/4 at the four corners; sum(W .* X) */
    double sum = 0.25 * X[0] + 0.25 * X[nx - 1] + 0.25 * X[(size_t)(ny - 1) * nx] +
                 0.25 * X[(size_t)(ny - 1) * nx + nx - 1];
    const double off = sum - x_border;
    const size_t n = (size_t)nx * ny;
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < n; k++) X[k] -= off;
}

/* ======================================================================
 * Convolution: ConvolutionPlanHelpers / ConvolutionPlan / conv! /
 * samesize_conv! with ExtendedBCSpace (src/convolutions.jl:1-15, 21-56,
 * 81-106, 134-143, 196-204).
 * ====================================================================== */
static void pad_to(cpx* P, const double* in, int nx, int ny, int Mx, int My) {
    memset(P, 0, sizeof(cpx) * (size_t)Mx * My);
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) P[i + (size_t)j * Mx].re = in[i + (size_t)j * nx];
}

/* kernel_fft = p_rfft * pad(kernel) (full complex spectrum here) */
/* K_0(z) for complex z with Re z > 0 (SpecialFunctions besselk(0, z) as the reference
 * calls it) from the integral K_0(z) = int_0^inf exp(-z cosh t) dt (Abramowitz &
 * Stegun 9.6.24) by the trapezoidal rule with step 1/20: the integrand is analytic and
 * decays doubly exponentially, so the rule converges geometrically (about 1e-15 relative
 * for |z| in [1e-5, 60] on the ray arg z = pi/4, checked against scipy). */
static double complex besselk0_(double complex z) {
    const double h = 0.05;
    double complex sum = 0.5 * cexp(-z);
    for (int k = 1; k < 4000; k++) {
        const double complex v = cexp(-z * cosh(k * h));
        sum += v;
        if (k * h > 1.0 && cabs(v) < 1e-18 * cabs(sum)) break;
    }
    return h * sum;
}

/* besselkei(x) = imag(besselk(0, x e^{i pi/4})), src/material.jl:370-373 */
double or_kei(double x) { return cimag(besselk0_(x * cexp(_Complex_I * M_PI / 4.0))); }

/* green_viscous(domain, rho_uppermantle, mean(litho_rigidity)) (src/material.jl:375-380,
 * src/tools.jl:53-58): -(L^2 / (2 pi D)) kei(max(R, 1) / L) dx dy with the flexural
 * length L = (D / (rho g))^(1/4), g = 9.81 (src/material.jl:396-399). */
static void build_viscous_green_(or_sim* s) {
    const size_t n = (size_t)s->nx * s->ny;
    double D = 0.0;
    for (size_t k = 0; k < n; k++) D += s->D[k];
    D /= (double)n;
    const double L = pow(D / (s->cfg.rho_uppermantle * 9.81), 0.25);
    for (int j = 0; j < s->ny; j++)
        for (int i = 0; i < s->nx; i++) {
            double R = sqrt(s->x[i] * s->x[i] + s->y[j] * s->y[j]);
            if (R < 1.0) R = 1.0;
            s->Gv[i + (size_t)j * s->nx] = -(L * L / (2.0 * M_PI * D) * or_kei(R / L)) * (s->dx * s->dy);
        }
}

static void conv_plan(or_sim* s, const double* kernel, cpx* khat) {
    pad_to(khat, kernel, s->nx, s->ny, s->Mx, s->My);
    fft2(&s->fMx, &s->fMy, khat, s->Mx, s->My, 0);
}

/* conv!(input, p, h): output_cropped = irfft(rfft(pad(input)) .* kernel_fft)[1:2nx-1, 1:2ny-1] */
static void conv_full_(or_sim* s, const double* input, const cpx* khat, double* cropped) {
    const int Mx = s->Mx, My = s->My, cx = 2 * s->nx - 1, cy = 2 * s->ny - 1;
    pad_to(s->convbuf, input, s->nx, s->ny, Mx, My);
    fft2(&s->fMx, &s->fMy, s->convbuf, Mx, My, 0);
    const size_t n = (size_t)Mx * My;
    for (size_t k = 0; k < n; k++) {
        cpx a = s->convbuf[k], b = khat[k];
        s->convbuf[k].re = a.re * b.re - a.im * b.im;
        s->convbuf[k].im = a.re * b.im + a.im * b.re;
    }
    fft2(&s->fMx, &s->fMy, s->convbuf, Mx, My, 1);
    for (int j = 0; j < cy; j++)
        for (int i = 0; i < cx; i++) cropped[i + (size_t)j * cx] = s->convbuf[i + (size_t)j * Mx].re;
}

/* samesize_conv!(output, input, p, h, domain, bc, ::ExtendedBCSpace) */
static void samesize_conv_ext(or_sim* s, double* output, const double* input, const cpx* khat,
                              double x_border) {
    const int cx = 2 * s->nx - 1, cy = 2 * s->ny - 1;
    conv_full_(s, input, khat, s->cropped);
    corner_bc(s->cropped, cx, cy, x_border);
    for (int j = 0; j < s->ny; j++)
        for (int i = 0; i < s->nx; i++)
            output[i + (size_t)j * s->nx] = s->cropped[(s->i1 - 1 + i) + (size_t)(s->j1 - 1 + j) * cx];
}

/* ======================================================================
 * Setup: domain (src/domain.jl:76-83, 151-163), derivatives in Fourier space
 * (src/derivatives.jl:201-223), channel scaling (src/material.jl:232-278),
 * Green's functions (src/material.jl:299-364, src/sealevel.jl:208-219,
 * src/utils.jl:118-187).
 * ====================================================================== */
static void fftint_(int N, double* f) {
    const int N2 = N / 2;
    int k = 0;
    for (int i = 0; i <= N2; i++) f[k++] = i;
    if (N % 2 == 0)
        for (int i = N2 - 1; i >= 1; i--) f[k++] = i;
    else
        for (int i = N2; i >= 1; i--) f[k++] = i;
}

static void samesize_conv_indices_(int N, int M, int* a, int* b) {
    *a = (N % 2 == 0) ? M : M + 1;
    *b = 2 * N - 1 - M;
}

static double loadgreen_(const or_sim* s, double r) {
    /* get_loadgreen, src/material.jl:318-332 */
    const double* rm = s->rm;
    const double* GE = s->GE;
    const int n = s->n_table;
    if (r < 0.01) return GE[0] / (rm[1] * 1e12);
    if (r > rm[n - 1]) return 0.0;
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        int mid = (lo + hi) / 2;
        if (rm[mid] <= r) lo = mid; else hi = mid;
    }
    const double w = (r - rm[lo]) / (rm[hi] - rm[lo]);
    const double v = (1.0 - w) * GE[lo] + w * GE[hi];
    return v / (r * 1e12);
}

static void gauss_legendre4_(double* x, double* w) {
    /* FastGaussQuadrature.gausslegendre(4), closed form */
    const double a = sqrt(3.0 / 7.0 - 2.0 / 7.0 * sqrt(6.0 / 5.0));
    const double b = sqrt(3.0 / 7.0 + 2.0 / 7.0 * sqrt(6.0 / 5.0));
    const double wa = (18.0 + sqrt(30.0)) / 36.0, wb = (18.0 - sqrt(30.0)) / 36.0;
    x[0] = -b; x[1] = -a; x[2] = a; x[3] = b;
    w[0] = wb; w[1] = wa; w[2] = wa; w[3] = wb;
}

static void build_elastic_green_(or_sim* s) {
    /* get_elastic_green, src/material.jl:340-364 with quadrature2D, utils.jl:146-165 */
    double qx[4], qw[4];
    gauss_legendre4_(qx, qw);
    const int nx = s->nx, ny = s->ny;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++) {
        for (int i = 0; i < nx; i++) {
            const int p = i - s->mx, q = j - s->my; /* i - mx - 1 with 1-based i */
            const double x1 = p * s->dx, x2 = (p + 1) * s->dx, y1 = q * s->dy, y2 = (q + 1) * s->dy;
            const double mx_ = 2.0 / (x2 - x1), px_ = -1.0 - mx_ * x1;
            const double my_ = 2.0 / (y2 - y1), py_ = -1.0 - my_ * y1;
            double sum = 0.0;
            for (int a = 0; a < 4; a++)
                for (int b = 0; b < 4; b++) {
                    const double xx = (qx[a] - px_) / mx_, yy = (qx[b] - py_) / my_;
                    sum = sum + loadgreen_(s, sqrt(xx * xx + yy * yy)) * qw[a] * qw[b] / mx_ / my_;
                }
            s->Ge[i + (size_t)j * nx] = sum;
        }
    }
}

static void build_geoid_green_(or_sim* s) {
    /* get_dz_ss_green / unbounded_dz_ssgreen, src/sealevel.jl:208-219 */
    const fi_config* c = &s->cfg;
    const double cap = c->r_pole / (2.0 * c->mE * sin((s->dx / 2) / (2.0 * c->r_pole)));
    for (int j = 0; j < s->ny; j++)
        for (int i = 0; i < s->nx; i++) {
            const double R = sqrt(s->x[i] * s->x[i] + s->y[j] * s->y[j]);
            double g = c->r_pole / (2.0 * c->mE * sin(R / (2.0 * c->r_pole)));
            if (!(g <= cap)) g = cap; /* min.(green, cap); R = 0 gives Inf */
            s->Gg[i + (size_t)j * s->nx] = g;
        }
}

static double channel_scaling_(double kappa, double T, double r) {
    /* channel_scaling, src/material.jl:232-262 (Tint = Float64) */
    const double C = cosh(T * kappa), S = sinh(T * kappa);
    double num = 0.0, den = 0.0;
    num += 2 * r * C * S;
    num += (1 - r * r) * T * T * kappa * kappa;
    num += r * r * S * S + C * C;
    den += (r + 1 / r) * C * S;
    den += (r - 1 / r) * T * kappa;
    den += S * S + C * C;
    return num / den;
}

/* ======================================================================
 * Lifecycle
 * ====================================================================== */
int or_create(const fi_config* cfg, or_sim** out) {
    if (!cfg || !out) return FI_ERR_ARG;
    if (cfg->nx < 4 || cfg->ny < 4 || !(cfg->Wx > 0) || !(cfg->Wy > 0)) return FI_ERR_ARG;
    or_sim* s = (or_sim*)calloc(1, sizeof(or_sim));
    s->cfg = *cfg;
    const int nx = cfg->nx, ny = cfg->ny;
    s->nx = nx; s->ny = ny;
    s->mx = nx / 2; s->my = ny / 2;
    s->dx = 2 * cfg->Wx / nx;
    s->dy = 2 * cfg->Wy / ny;
    s->A = s->dx * s->dy;
    s->rho_sw_ice = cfg->rho_seawater / cfg->rho_ice;
    s->x = dalloc(nx);
    s->y = dalloc(ny);
    {
        /* range(-W+dx, stop = W, length = n): correctly rounded linear spacing */
        const long double x0 = (long double)(-cfg->Wx + s->dx), x1 = cfg->Wx;
        for (int i = 0; i < nx; i++) s->x[i] = (double)(x0 + (x1 - x0) * (long double)i / (long double)(nx - 1));
        const long double y0 = (long double)(-cfg->Wy + s->dy), y1 = cfg->Wy;
        for (int j = 0; j < ny; j++) s->y[j] = (double)(y0 + (y1 - y0) * (long double)j / (long double)(ny - 1));
    }
    samesize_conv_indices_(nx, s->mx, &s->i1, &s->i2);
    samesize_conv_indices_(ny, s->my, &s->j1, &s->j2);
    s->Mx = or_nextfastfft(2 * nx - 1);
    s->My = or_nextfastfft(2 * ny - 1);
    fft_plan_init(&s->fx, nx);
    fft_plan_init(&s->fy, ny);
    fft_plan_init(&s->fMx, s->Mx);
    fft_plan_init(&s->fMy, s->My);
    const size_t n = (size_t)nx * ny, M = (size_t)s->Mx * s->My;
    double** fields[] = {&s->D, &s->eta, &s->R, &s->mask, &s->pseudodiff, &s->spinv, &s->Ge, &s->Gg,
                         &s->u_ref, &s->ue_ref, &s->dz_ss_ref, &s->z_b_ref, &s->H_ice_ref, &s->H_af_ref,
                         &s->z_ss_ref, &s->u, &s->ue, &s->dudt, &s->H_ice, &s->H_af, &s->z_b, &s->dz_ss,
                         &s->z_ss, &s->c_ice, &s->c_sw, &s->c_sed, &s->c_litho, &s->c_mantle, &s->c_load,
                         &s->c_full, &s->rhs, &s->bxx, &s->byy, &s->bx, &s->bxy, &s->Mxx, &s->Myy, &s->Mxy,
                         &s->buf, &s->H_water, &s->mask_gr, &s->mask_oc, &s->tau, &s->u_eq, &s->Gv};
    for (size_t k = 0; k < sizeof(fields) / sizeof(fields[0]); k++) *fields[k] = dalloc(n);
    for (size_t k = 0; k < n; k++) { s->R[k] = 1.0; s->mask[k] = 1.0; s->z_b_ref[k] = 1e6; s->tau[k] = 855.0; }
    s->Gv_hat = (cpx*)calloc(M, sizeof(cpx));
    s->fftU = (cpx*)calloc(n, sizeof(cpx));
    s->fftrhs = (cpx*)calloc(n, sizeof(cpx));
    s->convbuf = (cpx*)calloc(M, sizeof(cpx));
    s->Ge_hat = (cpx*)calloc(M, sizeof(cpx));
    s->Gg_hat = (cpx*)calloc(M, sizeof(cpx));
    s->cropped = dalloc((size_t)(2 * nx - 1) * (2 * ny - 1));
    *out = s;
    return FI_OK;
}

void or_destroy(or_sim* s) {
    if (!s) return;
    double* ptrs[] = {s->x, s->y, s->D, s->eta, s->R, s->mask, s->pseudodiff, s->spinv, s->Ge, s->Gg,
                      s->u_ref, s->ue_ref, s->dz_ss_ref, s->z_b_ref, s->H_ice_ref, s->H_af_ref, s->z_ss_ref,
                      s->u, s->ue, s->dudt, s->H_ice, s->H_af, s->z_b, s->dz_ss, s->z_ss, s->c_ice, s->c_sw,
                      s->c_sed, s->c_litho, s->c_mantle, s->c_load, s->c_full, s->rhs, s->bxx, s->byy, s->bx,
                      s->bxy, s->Mxx, s->Myy, s->Mxy, s->buf, s->cropped, s->rm, s->GE, s->t_ice, s->H_tab,
                      s->ch_ratio, s->ch_thick, s->tout_copy, s->H_water, s->mask_gr, s->mask_oc,
                      s->osurf_z, s->osurf_A, s->bslh_t, s->bslh_z, s->tau, s->u_eq, s->Gv};
    for (size_t k = 0; k < sizeof(ptrs) / sizeof(ptrs[0]); k++) free(ptrs[k]);
    free(s->fftrhs); free(s->convbuf); free(s->Ge_hat); free(s->Gg_hat); free(s->Gv_hat); free(s->fftU);
    fft_plan_free(&s->fx); fft_plan_free(&s->fy); fft_plan_free(&s->fMx); fft_plan_free(&s->fMy);
    or_integ* I = &s->I;
    free(I->u); free(I->uprev); free(I->k1); free(I->k2); free(I->k3); free(I->k4); free(I->tmp);
    free(I->utilde); free(I->tstops); free(I->replay); free(I->rec);
    free(s);
}

const char* or_last_error(const or_sim* s) { return s ? s->err : "null handle"; }

static double* field_ptr(or_sim* s, int32_t f, int for_set) {
    switch (f) {
        case FI_FIELD_LITHO_RIGIDITY: return s->D;
        case FI_FIELD_EFFECTIVE_VISCOSITY: return s->eta;
        case FI_FIELD_PSEUDODIFF_SCALING: if (for_set) s->R_given = 1; return s->R;
        case FI_FIELD_MASKACTIVE: return s->mask;
        case FI_FIELD_U_REF: return s->u_ref;
        case FI_FIELD_UE_REF: return s->ue_ref;
        case FI_FIELD_DZ_SS_REF: return s->dz_ss_ref;
        case FI_FIELD_Z_B_REF: return s->z_b_ref;
        case FI_FIELD_U: if (for_set) s->u_set = 1; return s->u;
        case FI_FIELD_UE: return s->ue;
        case FI_FIELD_DUDT: return s->dudt;
        case FI_FIELD_DZ_SS: return s->dz_ss;
        case FI_FIELD_H_ICE: return s->H_ice;
        case FI_FIELD_Z_SS: return s->z_ss;
        case FI_FIELD_Z_B: return s->z_b;
        case FI_FIELD_ELASTIC_GREEN: return for_set ? NULL : s->Ge;
        case FI_FIELD_DZ_SS_GREEN: return for_set ? NULL : s->Gg;
        case FI_FIELD_PSEUDODIFF: return for_set ? NULL : s->pseudodiff;
        case FI_FIELD_SCALED_PSEUDODIFF_INV: return for_set ? NULL : s->spinv;
        case FI_FIELD_COLUMNANOM_LOAD: return s->c_load;
        case FI_FIELD_COLUMNANOM_FULL: return s->c_full;
        case FI_FIELD_H_AF: return s->H_af;
        case FI_FIELD_MASKGROUNDED: return for_set ? NULL : s->mask_gr;
        case FI_FIELD_MASKOCEAN: return for_set ? NULL : s->mask_oc;
        case FI_FIELD_H_WATER: return for_set ? NULL : s->H_water;
        case FI_FIELD_COLUMNANOM_SEAWATER: return for_set ? NULL : s->c_sw;
        case FI_FIELD_TAU: return s->tau;
        case FI_FIELD_U_EQ: return for_set ? NULL : s->u_eq;
        default: return NULL;
    }
}

int or_set_field(or_sim* s, int32_t field, const double* host, size_t n) {
    if (!s || !host) return FI_ERR_ARG;
    if (n != (size_t)s->nx * s->ny) return set_err(s, FI_ERR_ARG, "field size %zu != nx*ny", n);
    double* p = field_ptr(s, field, 1);
    if (!p) return set_err(s, FI_ERR_ARG, "field %d is not settable", field);
    memcpy(p, host, n * sizeof(double));
    return FI_OK;
}

int or_get_field(or_sim* s, int32_t field, double* host, size_t n) {
    if (!s || !host) return FI_ERR_ARG;
    if (n != (size_t)s->nx * s->ny) return set_err(s, FI_ERR_ARG, "field size %zu != nx*ny", n);
    double* p = field_ptr(s, field, 0);
    if (!p) return set_err(s, FI_ERR_ARG, "unknown field %d", field);
    memcpy(host, p, n * sizeof(double));
    return FI_OK;
}

int or_set_ice_history(or_sim* s, int32_t K, const double* t, const double* H) {
    if (!s || K < 1 || !t || !H) return FI_ERR_ARG;
    for (int k = 1; k < K; k++)
        if (!(t[k] > t[k - 1])) return set_err(s, FI_ERR_ARG, "ice times must increase");
    const size_t n = (size_t)s->nx * s->ny;
    free(s->t_ice); free(s->H_tab);
    s->K = K;
    s->t_ice = dalloc(K);
    s->H_tab = dalloc((size_t)K * n);
    memcpy(s->t_ice, t, sizeof(double) * K);
    memcpy(s->H_tab, H, sizeof(double) * K * n);
    return FI_OK;
}

int or_set_elastic_table(or_sim* s, int32_t n, const double* rm, const double* GE) {
    if (!s || n < 2 || !rm || !GE) return FI_ERR_ARG;
    free(s->rm); free(s->GE);
    s->n_table = n;
    s->rm = dalloc(n);
    s->GE = dalloc(n);
    memcpy(s->rm, rm, sizeof(double) * n);
    memcpy(s->GE, GE, sizeof(double) * n);
    return FI_OK;
}

int or_set_channel_scaling(or_sim* s, int32_t n, const double* ratio, const double* thick) {
    if (!s || n < 0) return FI_ERR_ARG;
    free(s->ch_ratio); free(s->ch_thick);
    s->n_ch = n;
    s->ch_ratio = dalloc(n);
    s->ch_thick = dalloc(n);
    if (n) { memcpy(s->ch_ratio, ratio, sizeof(double) * n); memcpy(s->ch_thick, thick, sizeof(double) * n); }
    return FI_OK;
}

static int copy_table_(or_sim* s, int32_t n, const double* x, const double* y, int* n_out, double** xo, double** yo) {
    if (n < 2 || !x || !y) return set_err(s, FI_ERR_ARG, "a table needs >= 2 points");
    for (int k = 1; k < n; k++)
        if (!(x[k] > x[k - 1])) return set_err(s, FI_ERR_ARG, "table abscissae must increase");
    free(*xo); free(*yo);
    *xo = dalloc(n); *yo = dalloc(n);
    memcpy(*xo, x, sizeof(double) * n);
    memcpy(*yo, y, sizeof(double) * n);
    *n_out = n;
    return FI_OK;
}

int or_set_ocean_surface_table(or_sim* s, int32_t n, const double* z, const double* A) {
    if (!s) return FI_ERR_ARG;
    return copy_table_(s, n, z, A, &s->n_osurf, &s->osurf_z, &s->osurf_A);
}

int or_set_bsl_history(or_sim* s, int32_t n, const double* t, const double* z) {
    if (!s) return FI_ERR_ARG;
    return copy_table_(s, n, t, z, &s->n_bslh, &s->bslh_t, &s->bslh_z);
}

/* interpolate(x, ::TimeInterpolation0D) with flat_bc = false (src/interpolations.jl:20-40):
 * linear inside the table, an error outside */
static int interp0d_(const double* xs, const double* ys, int n, double x, double* y) {
    if (n < 2 || x < xs[0] || x > xs[n - 1]) return FI_ERR_FORCING_RANGE;
    int k = 0;
    while (k < n - 2 && xs[k + 1] < x) k++;
    const double w = (x - xs[k]) / (xs[k + 1] - xs[k]);
    *y = ys[k] + w * (ys[k + 1] - ys[k]);
    return FI_OK;
}

int or_get_sealevel(or_sim* s, fi_sealevel* out) {
    if (!s || !out) return FI_ERR_ARG;
    memset(out, 0, sizeof(*out));
    out->z_bsl = s->z_bsl; out->A_bsl = s->A_bsl;
    out->V_af = s->V_af; out->V_den = s->V_den; out->V_pov = s->V_pov; out->delta_V = s->delta_V;
    out->tracked = 1;
    return FI_OK;
}

/* update_V_af!, update_V_den!, update_V_pov! (src/sealevel.jl:275-332) on the current
 * H_af, H_ice, z_ss and z_b; returns the total volume */
static double update_volumes_(or_sim* s) {
    const fi_config* c = &s->cfg;
    const size_t n = (size_t)s->nx * s->ny;
    double saf = 0.0, sden = 0.0, spov = 0.0;
    for (size_t k = 0; k < n; k++) {
        saf += s->H_af[k] * s->A;
        sden += s->H_ice[k] * s->A;
        const double w = s->z_ss[k] - s->z_b[k];
        spov += (w > 0 ? w : 0.0) * s->A;
    }
    s->V_af = c->volume_contribution == FI_CONTRIB_GOELZER ? saf * c->rho_ice / c->rho_seawater : 0.0;
    s->V_den = c->density_contribution == FI_CONTRIB_GOELZER
                   ? sden * (c->rho_ice / c->rho_water - c->rho_ice / c->rho_seawater) : 0.0;
    s->V_pov = c->adjustment_contribution == FI_CONTRIB_GOELZER ? spov : 0.0;
    return s->V_af + s->V_den + s->V_pov;
}

/* internal_update_bsl! (src/sealevel.jl:242-262) with update_bsl! of each BSL
 * (src/barystatic_sealevel.jl:215-235) */
static int internal_update_bsl_(or_sim* s, double t) {
    const fi_config* c = &s->cfg;
    const double Vold = s->V_af + s->V_den + s->V_pov;
    s->delta_V = update_volumes_(s) - Vold;
    if (c->bsl_update != FI_BSL_UPDATE_INTERNAL) return FI_OK;
    const double dV = -s->delta_V;
    switch (c->bsl_mode) {
        case FI_BSL_CONSTANT: s->z_bsl = c->z_bsl; break;
        case FI_BSL_CONSTANT_OCEAN_SURFACE: s->A_bsl = c->bsl_ref_A; s->z_bsl += dV / s->A_bsl; break;
        case FI_BSL_PIECEWISE_CONSTANT: {
            s->z_bsl += dV / s->A_bsl;
            double A;
            if (interp0d_(s->osurf_z, s->osurf_A, s->n_osurf, s->z_bsl, &A))
                return set_err(s, FI_ERR_FORCING_RANGE, "BSL %g outside the ocean-surface table", s->z_bsl);
            s->A_bsl = A;
            break;
        }
        case FI_BSL_IMPOSED: {
            double z;
            if (interp0d_(s->bslh_t, s->bslh_z, s->n_bslh, t, &z))
                return set_err(s, FI_ERR_FORCING_RANGE, "t = %g outside the imposed BSL history", t);
            s->z_bsl = z;
            break;
        }
        default: return set_err(s, FI_ERR_ARG, "unknown BSL mode %d", c->bsl_mode);
    }
    return FI_OK;
}

/* update_maskgrounded!, update_maskocean!, watercolumn! and columnanom_water!
 * (src/topography.jl:1-28, src/loads.jl:56-85) on the current fields */
static void masks_water_(or_sim* s) {
    const fi_config* c = &s->cfg;
    const size_t n = (size_t)s->nx * s->ny;
    const int interactive = c->sealevel_load == FI_SEALEVEL_LOAD_INTERACTIVE;
    for (size_t k = 0; k < n; k++) {
        const int gr = s->H_af[k] > 0;
        const double w = s->z_ss[k] - s->z_b[k];
        const int oc = (w > 0) && !gr;
        s->mask_gr[k] = gr;
        s->mask_oc[k] = oc;
        const double wc = w > 0 ? w : 0.0;
        const double H = s->H_ice[k];
        s->H_water[k] = (H <= 1 ? wc : 0.0) + ((!gr && H > 1) ? wc - H * (c->rho_ice / c->rho_seawater) : 0.0);
        s->c_sw[k] = interactive ? c->rho_seawater * (s->z_ss[k] - s->z_ss_ref[k]) * oc * s->mask[k] : 0.0;
    }
}

/* interpolate!(X_out, t, ::TimeInterpolation2D), src/interpolations.jl:51-74 */
static int interp_ice_(or_sim* s, double t, double* H) {
    const size_t n = (size_t)s->nx * s->ny;
    const int K = s->K;
    if (K < 1) return set_err(s, FI_ERR_STATE, "no ice history");
    const double tmin = s->t_ice[0], tmax = s->t_ice[K - 1];
    if (t < tmin) {
        if (!s->cfg.ice_flat_bc) return set_err(s, FI_ERR_FORCING_RANGE, "TimeInterpolation2D out of range.");
        memcpy(H, s->H_tab, n * sizeof(double));
        return FI_OK;
    }
    if (t > tmax) {
        if (!s->cfg.ice_flat_bc) return set_err(s, FI_ERR_FORCING_RANGE, "TimeInterpolation2D out of range.");
        memcpy(H, s->H_tab + (size_t)(K - 1) * n, n * sizeof(double));
        return FI_OK;
    }
    /* searchsortedfirst: first index with t_ice[i] >= t */
    int i = 0;
    while (s->t_ice[i] < t) i++;
    if (s->t_ice[i] == t) {
        memcpy(H, s->H_tab + (size_t)i * n, n * sizeof(double));
        return FI_OK;
    }
    i -= 1;
    const double* a = s->H_tab + (size_t)i * n;
    const double* b = s->H_tab + (size_t)(i + 1) * n;
    const double dt = s->t_ice[i + 1] - s->t_ice[i], tt = t - s->t_ice[i];
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < n; k++) H[k] = a[k] + (b[k] - a[k]) / dt * tt;
    return FI_OK;
}

static double haf_(const or_sim* s, double H, double zb, double zss) {
    /* height_above_floatation / update_Haf!, src/topography.jl:36-39 */
    double m = zb - zss;
    if (m > 0) m = 0;
    double v = H + m * s->rho_sw_ice;
    return v > 0 ? v : 0.0;
}

/* ======================================================================
 * update_diagnostics!(dudt, u, sim, t), src/simulation.jl:335-393
 * ====================================================================== */
static int rhs_impl(or_sim* s, double t, double* u, double* dudt) {
    const fi_config* c = &s->cfg;
    const int nx = s->nx, ny = s->ny;
    const size_t n = (size_t)nx * ny;
    s->nf++;

    /* apply_bc!(u, viscous_displacement): CornerBC in RegularBCSpace */
    corner_bc(u, nx, ny, c->bc_viscous_border);
    /* update_bedrock!(sim, u), columnanom_mantle!(sim) */
    for (size_t k = 0; k < n; k++) {
        s->u[k] = u[k];
        s->z_b[k] = s->z_b_ref[k] + s->ue[k] + s->u[k];
        s->c_mantle[k] = c->rho_uppermantle * (s->u[k] - s->u_ref[k]);
    }
    /* apply_bc!(H_ice, t, ice_thickness) */
    if (c->ice_mode == FI_ICE_TIME_INTERPOLATED) {
        int rc = interp_ice_(s, t, s->H_ice);
        if (rc) return rc;
    }
    /* update_Haf!, columnanom_ice! */
    for (size_t k = 0; k < n; k++) {
        s->H_af[k] = haf_(s, s->H_ice[k], s->z_b[k], s->z_ss[k]);
        s->c_ice[k] = c->rho_ice * (s->H_af[k] - s->H_af_ref[k]);
    }
    const int gate = ((t - c->t0) / c->dt_sparse_diagnostics) >= (double)s->count_sparse;
    if (gate) {
        /* update_elasticresponse!, src/deformation.jl:175-189 */
        if (c->lithosphere == FI_LITHO_RIGID) {
            memset(s->ue, 0, n * sizeof(double));
        } else {
            for (size_t k = 0; k < n; k++) s->buf[k] = s->c_load[k]; /* * K^2, K == 1 */
            samesize_conv_ext(s, s->ue, s->buf, s->Ge_hat, c->bc_elastic_border);
        }
        /* columnanom_litho! */
        for (size_t k = 0; k < n; k++) s->c_litho[k] = c->rho_litho * (s->ue[k] - s->ue_ref[k]);
        /* internal_update_bsl!, src/sealevel.jl:242-262 */
        {
            int rc = internal_update_bsl_(s, t);
            if (rc) return rc;
        }
        /* update_dz_ss!(sim, surface), src/sealevel.jl:173-201 */
        if (c->sea_surface == FI_SEA_SURFACE_LATERALLY_VARIABLE) {
            if (c->lithosphere_column == FI_COLUMN_COMPRESSIBLE)
                for (size_t k = 0; k < n; k++) s->buf[k] = s->A * (s->c_load[k] + s->mask[k] * s->c_mantle[k]);
            else
                for (size_t k = 0; k < n; k++) s->buf[k] = s->A * s->c_full[k];
            samesize_conv_ext(s, s->dz_ss, s->buf, s->Gg_hat, c->bc_sea_surface_border);
        }
        /* update_z_ss!, update_Haf!, masks, columnanom_water!, columnanom_ice! */
        for (size_t k = 0; k < n; k++) {
            s->z_ss[k] = s->z_ss_ref[k] + s->dz_ss[k] + s->z_bsl;
            s->H_af[k] = haf_(s, s->H_ice[k], s->z_b[k], s->z_ss[k]);
        }
        masks_water_(s);
        for (size_t k = 0; k < n; k++) s->c_ice[k] = c->rho_ice * (s->H_af[k] - s->H_af_ref[k]);
        s->count_sparse += 1;
    }
    /* columnanom_load!, columnanom_full!, src/loads.jl:96-106 */
    for (size_t k = 0; k < n; k++) {
        s->c_load[k] = s->mask[k] * (s->c_ice[k] + s->c_sw[k] + s->c_sed[k]);
        s->c_full[k] = s->c_load[k] + s->mask[k] * (s->c_litho[k] + s->c_mantle[k]);
    }
    /* update_dudt!(dudt, u, sim, t, mantle, lithosphere), src/deformation.jl:21-103 */
    if (c->mantle == FI_MANTLE_RIGID) {
        memset(dudt, 0, n * sizeof(double)); /* RigidMantle: dudt .= 0 */
        memcpy(s->dudt, dudt, n * sizeof(double));
        return FI_OK;
    }
    if (c->mantle == FI_MANTLE_RELAXED) {
        if (c->lithosphere == FI_LITHO_LATERALLY_VARIABLE)
            return set_err(s, FI_ERR_UNSUPPORTED,
                           "Relaxed rheology is not implemented for laterally variable lithosphere.");
        /* ELRA (src/deformation.jl:29-45): u_eq = samesize_conv(-(load + litho) g K^2,
         * viscous Green) in the regular BC space, dudt = (u_eq - u) / tau */
        const int cx = 2 * nx - 1;
        for (size_t k = 0; k < n; k++) s->buf[k] = -(s->c_load[k] + s->c_litho[k]) * c->g;
        conv_full_(s, s->buf, s->Gv_hat, s->cropped);
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++)
                s->u_eq[i + (size_t)j * nx] = s->cropped[(s->i1 - 1 + i) + (size_t)(s->j1 - 1 + j) * cx];
        corner_bc(s->u_eq, nx, ny, c->bc_viscous_border);
        for (size_t k = 0; k < n; k++) dudt[k] = 1.0 / s->tau[k] * (s->u_eq[k] - s->u[k]);
        memcpy(s->dudt, dudt, n * sizeof(double));
        for (size_t k = 0; k < n; k++)
            if (!isfinite(dudt[k])) return set_err(s, FI_ERR_NONFINITE, "non-finite dudt");
        return FI_OK;
    }
    if (c->lithosphere == FI_LITHO_LATERALLY_CONSTANT) {
        /* MaxwellMantle with a laterally constant lithosphere (Bueler et al. 2007,
         * src/deformation.jl:52-89): one step of dt_min of the spectral scheme
         * U+ = ((nabla - dt/2 beta) U + dt F) / (nabla + dt/2 beta), nabla = 2 eta |k| R,
         * beta = rho_m g + D |k|^4, written into u in place; dudt is left as it is.
         * A rigid lithosphere keeps the laterally variable operator below with a zero
         * elastic response: src/deformation.jl:15 lists MaxwellMantle with
         * RigidLithosphere as not implemented, and the operator with u_e = 0 is the
         * behaviour both forms of this library share for it. */
        const double dt = c->dt_min * c->seconds_per_year;
        for (size_t k = 0; k < n; k++) {
            s->fftrhs[k].re = -(s->c_load[k] + s->c_litho[k]) * c->g; /* K == 1 */
            s->fftrhs[k].im = 0.0;
            s->fftU[k].re = u[k];
            s->fftU[k].im = 0.0;
        }
        fft2(&s->fx, &s->fy, s->fftrhs, nx, ny, 0);
        fft2(&s->fx, &s->fy, s->fftU, nx, ny, 0);
        for (size_t k = 0; k < n; k++) {
            const double pd = s->pseudodiff[k];
            const double nab = 2.0 * s->eta[k] * pd * s->R[k];
            const double beta = c->rho_uppermantle * c->g + s->D[k] * pd * pd * pd * pd;
            const double a = nab - dt / 2 * beta, b = nab + dt / 2 * beta;
            s->fftU[k].re = (a * s->fftU[k].re + dt * s->fftrhs[k].re) / b;
            s->fftU[k].im = (a * s->fftU[k].im + dt * s->fftrhs[k].im) / b;
        }
        fft2(&s->fx, &s->fy, s->fftU, nx, ny, 1);
        for (size_t k = 0; k < n; k++) u[k] = s->fftU[k].re;
        corner_bc(u, nx, ny, c->bc_viscous_border);
        memcpy(s->u, u, n * sizeof(double));
        memcpy(s->dudt, dudt, n * sizeof(double));
        return FI_OK;
    }
    /* update_dudt!(.., MaxwellMantle, LaterallyVariableLithosphere), deformation.jl:91-103 */
    /* update_deformation_rhs!(sim, u), deformation.jl:110-131 */
    const double nu = c->litho_poissonratio;
    for (size_t k = 0; k < n; k++) s->rhs[k] = -c->g * s->c_full[k];
    or_second_derivatives(nx, ny, s->dx, s->dy, u, s->bxx, s->byy, s->bx, s->bxy);
    for (size_t k = 0; k < n; k++) {
        s->Mxx[k] = -s->D[k] * (nu * s->byy[k] + s->bxx[k]);
        s->Myy[k] = -s->D[k] * (nu * s->bxx[k] + s->byy[k]);
        s->Mxy[k] = -s->D[k] * (1 - nu) * s->bxy[k];
    }
    dxx_(s->bxx, s->Mxx, nx, ny, s->dx);
    dyy_(s->byy, s->Myy, nx, ny, s->dy);
    dx_(s->bx, s->Mxy, nx, ny, s->dx);
    dy_(s->bxy, s->bx, nx, ny, s->dy);
    for (size_t k = 0; k < n; k++) s->rhs[k] += s->bxx[k] + (2 * s->bxy[k] + s->byy[k]);
    /* smooth_convo = EmptyConvolution: no-op */
    for (size_t k = 0; k < n; k++) {
        s->fftrhs[k].re = s->rhs[k] * 1.0 / (2 * s->eta[k]); /* K == 1 */
        s->fftrhs[k].im = 0.0;
    }
    fft2(&s->fx, &s->fy, s->fftrhs, nx, ny, 0);
    for (size_t k = 0; k < n; k++) { s->fftrhs[k].re *= s->spinv[k]; s->fftrhs[k].im *= s->spinv[k]; }
    fft2(&s->fx, &s->fy, s->fftrhs, nx, ny, 1);
    for (size_t k = 0; k < n; k++) dudt[k] = s->fftrhs[k].re * c->seconds_per_year;
    corner_bc(dudt, nx, ny, c->bc_viscous_border);
    memcpy(s->dudt, dudt, n * sizeof(double));
    for (size_t k = 0; k < n; k++)
        if (!isfinite(dudt[k])) return set_err(s, FI_ERR_NONFINITE, "non-finite dudt");
    return FI_OK;
}

static int rhs_cb(void* ctx, double t, double* u, double* du) { return rhs_impl((or_sim*)ctx, t, u, du); }

/* Simulation(...) tail (src/simulation.jl:129-156): GIATools, reference and current state. */
static int setup_(or_sim* s) {
    const fi_config* c = &s->cfg;
    const int nx = s->nx, ny = s->ny;
    const size_t n = (size_t)nx * ny;
    /* pseudodiff, src/domain.jl:151-155 and src/derivatives.jl:201-214 */
    double* fxv = dalloc(nx);
    double* fyv = dalloc(ny);
    fftint_(nx, fxv);
    fftint_(ny, fyv);
    const double mux = M_PI / c->Wx, muy = M_PI / c->Wy;
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            const double a = mux * fxv[i], b = muy * fyv[j];
            s->pseudodiff[i + (size_t)j * nx] = sqrt(a * a + b * b);
        }
    s->pseudodiff[0] = 1e-3 * ((s->pseudodiff[nx] + s->pseudodiff[1]) / 2);
    free(fxv); free(fyv);
    /* pseudodiff_scaling R (FreqDomainViscosityLumping) and scaled_pseudodiff_inv (solidearth.jl:222) */
    if (!s->R_given) {
        for (size_t k = 0; k < n; k++) s->R[k] = 1.0;
        for (int l = 0; l < s->n_ch; l++)
            for (size_t k = 0; k < n; k++) s->R[k] *= channel_scaling_(s->pseudodiff[k], s->ch_thick[l], s->ch_ratio[l]);
    }
    for (size_t k = 0; k < n; k++) s->spinv[k] = 1.0 / (s->R[k] * s->pseudodiff[k]);
    /* Green's functions and convolution plans, src/tools.jl:49-97 */
    if (c->lithosphere != FI_LITHO_RIGID) {
        if (s->n_table < 2) return set_err(s, FI_ERR_STATE, "elastic Green table not set");
        build_elastic_green_(s);
        conv_plan(s, s->Ge, s->Ge_hat);
    }
    build_geoid_green_(s);
    conv_plan(s, s->Gg, s->Gg_hat);
    if (c->mantle == FI_MANTLE_RELAXED) {
        build_viscous_green_(s);
        conv_plan(s, s->Gv, s->Gv_hat);
    }
    /* reference state, src/simulation.jl:132-151 */
    memset(s->H_ice_ref, 0, n * sizeof(double));
    if (c->ice_mode == FI_ICE_TIME_INTERPOLATED) {
        int rc = interp_ice_(s, c->t0, s->H_ice_ref);
        if (rc) return rc;
    }
    for (size_t k = 0; k < n; k++) {
        s->z_ss_ref[k] = c->z_bsl + s->dz_ss_ref[k];
        s->H_af_ref[k] = haf_(s, s->H_ice_ref[k], s->z_b_ref[k], s->z_ss_ref[k]);
    }
    /* CurrentState(domain, ref, z_bsl), src/state.jl:79-103 (u kept if set beforehand) */
    for (size_t k = 0; k < n; k++) {
        s->ue[k] = s->ue_ref[k];
        s->H_ice[k] = s->H_ice_ref[k];
        s->H_af[k] = s->H_af_ref[k];
        s->z_b[k] = s->z_b_ref[k];
        s->dz_ss[k] = 0.0;
        s->z_ss[k] = s->z_ss_ref[k];
        s->c_ice[k] = s->c_sw[k] = s->c_sed[k] = s->c_litho[k] = s->c_mantle[k] = s->c_load[k] = s->c_full[k] = 0.0;
        s->dudt[k] = 0.0;
    }
    /* ReferenceState masks and water column; CurrentState copies them */
    s->z_bsl = c->z_bsl;
    s->A_bsl = c->bsl_ref_A > 0 ? c->bsl_ref_A : 3.625e14;
    masks_water_(s);
    for (size_t k = 0; k < n; k++) s->c_sw[k] = 0.0; /* ColumnAnomalies start at zero */
    s->V_af = s->V_den = s->V_pov = s->delta_V = 0.0;
    s->count_sparse = 0;
    return FI_OK;
}

int or_init(or_sim* s) {
    if (!s) return FI_ERR_ARG;
    /* u defaults to copy(u_ref) unless set explicitly */
    const size_t n = (size_t)s->nx * s->ny;
    if (!s->u_set) memcpy(s->u, s->u_ref, n * sizeof(double));
    if (s->cfg.sealevel_load == FI_SEALEVEL_LOAD_INTERACTIVE) {
        double active = 0.0;
        for (size_t k = 0; k < n; k++) active += s->mask[k] != 0.0;
        if (active > 0.6 * (double)n)
            return set_err(s, FI_ERR_ARG, "Mask defining regions of active load must not cover more than 60%% "
                                          "of the cells when using an interactive sea level.");
    }
    int rc = setup_(s);
    if (rc) return rc;
    /* init_problem!: the volumes of the initial state, then the first
     * update_diagnostics! at t0 (forces the sparse update), src/simulation.jl:305-312 */
    update_volumes_(s);
    double* du = dalloc(n);
    rc = rhs_impl(s, s->cfg.t0, s->u, du);
    free(du);
    if (rc) return rc;
    s->initialized = 1;
    return FI_OK;
}

int or_rhs(or_sim* s, double t, double* u_inout, double* dudt_out) {
    if (!s || !u_inout || !dudt_out) return FI_ERR_ARG;
    if (!s->initialized) return set_err(s, FI_ERR_STATE, "or_init not called");
    return rhs_impl(s, t, u_inout, dudt_out);
}

/* ======================================================================
 * BS3 integrator with the OrdinaryDiffEq default adaptive machinery.
 * Tableau: src/integrators.jl:154-173 (Bogacki-Shampine 3(2)); controller,
 * initial dt, tstops and callback handling restate OrdinaryDiffEqCore:
 *   PIController(beta1 = 7/30, beta2 = 2/15), qmin = 1/5, qmax = 10, gamma = 9/10,
 *   qoldinit = 1e-4, EEst = RMS(utilde ./ (abstol + reltol*max(|uprev|,|u|))),
 *   accept iff EEst <= 1, initial dt by the Hairer-Norsett-Wanner heuristic.
 * ====================================================================== */
#define BS3_A21 0.5
#define BS3_A32 0.75
#define BS3_A41 (2.0 / 9.0)
#define BS3_A42 (1.0 / 3.0)
#define BS3_A43 (4.0 / 9.0)
#define BS3_C1 0.5
#define BS3_C2 0.75
#define BS3_BT1 (-5.0 / 72.0)
#define BS3_BT2 (1.0 / 12.0)
#define BS3_BT3 (1.0 / 9.0)
#define BS3_BT4 (-1.0 / 8.0)
#define PI_BETA1 (7.0 / 30.0)
#define PI_BETA2 (2.0 / 15.0)
#define CTRL_QMIN 0.2
#define CTRL_QMAX 10.0
#define CTRL_GAMMA 0.9
#define CTRL_QOLDINIT 1e-4

static inline double rms_(const double* a, int n) {
    double s = 0.0;
    for (int k = 0; k < n; k++) s += a[k] * a[k];
    return sqrt(s / n);
}

static double eps_(double x) { x = fabs(x); return nextafter(x, INFINITY) - x; }

static void integ_alloc(or_integ* I, int n) {
    I->n = n;
    double** bufs[] = {&I->u, &I->uprev, &I->k1, &I->k2, &I->k3, &I->k4, &I->tmp, &I->utilde};
    for (size_t k = 0; k < sizeof(bufs) / sizeof(bufs[0]); k++) {
        free(*bufs[k]);
        *bufs[k] = dalloc(n);
    }
}

static void tstop_add(or_integ* I, double ts) {
    if (!(ts > I->t0) || ts > I->t1) return;
    if (I->ntstops == I->captstops) {
        I->captstops = I->captstops ? 2 * I->captstops : 16;
        I->tstops = (double*)realloc(I->tstops, sizeof(double) * I->captstops);
    }
    int k = I->ntstops++;
    while (k > 0 && I->tstops[k - 1] > ts) { I->tstops[k] = I->tstops[k - 1]; k--; }
    I->tstops[k] = ts;
}

static void tstop_pop(or_integ* I) {
    memmove(I->tstops, I->tstops + 1, sizeof(double) * (I->ntstops - 1));
    I->ntstops--;
}

/* ode_determine_initdt (OrdinaryDiffEqCore initdt.jl), FSAL preamble first. */
static int integ_start(or_integ* I, const double* u0, double t0, double t1) {
    const int n = I->n;
    I->t0 = t0; I->t1 = t1; I->t = t0;
    I->dtmax = t1 - t0;
    I->dtmin = eps_(fabs(t0) > fabs(t1) ? t0 : t1);
    I->qold = CTRL_QOLDINIT; I->q11 = 1.0; I->EEst = 1.0;
    I->iter = 0; I->naccept = 0; I->nreject = 0;
    I->accept_step = 0; I->reeval_fsal = 0; I->u_modified = 0;
    I->ntstops = 0;
    tstop_add(I, t1);
    memcpy(I->u, u0, sizeof(double) * n);
    memcpy(I->uprev, u0, sizeof(double) * n);
    /* initialize!(integrator, ::BS3Cache): fsalfirst = f(uprev, t) */
    int rc = I->f(I->ctx, t0, I->uprev, I->k1);
    if (rc) return rc;
    if (I->euler) {
        /* solve(prob, Euler(); dt = dt_min, dtmin = dt_min, force_dtmin = true) */
        I->dt = I->dt_fixed;
        I->dtpropose = I->dt_fixed;
        I->initialized = 1;
        return FI_OK;
    }
    /* handle_dt! -> auto_dt_reset! -> ode_determine_initdt */
    double* sk = I->tmp;
    for (int k = 0; k < n; k++) sk[k] = I->abstol + fabs(I->u[k]) * I->reltol;
    rc = I->f(I->ctx, t0, I->u, I->k4); /* f0 into fsallast */
    if (rc) return rc;
    double d0 = 0.0, d1 = 0.0;
    for (int k = 0; k < n; k++) { double a = I->u[k] / sk[k]; d0 += a * a; a = I->k4[k] / sk[k]; d1 += a * a; }
    d0 = sqrt(d0 / n); d1 = sqrt(d1 / n);
    const double smalldt = 1e-6;
    double dt0 = (d0 < 1e-5 || d1 < 1e-5) ? smalldt : (d0 / d1) / 100;
    if (dt0 > I->dtmax) dt0 = I->dtmax;
    double dt;
    if (dt0 < 10 * 2.220446049250313e-16) {
        dt = smalldt > I->dtmin ? smalldt : I->dtmin;
    } else {
        double* u1 = I->utilde;
        double* f1 = I->k2;
        for (int k = 0; k < n; k++) u1[k] = I->u[k] + dt0 * I->k4[k];
        rc = I->f(I->ctx, t0 + dt0, u1, f1);
        if (rc) return rc;
        int same = 1;
        for (int k = 0; k < n; k++) if (f1[k] != I->k4[k]) { same = 0; break; }
        if (same) {
            dt = 100 * dt0 > I->dtmin ? 100 * dt0 : I->dtmin;
        } else {
            double d2 = 0.0;
            for (int k = 0; k < n; k++) { double a = (f1[k] - I->k4[k]) / sk[k]; d2 += a * a; }
            d2 = sqrt(d2 / n) / dt0;
            const double mx = d1 > d2 ? d1 : d2;
            double dt1;
            if (mx <= 1e-15) dt1 = (1e-6 > dt0 * 1e-3) ? 1e-6 : dt0 * 1e-3;
            else dt1 = pow(10.0, -(2 + log10(mx)) / 3.0);
            dt = 100 * dt0;
            if (dt1 < dt) dt = dt1;
            if (I->dtmax < dt) dt = I->dtmax;
            if (dt < I->dtmin) dt = I->dtmin;
        }
    }
    I->dt = dt;
    I->dtpropose = dt;
    I->initialized = 1;
    return FI_OK;
}

static double dtmin_at_(const or_integ* I) {
    const double e = eps_(I->t);
    return I->dtmin > e ? I->dtmin : e;
}

/* loopheader! + check_error! + perform_step!(BS3) + loopfooter! (one attempt) */
static int integ_attempt(or_integ* I) {
    const int n = I->n;
    int rc;
    /* _loopheader! */
    if (I->iter > 0) {
        if (I->accept_step) {
            /* apply_step!: uprev <- u, dt <- dtpropose, FSAL */
            memcpy(I->uprev, I->u, sizeof(double) * n);
            I->dt = I->dtpropose;
            if (I->reeval_fsal || I->u_modified) {
                rc = I->f(I->ctx, I->t, I->u, I->k1); /* reset_fsal! */
                if (rc) return rc;
            } else {
                memcpy(I->k1, I->k4, sizeof(double) * n);
            }
        } else {
            /* step_reject_controller!(PIController) */
            const double q = I->q11 / CTRL_GAMMA;
            I->dt /= (1.0 / CTRL_QMIN < q ? 1.0 / CTRL_QMIN : q);
        }
        /* a replayed sequence: this attempt takes the next recorded dt */
        if (I->replay_n > 0 && I->replay_i <= I->replay_n) {
            if (I->replay_i < I->replay_n) {
                I->dt = fabs(I->replay[I->replay_i]);
                I->dtpropose = I->dt;
            }
            I->replay_i++;
        }
    }
    I->iter += 1;
    /* fix_dt_at_bounds!, modify_dt_for_tstops! */
    if (I->dt > I->dtmax) I->dt = I->dtmax;
    {
        const double dm = dtmin_at_(I);
        if (I->dt < dm) I->dt = dm;
    }
    if (I->ntstops > 0) {
        const double rem = I->tstops[0] - I->t;
        if (rem < I->dt) I->dt = rem;
    }
    /* check_error! */
    if (I->max_steps > 0 && I->iter > I->max_steps) return FI_ERR_MAXITERS;
    if (!(I->dt == I->dt)) return FI_ERR_NONFINITE;
    if (I->dt <= I->dtmin) return FI_ERR_DT_UNDERFLOW;
    if (I->euler) {
        /* fixed step: the next attempt restarts from dt_min (dtcache), clipped at tstops */
        if (I->iter > 1 && !(I->replay_n > 0 && I->replay_i <= I->replay_n)) {
            I->dt = I->dt_fixed;
            if (I->ntstops > 0 && I->tstops[0] - I->t < I->dt) I->dt = I->tstops[0] - I->t;
        }
        /* perform_step!(integrator, ::EulerCache): u = uprev + dt k1; k4 = f(u, t + dt) (FSAL) */
        const double t = I->t, dt = I->dt;
        for (int k = 0; k < n; k++) I->u[k] = I->uprev[k] + dt * I->k1[k];
        if ((rc = I->f(I->ctx, t + dt, I->u, I->k4))) return rc;
        I->EEst = 0.0;
        I->reeval_fsal = 0;
        I->u_modified = 0;
        const double ttmp = I->t + I->dt;
        I->accept_step = 1;
        if (I->rec && I->rec_n < I->rec_cap) I->rec[I->rec_n] = I->dt;
        I->rec_n++;
        I->naccept++;
        if (I->ntstops > 0) {
            const double ts = I->tstops[0];
            const double big = I->t > ts ? I->t : ts;
            I->t = (fabs(ttmp - ts) < 100 * eps_(big)) ? ts : ttmp;
        } else {
            I->t = ttmp;
        }
        I->dtpropose = I->dt_fixed;
        if (I->nout > 0 && I->kout < I->nout && I->t >= I->tout[I->kout]) {
            if (I->record) I->record(I->ctx, I->kout, I->t);
            I->kout++;
            I->u_modified = 1;
            I->reeval_fsal = 1;
        }
        return FI_OK;
    }
    /* perform_step!(integrator, ::BS3Cache) */
    const double t = I->t, dt = I->dt;
    for (int k = 0; k < n; k++) I->tmp[k] = I->uprev[k] + dt * BS3_A21 * I->k1[k];
    if ((rc = I->f(I->ctx, t + BS3_C1 * dt, I->tmp, I->k2))) return rc;
    for (int k = 0; k < n; k++) I->tmp[k] = I->uprev[k] + dt * BS3_A32 * I->k2[k];
    if ((rc = I->f(I->ctx, t + BS3_C2 * dt, I->tmp, I->k3))) return rc;
    for (int k = 0; k < n; k++)
        I->u[k] = I->uprev[k] + dt * (BS3_A41 * I->k1[k] + BS3_A42 * I->k2[k] + BS3_A43 * I->k3[k]);
    if ((rc = I->f(I->ctx, t + dt, I->u, I->k4))) return rc;
    double acc = 0.0;
    for (int k = 0; k < n; k++) {
        const double ut = dt * (BS3_BT1 * I->k1[k] + BS3_BT2 * I->k2[k] + BS3_BT3 * I->k3[k] + BS3_BT4 * I->k4[k]);
        const double a = fabs(I->uprev[k]), b = fabs(I->u[k]);
        const double r = ut / (I->abstol + (a > b ? a : b) * I->reltol);
        acc += r * r;
    }
    I->EEst = sqrt(acc / n);
    if (!(I->EEst == I->EEst)) return FI_ERR_NONFINITE;
    /* _loopfooter! */
    I->reeval_fsal = 0;
    I->u_modified = 0;
    const double ttmp = I->t + I->dt;
    /* stepsize_controller!(PIController) */
    double q;
    if (I->EEst == 0.0) {
        q = 1.0 / CTRL_QMAX;
    } else {
        const double q11 = pow(I->EEst, PI_BETA1);
        q = q11 / pow(I->qold, PI_BETA2);
        I->q11 = q11;
        q = q / CTRL_GAMMA;
        if (q > 1.0 / CTRL_QMIN) q = 1.0 / CTRL_QMIN;
        if (q < 1.0 / CTRL_QMAX) q = 1.0 / CTRL_QMAX;
    }
    /* replay: this attempt took replay[replay_i - 1]; its sign is the decision */
    const int replay = I->replay_n > 0 && I->replay_i <= I->replay_n;
    I->accept_step = replay ? (I->replay[I->replay_i - 1] > 0.0) : (I->EEst <= 1.0);
    if (I->rec && I->rec_n < I->rec_cap) I->rec[I->rec_n] = I->accept_step ? I->dt : -I->dt;
    I->rec_n++;
    if (I->accept_step) {
        I->naccept++;
        /* step_accept_controller! */
        if (q == 1.0) q = 1.0;
        I->qold = I->EEst > CTRL_QOLDINIT ? I->EEst : CTRL_QOLDINIT;
        const double dtnew = I->dt / q;
        /* t update with snapping to the next tstop */
        if (I->ntstops > 0) {
            const double ts = I->tstops[0];
            const double big = I->t > ts ? I->t : ts;
            I->t = (fabs(ttmp - ts) < 100 * eps_(big)) ? ts : ttmp;
        } else {
            I->t = ttmp;
        }
        /* calc_dt_propose! */
        double dp = dtnew < I->dtmax ? dtnew : I->dtmax;
        const double dm = dtmin_at_(I);
        I->dtpropose = dp > dm ? dp : dm;
        /* handle_callbacks!: nout_condition / nout_affect! (src/simulation.jl:194-225) */
        if (I->nout > 0 && I->kout < I->nout && I->t >= I->tout[I->kout]) {
            if (I->record) I->record(I->ctx, I->kout, I->t);
            I->kout++;
            I->u_modified = 1;
            I->reeval_fsal = 1;
        }
    } else {
        I->nreject++;
    }
    return FI_OK;
}

/* solve!(integrator): step until every tstop is consumed */
static int integ_solve(or_integ* I) {
    while (I->ntstops > 0) {
        while (I->t < I->tstops[0]) {
            int rc = integ_attempt(I);
            if (rc) return rc;
        }
        while (I->ntstops > 0 && I->t == I->tstops[0]) tstop_pop(I); /* handle_tstop! */
        if (I->ntstops > 0 && I->t > I->tstops[0]) return FI_ERR_STATE;
    }
    return FI_OK;
}

/* step!(integrator, dt, true), SciMLBase: add a tstop and take accepted steps to it */
static int integ_step_to(or_integ* I, double dt) {
    const double next_t = I->t + dt;
    if (next_t > I->t1) return FI_ERR_ARG;
    tstop_add(I, next_t);
    while (I->t < next_t) {
        int rc;
        do {
            rc = integ_attempt(I);
            if (rc) return rc;
        } while (!I->accept_step);
        while (I->ntstops > 0 && I->t == I->tstops[0]) tstop_pop(I);
    }
    return FI_OK;
}

static void record_(void* ctx, int k, double t) {
    or_sim* s = (or_sim*)ctx;
    const size_t n = (size_t)s->nx * s->ny;
    if (s->out_t) s->out_t[k] = t;
    if (s->out_u) memcpy(s->out_u + (size_t)k * n, s->u, n * sizeof(double));
    if (s->out_ue) memcpy(s->out_ue + (size_t)k * n, s->ue, n * sizeof(double));
    if (s->out_dudt) memcpy(s->out_dudt + (size_t)k * n, s->dudt, n * sizeof(double));
    if (s->out_dz_ss) memcpy(s->out_dz_ss + (size_t)k * n, s->dz_ss, n * sizeof(double));
}

static int start_integrator_at_(or_sim* s, double t_start, int32_t n_tstops, const double* tstops);

static int start_integrator_(or_sim* s, int32_t n_tstops, const double* tstops) {
    return start_integrator_at_(s, s->cfg.t0, n_tstops, tstops);
}

static int start_integrator_at_(or_sim* s, double t_start, int32_t n_tstops, const double* tstops) {
    or_integ* I = &s->I;
    integ_alloc(I, s->nx * s->ny);
    I->f = rhs_cb;
    I->ctx = s;
    I->reltol = s->cfg.reltol;
    I->abstol = s->cfg.abstol;
    I->euler = s->cfg.alg == FI_ALG_EULER;
    I->dt_fixed = s->cfg.dt_min;
    if (I->euler && !(I->dt_fixed > 0))
        return set_err(s, FI_ERR_ARG, "The `dt_min` option is only compatible with the Euler algorithm.");
    I->max_steps = s->cfg.max_steps;
    I->record = record_;
    I->kout = 0;
    /* run! constructs the ODEProblem on sim.now.u after init_problem! */
    int rc = integ_start(I, s->u, t_start, s->cfg.t1);
    if (rc) return rc;
    for (int k = 0; k < n_tstops; k++) tstop_add(I, tstops[k]);
    return FI_OK;
}

int or_run(or_sim* s, int32_t n_out, const double* t_out, double* out_t, double* out_u, double* out_ue,
           double* out_dudt, double* out_dz_ss) {
    if (!s || n_out < 0 || (n_out > 0 && !t_out)) return FI_ERR_ARG;
    if (!s->initialized) return set_err(s, FI_ERR_STATE, "or_init not called");
    for (int k = 1; k < n_out; k++)
        if (t_out[k] < t_out[k - 1]) return set_err(s, FI_ERR_ARG, "t_out must be sorted");
    s->out_t = out_t; s->out_u = out_u; s->out_ue = out_ue; s->out_dudt = out_dudt; s->out_dz_ss = out_dz_ss;
    or_integ* I = &s->I;
    I->nout = n_out;
    I->tout = t_out;
    int rc = start_integrator_(s, n_out, t_out);
    if (rc) return set_err(s, rc, "integrator start failed (%d): %s", rc, s->err);
    rc = integ_solve(I);
    s->out_t = NULL; s->out_u = s->out_ue = s->out_dudt = s->out_dz_ss = NULL;
    I->nout = 0;
    if (rc) return set_err(s, rc, "run failed at t=%g (code %d) %s", I->t, rc, s->err);
    return FI_OK;
}

int or_init_integrator(or_sim* s, int32_t n_tstops, const double* tstops) {
    if (!s) return FI_ERR_ARG;
    if (!s->initialized) return set_err(s, FI_ERR_STATE, "or_init not called");
    /* init(prob; tstops = nout.t, callback): the output callback fires at the tstops
     * (forcing the FSAL re-evaluation) although nothing is recorded */
    free(s->tout_copy);
    s->tout_copy = dalloc(n_tstops);
    if (n_tstops) memcpy(s->tout_copy, tstops, sizeof(double) * n_tstops);
    s->out_t = NULL; s->out_u = s->out_ue = s->out_dudt = s->out_dz_ss = NULL;
    int rc = start_integrator_(s, n_tstops, tstops);
    s->I.nout = n_tstops;
    s->I.tout = s->tout_copy;
    s->I.kout = 0;
    return rc;
}

/* Resume at time t from a state computed elsewhere (u, ue, dz_ss and the sparse-update
 * count at t): the diagnostics of the last update_diagnostics! call at (t, u) are
 * rebuilt with the sparse gate held shut, then the integrator starts at t as
 * init_integrator does at t0 (initial dt heuristic, tstops with output callbacks).
 * Test infrastructure: times the oracle over a window that starts late in a run. */
int or_resume(or_sim* s, double t, int64_t count_sparse, const double* u, const double* ue, const double* dz_ss,
              int32_t n_tstops, const double* tstops) {
    if (!s || !u || !ue || !dz_ss || n_tstops < 0 || (n_tstops > 0 && !tstops)) return FI_ERR_ARG;
    if (!s->initialized) return set_err(s, FI_ERR_STATE, "or_init not called");
    const fi_config* c = &s->cfg;
    const size_t n = (size_t)s->nx * s->ny;
    memcpy(s->ue, ue, n * sizeof(double));
    memcpy(s->dz_ss, dz_ss, n * sizeof(double));
    for (size_t k = 0; k < n; k++) {
        s->c_litho[k] = c->rho_litho * (s->ue[k] - s->ue_ref[k]);
        s->z_ss[k] = s->z_ss_ref[k] + s->dz_ss[k] + c->z_bsl;
    }
    double* uu = dalloc(n);
    double* du = dalloc(n);
    memcpy(uu, u, n * sizeof(double));
    s->count_sparse = INT64_MAX; /* gate shut for the rebuild */
    int rc = rhs_impl(s, t, uu, du);
    s->count_sparse = count_sparse;
    free(uu);
    free(du);
    if (rc) return rc;
    free(s->tout_copy);
    s->tout_copy = dalloc(n_tstops);
    if (n_tstops) memcpy(s->tout_copy, tstops, sizeof(double) * n_tstops);
    s->out_t = NULL; s->out_u = s->out_ue = s->out_dudt = s->out_dz_ss = NULL;
    rc = start_integrator_at_(s, t, n_tstops, tstops);
    s->I.nout = n_tstops;
    s->I.tout = s->tout_copy;
    s->I.kout = 0;
    return rc;
}

int or_step(or_sim* s, double dt) {
    if (!s || !(dt > 0)) return FI_ERR_ARG;
    if (!s->I.initialized) return set_err(s, FI_ERR_STATE, "or_init_integrator not called");
    return integ_step_to(&s->I, dt);
}

int or_record_steps(or_sim* s, int64_t cap) {
    if (!s || cap < 0) return FI_ERR_ARG;
    if (!s->I.initialized) return set_err(s, FI_ERR_STATE, "or_init_integrator not called");
    free(s->I.rec);
    s->I.rec = cap > 0 ? dalloc((size_t)cap) : NULL;
    s->I.rec_cap = cap;
    s->I.rec_n = 0;
    return FI_OK;
}

int or_get_step_record(or_sim* s, double* dts, int64_t cap, int64_t* n) {
    if (!s || !n || cap < 0 || (cap > 0 && !dts)) return FI_ERR_ARG;
    int64_t k = s->I.rec_n < s->I.rec_cap ? s->I.rec_n : s->I.rec_cap;
    if (k > cap) k = cap;
    if (k > 0) memcpy(dts, s->I.rec, (size_t)k * sizeof(double));
    *n = s->I.rec_n;
    return FI_OK;
}

int or_set_step_replay(or_sim* s, int64_t n, const double* dts) {
    if (!s || n < 0 || (n > 0 && !dts)) return FI_ERR_ARG;
    if (!s->I.initialized) return set_err(s, FI_ERR_STATE, "or_init_integrator not called");
    free(s->I.replay);
    s->I.replay = NULL;
    if (n > 0) {
        s->I.replay = dalloc((size_t)n);
        memcpy(s->I.replay, dts, (size_t)n * sizeof(double));
        s->I.dt = fabs(dts[0]);
        s->I.dtpropose = fabs(dts[0]);
    }
    s->I.replay_n = n;
    s->I.replay_i = n > 0 ? 1 : 0;
    return FI_OK;
}

int or_get_stats(or_sim* s, fi_stats* st) {
    if (!s || !st) return FI_ERR_ARG;
    memset(st, 0, sizeof(*st));
    st->t = s->I.initialized ? s->I.t : s->cfg.t0;
    st->dt = s->I.dtpropose;
    st->nf = s->nf;
    st->naccept = s->I.naccept;
    st->nreject = s->I.nreject;
    st->nsparse = s->count_sparse;
    st->status = 0;
    st->form = -1;
    return FI_OK;
}

/* ======================================================================
 * Known-answer helpers
 * ====================================================================== */
int or_fft2(int32_t nx, int32_t ny, const double* in_re, const double* in_im, double* out_re, double* out_im,
            int32_t inverse) {
    or_fft px, py;
    fft_plan_init(&px, nx);
    fft_plan_init(&py, ny);
    const size_t n = (size_t)nx * ny;
    cpx* a = (cpx*)malloc(sizeof(cpx) * n);
    for (size_t k = 0; k < n; k++) { a[k].re = in_re[k]; a[k].im = in_im ? in_im[k] : 0.0; }
    fft2(&px, &py, a, nx, ny, inverse);
    for (size_t k = 0; k < n; k++) { out_re[k] = a[k].re; out_im[k] = a[k].im; }
    free(a);
    fft_plan_free(&px);
    fft_plan_free(&py);
    return FI_OK;
}

int or_conv_full(int32_t nx, int32_t ny, const double* kernel, const double* input, double* out) {
    fi_config cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.nx = nx; cfg.ny = ny; cfg.Wx = 1.0; cfg.Wy = 1.0;
    or_sim* s = NULL;
    int rc = or_create(&cfg, &s);
    if (rc) return rc;
    conv_plan(s, kernel, s->Ge_hat);
    conv_full_(s, input, s->Ge_hat, out);
    or_destroy(s);
    return FI_OK;
}

typedef struct { double lambda; } decay_ctx;
static int decay_f(void* ctx, double t, double* u, double* du) {
    (void)t;
    du[0] = ((decay_ctx*)ctx)->lambda * u[0];
    return FI_OK;
}
typedef struct { double* u_out; or_integ* I; } decay_rec;

int or_bs3_decay(double lambda, double u0, double t1, double reltol, double abstol, int32_t n_out,
                 const double* t_out, double* u_out, int64_t* nsteps) {
    or_integ I;
    memset(&I, 0, sizeof(I));
    integ_alloc(&I, 1);
    decay_ctx ctx = {lambda};
    I.f = decay_f;
    I.ctx = &ctx;
    I.reltol = reltol;
    I.abstol = abstol;
    double u = u0;
    int rc = integ_start(&I, &u, 0.0, t1);
    for (int k = 0; k < n_out && !rc; k++) {
        if (t_out[k] > I.t) rc = integ_step_to(&I, t_out[k] - I.t);
        u_out[k] = I.u[0];
    }
    if (nsteps) *nsteps = I.naccept + I.nreject;
    free(I.u); free(I.uprev); free(I.k1); free(I.k2); free(I.k3); free(I.k4); free(I.tmp); free(I.utilde);
    free(I.tstops);
    return rc;
}
