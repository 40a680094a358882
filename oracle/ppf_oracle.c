/*
 * ppf_oracle.c -- CPU restatement of the PaScaL_POISSON_FFT solve path.
 *
 * TEST INFRASTRUCTURE ONLY (the parity checker).  tests/, smoke() and the
 * CPU-baseline leg of bench.py load this library; the CUDA product never
 * does.  Each routine names the reference file:line it restates.
 *
 * The reference delegates its FFTs to FFTW (CPU, Intel MKL wrappers,
 * 01_Fortran/examples/Makefile:28-30) and cuFFT (GPU,
 * 01_Fortran/src/fft_3d_poisson.f90:195-286).  Neither is vendored, so this
 * file carries its own unnormalised DFT (Stockham, radix 2/3/4/5 plus a
 * generic prime butterfly) with the same sign and scaling conventions:
 * forward e^{-2 pi i jk/n}, backward e^{+2 pi i jk/n}, no 1/n.
 */
#include "ppf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { double re, im; } cd;

static const long double PI_L = 3.141592653589793238462643383279502884L;
static const double PI_D = 3.141592653589793238462643383279502884;

/* ------------------------------------------------------------------------ */
/* mesh: 01_Fortran/examples/mpi_subdomain.f90:397-472                      */
/* ------------------------------------------------------------------------ */
void ora_mesh(int nm, double L, int uniform, double gamma, int pbc,
              double *x, double *dx, double *dmx)
{
    const int n = nm + 1;
    /* calculate_x: idx = sta-1 .. end+1 with sta=1, end=nm -> x(0..nm+1) */
    for (int idx = 0; idx <= nm + 1; ++idx) {
        if (uniform) {
            /* uniform_grid :440-450 */
            x[idx] = (double)(idx - 1) * L / (double)nm;
        } else {
            /* non_uniform_channel_grid :426-438 */
            x[idx] = L * 0.5 * (1.0 + tanh(0.5 * gamma * (2.0 * (double)(idx - 1) / (double)nm - 1.0))
                                          / tanh(gamma * 0.5));
        }
    }
    if (!pbc) x[0] = x[1];                                   /* :415 */

    /* calculate_dx_dmx :452-472 at one rank */
    for (int i = 0; i <= n; ++i) { dx[i] = 0.0; dmx[i] = 0.0; }
    for (int i = 1; i <= nm; ++i) dx[i] = x[i + 1] - x[i];
    if (pbc) { dx[0] = dx[nm]; dx[n] = dx[1]; }              /* ghostcell_1d :783-798 */
    else     { dx[0] = 0.0;    dx[n] = 0.0; }
    for (int i = 1; i <= nm; ++i) dmx[i] = 0.5 * (dx[i - 1] + dx[i]);
    if (pbc) { dmx[0] = dmx[nm]; dmx[n] = dmx[1]; }
    else     { dmx[n] = 0.5 * (dx[nm] + dx[n]); }
}

/* ------------------------------------------------------------------------ */
/* modified wavenumbers: 01_Fortran/src/fft_3d_poisson.f90:288-351          */
/* ------------------------------------------------------------------------ */
static double wn_dct(int m, int n, double h)
{
    double s = sin(0.5 * (double)m * PI_D / (double)n);
    return 4.0 * (s * s) / (h * h);
}
static double wn_fft(int m, int n, double h)
{
    return 2.0 * (1.0 - cos(2.0 * (double)m * PI_D / (double)n)) / (h * h);
}

void ora_wavenumbers(int n1m, int n2m, double L1, double L2, int pbc1, int pbc2,
                     double *dxk2, double *dyk2)
{
    const double h1 = L1 / (double)n1m, h2 = L2 / (double)n2m;
    for (int i = 1; i <= n1m; ++i)
        dxk2[i - 1] = pbc1 ? wn_fft(i - 1, n1m, h1) : wn_dct(i - 1, n1m, h1);
    for (int j = 1; j <= n2m; ++j) {
        if (!pbc2) { dyk2[j - 1] = wn_dct(j - 1, n2m, h2); continue; }
        int jm = j - 1;
        /* the periodic-periodic branch folds j > n2m/2+1 (:339-346);
           the Neumann-periodic branch does not (:316-320) */
        if (pbc1 && j > n2m / 2 + 1) jm = n2m - j + 1;
        dyk2[j - 1] = wn_fft(jm, n2m, h2);
    }
}

/* ------------------------------------------------------------------------ */
/* Thomas solvers: 01_Fortran/PaScaL_TDMA/src/tdmas.f90                      */
/* ------------------------------------------------------------------------ */
#define A2(arr, i, j) arr[(size_t)(j) * (size_t)n_sys + (size_t)(i)]

void ora_tdma_many(double *a, double *b, double *c, double *d, int n_sys, int n_row)
{
    /* tdmas.f90:114-147 */
    for (int i = 0; i < n_sys; ++i) {
        A2(d, i, 0) = A2(d, i, 0) / A2(b, i, 0);
        A2(c, i, 0) = A2(c, i, 0) / A2(b, i, 0);
    }
    for (int j = 1; j < n_row; ++j)
        for (int i = 0; i < n_sys; ++i) {
            double r = 1.0 / (A2(b, i, j) - A2(a, i, j) * A2(c, i, j - 1));
            A2(d, i, j) = r * (A2(d, i, j) - A2(a, i, j) * A2(d, i, j - 1));
            A2(c, i, j) = r * A2(c, i, j);
        }
    for (int j = n_row - 2; j >= 0; --j)
        for (int i = 0; i < n_sys; ++i)
            A2(d, i, j) = A2(d, i, j) - A2(c, i, j) * A2(d, i, j + 1);
}

void ora_tdma_cycl_many(double *a, double *b, double *c, double *d, int n_sys, int n_row)
{
    /* tdmas.f90:160-213 */
    const int n2 = n_row;
    double *e = (double *)calloc((size_t)n_sys * (size_t)n_row, sizeof(double));
    for (int i = 0; i < n_sys; ++i) {
        A2(e, i, 1) = -A2(a, i, 1);
        A2(e, i, n2 - 1) = -A2(c, i, n2 - 1);
    }
    for (int i = 0; i < n_sys; ++i) {
        A2(d, i, 1) = A2(d, i, 1) / A2(b, i, 1);
        A2(e, i, 1) = A2(e, i, 1) / A2(b, i, 1);
        A2(c, i, 1) = A2(c, i, 1) / A2(b, i, 1);
    }
    for (int j = 2; j < n2; ++j)
        for (int i = 0; i < n_sys; ++i) {
            double rr = 1.0 / (A2(b, i, j) - A2(a, i, j) * A2(c, i, j - 1));
            A2(d, i, j) = rr * (A2(d, i, j) - A2(a, i, j) * A2(d, i, j - 1));
            A2(e, i, j) = rr * (A2(e, i, j) - A2(a, i, j) * A2(e, i, j - 1));
            A2(c, i, j) = rr * A2(c, i, j);
        }
    for (int j = n2 - 2; j >= 1; --j)
        for (int i = 0; i < n_sys; ++i) {
            A2(d, i, j) = A2(d, i, j) - A2(c, i, j) * A2(d, i, j + 1);
            A2(e, i, j) = A2(e, i, j) - A2(c, i, j) * A2(e, i, j + 1);
        }
    for (int i = 0; i < n_sys; ++i)
        A2(d, i, 0) = (A2(d, i, 0) - A2(a, i, 0) * A2(d, i, n2 - 1) - A2(c, i, 0) * A2(d, i, 1))
                    / (A2(b, i, 0) + A2(a, i, 0) * A2(e, i, n2 - 1) + A2(c, i, 0) * A2(e, i, 1));
    for (int j = 1; j < n2; ++j)
        for (int i = 0; i < n_sys; ++i)
            A2(d, i, j) = A2(d, i, j) + A2(d, i, 0) * A2(e, i, j);
    free(e);
}
#undef A2

/* ------------------------------------------------------------------------ */
/* DFT (stand-in for FFTW / cuFFT)                                          */
/* ------------------------------------------------------------------------ */
typedef struct {
    int n, nf;
    int f[40];
    cd *tw;           /* tw[k] = exp(-2 pi i k / n), k = 0..n-1 */
} fft_plan;

static void exp_table(int n, cd *tw)
{
    for (int k = 0; k < n; ++k) {
        long double a = -2.0L * PI_L * (long double)k / (long double)n;
        tw[k].re = (double)cosl(a);
        tw[k].im = (double)sinl(a);
    }
}

static int fft_plan_init(fft_plan *p, int n)
{
    if (n < 1) return -1;
    p->n = n; p->nf = 0;
    int m = n;
    while (m % 4 == 0) { p->f[p->nf++] = 4; m /= 4; }
    while (m % 2 == 0) { p->f[p->nf++] = 2; m /= 2; }
    while (m % 3 == 0) { p->f[p->nf++] = 3; m /= 3; }
    while (m % 5 == 0) { p->f[p->nf++] = 5; m /= 5; }
    for (int q = 7; m > 1; q += 2)
        while (m % q == 0) { p->f[p->nf++] = q; m /= q; }
    p->tw = (cd *)malloc(sizeof(cd) * (size_t)n);
    if (!p->tw) return -1;
    exp_table(n, p->tw);
    return 0;
}
static void fft_plan_free(fft_plan *p) { free(p->tw); p->tw = NULL; }

static inline cd cmul(cd a, cd b) { cd r = { a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re }; return r; }
static inline cd cconj(cd a) { cd r = { a.re, -a.im }; return r; }

/* One Stockham autosort pass of radix R over a length-n sequence.
 * Ns = product of the radices already applied. */
static void fft_pass(const cd *in, cd *out, const fft_plan *p, int R, int Ns, int sign)
{
    const int n = p->n, nb = n / R;
    const long long tstep = n / (Ns * R);
    cd v[R], V[R];   /* R <= n: variable-length arrays */
    for (int j = 0; j < nb; ++j) {
        const int k = j % Ns;
        for (int q = 0; q < R; ++q) {
            cd w = p->tw[(long long)q * k * tstep % n];
            if (sign > 0) w = cconj(w);
            v[q] = cmul(in[j + q * nb], w);
        }
        if (R == 2) {
            V[0].re = v[0].re + v[1].re; V[0].im = v[0].im + v[1].im;
            V[1].re = v[0].re - v[1].re; V[1].im = v[0].im - v[1].im;
        } else {
            for (int pp = 0; pp < R; ++pp) {
                cd s = { 0.0, 0.0 };
                for (int q = 0; q < R; ++q) {
                    cd w = p->tw[(long long)((pp * q) % R) * nb];
                    if (sign > 0) w = cconj(w);
                    cd t = cmul(v[q], w);
                    s.re += t.re; s.im += t.im;
                }
                V[pp] = s;
            }
        }
        const int base = (j / Ns) * Ns * R + k;
        for (int pp = 0; pp < R; ++pp) out[base + pp * Ns] = V[pp];
    }
}

/* in-place transform of a contiguous complex sequence; work has n entries */
static void fft_exec(const fft_plan *p, cd *x, cd *work, int sign)
{
    cd *src = x, *dst = work;
    int Ns = 1;
    for (int s = 0; s < p->nf; ++s) {
        fft_pass(src, dst, p, p->f[s], Ns, sign);
        Ns *= p->f[s];
        cd *t = src; src = dst; dst = t;
    }
    if (src != x) memcpy(x, src, sizeof(cd) * (size_t)p->n);
}

int ora_fft_c2c(double *data, int n, int sign)
{
    fft_plan p;
    if (fft_plan_init(&p, n)) return -1;
    cd *w = (cd *)malloc(sizeof(cd) * (size_t)n);
    fft_exec(&p, (cd *)data, w, sign);
    free(w);
    fft_plan_free(&p);
    return 0;
}

/* Per-thread workspace for the line transforms of one axis length n. */
typedef struct {
    int n;              /* real length (even) */
    fft_plan half;      /* complex FFT of length n/2 (real transforms) */
    fft_plan full;      /* complex FFT of length n (complex lines) */
    cd *tw_n;           /* exp(-2 pi i k / n), k = 0..n-1 */
    cd *buf, *work;     /* n entries each */
    double *rbuf;       /* n+1 reals */
    cd *cs;             /* n/2+1 complex: half spectrum of the DCT lines */
    double *ry;         /* n reals: line scratch */
} axis_ws;

static int axis_ws_init(axis_ws *w, int n)
{
    memset(w, 0, sizeof(*w));
    w->n = n;
    if (fft_plan_init(&w->half, n / 2) || fft_plan_init(&w->full, n)) return -1;
    w->tw_n = (cd *)malloc(sizeof(cd) * (size_t)n);
    w->buf = (cd *)malloc(sizeof(cd) * (size_t)(n + 1));
    w->work = (cd *)malloc(sizeof(cd) * (size_t)(n + 1));
    w->rbuf = (double *)malloc(sizeof(double) * (size_t)(n + 2));
    w->cs = (cd *)malloc(sizeof(cd) * (size_t)(n / 2 + 1));
    w->ry = (double *)malloc(sizeof(double) * (size_t)n);
    exp_table(n, w->tw_n);
    return 0;
}
static void axis_ws_free(axis_ws *w)
{
    fft_plan_free(&w->half); fft_plan_free(&w->full);
    free(w->tw_n); free(w->buf); free(w->work); free(w->rbuf);
    free(w->cs); free(w->ry);
}

/* unnormalised real-to-complex transform of a strided real line:
 * X_k = sum_j x_j e^{-2 pi i jk/n}, k = 0..n/2 (cuFFT D2Z / FFTW r2c) */
static void r2c_line(axis_ws *w, const double *x, long sx, cd *X, long sX)
{
    const int n = w->n, m = n / 2;
    cd *z = w->buf;
    for (int j = 0; j < m; ++j) { z[j].re = x[(2 * j) * sx]; z[j].im = x[(2 * j + 1) * sx]; }
    fft_exec(&w->half, z, w->work, -1);
    for (int k = 0; k <= m; ++k) {
        cd zk = z[k % m], zc = cconj(z[(m - k) % m]);
        cd E = { 0.5 * (zk.re + zc.re), 0.5 * (zk.im + zc.im) };
        cd D = { zk.re - zc.re, zk.im - zc.im };          /* = 2 i O_k */
        cd O = { 0.5 * D.im, -0.5 * D.re };               /* D / (2i) */
        cd t = cmul(w->tw_n[k % n], O);
        X[k * sX].re = E.re + t.re;
        X[k * sX].im = E.im + t.im;
    }
}

/* unnormalised complex-to-real transform (cuFFT Z2D / FFTW c2r):
 * x_j = sum_{k=0}^{n-1} X_k e^{+2 pi i jk/n} with X_{n-k} = conj(X_k);
 * the imaginary parts of X_0 and X_{n/2} are ignored. */
static void c2r_line(axis_ws *w, const cd *X, long sX, double *x, long sx)
{
    const int n = w->n, m = n / 2;
    cd *Z = w->buf;
    for (int k = 0; k < m; ++k) {
        cd xk = X[k * sX], xc = cconj(X[(m - k) * sX]);
        if (k == 0) { xk.im = 0.0; xc.im = 0.0; }
        cd E = { xk.re + xc.re, xk.im + xc.im };
        cd D = { xk.re - xc.re, xk.im - xc.im };
        cd O = cmul(D, cconj(w->tw_n[k]));                 /* 2 O_k */
        Z[k].re = E.re - O.im;                             /* E + i O */
        Z[k].im = E.im + O.re;
    }
    fft_exec(&w->half, Z, w->work, +1);
    for (int j = 0; j < m; ++j) { x[(2 * j) * sx] = Z[j].re; x[(2 * j + 1) * sx] = Z[j].im; }
}

/* DCT-II by Makhoul's reordering:
 * cuda_Poisson_DCT_f_pre (fft_3d_poisson.f90:915-935), D2Z, and
 * cuda_Poisson_DCT_f_post (:937-969).  X_k = 2 sum_j x_j cos(pi k (2j+1)/(2n)). */
static void dct2_line(axis_ws *w, const double *x, long sx, double *X, long sX)
{
    const int n = w->n, h = n / 2;
    double *v = w->rbuf;
    for (int i = 1; i <= h; ++i) {
        v[i - 1] = x[(2 * i - 1 - 1) * sx];
        v[i + h - 1] = x[(2 * (n - (i + h) + 1) - 1) * sx];
    }
    cd *Vs = w->cs;
    r2c_line(w, v, 1, Vs, 1);
    for (int i = 1; i <= h; ++i) {
        double arg = -PI_D * (double)(i - 1) / (2.0 * (double)n);
        X[(i - 1) * sX] = 2.0 * (cos(arg) * Vs[i - 1].re - sin(arg) * Vs[i - 1].im);
    }
    for (int i = h + 1; i <= n; ++i) {
        double arg = -PI_D * (double)(i - 1) / (2.0 * (double)n);
        X[(i - 1) * sX] = 2.0 * (cos(arg) * Vs[n - i + 1].re + sin(arg) * Vs[n - i + 1].im);
    }
}

/* Inverse DCT without the 1/(2n) factor:
 * cuda_Poisson_DCT_b_pre (fft_3d_poisson.f90:971-1011), Z2D, and
 * cuda_Poisson_DCT_b_post (:1013-1033). */
static void idct_line(axis_ws *w, const double *X, long sX, double *x, long sx)
{
    const int n = w->n, h = n / 2;
    double *in2 = w->rbuf;
    for (int i = 0; i < n; ++i) in2[i] = X[i * sX];
    in2[n] = 0.0;
    cd *Zs = w->cs;
    for (int i = 1; i <= h + 1; ++i) {
        double arg = -PI_D * (double)(i - 1) / (2.0 * (double)n);
        Zs[i - 1].re = cos(arg) * in2[i - 1] - sin(arg) * in2[n + 2 - i - 1];
        Zs[i - 1].im = -sin(arg) * in2[i - 1] - cos(arg) * in2[n + 2 - i - 1];
    }
    double *y = w->ry;
    c2r_line(w, Zs, 1, y, 1);
    for (int i = 1; i <= h; ++i) {
        x[(2 * i - 1 - 1) * sx] = y[i - 1];
        x[(2 * (n - (i + h) + 1) - 1) * sx] = y[i + h - 1];
    }
}

/* complex transform of a strided complex line */
static void c2c_line(axis_ws *w, cd *X, long sX, int sign)
{
    const int n = w->n;
    cd *z = w->buf;
    for (int j = 0; j < n; ++j) z[j] = X[j * sX];
    fft_exec(&w->full, z, w->work, sign);
    for (int j = 0; j < n; ++j) X[j * sX] = z[j];
}

/* ------------------------------------------------------------------------ */
/* ghost cells: fft_3d_poisson.f90:798-852 then :666-796                     */
/* ------------------------------------------------------------------------ */
void ora_fill_ghosts(int n1m, int n2m, int n3m, int pbc1, int pbc2, int pbc3,
                     double *P, const double *dmx1, const double *dmx2,
                     const double *dmx3)
{
    const int n1 = n1m + 1, n2 = n2m + 1, n3 = n3m + 1;
    const long s1 = 1, s2 = (long)(n1 + 1), s3 = (long)(n1 + 1) * (n2 + 1);
#define PX(i, j, k) P[(long)(i) * s1 + (long)(j) * s2 + (long)(k) * s3]
    const int pbc[3] = { pbc1, pbc2, pbc3 };
    const int nsub[3] = { n1, n2, n3 };
    const double *dmx[3] = { dmx1, dmx2, dmx3 };
    /* apply_bc_on_direction for non-periodic axes, in x, y, z order */
    for (int dir = 0; dir < 3; ++dir) {
        if (pbc[dir]) continue;
        const double *dm = dmx[dir];
        const int na = nsub[dir], nma = na - 1;
        double sl = dm[1] + dm[2];
        double a_lo = (sl * sl) / ((sl * sl) - dm[1] * dm[1]);
        double b_lo = (dm[1] * dm[1]) / ((sl * sl) - dm[1] * dm[1]);
        double su = dm[na] + dm[nma];
        double a_hi = (su * su) / ((su * su) - dm[na] * dm[na]);
        double b_hi = (dm[na] * dm[na]) / ((su * su) - dm[na] * dm[na]);
        if (dir == 0) {
            for (int c = 0; c <= n3; ++c) for (int b = 0; b <= n2; ++b) {
                PX(0, b, c) = a_lo * PX(1, b, c) - b_lo * PX(2, b, c);
                PX(na, b, c) = a_hi * PX(nma, b, c) - b_hi * PX(na - 2, b, c);
            }
        } else if (dir == 1) {
            for (int c = 0; c <= n3; ++c) for (int b = 0; b <= n1; ++b) {
                PX(b, 0, c) = a_lo * PX(b, 1, c) - b_lo * PX(b, 2, c);
                PX(b, na, c) = a_hi * PX(b, nma, c) - b_hi * PX(b, na - 2, c);
            }
        } else {
            for (int c = 0; c <= n2; ++c) for (int b = 0; b <= n1; ++b) {
                PX(b, c, 0) = a_lo * PX(b, c, 1) - b_lo * PX(b, c, 2);
                PX(b, c, na) = a_hi * PX(b, c, nma) - b_hi * PX(b, c, na - 2);
            }
        }
    }
    /* ghostcell_update_on_direction for periodic axes at nprocs=1:
       ghost 0 <- plane n-1, ghost n <- plane 1 (x, y, z order) */
    for (int dir = 0; dir < 3; ++dir) {
        if (!pbc[dir]) continue;
        const int na = nsub[dir];
        if (dir == 0) {
            for (int c = 0; c <= n3; ++c) for (int b = 0; b <= n2; ++b) {
                double s0 = PX(1, b, c), s1v = PX(na - 1, b, c);
                PX(0, b, c) = s1v; PX(na, b, c) = s0;
            }
        } else if (dir == 1) {
            for (int c = 0; c <= n3; ++c) for (int b = 0; b <= n1; ++b) {
                double s0 = PX(b, 1, c), s1v = PX(b, na - 1, c);
                PX(b, 0, c) = s1v; PX(b, na, c) = s0;
            }
        } else {
            for (int c = 0; c <= n2; ++c) for (int b = 0; b <= n1; ++b) {
                double s0 = PX(b, c, 1), s1v = PX(b, c, na - 1);
                PX(b, c, 0) = s1v; PX(b, c, na) = s0;
            }
        }
    }
#undef PX
}

/* ------------------------------------------------------------------------ */
/* the solve: cuda_Poisson_FFT_1D, fft_3d_poisson.f90:353-626                 */
/* ------------------------------------------------------------------------ */

/* z-direction coefficients of cuda_Poisson_TDMA_z_{real,complex}
 * (:1137-1161, :1215-1254): am at k=1 and ap at k=n3m are zero at one rank
 * whether or not z is periodic. */
static void z_coeffs(int n3m, const double *dx3, const double *dmx3, double *am, double *ap)
{
    for (int k = 1; k <= n3m; ++k) {
        am[k - 1] = 1.0 / dx3[k] / dmx3[k];
        ap[k - 1] = 1.0 / dx3[k] / dmx3[k + 1];
        if (k == 1) am[k - 1] = 0.0;
        if (k == n3m) ap[k - 1] = 0.0;
    }
}

/* Solve one block of systems (system index fastest, nz rows) whose diagonal
 * is ac - lx[s] - ly[s] (evaluated left to right, as
 * `b = ac - dxk2(i) - dyk2(j)` at fft_3d_poisson.f90:1146, 1233, 1294);
 * pin applies to system `pin_sys` (or none if < 0).  d is overwritten with
 * the solution.  pbc3 selects the cyclic solver (cuda_ptdma_core :898-913). */
static void solve_block(int nsys, int nz, const double *am, const double *ap,
                        const double *lx, const double *ly, int pin_sys, int pbc3, double *d)
{
    size_t N = (size_t)nsys * nz;
    double *a = (double *)malloc(N * sizeof(double));
    double *b = (double *)malloc(N * sizeof(double));
    double *c = (double *)malloc(N * sizeof(double));
    for (int k = 0; k < nz; ++k) {
        const double ac = -am[k] - ap[k];
        for (int s = 0; s < nsys; ++s) {
            size_t id = (size_t)k * nsys + s;
            a[id] = am[k];
            b[id] = ac - lx[s] - ly[s];
            c[id] = ap[k];
        }
    }
    if (pin_sys >= 0) {
        a[pin_sys] = 0.0; b[pin_sys] = 1.0; c[pin_sys] = 0.0; d[pin_sys] = 0.0;
    }
    if (pbc3) ora_tdma_cycl_many(a, b, c, d, nsys, nz);
    else      ora_tdma_many(a, b, c, d, nsys, nz);
    free(a); free(b); free(c);
}

static int nthreads_set(int nt)
{
#ifdef _OPENMP
    if (nt > 0) omp_set_num_threads(nt);
    return omp_get_max_threads();
#else
    (void)nt; return 1;
#endif
}

#ifdef _OPENMP
#define OMP_FOR _Pragma("omp for schedule(static)")
#define OMP_PARALLEL _Pragma("omp parallel")
#else
#define OMP_FOR
#define OMP_PARALLEL
#endif

/* Wall-clock stamps of the last ora_poisson_solve: start, then before each of
 * its parallel regions (forward transforms, z solves, inverse transforms),
 * before the mean removal and at the end.  ora_last_stage_seconds() turns
 * them into the reference's timer stages (01_Fortran/examples/main.f90:65-78:
 * build TDMA + transforms, TDMA, update solution). */
static double g_stamps[16];
static int g_nstamp = 0;
#ifdef _OPENMP
#define ORA_STAMP() do { if (g_nstamp < 16) g_stamps[g_nstamp++] = omp_get_wtime(); } while (0)
#else
#define ORA_STAMP() do { } while (0)
#endif

/* Seconds of the last solve per stage: [0] set-up (wavenumbers, z
 * coefficients), [1] forward x/y transforms, [2] z tridiagonal solves,
 * [3] inverse y/x transforms, [4] mean removal and ghost cells.  Returns the
 * number of stamps taken (6 when every stage was seen). */
int ora_last_stage_seconds(double *out)
{
    for (int i = 0; i < 5; ++i) out[i] = 0.0;
    if (g_nstamp != 6) return g_nstamp;
    /* stamps: start, before the forward transforms, the z solves, the inverse
       transforms, the mean removal, and the end */
    for (int i = 0; i < 5; ++i) out[i] = g_stamps[i + 1] - g_stamps[i];
    return g_nstamp;
}

int ora_poisson_solve(int n1m, int n2m, int n3m, double L1, double L2,
                      int pbc1, int pbc2, int pbc3,
                      const double *f, double *P,
                      const double *dmx1, const double *dmx2,
                      const double *dmx3, const double *dx3,
                      int cpu_fft1_imag_zero, int nthreads)
{
    if (n1m < 2 || n2m < 2 || n3m < 3 || (n1m & 1) || (n2m & 1)) return -1;
    nthreads_set(nthreads);
    g_nstamp = 0;
    ORA_STAMP();
    const long nx = n1m, ny = n2m, nz = n3m;
    const long ncell = nx * ny * nz;
    double *dxk2 = (double *)malloc(sizeof(double) * nx);
    double *dyk2 = (double *)malloc(sizeof(double) * ny);
    double *am = (double *)malloc(sizeof(double) * nz);
    double *ap = (double *)malloc(sizeof(double) * nz);
    ora_wavenumbers(n1m, n2m, L1, L2, pbc1, pbc2, dxk2, dyk2);
    z_coeffs(n3m, dx3, dmx3, am, ap);

    double *tmp = (double *)malloc(sizeof(double) * ncell);   /* PRHS_d scratch */
    int rc = 0;

    if (!pbc1 && !pbc2) {
        /* ---- N-N : real DCT in x, real DCT in y, real TDMA ---- */
        double *X = (double *)malloc(sizeof(double) * ncell);  /* (i,j,k) */
        ORA_STAMP();
        OMP_PARALLEL
        {
            axis_ws wx, wy;
            axis_ws_init(&wx, n1m); axis_ws_init(&wy, n2m);
            OMP_FOR
            for (long jk = 0; jk < ny * nz; ++jk)             /* F_x :380-392 */
                dct2_line(&wx, f + jk * nx, 1, X + jk * nx, 1);
            OMP_FOR
            for (long ik = 0; ik < nx * nz; ++ik) {           /* F_y :424-444 */
                long i = ik % nx, k = ik / nx;
                double *col = X + k * nx * ny + i;
                double *t = wy.ry;   /* dct2_line reads its input before writing t */
                dct2_line(&wy, col, nx, t, 1);
                for (long j = 0; j < ny; ++j) col[j * nx] = t[j];
            }
            axis_ws_free(&wx); axis_ws_free(&wy);
        }
        /* TDMA-z (cuda_Poisson_TDMA_z_real :1121-1170): systems (i,j), i fastest.
           Solved per j-row block of n1m systems (independent systems). */
        ORA_STAMP();
        OMP_PARALLEL
        {
            double *lam = (double *)malloc(sizeof(double) * nx);
            double *d = (double *)malloc(sizeof(double) * nx * nz);
            OMP_FOR
            for (long j = 0; j < ny; ++j) {
                for (long i = 0; i < nx; ++i) lam[i] = dyk2[j];
                for (long k = 0; k < nz; ++k)
                    for (long i = 0; i < nx; ++i) d[k * nx + i] = X[k * nx * ny + j * nx + i];
                solve_block((int)nx, (int)nz, am, ap, dxk2, lam, j == 0 ? 0 : -1, pbc3, d);
                for (long k = 0; k < nz; ++k)
                    for (long i = 0; i < nx; ++i) X[k * nx * ny + j * nx + i] = d[k * nx + i];
            }
            free(lam); free(d);
        }
        ORA_STAMP();
        OMP_PARALLEL
        {
            axis_ws wx, wy;
            axis_ws_init(&wx, n1m); axis_ws_init(&wy, n2m);
            const double sy = 1.0 / (double)(2 * n2m), sx = 1.0 / (double)(2 * n1m);
            OMP_FOR
            for (long ik = 0; ik < nx * nz; ++ik) {           /* B_y :497-518 */
                long i = ik % nx, k = ik / nx;
                double *col = X + k * nx * ny + i;
                double *t = (double *)wy.work;  /* idct_line does not touch work after c2r */
                idct_line(&wy, col, nx, t, 1);
                for (long j = 0; j < ny; ++j) col[j * nx] = t[j] * sy;
            }
            OMP_FOR
            for (long jk = 0; jk < ny * nz; ++jk) {           /* B_x :562-579 */
                idct_line(&wx, X + jk * nx, 1, tmp + jk * nx, 1);
                for (long i = 0; i < nx; ++i) tmp[jk * nx + i] *= sx;
            }
            axis_ws_free(&wx); axis_ws_free(&wy);
        }
        free(X);
    } else if (!pbc1 && pbc2) {
        /* ---- N-P : real DCT in x, R2C in y, complex TDMA ---- */
        const long hy = ny / 2 + 1;
        double *X = (double *)malloc(sizeof(double) * ncell);
        cd *C = (cd *)malloc(sizeof(cd) * nx * hy * nz);      /* (i, jy, k) */
        ORA_STAMP();
        OMP_PARALLEL
        {
            axis_ws wx, wy;
            axis_ws_init(&wx, n1m); axis_ws_init(&wy, n2m);
            OMP_FOR
            for (long jk = 0; jk < ny * nz; ++jk)             /* F_x :380-392 */
                dct2_line(&wx, f + jk * nx, 1, X + jk * nx, 1);
            OMP_FOR
            for (long ik = 0; ik < nx * nz; ++ik) {           /* F_y :446-459 */
                long i = ik % nx, k = ik / nx;
                r2c_line(&wy, X + k * nx * ny + i, nx, C + k * nx * hy + i, nx);
            }
            axis_ws_free(&wx); axis_ws_free(&wy);
        }
        ORA_STAMP();
        OMP_PARALLEL
        {
            double *lam = (double *)malloc(sizeof(double) * nx);
            double *dr = (double *)malloc(sizeof(double) * nx * nz);
            double *di = (double *)malloc(sizeof(double) * nx * nz);
            OMP_FOR
            for (long j = 0; j < hy; ++j) {                   /* :1276-1334 */
                for (long i = 0; i < nx; ++i) lam[i] = dyk2[j];
                for (long k = 0; k < nz; ++k)
                    for (long i = 0; i < nx; ++i) {
                        cd v = C[k * nx * hy + j * nx + i];
                        dr[k * nx + i] = v.re; di[k * nx + i] = v.im;
                    }
                solve_block((int)nx, (int)nz, am, ap, dxk2, lam, j == 0 ? 0 : -1, pbc3, dr);
                solve_block((int)nx, (int)nz, am, ap, dxk2, lam, j == 0 ? 0 : -1, pbc3, di);
                for (long k = 0; k < nz; ++k)
                    for (long i = 0; i < nx; ++i) {
                        cd v = { dr[k * nx + i], di[k * nx + i] };
                        C[k * nx * hy + j * nx + i] = v;
                    }
            }
            free(lam); free(dr); free(di);
        }
        ORA_STAMP();
        OMP_PARALLEL
        {
            axis_ws wx, wy;
            axis_ws_init(&wx, n1m); axis_ws_init(&wy, n2m);
            const double sy = 1.0 / (double)n2m, sx = 1.0 / (double)(2 * n1m);
            OMP_FOR
            for (long ik = 0; ik < nx * nz; ++ik) {           /* B_y :520-533 */
                long i = ik % nx, k = ik / nx;
                double *col = X + k * nx * ny + i;
                c2r_line(&wy, C + k * nx * hy + i, nx, col, nx);
                for (long j = 0; j < ny; ++j) col[j * nx] *= sy;
            }
            OMP_FOR
            for (long jk = 0; jk < ny * nz; ++jk) {           /* B_x :562-579 */
                idct_line(&wx, X + jk * nx, 1, tmp + jk * nx, 1);
                for (long i = 0; i < nx; ++i) tmp[jk * nx + i] *= sx;
            }
            axis_ws_free(&wx); axis_ws_free(&wy);
        }
        free(X); free(C);
    } else if (pbc1 && !pbc2) {
        /* ---- P-N : real DCT in y first, R2C in x, complex TDMA ---- */
        const long hx = nx / 2 + 1;
        double *Y = (double *)malloc(sizeof(double) * ncell);  /* (i,j,k) */
        cd *C = (cd *)malloc(sizeof(cd) * hx * ny * nz);      /* (ix, j, k) */
        ORA_STAMP();
        OMP_PARALLEL
        {
            axis_ws wx, wy;
            axis_ws_init(&wx, n1m); axis_ws_init(&wy, n2m);
            OMP_FOR
            for (long ik = 0; ik < nx * nz; ++ik) {           /* F_x (Y-R2R) :394-410 */
                long i = ik % nx, k = ik / nx;
                dct2_line(&wy, f + k * nx * ny + i, nx, Y + k * nx * ny + i, nx);
            }
            OMP_FOR
            for (long jk = 0; jk < ny * nz; ++jk)             /* F_y (X-R2C) :461-469 */
                r2c_line(&wx, Y + jk * nx, 1, C + jk * hx, 1);
            axis_ws_free(&wx); axis_ws_free(&wy);
        }
        ORA_STAMP();
        OMP_PARALLEL
        {
            double *lam = (double *)malloc(sizeof(double) * ny);
            double *dr = (double *)malloc(sizeof(double) * ny * nz);
            double *di = (double *)malloc(sizeof(double) * ny * nz);
            OMP_FOR
            for (long i = 0; i < hx; ++i) {                   /* :1215-1272, systems (j,i) */
                for (long j = 0; j < ny; ++j) lam[j] = dxk2[i];
                for (long k = 0; k < nz; ++k)
                    for (long j = 0; j < ny; ++j) {
                        cd v = C[k * hx * ny + j * hx + i];
                        dr[k * ny + j] = v.re; di[k * ny + j] = v.im;
                    }
                solve_block((int)ny, (int)nz, am, ap, lam, dyk2, i == 0 ? 0 : -1, pbc3, dr);
                solve_block((int)ny, (int)nz, am, ap, lam, dyk2, i == 0 ? 0 : -1, pbc3, di);
                for (long k = 0; k < nz; ++k)
                    for (long j = 0; j < ny; ++j) {
                        cd v = { dr[k * ny + j], di[k * ny + j] };
                        C[k * hx * ny + j * hx + i] = v;
                    }
            }
            free(lam); free(dr); free(di);
        }
        ORA_STAMP();
        OMP_PARALLEL
        {
            axis_ws wx, wy;
            axis_ws_init(&wx, n1m); axis_ws_init(&wy, n2m);
            const double sx = 1.0 / (double)n1m, sy = 1.0 / (double)(2 * n2m);
            OMP_FOR
            for (long jk = 0; jk < ny * nz; ++jk) {           /* B_y (X-C2R) :535-545 */
                c2r_line(&wx, C + jk * hx, 1, Y + jk * nx, 1);
                for (long i = 0; i < nx; ++i) Y[jk * nx + i] *= sx;
            }
            OMP_FOR
            for (long ik = 0; ik < nx * nz; ++ik) {           /* B_x (Y-R2R) :581-603 */
                long i = ik % nx, k = ik / nx;
                double *col = tmp + k * nx * ny + i;
                idct_line(&wy, Y + k * nx * ny + i, nx, col, nx);
                for (long j = 0; j < ny; ++j) col[j * nx] *= sy;
            }
            axis_ws_free(&wx); axis_ws_free(&wy);
        }
        free(Y); free(C);
    } else {
        /* ---- P-P : R2C in x, C2C in y, complex TDMA ---- */
        const long hx = nx / 2 + 1;
        cd *C = (cd *)malloc(sizeof(cd) * hx * ny * nz);      /* (ix, j, k) */
        ORA_STAMP();
        OMP_PARALLEL
        {
            axis_ws wx, wy;
            axis_ws_init(&wx, n1m); axis_ws_init(&wy, n2m);
            OMP_FOR
            for (long jk = 0; jk < ny * nz; ++jk)             /* F_x (X-R2C) :412-417 */
                r2c_line(&wx, f + jk * nx, 1, C + jk * hx, 1);
            OMP_FOR
            for (long ik = 0; ik < hx * nz; ++ik) {           /* F_y (Y-C2C) :471-481 */
                long i = ik % hx, k = ik / hx;
                c2c_line(&wy, C + k * hx * ny + i, hx, -1);
            }
            axis_ws_free(&wx); axis_ws_free(&wy);
        }
        ORA_STAMP();
        OMP_PARALLEL
        {
            double *lam = (double *)malloc(sizeof(double) * ny);
            double *dr = (double *)malloc(sizeof(double) * ny * nz);
            double *di = (double *)malloc(sizeof(double) * ny * nz);
            OMP_FOR
            for (long i = 0; i < hx; ++i) {                   /* :1215-1272, systems (j,i) */
                for (long j = 0; j < ny; ++j) lam[j] = dxk2[i];
                for (long k = 0; k < nz; ++k)
                    for (long j = 0; j < ny; ++j) {
                        cd v = C[k * hx * ny + j * hx + i];
                        dr[k * ny + j] = v.re; di[k * ny + j] = v.im;
                    }
                solve_block((int)ny, (int)nz, am, ap, lam, dyk2, i == 0 ? 0 : -1, pbc3, dr);
                solve_block((int)ny, (int)nz, am, ap, lam, dyk2, i == 0 ? 0 : -1, pbc3, di);
                if (cpu_fft1_imag_zero && i == 0) {
                    /* module_solve_poisson.f90:389-397 */
                    for (long k = 0; k < nz; ++k) { di[k * ny + 0] = 0.0; di[k * ny + ny / 2] = 0.0; }
                }
                for (long k = 0; k < nz; ++k)
                    for (long j = 0; j < ny; ++j) {
                        cd v = { dr[k * ny + j], di[k * ny + j] };
                        C[k * hx * ny + j * hx + i] = v;
                    }
            }
            free(lam); free(dr); free(di);
        }
        ORA_STAMP();
        OMP_PARALLEL
        {
            axis_ws wx, wy;
            axis_ws_init(&wx, n1m); axis_ws_init(&wy, n2m);
            const double sy = 1.0 / (double)n2m, sx = 1.0 / (double)n1m;
            OMP_FOR
            for (long ik = 0; ik < hx * nz; ++ik) {           /* B_y (Y-C2C) :547-559 */
                long i = ik % hx, k = ik / hx;
                cd *col = C + k * hx * ny + i;
                c2c_line(&wy, col, hx, +1);
                for (long j = 0; j < ny; ++j) { col[j * hx].re *= sy; col[j * hx].im *= sy; }
            }
            OMP_FOR
            for (long jk = 0; jk < ny * nz; ++jk) {           /* B_x (X-C2R) :605-614 */
                c2r_line(&wx, C + jk * hx, 1, tmp + jk * nx, 1);
                for (long i = 0; i < nx; ++i) tmp[jk * nx + i] *= sx;
            }
            axis_ws_free(&wx); axis_ws_free(&wy);
        }
        free(C);
    }

    ORA_STAMP();
    /* cuda_Poisson_average_elimination :628-664 (arithmetic mean) */
    double aver = 0.0;
    for (long q = 0; q < ncell; ++q) aver += tmp[q];
    aver = aver / (double)n1m / (double)n2m / (double)n3m;
    const long s2 = nx + 2, s3 = (nx + 2) * (ny + 2);
    OMP_PARALLEL
    {
        OMP_FOR
        for (long k = 0; k < nz; ++k)
            for (long j = 0; j < ny; ++j)
                for (long i = 0; i < nx; ++i)
                    P[(i + 1) + (j + 1) * s2 + (k + 1) * s3] = tmp[i + j * nx + k * nx * ny] - aver;
    }
    ora_fill_ghosts(n1m, n2m, n3m, pbc1, pbc2, pbc3, P, dmx1, dmx2, dmx3);

    ORA_STAMP();
    free(tmp); free(dxk2); free(dyk2); free(am); free(ap);
    return rc;
}

/* ------------------------------------------------------------------------ */
void ora_residual(int n1m, int n2m, int n3m, double L1, double L2,
                  int pbc1, int pbc2, const double *f, const double *P,
                  const double *dmx3, const double *dx3, double *r)
{
    const long nx = n1m, ny = n2m, nz = n3m;
    const double hx = L1 / (double)n1m, hy = L2 / (double)n2m;
    const double ix2 = 1.0 / (hx * hx), iy2 = 1.0 / (hy * hy);
    const long s2 = nx + 2, s3 = (nx + 2) * (ny + 2);
#define U(i, j, k) P[((i) + 1) + ((j) + 1) * s2 + ((k) + 1) * s3]
    OMP_PARALLEL
    {
        OMP_FOR
        for (long k = 0; k < nz; ++k) {
            double am = (k == 0) ? 0.0 : 1.0 / dx3[k + 1] / dmx3[k + 1];
            double ap = (k == nz - 1) ? 0.0 : 1.0 / dx3[k + 1] / dmx3[k + 2];
            for (long j = 0; j < ny; ++j)
                for (long i = 0; i < nx; ++i) {
                    double u = U(i, j, k);
                    long im = i - 1, ip = i + 1, jm = j - 1, jp = j + 1;
                    double uxm, uxp, uym, uyp;
                    if (pbc1) { uxm = U((im + nx) % nx, j, k); uxp = U(ip % nx, j, k); }
                    else { uxm = (im < 0) ? u : U(im, j, k); uxp = (ip >= nx) ? u : U(ip, j, k); }
                    if (pbc2) { uym = U(i, (jm + ny) % ny, k); uyp = U(i, jp % ny, k); }
                    else { uym = (jm < 0) ? u : U(i, jm, k); uyp = (jp >= ny) ? u : U(i, jp, k); }
                    double uzm = (k == 0) ? u : U(i, j, k - 1);
                    double uzp = (k == nz - 1) ? u : U(i, j, k + 1);
                    double lu = (uxm - 2.0 * u + uxp) * ix2 + (uym - 2.0 * u + uyp) * iy2
                              + am * (uzm - u) + ap * (uzp - u);
                    r[i + j * nx + k * nx * ny] = f[i + j * nx + k * nx * ny] - lu;
                }
        }
    }
#undef U
}
