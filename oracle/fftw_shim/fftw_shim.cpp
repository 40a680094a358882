// fftw_shim.cpp -- the FFTW 3 calls of fftw3.h (test infrastructure only).
//
// Each transform is the DFT by its definition, X_k = sum_j x_j
// exp(sign 2 pi i j k / n), summed in long double with the angle reduced
// to (j k mod n) / n, so every output is exact to a few units of the last
// place of a double at the oracle's sizes.  A plan records the geometry;
// execution gathers each line through a scratch vector, so in-place and
// out-of-place calls agree.
#include "fftw3.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

struct ppf_fftw_plan_s {
    int kind;          // 0 complex, 1 r2c, 2 c2r
    int n, howmany, istride, idist, ostride, odist, sign;
    void* in;
    void* out;
};

namespace {

[[noreturn]] void die(const char* what)
{
    std::fprintf(stderr, "FFTW shim: %s\n", what);
    std::abort();
}

fftw_plan make(int kind, int rank, const int* n, int howmany, void* in, int istride, int idist, void* out,
               int ostride, int odist, int sign)
{
    if (rank != 1) die("only rank-1 transforms are provided");
    if (n[0] < 1 || howmany < 0) die("bad transform size");
    return new ppf_fftw_plan_s{ kind, n[0], howmany, istride, idist, ostride, odist, sign, in, out };
}

// y_k = sum_j x_j exp(sign 2 pi i j k / n), all n outputs
void dft(const std::vector<long double>& xr, const std::vector<long double>& xi, int sign,
         std::vector<long double>& yr, std::vector<long double>& yi)
{
    const long n = (long)xr.size();
    const long double two_pi = 6.283185307179586476925286766559005768L;
    std::vector<long double> c((size_t)n), s((size_t)n);
    for (long m = 0; m < n; ++m) {
        c[(size_t)m] = std::cos(two_pi * (long double)m / (long double)n);
        s[(size_t)m] = std::sin(two_pi * (long double)m / (long double)n) * (long double)sign;
    }
    yr.assign((size_t)n, 0.0L);
    yi.assign((size_t)n, 0.0L);
    for (long k = 0; k < n; ++k) {
        long double ar = 0.0L, ai = 0.0L;
        for (long j = 0; j < n; ++j) {
            const size_t m = (size_t)((j * k) % n);
            ar += xr[(size_t)j] * c[m] - xi[(size_t)j] * s[m];
            ai += xr[(size_t)j] * s[m] + xi[(size_t)j] * c[m];
        }
        yr[(size_t)k] = ar;
        yi[(size_t)k] = ai;
    }
}

void run(const ppf_fftw_plan_s* p, void* in_, void* out_)
{
    const int n = p->n;
    std::vector<long double> xr((size_t)n), xi((size_t)n), yr, yi;
    for (int t = 0; t < p->howmany; ++t) {
        if (p->kind == 0) {
            const fftw_complex* in = static_cast<const fftw_complex*>(in_) + (long)t * p->idist;
            for (int j = 0; j < n; ++j) {
                xr[(size_t)j] = in[(long)j * p->istride][0];
                xi[(size_t)j] = in[(long)j * p->istride][1];
            }
            dft(xr, xi, p->sign, yr, yi);
            fftw_complex* out = static_cast<fftw_complex*>(out_) + (long)t * p->odist;
            for (int k = 0; k < n; ++k) {
                out[(long)k * p->ostride][0] = (double)yr[(size_t)k];
                out[(long)k * p->ostride][1] = (double)yi[(size_t)k];
            }
        } else if (p->kind == 1) {
            const double* in = static_cast<const double*>(in_) + (long)t * p->idist;
            for (int j = 0; j < n; ++j) {
                xr[(size_t)j] = in[(long)j * p->istride];
                xi[(size_t)j] = 0.0L;
            }
            dft(xr, xi, FFTW_FORWARD, yr, yi);
            fftw_complex* out = static_cast<fftw_complex*>(out_) + (long)t * p->odist;
            for (int k = 0; k <= n / 2; ++k) {
                out[(long)k * p->ostride][0] = (double)yr[(size_t)k];
                out[(long)k * p->ostride][1] = (double)yi[(size_t)k];
            }
        } else {
            // the Hermitian extension of the n/2+1 inputs; the imaginary
            // parts of X_0 and (n even) X_{n/2} do not enter a real output
            const fftw_complex* in = static_cast<const fftw_complex*>(in_) + (long)t * p->idist;
            for (int k = 0; k <= n / 2; ++k) {
                xr[(size_t)k] = in[(long)k * p->istride][0];
                xi[(size_t)k] = in[(long)k * p->istride][1];
            }
            xi[0] = 0.0L;
            if (n % 2 == 0) xi[(size_t)(n / 2)] = 0.0L;
            for (int k = n / 2 + 1; k < n; ++k) {
                xr[(size_t)k] = xr[(size_t)(n - k)];
                xi[(size_t)k] = -xi[(size_t)(n - k)];
            }
            dft(xr, xi, FFTW_BACKWARD, yr, yi);
            double* out = static_cast<double*>(out_) + (long)t * p->odist;
            for (int j = 0; j < n; ++j) out[(long)j * p->ostride] = (double)yr[(size_t)j];
        }
    }
}

}  // namespace

fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany, fftw_complex* in, const int*, int istride,
                             int idist, fftw_complex* out, const int*, int ostride, int odist, int sign, unsigned)
{
    return make(0, rank, n, howmany, in, istride, idist, out, ostride, odist, sign);
}
fftw_plan fftw_plan_many_dft_r2c(int rank, const int* n, int howmany, double* in, const int*, int istride, int idist,
                                 fftw_complex* out, const int*, int ostride, int odist, unsigned)
{
    return make(1, rank, n, howmany, in, istride, idist, out, ostride, odist, FFTW_FORWARD);
}
fftw_plan fftw_plan_many_dft_c2r(int rank, const int* n, int howmany, fftw_complex* in, const int*, int istride,
                                 int idist, double* out, const int*, int ostride, int odist, unsigned)
{
    return make(2, rank, n, howmany, in, istride, idist, out, ostride, odist, FFTW_BACKWARD);
}
void fftw_execute(const fftw_plan p) { run(p, p->in, p->out); }
void fftw_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out) { run(p, in, out); }
void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out) { run(p, in, out); }
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out) { run(p, in, out); }
void fftw_destroy_plan(fftw_plan p) { delete p; }
