// ppf_cxx_driver.cpp -- the C++ example driver's solve calls on libppf.
//
// mpi_poisson::mpi_Poisson_FFT{1..5}(dx2, dmx2) (00_C/examples/modules.hpp:
// 223-232) read the right-hand side from mpi_subdomain::PRHS and write the
// ghosted solution into mpi_poisson::P (00_C/examples/module_solve_poisson.
// cpp:47-52); the globals are the caller's, declared here as the reference
// declares them.  The C++ driver's axes are (x1, x2, x3) with x2 the
// wall-normal axis of the tridiagonal solves; libppf solves along its third
// axis, so each call permutes the two outer axes of PRHS on the host
// (x1-lines are contiguous in both layouts and are copied whole), solves
// with ppf_solve_host (copy in, solve, copy out) and permutes the ghosted
// solution back into P.  The plan and the host staging persist between
// calls, like the reference's module-level FFTW and TDMA plans.
#include "../../include/ppf.h"
#include "../../include/ppf_cxx_driver.h"

#include <cstdio>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

// The caller's globals (00_C/examples/modules.hpp:14-34, 68-77, 186-190).
namespace global {
extern int n1m, n2m, n3m;
extern int np1, np2, np3;
extern bool pbc1, pbc2, pbc3;
extern double L1, L2, L3;
}  // namespace global
namespace mpi_subdomain {
extern int n1msub, n2msub, n3msub;
extern std::vector<double> PRHS;
extern std::vector<double> dmx1_sub, dmx3_sub;
}  // namespace mpi_subdomain
namespace mpi_poisson {
extern std::vector<double> P;
}  // namespace mpi_poisson

namespace {

thread_local std::string g_msg;

struct DriverError : std::runtime_error {
    int code;
    DriverError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

struct Driver {
    ppf_plan* plan = nullptr;
    ppf_desc desc{};
    int precision = PPF_FP64;
    int max_sweeps = 0;
    std::vector<double> f;   // PRHS in libppf's axis order
    std::vector<double> p;   // ghosted solution in libppf's axis order
};

std::mutex g_mu;
Driver g_drv;

void check(int rc, const char* what)
{
    if (rc != PPF_OK) throw DriverError(rc, std::string(what) + ": " + ppf_last_error());
}

bool same(const ppf_desc& a, const ppf_desc& b)
{
    return a.n1m == b.n1m && a.n2m == b.n2m && a.n3m == b.n3m && a.L1 == b.L1 && a.L2 == b.L2 &&
           a.pbc1 == b.pbc1 && a.pbc2 == b.pbc2 && a.pbc3 == b.pbc3 && a.precision == b.precision &&
           a.max_sweeps == b.max_sweeps;
}

void need(bool ok, const std::string& msg)
{
    if (!ok) throw DriverError(PPF_ERR_INVALID, "mpi_Poisson_FFT: " + msg);
}

void solve(const std::vector<double>& dx2, const std::vector<double>& dmx2)
{
    using namespace mpi_subdomain;
    std::lock_guard<std::mutex> lk(g_mu);
    Driver& d = g_drv;
    need(global::np1 * global::np2 * global::np3 == 1, "libppf solves one subdomain per GPU (np1 = np2 = np3 = 1)");
    const long nx = n1msub, nw = n2msub, nk = n3msub;   // x1, x2 (walls), x3
    need(nx == global::n1m && nw == global::n2m && nk == global::n3m, "subdomain sizes differ from the global grid");
    need((long)PRHS.size() == nx * nw * nk, "PRHS holds " + std::to_string(PRHS.size()) + " values, expected n1msub*n2msub*n3msub");
    need((long)dx2.size() >= nw + 2 && (long)dmx2.size() >= nw + 2, "dx2/dmx2 need n2sub + 1 values");
    need((long)dmx1_sub.size() >= nx + 2 && (long)dmx3_sub.size() >= nk + 2, "dmx1_sub/dmx3_sub need n1sub + 1 / n3sub + 1 values");

    // libppf axes: x = x1, y = x3, z = x2 (the tridiagonal direction)
    ppf_desc want{};
    want.n1m = (int)nx; want.n2m = (int)nk; want.n3m = (int)nw;
    want.L1 = global::L1; want.L2 = global::L3;
    want.pbc1 = global::pbc1 ? 1 : 0; want.pbc2 = global::pbc3 ? 1 : 0; want.pbc3 = global::pbc2 ? 1 : 0;
    want.precision = d.precision;
    want.max_sweeps = d.precision == PPF_MIXED ? d.max_sweeps : 0;
    if (!d.plan || !same(d.desc, want)) {
        if (d.plan) ppf_plan_destroy(d.plan);
        d.plan = nullptr;
        check(ppf_plan_create(&want, &d.plan), "ppf_plan_create");
        d.desc = want;
    }
    const long gx = nx + 2, gw = nw + 2, gk = nk + 2;
    d.f.resize((size_t)(nx * nw * nk));
    d.p.resize((size_t)(gx * gw * gk));
    if ((long)mpi_poisson::P.size() != gx * gw * gk) mpi_poisson::P.assign((size_t)(gx * gw * gk), 0.0);

    // PRHS (k, j, i) -> f (j, k, i), whole x1-lines
    const double* src = PRHS.data();
    double* f = d.f.data();
#pragma omp parallel for collapse(2) schedule(static)
    for (long j = 0; j < nw; ++j)
        for (long k = 0; k < nk; ++k)
            std::memcpy(f + (j * nk + k) * nx, src + (k * nw + j) * nx, sizeof(double) * nx);

    check(ppf_solve_host(d.plan, d.f.data(), d.p.data(), dmx1_sub.data(), dmx3_sub.data(), dmx2.data(),
                         dx2.data(), nullptr),
          "ppf_solve_host");

    // ghosted p (j, k, i) -> P (k, j, i)
    const double* q = d.p.data();
    double* P = mpi_poisson::P.data();
#pragma omp parallel for collapse(2) schedule(static)
    for (long k = 0; k < gk; ++k)
        for (long j = 0; j < gw; ++j)
            std::memcpy(P + (k * gw + j) * gx, q + (j * gk + k) * gx, sizeof(double) * gx);
}

}  // namespace

namespace mpi_poisson {
void mpi_Poisson_FFT1(const std::vector<double>& dx2, const std::vector<double>& dmx2) { solve(dx2, dmx2); }
void mpi_Poisson_FFT2(const std::vector<double>& dx2, const std::vector<double>& dmx2) { solve(dx2, dmx2); }
void mpi_Poisson_FFT3(const std::vector<double>& dx2, const std::vector<double>& dmx2) { solve(dx2, dmx2); }
void mpi_Poisson_FFT4(const std::vector<double>& dx2, const std::vector<double>& dmx2) { solve(dx2, dmx2); }
void mpi_Poisson_FFT5(const std::vector<double>& dx2, const std::vector<double>& dmx2) { solve(dx2, dmx2); }
}  // namespace mpi_poisson

extern "C" {

int ppf_cxx_poisson_fft(int variant, const double* dx2, const double* dmx2, int n)
{
    g_msg.clear();
    if (variant < 1 || variant > 5 || !dx2 || !dmx2 || n < 0) {
        g_msg = "ppf_cxx_poisson_fft: variant must be 1..5 and dx2, dmx2 non-null";
        return PPF_ERR_INVALID;
    }
    try {
        const std::vector<double> a(dx2, dx2 + n), b(dmx2, dmx2 + n);
        switch (variant) {
        case 1: mpi_poisson::mpi_Poisson_FFT1(a, b); break;
        case 2: mpi_poisson::mpi_Poisson_FFT2(a, b); break;
        case 3: mpi_poisson::mpi_Poisson_FFT3(a, b); break;
        case 4: mpi_poisson::mpi_Poisson_FFT4(a, b); break;
        default: mpi_poisson::mpi_Poisson_FFT5(a, b); break;
        }
    } catch (const DriverError& e) {
        g_msg = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_msg = e.what();
        return PPF_ERR_INVALID;
    }
    return PPF_OK;
}

int ppf_cxx_set_precision(int precision, int max_sweeps)
{
    g_msg.clear();
    if ((precision != PPF_FP64 && precision != PPF_MIXED) || max_sweeps < 0 || max_sweeps > 8) {
        g_msg = "ppf_cxx_set_precision: PPF_FP64 or PPF_MIXED with 0..8 sweeps";
        return PPF_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    g_drv.precision = precision;
    g_drv.max_sweeps = max_sweeps;
    return PPF_OK;
}

int ppf_cxx_release(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_drv.plan) ppf_plan_destroy(g_drv.plan);
    g_drv.plan = nullptr;
    std::vector<double>().swap(g_drv.f);
    std::vector<double>().swap(g_drv.p);
    return PPF_OK;
}

const char* ppf_cxx_last_error(void) { return g_msg.c_str(); }

}  // extern "C"
