// ref_cxx_poisson.cpp -- runs the reference's own C++ Poisson solve
// (00_C/examples/module_solve_poisson.cpp, mpi_Poisson_FFT1..5) as one
// rank: test infrastructure that shows how that solve discretises the
// problem.  Built by oracle/Makefile from the reference sources where they
// lie, with the one-rank MPI of mpi_stub/ and the FFTW 3 calls restated in
// fftw_shim/.  (Its wall-normal discretisation is not the Fortran module's
// that libppf and the oracle implement -- FFT2..5 close the walls with a
// Dirichlet ghost row and uniform-spacing coefficients, FFT1 reads the ghost
// entry of dx2 at one rank -- so it is not a known-answer oracle for the
// solve path; tests/test_ref_cxx_port.py records this.)
//
// One call does what the reference's example driver does for one solve
// (00_C/examples/main.cpp:13-62, 159-201): the input parameters through
// global_inputpara (from a parameter file this call writes), the topology,
// subdomain, mesh, index, datatype, allocation, transpose, wavenumber and
// ghost-cell set-up, the timers, the right-hand side (the caller's, or the
// reference's mpi_poisson_RHS), the solve, and the clean-up of the plans
// and modules.
#include "modules.hpp"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unistd.h>
#include <vector>

namespace {

std::string g_err;

bool write_params(const std::string& path, int n1m, int n2m, int n3m, double a1, double a2, double a3, int pbc1,
                  int pbc2, int pbc3, int uniform2, double gamma2)
{
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return false;
    auto tf = [](int b) { return b ? ".true." : ".false."; };
    std::fprintf(f, "&MESHES\n n1m = %d\n n2m = %d\n n3m = %d\n/\n", n1m, n2m, n3m);
    std::fprintf(f, "&MPI_PROCS\n np1 = 1\n np2 = 1\n np3 = 1\n/\n");
    std::fprintf(f, "&PERIODIC_BOUNDARY\n pbc1 = %s\n pbc2 = %s\n pbc3 = %s\n/\n", tf(pbc1), tf(pbc2), tf(pbc3));
    std::fprintf(f, "&UNIFORM_MESH\n uniform1 = 1\n uniform2 = %d\n uniform3 = 1\n/\n", uniform2);
    std::fprintf(f, "&MESH_STRETCH\n gamma1 = 0.0\n gamma2 = %.17g\n gamma3 = 0.0\n/\n", gamma2);
    std::fprintf(f, "&ASPECT_RATIO\n H = 1.0\n Aspect1 = %.17g\n Aspect2 = %.17g\n Aspect3 = %.17g\n/\n", a1, a2, a3);
    std::fprintf(f, "&SIM_CONTINUE\n ContinueFilein = 0\n ContinueFileout = 0\n/\n");
    return std::fclose(f) == 0;
}

}  // namespace

extern "C" {

__attribute__((visibility("default"))) const char* ref_cxx_last_error(void) { return g_err.c_str(); }

// variant 1..5: mpi_Poisson_FFT<variant>.  Axes as the reference's: x1
// (n1m, real FFT), x2 (n2m, the tridiagonal direction, walls unless pbc2),
// x3 (n3m, complex FFT); domain H = 1 times the aspect ratios; x2 uniform
// (uniform2 = 1) or stretched with gamma2.  prhs: n1m*n2m*n3m values,
// index (k*n2m + j)*n1m + i, or null for the reference's own manufactured
// right-hand side (mpi_poisson_RHS), whose exact solution
// (mpi_poisson_exact_sol) then goes to `exact` when it is given.  Outputs:
// p ((n1m+2)*(n2m+2)*(n3m+2) values, mpi_poisson::P as the solve leaves
// it; `exact` in the same layout), dx2 and dmx2 (n2m+2 values each, the x2
// metric the solve used).  Returns 0, or -1 with ref_cxx_last_error.
__attribute__((visibility("default"))) int ref_cxx_poisson(int variant, int n1m, int n2m, int n3m, double aspect1,
                                                           double aspect2, double aspect3, int pbc1, int pbc2,
                                                           int pbc3, int uniform2, double gamma2, const double* prhs,
                                                           double* p, double* dx2, double* dmx2, double* exact)
{
    g_err.clear();
    if (variant < 1 || variant > 5 || n1m < 2 || n2m < 3 || n3m < 2 || !p || !dx2 || !dmx2) {
        g_err = "bad argument";
        return -1;
    }
    char path[] = "/tmp/ppf_ref_paraXXXXXX";
    const int fd = mkstemp(path);
    if (fd < 0) {
        g_err = "cannot create the parameter file";
        return -1;
    }
    close(fd);
    const bool ok = write_params(path, n1m, n2m, n3m, aspect1, aspect2, aspect3, pbc1, pbc2, pbc3, uniform2, gamma2);
    try {
        if (!ok) throw std::runtime_error("cannot write the parameter file");
        MPI_Init(nullptr, nullptr);
        MPI_Comm_size(MPI_COMM_WORLD, &mpi_topology::nprocs);
        MPI_Comm_rank(MPI_COMM_WORLD, &mpi_topology::myrank);
        global::global_inputpara(path);
        mpi_topology::mpi_topology_make();
        mpi_subdomain::mpi_subdomain_make();
        mpi_subdomain::mpi_subdomain_mesh();
        mpi_subdomain::mpi_subdomain_indices();
        mpi_subdomain::mpi_subdomain_DDT_ghostcell();
        mpi_poisson::mpi_poisson_allocation();
        // transpose scheme 1 (FFT1) moves spectra with the I-to-K datatypes
        // of DDT_transpose1; every scheme uses the FFT and TDMA plans that
        // DDT_transpose2 creates
        if (variant == 1) mpi_subdomain::mpi_subdomain_DDT_transpose1();
        mpi_subdomain::mpi_subdomain_DDT_transpose2();
        mpi_poisson::mpi_poisson_wave_number();
        mpi_subdomain::mpi_subdomain_ghostcell_update(mpi_poisson::P.data());
        std::vector<std::string> names(13, "timer");
        timer::timer_init(13, names);

        const size_t cells = (size_t)n1m * n2m * n3m;
        if (mpi_subdomain::PRHS.size() != cells) throw std::runtime_error("PRHS size differs from the grid");
        if (prhs) std::memcpy(mpi_subdomain::PRHS.data(), prhs, sizeof(double) * cells);
        else mpi_poisson::mpi_poisson_RHS();
        switch (variant) {
            case 1: mpi_poisson::mpi_Poisson_FFT1(mpi_subdomain::dx2_sub, mpi_subdomain::dmx2_sub); break;
            case 2: mpi_poisson::mpi_Poisson_FFT2(mpi_subdomain::dx2_sub, mpi_subdomain::dmx2_sub); break;
            case 3: mpi_poisson::mpi_Poisson_FFT3(mpi_subdomain::dx2_sub, mpi_subdomain::dmx2_sub); break;
            case 4: mpi_poisson::mpi_Poisson_FFT4(mpi_subdomain::dx2_sub, mpi_subdomain::dmx2_sub); break;
            default: mpi_poisson::mpi_Poisson_FFT5(mpi_subdomain::dx2_sub, mpi_subdomain::dmx2_sub); break;
        }
        const size_t ghosted = (size_t)(n1m + 2) * (n2m + 2) * (n3m + 2);
        if (mpi_poisson::P.size() != ghosted) throw std::runtime_error("P size differs from the ghosted grid");
        std::memcpy(p, mpi_poisson::P.data(), sizeof(double) * ghosted);
        if (!prhs && exact) {
            mpi_poisson::mpi_poisson_exact_sol();
            if (mpi_poisson::exact_sol.size() != ghosted) throw std::runtime_error("exact_sol size differs");
            std::memcpy(exact, mpi_poisson::exact_sol.data(), sizeof(double) * ghosted);
        }
        if (mpi_subdomain::dx2_sub.size() < (size_t)n2m + 2 || mpi_subdomain::dmx2_sub.size() < (size_t)n2m + 2)
            throw std::runtime_error("x2 metric shorter than n2m + 2");
        std::memcpy(dx2, mpi_subdomain::dx2_sub.data(), sizeof(double) * (n2m + 2));
        std::memcpy(dmx2, mpi_subdomain::dmx2_sub.data(), sizeof(double) * (n2m + 2));

        // the clean-up of the reference's driver (main.cpp:123-137, 187-201)
        fftw_destroy_plan(mpi_subdomain::plan_fft_x);
        fftw_destroy_plan(mpi_subdomain::plan_fft_z);
        fftw_destroy_plan(mpi_subdomain::plan_ifft_x);
        fftw_destroy_plan(mpi_subdomain::plan_ifft_z);
        PaScaL_TDMA_plan_many_destroy(&mpi_subdomain::plan_tdma, mpi_topology::comm_1d_x2.nprocs);
        PaScaL_TDMA_plan_many_destroy(&mpi_subdomain::plan_tdma_modified, mpi_topology::comm_1d_x2.nprocs);
        mpi_poisson::mpi_poisson_clean();
        mpi_subdomain::mpi_subdomain_indices_clean();
        mpi_subdomain::mpi_subdomain_clean();
        mpi_topology::mpi_topology_clean();
        MPI_Finalize();
    } catch (const std::exception& e) {
        g_err = e.what();
    }
    unlink(path);
    return g_err.empty() ? 0 : -1;
}

}  // extern "C"
