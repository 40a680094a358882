// Test harness of libppf_cxx.so: defines the C++ example driver's globals
// that mpi_poisson::mpi_Poisson_FFT{1..5} read and write (in the driver they
// live in module_global.cpp, module_mpi_subdomain.cpp and
// module_solve_poisson.cpp; 00_C/examples/modules.hpp:14-34, 68-77, 186-190)
// and gives ctypes plain C accessors to them.  Test infrastructure only.
#include <algorithm>
#include <vector>

namespace global {
int n1m = 0, n2m = 0, n3m = 0;
int np1 = 1, np2 = 1, np3 = 1;
bool pbc1 = true, pbc2 = false, pbc3 = true;
double L1 = 1.0, L2 = 1.0, L3 = 1.0;
}  // namespace global
namespace mpi_subdomain {
int n1msub = 0, n2msub = 0, n3msub = 0;
std::vector<double> PRHS, dmx1_sub, dmx3_sub;
}  // namespace mpi_subdomain
namespace mpi_poisson {
std::vector<double> P;
}  // namespace mpi_poisson

extern "C" {

// grid of the driver's axes (x1, x2 = walls, x3) and its metrics
void harness_setup(int n1m, int n2m, int n3m, double L1, double L2, double L3, int pbc1, int pbc2, int pbc3,
                   int np1, const double* dmx1, const double* dmx3)
{
    global::n1m = n1m; global::n2m = n2m; global::n3m = n3m;
    global::L1 = L1; global::L2 = L2; global::L3 = L3;
    global::pbc1 = pbc1 != 0; global::pbc2 = pbc2 != 0; global::pbc3 = pbc3 != 0;
    global::np1 = np1; global::np2 = 1; global::np3 = 1;
    mpi_subdomain::n1msub = n1m; mpi_subdomain::n2msub = n2m; mpi_subdomain::n3msub = n3m;
    mpi_subdomain::dmx1_sub.assign(dmx1, dmx1 + n1m + 2);
    mpi_subdomain::dmx3_sub.assign(dmx3, dmx3 + n3m + 2);
    mpi_poisson::P.assign((size_t)(n1m + 2) * (n2m + 2) * (n3m + 2), 0.0);
}

void harness_set_prhs(const double* f, long n) { mpi_subdomain::PRHS.assign(f, f + n); }

long harness_get_p(double* out, long n)
{
    const long m = std::min<long>(n, (long)mpi_poisson::P.size());
    std::copy(mpi_poisson::P.begin(), mpi_poisson::P.begin() + m, out);
    return (long)mpi_poisson::P.size();
}

}  // extern "C"
