/*
 * ppf_cxx_driver.h -- drop-in replacement of the C++ example driver's solve
 * calls (00_C/examples/modules.hpp:223-232), library
 * pascal_poisson_fft_b200/libppf_cxx.so (links libppf.so).
 *
 * The reference declares, in namespace mpi_poisson,
 *     void mpi_Poisson_FFT1(const std::vector<double>& dx2,
 *                           const std::vector<double>& dmx2);   (and FFT2..FFT5)
 * which read the right-hand side from the global mpi_subdomain::PRHS and
 * write the ghosted solution into the global mpi_poisson::P
 * (00_C/examples/module_solve_poisson.cpp:47-52).  libppf_cxx.so defines
 * those five functions with the same signatures, reading and writing the
 * same globals, which the caller's own translation units define as before
 * (module_global.cpp, module_mpi_subdomain.cpp and module_solve_poisson.cpp
 * with its mpi_Poisson_FFT bodies removed).
 *
 * Axes follow the C++ driver: x1 (i, fastest) and x3 (k, slowest) are the
 * transform axes, x2 (j) is the wall-normal axis of the tridiagonal solves.
 *   PRHS[(k * n2msub + j) * n1msub + i]           interior, FP64, host
 *   P[(k * (n2sub + 1) + j) * (n1sub + 1) + i]     with ghost cells, FP64, host
 *   dx2, dmx2 (0..n2sub), mpi_subdomain::dmx1_sub (0..n1sub), dmx3_sub (0..n3sub)
 * The solve is libppf's (the Fortran solver's discretisation: Neumann walls
 * on a non-periodic axis with the zero mode pinned, arithmetic-mean removal,
 * the reference's ghost-cell update); the five variants, which in the
 * reference differ only in their MPI transpose schemes, are the same call.
 * One rank (np1 = np2 = np3 = 1).  Errors are thrown as std::runtime_error.
 */
#ifndef PPF_CXX_DRIVER_H
#define PPF_CXX_DRIVER_H

#if defined(__GNUC__)
#define PPF_CXX_API __attribute__((visibility("default")))
#else
#define PPF_CXX_API
#endif

#ifdef __cplusplus
#include <vector>

namespace mpi_poisson {
/* 00_C/examples/modules.hpp:223-232 */
PPF_CXX_API void mpi_Poisson_FFT1(const std::vector<double>& dx2, const std::vector<double>& dmx2);
PPF_CXX_API void mpi_Poisson_FFT2(const std::vector<double>& dx2, const std::vector<double>& dmx2);
PPF_CXX_API void mpi_Poisson_FFT3(const std::vector<double>& dx2, const std::vector<double>& dmx2);
PPF_CXX_API void mpi_Poisson_FFT4(const std::vector<double>& dx2, const std::vector<double>& dmx2);
PPF_CXX_API void mpi_Poisson_FFT5(const std::vector<double>& dx2, const std::vector<double>& dmx2);
}  // namespace mpi_poisson

extern "C" {
#endif

/* C-callable form of mpi_Poisson_FFT<variant> (variant 1..5) for hosts that
 * cannot call C++ (ctypes, Fortran, C): dx2 and dmx2 hold n values each
 * (n = n2msub + 2).  Returns 0, or a negative libppf status with the message
 * in ppf_cxx_last_error().  No reference counterpart (the reference's call is
 * C++ only). */
PPF_CXX_API int ppf_cxx_poisson_fft(int variant, const double *dx2, const double *dmx2, int n);

/* Precision of the driver's solves (PPF_FP64, the reference's and the
 * default, or PPF_MIXED with `max_sweeps` FP64 refinement sweeps).  No
 * reference counterpart. */
PPF_CXX_API int ppf_cxx_set_precision(int precision, int max_sweeps);

/* Releases the driver's plan and host staging (they are otherwise kept
 * between calls, like the reference's module-level FFT plans).  No
 * reference counterpart. */
PPF_CXX_API int ppf_cxx_release(void);

/* Thread-local message of the calling thread's last error ("" if none). */
PPF_CXX_API const char *ppf_cxx_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* PPF_CXX_DRIVER_H */
