/* The part of FFTW 3's API (FFTW 3.3.x, fftw3.h) that the reference's C++
 * Poisson solve calls, restated for the oracle builds (test infrastructure
 * only; FFTW itself is not in this image).  fftw_shim.cpp computes the
 * transforms FFTW defines for these calls: the unnormalised complex DFT
 * with sign -1 (FFTW_FORWARD) or +1 (FFTW_BACKWARD), the real-to-complex
 * forward DFT returning the n/2+1 non-redundant outputs, and the
 * complex-to-real backward DFT of a Hermitian half spectrum; rank-1
 * transforms of the advanced interface (howmany transforms, element j of
 * transform t at t*dist + j*stride). */
#ifndef PPF_ORACLE_FFTW3_SHIM_H
#define PPF_ORACLE_FFTW3_SHIM_H

typedef double fftw_complex[2];
typedef struct ppf_fftw_plan_s* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_PRESERVE_INPUT (1U << 4)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_many_dft(int rank, const int* n, int howmany, fftw_complex* in, const int* inembed, int istride,
                             int idist, fftw_complex* out, const int* onembed, int ostride, int odist, int sign,
                             unsigned flags);
fftw_plan fftw_plan_many_dft_r2c(int rank, const int* n, int howmany, double* in, const int* inembed, int istride,
                                 int idist, fftw_complex* out, const int* onembed, int ostride, int odist,
                                 unsigned flags);
fftw_plan fftw_plan_many_dft_c2r(int rank, const int* n, int howmany, fftw_complex* in, const int* inembed,
                                 int istride, int idist, double* out, const int* onembed, int ostride, int odist,
                                 unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out);
void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out);
void fftw_destroy_plan(fftw_plan p);

#endif
