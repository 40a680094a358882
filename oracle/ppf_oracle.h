/*
 * ppf_oracle.h -- CPU restatement of the PaScaL_POISSON_FFT solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker: tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / --impl reference leg
 * load it.  The product (libppf.so, the CUDA path) never links, calls or
 * falls back to it.
 *
 * Every routine cites the reference file:line it restates (paths relative
 * to the reference project root).  Arrays are Fortran column-major, first
 * index fastest, exactly as the reference lays them out.
 */
#ifndef PPF_ORACLE_H
#define PPF_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Grid faces, cell widths and centre spacings along one axis at one rank.
 * Restates 01_Fortran/examples/mpi_subdomain.f90:397-472
 * (calculate_x, non_uniform_channel_grid, uniform_grid, calculate_dx_dmx,
 * mpi_subdomain_ghostcell_1d at nprocs=1).
 *   nm      cells along the axis (n = nm+1 faces)
 *   x       faces,            indices 0..nm+1 (size nm+2)
 *   dx,dmx  widths / spacings, indices 0..nm+1 (size nm+2; index n=nm+1 is the
 *           upper ghost, index 0 the lower ghost)
 * uniform=1 -> x_i = (i-1) L/nm; uniform=0 -> tanh stretching with gamma. */
void ora_mesh(int nm, double L, int uniform, double gamma, int pbc,
              double *x, double *dx, double *dmx);

/* Modified wavenumbers dxk2(1:n1m), dyk2(1:n2m) for the four x/y boundary
 * combinations.  Restates 01_Fortran/src/fft_3d_poisson.f90:288-351. */
void ora_wavenumbers(int n1m, int n2m, double L1, double L2, int pbc1, int pbc2,
                     double *dxk2, double *dyk2);

/* Batched Thomas solves, system index fastest: a(n_sys, n_row).
 * Restates 01_Fortran/PaScaL_TDMA/src/tdmas.f90:114-147 (tdma_many) and
 * :160-213 (tdma_cycl_many).  In place: d <- x, c overwritten. */
void ora_tdma_many(double *a, double *b, double *c, double *d, int n_sys, int n_row);
void ora_tdma_cycl_many(double *a, double *b, double *c, double *d, int n_sys, int n_row);

/* Complex FFT (unnormalised), sign -1 forward / +1 inverse, interleaved
 * re/im doubles, n any positive integer (radix 2,3,4,5 + generic prime).
 * Stands in for FFTW/cuFFT (third-party, not vendored in the reference). */
int ora_fft_c2c(double *data, int n, int sign);

/* The full one-rank GPU solve path, cuda_Poisson_FFT_1D
 * (01_Fortran/src/fft_3d_poisson.f90:353-626):
 *   f     PRHS(1:n1m,1:n2m,1:n3m)   input, not modified
 *   P     P(0:n1m+1,0:n2m+1,0:n3m+1) output incl. ghost cells
 *   dmx1,dmx2,dmx3,dx3  metric arrays with indices 0..nm+1
 * pbc* select periodic (1) or Neumann (0) per axis.
 * cpu_fft1_imag_zero=1 additionally zeroes the imaginary part of the
 * (kx=0, ky in {0,Ny/2}) modes as the CPU solver does
 * (01_Fortran/src/module_solve_poisson.f90:389-397) -- periodic-periodic only.
 * Returns 0 on success, <0 on bad arguments. */
int ora_poisson_solve(int n1m, int n2m, int n3m, double L1, double L2,
                      int pbc1, int pbc2, int pbc3,
                      const double *f, double *P,
                      const double *dmx1, const double *dmx2,
                      const double *dmx3, const double *dx3,
                      int cpu_fft1_imag_zero, int nthreads);

/* Ghost-cell fill of a ghosted field in the reference's order:
 * Neumann extrapolation along every non-periodic axis (x, y, z), then the
 * periodic copies along every periodic axis (x, y, z).
 * Restates fft_3d_poisson.f90:798-852 (cuda_neumann_BC) and :666-796
 * (cuda_ghostcell_update at nprocs=1). */
void ora_fill_ghosts(int n1m, int n2m, int n3m, int pbc1, int pbc2, int pbc3,
                     double *P, const double *dmx1, const double *dmx2,
                     const double *dmx3);

/* 7-point FP64 residual r = f - L_h u of the operator the solve inverts
 * (3-point periodic / mirror-Neumann second differences in x,y with uniform
 * spacing L/N; finite-volume z stencil with am=1/(dx3_k dmx3_k),
 * ap=1/(dx3_k dmx3_{k+1}), am_1 = ap_n3m = 0).  u is read from the interior
 * of the ghosted array P.  No reference counterpart (a residual check). */
/* Seconds of the last ora_poisson_solve per stage: set-up, forward
 * transforms, z solves, inverse transforms, mean removal + ghosts (the
 * reference's timer stages, 01_Fortran/examples/main.f90:65-78).  Returns
 * the number of stamps (6 = complete). */
int ora_last_stage_seconds(double *out);

void ora_residual(int n1m, int n2m, int n3m, double L1, double L2,
                  int pbc1, int pbc2, const double *f, const double *P,
                  const double *dmx3, const double *dx3, double *r);

#ifdef __cplusplus
}
#endif
#endif
