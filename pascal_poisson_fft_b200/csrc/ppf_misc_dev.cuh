// ppf_misc_dev.cuh -- device bodies of the small solve steps, shared by
// their kernels (ppf_ghost.cu, ppf_tdma.cu) and the persistent batch kernel
// (ppf_batch.cu): the ghost-cell update of one axis, the refinement gate and
// the z coefficients.
//
// The reference fills the ghost cells in a fixed order: quadratic Neumann
// extrapolation along every non-periodic axis (apply_bc_on_direction,
// 01_Fortran/src/fft_3d_poisson.f90:798-852, x then y then z), then the
// periodic copies along every periodic axis (ghostcell_update_on_direction
// at one rank, :709-796, x then y then z).  Each step covers the whole face
// including the other axes' ghost lines, so later steps read values written
// by earlier ones; the same order is kept, one step per axis.
#pragma once
#include "ppf_kernels.cuh"

#include <math.h>

namespace ppf {

// face elements idx0, idx0 + stride, ... of axis dir
__device__ __forceinline__ void ghost_axis(double* __restrict__ P, int dir, int neumann, int n1m, int n2m, int n3m,
                                           long sy, long sz, const double* __restrict__ dmx, int faces, long idx0,
                                           long stride)
{
    const int N1 = n1m + 2, N2 = n2m + 2, N3 = n3m + 2;
    int nb, nm;
    long sa, sb, sc;
    if (dir == 0)      { nb = N2; sa = 1;  sb = sy; sc = sz; nm = n1m; }
    else if (dir == 1) { nb = N1; sa = sy; sb = 1;  sc = sz; nm = n2m; }
    else               { nb = N1; sa = sz; sb = 1;  sc = sy; nm = n3m; }
    const int nc = (dir == 2) ? N2 : N3;
    const int na = nm + 1;  // upper ghost index
    double alo = 0, blo = 0, ahi = 0, bhi = 0;
    if (neumann) {
        const double d1 = dmx[1], d2 = dmx[2], dn = dmx[na], dn1 = dmx[nm];
        const double sl = d1 + d2, su = dn + dn1;
        alo = (sl * sl) / ((sl * sl) - d1 * d1);
        blo = (d1 * d1) / ((sl * sl) - d1 * d1);
        ahi = (su * su) / ((su * su) - dn * dn);
        bhi = (dn * dn) / ((su * su) - dn * dn);
    }
    const long total = (long)nb * nc;
    for (long idx = idx0; idx < total; idx += stride) {
        const long ib = idx % nb, ic = idx / nb;
        const long base = ib * sb + ic * sc;
        if (neumann) {
            if (faces & 1) P[base] = alo * P[base + sa] - blo * P[base + 2 * sa];
            if (faces & 2) P[base + na * sa] = ahi * P[base + nm * sa] - bhi * P[base + (na - 2) * sa];
        } else {
            const double v0 = P[base + sa], v1 = P[base + nm * sa];
            P[base] = v1;
            P[base + na * sa] = v0;
        }
    }
}

// After an x-inverse pass that wrote per-block partial sums: reduce them in
// a fixed order (deterministic), keep mean(u) for the next accumulate pass,
// and after a refinement sweep count it, record ||du||/||u|| and close the
// gate for the remaining sweeps once it is below tol.  A sweep that was
// skipped (gate already closed) leaves everything unchanged.
// (one CTA of a power-of-two size up to 512 threads)
__device__ __forceinline__ void sweep_gate(const double* __restrict__ partials, long nblocks, double ncell,
                                           double* mean_prev, int* skip, int* sweeps_done, double* last_rel,
                                           double tol, int initial)
{
    __shared__ double red[3][512];
    if (*skip) return;
    double a = 0.0, b = 0.0, c = 0.0;
    for (long i = threadIdx.x; i < nblocks; i += blockDim.x) {
        a += partials[3 * i + 0];
        b += partials[3 * i + 1];
        c += partials[3 * i + 2];
    }
    red[0][threadIdx.x] = a; red[1][threadIdx.x] = b; red[2][threadIdx.x] = c;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            red[0][threadIdx.x] += red[0][threadIdx.x + o];
            red[1][threadIdx.x] += red[1][threadIdx.x + o];
            red[2][threadIdx.x] += red[2][threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    *mean_prev = red[2][0] / ncell;
    if (initial) return;
    *sweeps_done += 1;
    const double du = red[0][0], u = red[1][0];
    const double rel = (u > 0.0) ? sqrt(du / u) : (du > 0.0 ? INFINITY : 0.0);
    *last_rel = rel;
    if (tol > 0.0 && rel < tol) *skip = 1;
}

// z coefficients of cuda_Poisson_TDMA_z_* (fft_3d_poisson.f90:1139-1142):
// am_k = 1/dx3_k/dmx3_k, ap_k = 1/dx3_k/dmx3_{k+1}, am_1 = ap_n3m = 0; plus
// min_k dx3_k^2 for the low-wavenumber precision switch (a system is
// near-singular when lam dz^2 << 1 at the finest spacing).  One CTA.
__device__ __forceinline__ void zcoef(const double* __restrict__ dx3, const double* __restrict__ dmx3, int nz,
                                      double* __restrict__ am, double* __restrict__ ap, double* __restrict__ dzmin2)
{
    __shared__ double red[512];   // one CTA of a power-of-two size up to 512 threads
    double mn = INFINITY;
    for (int k = threadIdx.x; k < nz; k += blockDim.x) {
        const int kk = k + 1;
        double av = __ddiv_rn(__ddiv_rn(1.0, dx3[kk]), dmx3[kk]);
        double cv = __ddiv_rn(__ddiv_rn(1.0, dx3[kk]), dmx3[kk + 1]);
        if (k == 0) av = 0.0;
        if (k == nz - 1) cv = 0.0;
        am[k] = av;
        ap[k] = cv;
        mn = fmin(mn, dx3[kk] * dx3[kk]);
    }
    red[threadIdx.x] = mn;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] = fmin(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *dzmin2 = red[0];
}

}  // namespace ppf
