// ppf_ghost.cu -- ghost-cell update of the ghosted solution (sm_100a), and
// the device-side refinement gate.
//
// The reference fills the ghost cells in a fixed order: quadratic Neumann
// extrapolation along every non-periodic axis (apply_bc_on_direction,
// 01_Fortran/src/fft_3d_poisson.f90:798-852, x then y then z), then the
// periodic copies along every periodic axis (ghostcell_update_on_direction
// at one rank, :709-796, x then y then z).  Each step covers the whole face
// including the other axes' ghost lines, so later steps read values written
// by earlier ones; the same order is kept here, one launch per axis.
#include "ppf_kernels.cuh"

#include <math.h>

namespace ppf {

__global__ void k_ghost_axis(double* __restrict__ P, int dir, int neumann, int n1m, int n2m, int n3m,
                             long sy, long sz, const double* __restrict__ dmx, int faces)
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
    for (long idx = threadIdx.x + (long)blockIdx.x * blockDim.x; idx < total; idx += (long)blockDim.x * gridDim.x) {
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

cudaError_t launch_ghosts(double* P, const Geom& g, const double* dmx1, const double* dmx2, const double* dmx3,
                          cudaStream_t st, int zfaces)
{
    const int per[3] = { g.px, g.py, g.pz };
    const double* dmx[3] = { dmx1, dmx2, dmx3 };
    const long face[3] = { (long)(g.ny + 2) * (g.nz + 2), (long)(g.nx + 2) * (g.nz + 2),
                           (long)(g.nx + 2) * (g.ny + 2) };
    for (int pass = 0; pass < 2; ++pass) {          // Neumann axes first, then periodic axes
        for (int d = 0; d < 3; ++d) {
            const bool neumann = !per[d];
            if ((pass == 0) != neumann) continue;
            // z of a slab: walls only at the global ends (zfaces), the
            // planes between slabs come from the neighbouring ranks
            const int faces = (d == 2) ? zfaces : 3;
            if (faces == 0) continue;
            const int blocks = (int)((face[d] + 255) / 256);
            k_ghost_axis<<<blocks, 256, 0, st>>>(P, d, neumann ? 1 : 0, g.nx, g.ny, g.nz, g.pstride_y,
                                                 g.pstride_z, dmx[d], faces);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

// After an x-inverse pass that wrote per-block partial sums: reduce them in
// a fixed order (deterministic), keep mean(u) for the next accumulate pass,
// and after a refinement sweep count it, record ||du||/||u|| and close the
// gate for the remaining sweeps once it is below tol.  A sweep that was
// skipped (gate already closed) leaves everything unchanged.
__global__ void __launch_bounds__(512) k_sweep_gate(const double* __restrict__ partials, long nblocks, double ncell,
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

cudaError_t launch_sweep_gate(const double* partials, long nblocks, double ncell, double* mean_prev, int* skip_flag,
                              int* sweeps_done, double* last_rel, double tol, int initial, cudaStream_t st)
{
    k_sweep_gate<<<1, 512, 0, st>>>(partials, nblocks, ncell, mean_prev, skip_flag, sweeps_done, last_rel, tol,
                                    initial);
    return cudaGetLastError();
}

}  // namespace ppf
