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
#include "ppf_misc_dev.cuh"

#include <math.h>

namespace ppf {

__global__ void k_ghost_axis(double* __restrict__ P, int dir, int neumann, int n1m, int n2m, int n3m,
                             long sy, long sz, const double* __restrict__ dmx, int faces)
{
    ghost_axis(P, dir, neumann, n1m, n2m, n3m, sy, sz, dmx, faces, threadIdx.x + (long)blockIdx.x * blockDim.x,
               (long)blockDim.x * gridDim.x);
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

__global__ void __launch_bounds__(512) k_sweep_gate(const double* __restrict__ partials, long nblocks, double ncell,
                                                    double* mean_prev, int* skip, int* sweeps_done, double* last_rel,
                                                    double tol, int initial)
{
    sweep_gate(partials, nblocks, ncell, mean_prev, skip, sweeps_done, last_rel, tol, initial);
}

cudaError_t launch_sweep_gate(const double* partials, long nblocks, double ncell, double* mean_prev, int* skip_flag,
                              int* sweeps_done, double* last_rel, double tol, int initial, cudaStream_t st)
{
    k_sweep_gate<<<1, 512, 0, st>>>(partials, nblocks, ncell, mean_prev, skip_flag, sweeps_done, last_rel, tol,
                                    initial);
    return cudaGetLastError();
}

}  // namespace ppf
