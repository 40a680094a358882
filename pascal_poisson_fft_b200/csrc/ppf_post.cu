// ppf_post.cu -- device-side steps of the example drivers' field IO (sm_100a):
// the ghost-cell update of a ghosted field outside a solve, and the
// cell-to-node interpolation of the 3-D instant-field dump.
#include "ppf_misc_dev.cuh"

namespace ppf {

// Node (i, j, k), i = 1..n1m, j = 1..n2m, k = 1..n3m (Fortran indices), from
// the eight cells around it: calc_C2g of 01_Fortran/examples/cuda_post.f90:
// 338-353, the same weighted averages in the same order (z first, then x,
// then y).  P ghosted (0:n1m+1, 0:n2m+1, 0:n3m+1), G (n1m, n2m, n3m), x
// fastest; dx* (0:n*m+1).
__global__ void __launch_bounds__(256) k_cell_to_node(const double* __restrict__ P, int n1m, int n2m, int n3m,
                                                      const double* __restrict__ dx1, const double* __restrict__ dx2,
                                                      const double* __restrict__ dx3, double* __restrict__ G)
{
    const long total = (long)n1m * n2m * n3m;
    const long sy = n1m + 2, sz = (long)(n1m + 2) * (n2m + 2);
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
        const int i = (int)(q % n1m) + 1, j = (int)((q / n1m) % n2m) + 1, k = (int)(q / ((long)n1m * n2m)) + 1;
        const int im = i - 1, jm = j - 1, km = k - 1;
        auto X = [&](int a, int b, int c) { return P[a + b * sy + c * sz]; };
        // (p * wp + q * wq) / w with each product and sum rounded on its own
        // (no fused multiply-add), as the CPU evaluates it
        auto lerp = [](double p, double wp, double q, double wq, double w) {
            return __dadd_rn(__dmul_rn(p, wp), __dmul_rn(q, wq)) / w;
        };
        const double wz = __dadd_rn(dx3[k], dx3[km]), wx = __dadd_rn(dx1[i], dx1[im]);
        double X1 = lerp(X(im, jm, k), dx3[km], X(im, jm, km), dx3[k], wz);
        double X2 = lerp(X(i, jm, k), dx3[km], X(i, jm, km), dx3[k], wz);
        const double Xy1 = lerp(X2, dx1[im], X1, dx1[i], wx);
        X1 = lerp(X(im, j, k), dx3[km], X(im, j, km), dx3[k], wz);
        X2 = lerp(X(i, j, k), dx3[km], X(i, j, km), dx3[k], wz);
        const double Xy2 = lerp(X2, dx1[im], X1, dx1[i], wx);
        G[q] = lerp(Xy2, dx2[jm], Xy1, dx2[j], __dadd_rn(dx2[j], dx2[jm]));
    }
}

__global__ void k_ghost_axis_post(double* __restrict__ P, int dir, int neumann, int n1m, int n2m, int n3m, long sy,
                                  long sz, const double* __restrict__ dmx)
{
    ghost_axis(P, dir, neumann, n1m, n2m, n3m, sy, sz, dmx, 3, threadIdx.x + (long)blockIdx.x * blockDim.x,
               (long)blockDim.x * gridDim.x);
}

cudaError_t launch_ghost_update(double* P, int n1m, int n2m, int n3m, const int* per, const double* const* dmx,
                                int walls, cudaStream_t st)
{
    const long sy = n1m + 2, sz = (long)(n1m + 2) * (n2m + 2);
    const long face[3] = { (long)(n2m + 2) * (n3m + 2), (long)(n1m + 2) * (n3m + 2), (long)(n1m + 2) * (n2m + 2) };
    for (int pass = 0; pass < 2; ++pass)   // walls first, then the periodic copies
        for (int d = 0; d < 3; ++d) {
            const bool neumann = !per[d];
            if ((pass == 0) != neumann) continue;
            if (neumann && !walls) continue;
            const int blocks = (int)((face[d] + 255) / 256);
            k_ghost_axis_post<<<blocks, 256, 0, st>>>(P, d, neumann ? 1 : 0, n1m, n2m, n3m, sy, sz, dmx[d]);
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return e;
        }
    return cudaSuccess;
}

cudaError_t launch_cell_to_node(const double* P, int n1m, int n2m, int n3m, const double* dx1, const double* dx2,
                                const double* dx3, double* G, cudaStream_t st)
{
    const long total = (long)n1m * n2m * n3m;
    const long want = (total + 255) / 256;
    const int blocks = (int)(want < 148L * 32 ? want : 148L * 32);
    k_cell_to_node<<<blocks, 256, 0, st>>>(P, n1m, n2m, n3m, dx1, dx2, dx3, G);
    return cudaGetLastError();
}

}  // namespace ppf
