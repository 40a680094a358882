// ppf_slab.cu -- pieces of the z-slab (multi-rank) Poisson solve (sm_100a).
//
// With np3 > 1 the reference splits z over ranks: the x and y transforms
// stay local, and the z systems of every (kx, ky) are solved by PaScaL's
// multi-rank TDMA on coefficient arrays built per rank
// (cuda_Poisson_FFT_1D and cuda_Poisson_TDMA_z_*,
// 01_Fortran/src/fft_3d_poisson.f90:353-626, 1121-1344; the multi-rank
// PaScaL_TDMA_many_solve_cuda, PaScaL_TDMA/src/pascal_tdma_cuda.f90:243-266),
// the mean is removed with a global reduction (:628-664) and the ghost
// planes between ranks come from the neighbours (:666-796).  The kernels
// here are the rank-local steps around that exchange: the coefficient
// arrays of this rank's z rows, the interior sum, the mean shift, and the
// ghost update with z walls only at the global ends.
#include "ppf_kernels.cuh"

#include <algorithm>

namespace ppf {

namespace {

constexpr int SL_TPB = 256;

// Coefficients of this rank's rows z0 .. z0+nzl-1 of the global z operator
// for every spectral system s (re/im parts are separate systems with the
// same coefficients when the spectrum is complex); the right-hand side
// (the spectrum, in place) is scaled by the transforms' normalisation; the
// pin (a,b,c,d) = (0,1,0,0) at the global first row of (kx,ky) = (0,0)
// (fft_3d_poisson.f90:1152-1157, :1240-1249); padding columns solve to 0.
__global__ void __launch_bounds__(SL_TPB) k_slab_coef(double* __restrict__ a, double* __restrict__ b,
                                                      double* __restrict__ c, double* __restrict__ d, long ns,
                                                      int nzl, int cplx, long pitch, int mx,
                                                      const double* __restrict__ lamx,
                                                      const double* __restrict__ lamy,
                                                      const double* __restrict__ dx3, const double* __restrict__ dmx3,
                                                      int z0, int nzg, double scale)
{
    const long s = (long)blockIdx.x * SL_TPB + threadIdx.x;
    const int zl = blockIdx.y;
    if (s >= ns || zl >= nzl) return;
    const long col = cplx ? (s >> 1) : s;
    const int kx = (int)(col % pitch), ky = (int)(col / pitch);
    const int zg = z0 + zl;
    const long o = (long)zl * ns + s;
    if (kx >= mx) {
        a[o] = 0.0; b[o] = 1.0; c[o] = 0.0; d[o] = 0.0;
        return;
    }
    if (zg == 0 && kx == 0 && ky == 0) {
        a[o] = 0.0; b[o] = 1.0; c[o] = 0.0; d[o] = 0.0;
        return;
    }
    const int kk = zg + 1;
    double am = __ddiv_rn(__ddiv_rn(1.0, dx3[kk]), dmx3[kk]);
    double ap = __ddiv_rn(__ddiv_rn(1.0, dx3[kk]), dmx3[kk + 1]);
    if (zg == 0) am = 0.0;
    if (zg == nzg - 1) ap = 0.0;
    a[o] = am;
    c[o] = ap;
    b[o] = __dsub_rn(__dsub_rn(__dsub_rn(-am, ap), lamx[kx]), lamy[ky]);
    d[o] = d[o] * scale;
}

// per-(chunk, level) partial sums of the interior of the ghosted field
__global__ void __launch_bounds__(SL_TPB) k_slab_part(const double* __restrict__ P, int nx, int ny, long sy,
                                                      long sz, long chunk, int nchunk, double* __restrict__ part)
{
    __shared__ double red[SL_TPB / 32];
    const int k = blockIdx.y;
    const long plane = (long)nx * ny;
    const long i0 = (long)blockIdx.x * chunk, i1 = min(plane, i0 + chunk);
    double v = 0.0;
    for (long e = i0 + threadIdx.x; e < i1; e += SL_TPB) {
        const long j = e / nx, i = e - j * nx;
        v += P[(i + 1) + (j + 1) * sy + (long)(k + 1) * sz];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < SL_TPB / 32; ++q) t += red[q];
        part[(long)k * nchunk + blockIdx.x] = t;
    }
}

__global__ void k_slab_total(const double* __restrict__ part, long n, double* __restrict__ sum)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double t = 0.0;
    for (long q = 0; q < n; ++q) t += part[q];
    *sum = t;
}

__global__ void __launch_bounds__(SL_TPB) k_slab_shift(double* __restrict__ P, int nx, int ny, int nz, long sy,
                                                       long sz, const double* __restrict__ shift)
{
    const long total = (long)nx * ny * nz;
    const double m = *shift;
    for (long e = (long)blockIdx.x * SL_TPB + threadIdx.x; e < total; e += (long)gridDim.x * SL_TPB) {
        const long i = e % nx, r = e / nx, j = r % ny, k = r / ny;
        P[(i + 1) + (j + 1) * sy + (k + 1) * sz] -= m;
    }
}

}  // namespace

cudaError_t launch_slab_coef(double* a, double* b, double* c, double* d, long ns, int nzl, int cplx, long pitch,
                             int mx, const double* lamx, const double* lamy, const double* dx3, const double* dmx3,
                             int z0, int nzg, double scale, cudaStream_t st)
{
    dim3 grid((unsigned)((ns + SL_TPB - 1) / SL_TPB), (unsigned)nzl);
    k_slab_coef<<<grid, SL_TPB, 0, st>>>(a, b, c, d, ns, nzl, cplx, pitch, mx, lamx, lamy, dx3, dmx3, z0, nzg,
                                         scale);
    return cudaGetLastError();
}

long slab_sum_parts(const Geom& g) { return (long)g.nz * ((((long)g.nx * g.ny) + 16383) / 16384); }

cudaError_t launch_slab_sum(const double* P, const Geom& g, double* part, double* sum, cudaStream_t st)
{
    const long plane = (long)g.nx * g.ny;
    const int nchunk = (int)((plane + 16383) / 16384);
    const long chunk = (plane + nchunk - 1) / nchunk;
    k_slab_part<<<dim3(nchunk, g.nz), SL_TPB, 0, st>>>(P, g.nx, g.ny, g.pstride_y, g.pstride_z, chunk, nchunk, part);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_slab_total<<<1, 32, 0, st>>>(part, (long)nchunk * g.nz, sum);
    return cudaGetLastError();
}

cudaError_t launch_slab_shift(double* P, const Geom& g, const double* shift, cudaStream_t st)
{
    const long total = (long)g.nx * g.ny * g.nz;
    const unsigned blocks = (unsigned)std::min<long>((total + SL_TPB - 1) / SL_TPB, 148L * 16);
    k_slab_shift<<<blocks, SL_TPB, 0, st>>>(P, g.nx, g.ny, g.nz, g.pstride_y, g.pstride_z, shift);
    return cudaGetLastError();
}

}  // namespace ppf
