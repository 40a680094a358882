// ppf_adjoint.cu -- transpose of the solve map and the z-metric gradient
// (sm_100a).  The reference has no adjoint; this is the differentiation
// addition to its solve path.
//
// The solve is u = P0 M' f (transforms in x and y, one z system per
// (kx, ky) with the zero mode pinned, inverse transforms, arithmetic-mean
// removal P0).  The x and y operators are symmetric (uniform 3-point,
// periodic or mirror-Neumann); the z operator T = V^-1 S (V = diag(dx3),
// S symmetric: S_{k,k+1} = 1/dmx3_{k+1}), so T^-T = V T^-1 V^-1 for every
// system but the pinned zero mode.  The transpose is therefore
//     M^T g = V M (V^-1 g) + c(z),
// one ordinary solve (any precision, refinement included) between two
// diagonal scalings, plus a per-level constant c that replaces the zero
// mode of V M V^-1 by the transposed pinned system, solved here in FP64
// from the plane sums of g.  Each level's plane mean is removed from g
// before the scaling: that changes only the zero mode (replaced anyway) and
// makes the scaled right-hand side compatible, so the FP64 residual of a
// mixed-precision solve can converge.  With the forward solution u given, the
// gradient of J = <g, u> (g = dJ/du) with respect to the z coefficients is
//     dJ/dam_k = -sum_xy df_k (u_{k-1} - u_k),  dJ/dap_k = -sum_xy df_k (u_{k+1} - u_k),
// with df = M^T g, minus the zero-mode part of the pinned row
// (+ sum_xy df_0 * (sum_xy u_1 - sum_xy u_0) / (nx ny) on ap_0), chained
// to dx3 and dmx3 through am_k = 1/dx3_k/dmx3_k, ap_k = 1/dx3_k/dmx3_{k+1}
// (fft_3d_poisson.f90:1139-1144).  Every reduction is per block in a fixed
// order, then across blocks in a fixed order: the results are deterministic.
#include "ppf_kernels.cuh"

namespace ppf {

namespace {

constexpr int ADJ_TPB = 256;

__device__ __forceinline__ double block_sum(double v, double* red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) s += red[q];
    __syncthreads();
    return s;  // valid in thread 0
}

// per-(chunk, level) partial sums of g
__global__ void __launch_bounds__(ADJ_TPB) k_adj_sum(const double* __restrict__ g, long plane, long chunk,
                                                      int nchunk, double* __restrict__ colpart)
{
    __shared__ double red[ADJ_TPB / 32];
    const int k = blockIdx.y;
    const long i0 = (long)blockIdx.x * chunk;
    const long i1 = min(plane, i0 + chunk);
    const double* gk = g + (long)k * plane;
    double s = 0.0;
    for (long i = i0 + threadIdx.x; i < i1; i += blockDim.x) s += gk[i];
    s = block_sum(s, red);
    if (threadIdx.x == 0) colpart[(long)k * nchunk + blockIdx.x] = s;
}

// h = (g - plane mean of g) / dx3_k (dense; h may alias g)
__global__ void __launch_bounds__(ADJ_TPB) k_adj_rhs(const double* g, double* h, const double* __restrict__ dx3,
                                                      long plane, long chunk, int nchunk,
                                                      const double* __restrict__ colpart)
{
    __shared__ double mean;
    const int k = blockIdx.y;
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int c = 0; c < nchunk; ++c) s += colpart[(long)k * nchunk + c];
        mean = s / (double)plane;
    }
    __syncthreads();
    const long i0 = (long)blockIdx.x * chunk;
    const long i1 = min(plane, i0 + chunk);
    const double inv = 1.0 / dx3[k + 1], m = mean;
    const long base = (long)k * plane;
    for (long i = i0 + threadIdx.x; i < i1; i += blockDim.x) h[base + i] = (g[base + i] - m) * inv;
}

// Zero-mode correction c(z) (one block; the serial solve runs in thread 0)
__global__ void __launch_bounds__(ADJ_TPB) k_adj_corr(const double* __restrict__ colpart, int nchunk, int nz,
                                                       const double* __restrict__ am, const double* __restrict__ ap,
                                                       double nxy, double* __restrict__ corr,
                                                       double* __restrict__ wk)
{
    // wk: 3 * nz doubles of scratch (plane sums, factors, solution)
    double* cs = wk;
    double* cp = wk + nz;
    double* x2 = wk + 2 * nz;
    for (int k = threadIdx.x; k < nz; k += blockDim.x) {
        double s = 0.0;
        for (int c = 0; c < nchunk; ++c) s += colpart[(long)k * nchunk + c];
        cs[k] = s;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    double tot = 0.0;
    for (int k = 0; k < nz; ++k) tot += cs[k];
    // zero mode of M^T g: T00^T x = cs - mean, T00^T having sub-diagonal
    // c_{k-1} (c_0 = 0 at the pin), super-diagonal a_{k+1}, diagonal b_k (b_0 = 1);
    // the scaled right-hand side has no zero mode, so nothing is subtracted
    const double mean = tot / (double)nz;
    double cprev = 0.0, dprev = 0.0;
    for (int k = 0; k < nz; ++k) {
        const double a = (k >= 2) ? ap[k - 1] : 0.0;
        const double c = (k + 1 < nz) ? am[k + 1] : 0.0;
        const double b = (k == 0) ? 1.0 : (-am[k] - ap[k]);
        const double r = 1.0 / (b - a * cprev);
        cprev = c * r;
        dprev = ((cs[k] - mean) - a * dprev) * r;
        cp[k] = cprev;
        x2[k] = dprev;
    }
    for (int k = nz - 2; k >= 0; --k) x2[k] -= cp[k] * x2[k + 1];
    for (int k = 0; k < nz; ++k) corr[k] = x2[k] / nxy;
}

// df = dx3_k * W + c_k (W: ghosted solution of the scaled right-hand side);
// with u: per-(chunk, level) partial sums of df (u_{k-1} - u_k),
// df (u_{k+1} - u_k), df and u.
__global__ void __launch_bounds__(ADJ_TPB) k_adj_out(const double* __restrict__ W, double* __restrict__ df,
                                                      const double* __restrict__ dx3, const double* __restrict__ corr,
                                                      const double* __restrict__ u, int nx, int ny, int nz, long sy,
                                                      long sz, long chunk, int nchunk, double* __restrict__ mpart)
{
    __shared__ double red[ADJ_TPB / 32];
    const int k = blockIdx.y;
    const long plane = (long)nx * ny;
    const long i0 = (long)blockIdx.x * chunk;
    const long i1 = min(plane, i0 + chunk);
    const double s3 = dx3[k + 1], ck = corr[k];
    double sm = 0.0, sp = 0.0, sd = 0.0, su = 0.0;
    for (long e = i0 + threadIdx.x; e < i1; e += blockDim.x) {
        const long j = e / nx, i = e - j * nx;
        const long o = (i + 1) + (j + 1) * sy + (long)(k + 1) * sz;
        const double v = s3 * W[o] + ck;
        df[(long)k * plane + e] = v;
        if (u) {
            const double uc = u[o];
            if (k > 0) sm += v * (u[o - sz] - uc);
            if (k < nz - 1) sp += v * (u[o + sz] - uc);
            sd += v;
            su += uc;
        }
    }
    if (!u) return;
    sm = block_sum(sm, red);
    sp = block_sum(sp, red);
    sd = block_sum(sd, red);
    su = block_sum(su, red);
    if (threadIdx.x == 0) {
        const long q = (long)nz * nchunk, at = (long)k * nchunk + blockIdx.x;
        mpart[at] = sm;
        mpart[q + at] = sp;
        mpart[2 * q + at] = sd;
        mpart[3 * q + at] = su;
    }
}

// reduce the partials per level and chain dJ/dam, dJ/dap to dx3, dmx3
// (Fortran index j = 0..nz+1; cell k is j = k+1)
__global__ void __launch_bounds__(ADJ_TPB) k_adj_metric(const double* __restrict__ mpart, int nchunk, int nz,
                                                         double nxy, const double* __restrict__ am,
                                                         const double* __restrict__ ap, const double* __restrict__ dx3,
                                                         const double* __restrict__ dmx3, double* __restrict__ ddx3,
                                                         double* __restrict__ ddmx3, double* __restrict__ wk)
{
    double* dam = wk;
    double* dap = wk + nz;
    double* sdu = wk + 2 * nz;  // [0] sum df_0, [1] sum u_0, [2] sum u_1
    const long q = (long)nz * nchunk;
    for (int k = threadIdx.x; k < nz; k += blockDim.x) {
        double a = 0.0, b = 0.0, d = 0.0, s = 0.0;
        for (int c = 0; c < nchunk; ++c) {
            const long at = (long)k * nchunk + c;
            a += mpart[at];
            b += mpart[q + at];
            d += mpart[2 * q + at];
            s += mpart[3 * q + at];
        }
        dam[k] = (k == 0) ? 0.0 : -a;
        dap[k] = (k == nz - 1) ? 0.0 : -b;
        if (k == 0) { sdu[0] = d; sdu[1] = s; }
        if (k == 1) sdu[2] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0 && nz > 1) dap[0] += sdu[0] * (sdu[2] - sdu[1]) / nxy;
    __syncthreads();
    for (int j = threadIdx.x; j < nz + 2; j += blockDim.x) {
        double gx = 0.0, gm = 0.0;
        if (j >= 1 && j <= nz) {
            const int k = j - 1;
            gx = -(dam[k] * am[k] + dap[k] * ap[k]) / dx3[j];
            gm -= dam[k] * am[k] / dmx3[j];
        }
        if (j >= 2 && j <= nz + 1) {
            const int k = j - 2;
            gm -= dap[k] * ap[k] / dmx3[j];
        }
        if (ddx3) ddx3[j] = gx;
        if (ddmx3) ddmx3[j] = gm;
    }
}

}  // namespace

int adjoint_chunks(long plane, long* chunk)
{
    const long target = 16384;
    int n = (int)((plane + target - 1) / target);
    if (n < 1) n = 1;
    if (n > 64) n = 64;
    long c = (plane + n - 1) / n;
    c = (c + ADJ_TPB - 1) / ADJ_TPB * ADJ_TPB;
    *chunk = c;
    return (int)((plane + c - 1) / c);
}

cudaError_t launch_adj_rhs(const double* g, double* h, const double* dx3, const Geom& gm, long chunk, int nchunk,
                           double* colpart, cudaStream_t st)
{
    const long plane = (long)gm.nx * gm.ny;
    k_adj_sum<<<dim3(nchunk, gm.nz), ADJ_TPB, 0, st>>>(g, plane, chunk, nchunk, colpart);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_adj_rhs<<<dim3(nchunk, gm.nz), ADJ_TPB, 0, st>>>(g, h, dx3, plane, chunk, nchunk, colpart);
    return cudaGetLastError();
}

cudaError_t launch_adj_corr(const double* colpart, int nchunk, const Geom& gm, const double* am, const double* ap,
                            double* corr, double* wk, cudaStream_t st)
{
    k_adj_corr<<<1, ADJ_TPB, 0, st>>>(colpart, nchunk, gm.nz, am, ap, (double)gm.nx * gm.ny, corr, wk);
    return cudaGetLastError();
}

cudaError_t launch_adj_out(const double* W, double* df, const double* dx3, const double* corr, const double* u,
                           const Geom& gm, long chunk, int nchunk, double* mpart, cudaStream_t st)
{
    k_adj_out<<<dim3(nchunk, gm.nz), ADJ_TPB, 0, st>>>(W, df, dx3, corr, u, gm.nx, gm.ny, gm.nz, gm.pstride_y,
                                                      gm.pstride_z, chunk, nchunk, mpart);
    return cudaGetLastError();
}

cudaError_t launch_adj_metric(const double* mpart, int nchunk, const Geom& gm, const double* am, const double* ap,
                              const double* dx3, const double* dmx3, double* ddx3, double* ddmx3, double* wk,
                              cudaStream_t st)
{
    k_adj_metric<<<1, ADJ_TPB, 0, st>>>(mpart, nchunk, gm.nz, (double)gm.nx * gm.ny, am, ap, dx3, dmx3, ddx3,
                                        ddmx3, wk);
    return cudaGetLastError();
}

}  // namespace ppf
