// ppf_tdma.cu -- batched tridiagonal solves (sm_100a).
//
// One CTA owns S consecutive systems (consecutive wavenumbers / system
// indices, so a warp's loads of one row are contiguous) and splits every
// system's rows into P partitions of M rows, one partition per thread,
// held in registers.  This is PaScaL_TDMA's distributed algorithm
// (01_Fortran/PaScaL_TDMA/src/pascal_tdma_cuda.f90:230-269, 332-520:
// partition-local elimination -> reduced system of 2 rows per partition ->
// solution update) with the MPI ranks replaced by threads:
//   1. each thread eliminates its interior rows 1..M-2 and expresses them
//      through its own first and last unknowns
//      (x_i = h_i - al_i x_0 - ga_i x_{M-1});
//   2. the 2P-row reduced system of each system is solved by parallel
//      cyclic reduction in shared memory;
//   3. each thread updates its rows and stores them.
// The right-hand side is read once and the solution written once.
//
// k_tdma_z is the Poisson z-solve.  The coefficients of the reference's
// cuda_Poisson_TDMA_z_{real,complex} (01_Fortran/src/fft_3d_poisson.f90:
// 1121-1344) -- am = 1/(dx3_k dmx3_k), ap = 1/(dx3_k dmx3_{k+1}),
// b = -am - ap - dxk2 - dyk2, the pin at (kx,ky,k) = (0,0,1) -- are
// generated in registers instead of being materialised as six N-sized
// arrays, and real and imaginary parts share one sweep.  The zero-mode mean
// removal (cuda_Poisson_average_elimination, :628-664) and the normalisation
// of the unnormalised inverse transforms are applied here, in spectral
// space.  k_tdma_arr solves systems given as coefficient arrays (the
// PaScaL_TDMA_many_solve[_cycle] replacement).
#include "ppf_kernels.cuh"

#include <math.h>

namespace ppf {

namespace {

constexpr int TDMA_M = 16;  // rows per partition (per thread)

template <typename T, bool CPLX> struct Elem;
template <typename T> struct Elem<T, true> { using type = cx<T>; };
template <typename T> struct Elem<T, false> { using type = T; };

template <typename T> __device__ __forceinline__ void ld_elem(const cx<T>* p, double& r, double& i)
{
    cx<T> v = *p;
    r = (double)v.x;
    i = (double)v.y;
}
template <typename T> __device__ __forceinline__ void ld_elem(const T* p, double& r, double& i)
{
    r = (double)*p;
    i = 0.0;
}
template <typename T> __device__ __forceinline__ void st_elem(cx<T>* p, double r, double i)
{
    *p = mk<T>((T)r, (T)i);
}
template <typename T> __device__ __forceinline__ void st_elem(T* p, double r, double)
{
    *p = (T)r;
}

// Poisson coefficients: generated from the z tables and the wavenumbers.
struct Coef {
    const double* am;
    const double* ap;
    int nz;
    double lx, ly;
    bool pin;
    __device__ __forceinline__ void get(int zr, double& a, double& b, double& cc) const
    {
        if (zr >= nz || (pin && zr == 0)) {
            a = 0.0; b = 1.0; cc = 0.0;
            return;
        }
        const double am_ = __ldg(am + zr), ap_ = __ldg(ap + zr);
        a = am_;
        cc = ap_;
        b = ((-am_ - ap_) - lx) - ly;
    }
};

// Coefficient arrays, element (sys, row) at [row * nsys + sys]; rows
// [row0, row0 + nrow) of the stored system are solved.  The sub-diagonal
// of the first and the super-diagonal of the last solved row are taken as
// zero (tdma_many never reads them; the cyclic solver moves them into its
// second right-hand side).
struct CoefArr {
    const double* a;
    const double* b;
    const double* c;
    long nsys, sys;
    int row0, nrow;
    __device__ __forceinline__ void get(int zr, double& av, double& bv, double& cv) const
    {
        if (zr >= nrow) {
            av = 0.0; bv = 1.0; cv = 0.0;
            return;
        }
        const long o = (long)(zr + row0) * nsys + sys;
        av = (zr == 0) ? 0.0 : __ldg(a + o);
        bv = __ldg(b + o);
        cv = (zr == nrow - 1) ? 0.0 : __ldg(c + o);
    }
};

// Partition-local elimination in arithmetic type CT.  On return dr/di hold
// h, al holds alpha, ga holds gamma for rows 1..M-2, and the two reduced
// rows (F: first, L: last; sub, diag, super, rhs_re, rhs_im) are returned.
template <typename CT, int M, bool CPLX, typename CO>
__device__ __forceinline__ void eliminate(const CO& co, int z0, double* dr, double* di, double* al, double* ga,
                                          double* F, double* L)
{
    double a0, b0, c0, a1, b1, c1;
    co.get(z0, a0, b0, c0);
    co.get(z0 + 1, a1, b1, c1);
    {
        const CT ib = (CT)1 / (CT)b1;
        ga[1] = (double)((CT)c1 * ib);
        al[1] = (double)((CT)a1 * ib);
        dr[1] = (double)((CT)dr[1] * ib);
        if (CPLX) di[1] = (double)((CT)di[1] * ib);
    }
#pragma unroll
    for (int r = 2; r <= M - 2; ++r) {
        double a, b, c;
        co.get(z0 + r, a, b, c);
        const CT rr = (CT)1 / ((CT)b - (CT)a * (CT)ga[r - 1]);
        dr[r] = (double)(rr * ((CT)dr[r] - (CT)a * (CT)dr[r - 1]));
        if (CPLX) di[r] = (double)(rr * ((CT)di[r] - (CT)a * (CT)di[r - 1]));
        ga[r] = (double)(rr * (CT)c);
        al[r] = (double)(-rr * (CT)a * (CT)al[r - 1]);
    }
    double aL, bL, cL;
    co.get(z0 + M - 1, aL, bL, cL);
#pragma unroll
    for (int r = M - 3; r >= 1; --r) {
        const CT e = (CT)ga[r];
        dr[r] = (double)((CT)dr[r] - e * (CT)dr[r + 1]);
        if (CPLX) di[r] = (double)((CT)di[r] - e * (CT)di[r + 1]);
        al[r] = (double)((CT)al[r] - e * (CT)al[r + 1]);
        ga[r] = (double)(-e * (CT)ga[r + 1]);
    }
    // F couples (L_{p-1}, x_0, x_{M-1}); L couples (x_0, x_{M-1}, F_{p+1})
    F[0] = a0;
    F[1] = (double)((CT)b0 - (CT)c0 * (CT)al[1]);
    F[2] = (double)(-(CT)c0 * (CT)ga[1]);
    F[3] = (double)((CT)dr[0] - (CT)c0 * (CT)dr[1]);
    F[4] = CPLX ? (double)((CT)di[0] - (CT)c0 * (CT)di[1]) : 0.0;
    L[0] = (double)(-(CT)aL * (CT)al[M - 2]);
    L[1] = (double)((CT)bL - (CT)aL * (CT)ga[M - 2]);
    L[2] = cL;
    L[3] = (double)((CT)dr[M - 1] - (CT)aL * (CT)dr[M - 2]);
    L[4] = CPLX ? (double)((CT)di[M - 1] - (CT)aL * (CT)di[M - 2]) : 0.0;
}

// Parallel cyclic reduction of the 2P-row reduced systems of S systems in
// shared memory (two buffers of 4 * 2P * S doubles; rows stored with a unit
// diagonal).  Thread (sl, p) supplies rows 2p (F) and 2p+1 (L) and receives
// their solutions.  Returns the buffer that does not hold the result.
__device__ __forceinline__ double* reduced_solve(double* sh, int p, int sl, int S, int P, const double* F,
                                                 const double* L, double& x0r, double& x0i, double& xLr,
                                                 double& xLi)
{
    const int n2 = 2 * P;
    const int NS = n2 * S;
    double* src = sh;
    double* dst = sh + 4 * NS;
    {
        const double iF = 1.0 / F[1], iL = 1.0 / L[1];
        const int qF = (2 * p) * S + sl, qL = (2 * p + 1) * S + sl;
        src[qF] = F[0] * iF; src[NS + qF] = F[2] * iF; src[2 * NS + qF] = F[3] * iF; src[3 * NS + qF] = F[4] * iF;
        src[qL] = L[0] * iL; src[NS + qL] = L[2] * iL; src[2 * NS + qL] = L[3] * iL; src[3 * NS + qL] = L[4] * iL;
    }
    __syncthreads();
    for (int d = 1; d < n2; d <<= 1) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int i = 2 * p + h;
            const int q = i * S + sl;
            const double ai = src[q], ci = src[NS + q], dri = src[2 * NS + q], dii = src[3 * NS + q];
            double am_ = 0, cm_ = 0, drm = 0, dim_ = 0, ap_ = 0, cp_ = 0, drp = 0, dip = 0;
            if (i - d >= 0) {
                const int qm = (i - d) * S + sl;
                am_ = src[qm]; cm_ = src[NS + qm]; drm = src[2 * NS + qm]; dim_ = src[3 * NS + qm];
            }
            if (i + d < n2) {
                const int qp = (i + d) * S + sl;
                ap_ = src[qp]; cp_ = src[NS + qp]; drp = src[2 * NS + qp]; dip = src[3 * NS + qp];
            }
            const double ib = 1.0 / (1.0 - ai * cm_ - ci * ap_);
            dst[q] = -ai * am_ * ib;
            dst[NS + q] = -ci * cp_ * ib;
            dst[2 * NS + q] = (dri - ai * drm - ci * drp) * ib;
            dst[3 * NS + q] = (dii - ai * dim_ - ci * dip) * ib;
        }
        __syncthreads();
        double* t = src; src = dst; dst = t;
    }
    x0r = src[2 * NS + (2 * p) * S + sl];
    x0i = src[3 * NS + (2 * p) * S + sl];
    xLr = src[2 * NS + (2 * p + 1) * S + sl];
    xLi = src[3 * NS + (2 * p + 1) * S + sl];
    return dst;
}

template <int M, bool CPLX>
__device__ __forceinline__ void update_rows(double* dr, double* di, const double* al, const double* ga, double x0r,
                                            double x0i, double xLr, double xLi)
{
    dr[0] = x0r; di[0] = x0i;
#pragma unroll
    for (int r = 1; r <= M - 2; ++r) {
        dr[r] = dr[r] - al[r] * x0r - ga[r] * xLr;
        if (CPLX) di[r] = di[r] - al[r] * x0i - ga[r] * xLi;
    }
    dr[M - 1] = xLr; di[M - 1] = xLi;
}

// Partitions / systems per CTA for n rows: P = ceil(n/M) partitions, S a
// power of two with S*P <= 256.
inline bool tdma_shape(int nrows, int& P, int& S, int& lgS)
{
    P = (nrows + TDMA_M - 1) / TDMA_M;
    if (P > 64 || P < 1) return false;
    S = 1;
    while (S * 2 * P <= 256 && S < 128) S *= 2;
    lgS = 0;
    while ((1 << lgS) < S) ++lgS;
    return true;
}

}  // namespace

template <typename T, bool CPLX>
__global__ void __launch_bounds__(256) k_tdma_z(void* __restrict__ data_, ZSys z, int lgS,
                                                const int* __restrict__ skip, int* __restrict__ err)
{
    constexpr int M = TDMA_M;
    if (skip && *skip) return;
    extern __shared__ double sh[];
    using E = typename Elem<T, CPLX>::type;
    E* data = reinterpret_cast<E*>(data_);

    const int S = 1 << lgS;
    const int P = blockDim.x >> lgS;
    const int sl = threadIdx.x & (S - 1), p = threadIdx.x >> lgS;
    const long sys = (long)blockIdx.x * S + sl;
    const int kx = (int)(sys % z.pitch), ky = (int)(sys / z.pitch);
    const bool valid = (kx < z.mx) && (ky < z.my);

    Coef co;
    co.am = z.am; co.ap = z.ap; co.nz = z.nz;
    co.lx = valid ? z.lamx[kx] : 0.0;
    co.ly = valid ? z.lamy[ky] : 0.0;
    co.pin = valid && kx == 0 && ky == 0;

    const int z0 = p * M;
    double dr[M], di[M], al[M], ga[M];
#pragma unroll
    for (int r = 0; r < M; ++r) {
        const int zr = z0 + r;
        dr[r] = 0.0; di[r] = 0.0;
        if (valid && zr < z.nz && !(co.pin && zr == 0)) ld_elem<T>(data + (long)zr * z.plane + sys, dr[r], di[r]);
    }

    double F[5], L[5];
    const bool fp64 = (sizeof(T) == 8) || ((co.lx + co.ly) * __ldg(z.dzmax2) < z.lowk);
    if (fp64) eliminate<double, M, CPLX, Coef>(co, z0, dr, di, al, ga, F, L);
    else      eliminate<float, M, CPLX, Coef>(co, z0, dr, di, al, ga, F, L);

    double x0r, x0i, xLr, xLi;
    double* freebuf = reduced_solve(sh, p, sl, S, P, F, L, x0r, x0i, xLr, xLi);
    update_rows<M, CPLX>(dr, di, al, ga, x0r, x0i, xLr, xLi);

    // zero mode: subtract the z-average of (kx,ky)=(0,0), i.e. the
    // arithmetic mean of u over all cells
    if (blockIdx.x == 0) {
        double part = 0.0;
        if (sl == 0) {
#pragma unroll
            for (int r = 0; r < M; ++r)
                if (z0 + r < z.nz) part += dr[r];
            freebuf[p] = part;
        }
        __syncthreads();
        if (sl == 0) {
            double tot = 0.0;
            for (int q = 0; q < P; ++q) tot += freebuf[q];
            const double mean = tot / (double)z.nz;
#pragma unroll
            for (int r = 0; r < M; ++r) dr[r] -= mean;
        }
    }

    bool bad = false;
#pragma unroll
    for (int r = 0; r < M; ++r) {
        const int zr = z0 + r;
        if (valid && zr < z.nz) {
            const double vr = dr[r] * z.scale, vi = di[r] * z.scale;
            if (!isfinite(vr) || !isfinite(vi)) bad = true;
            st_elem<T>(data + (long)zr * z.plane + sys, vr, vi);
        }
    }
    if (bad && err) atomicOr(err, 1);
}

template <typename T, bool CPLX>
cudaError_t launch_tdma_z(void* data, const ZSys& z, const int* skip_flag, int* err_flag, cudaStream_t st)
{
    int P, S, lgS;
    if (!tdma_shape(z.nz, P, S, lgS)) return cudaErrorInvalidConfiguration;  // nz <= 1024
    const int threads = S * P;
    const size_t smem = (size_t)2 * 4 * (2 * P) * S * sizeof(double);
    const long nsys = z.plane;  // pitch * my systems incl. padding columns
    dim3 grid((unsigned)((nsys + S - 1) / S));
    auto kern = k_tdma_z<T, CPLX>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kern<<<grid, threads, smem, st>>>(data, z, lgS, skip_flag, err_flag);
    return cudaGetLastError();
}

template cudaError_t launch_tdma_z<double, true>(void*, const ZSys&, const int*, int*, cudaStream_t);
template cudaError_t launch_tdma_z<double, false>(void*, const ZSys&, const int*, int*, cudaStream_t);
template cudaError_t launch_tdma_z<float, true>(void*, const ZSys&, const int*, int*, cudaStream_t);
template cudaError_t launch_tdma_z<float, false>(void*, const ZSys&, const int*, int*, cudaStream_t);

// --------------------------------------------------------------------------
// Coefficient-array solves (PaScaL_TDMA_many_solve / _cycle replacement).
//   non-cyclic: rows 0..n-1, right-hand side d.
//   cyclic    : the method of tdma_cycl_many (01_Fortran/PaScaL_TDMA/src/
//               tdmas.f90:160-213): rows 1..n-1 are solved for two
//               right-hand sides, d and e (e_1 = -a_1, e_{n-1} = -c_{n-1}),
//               then x_0 = (d_0 - a_0 d'_{n-1} - c_0 d'_1) /
//                          (b_0 + a_0 e'_{n-1} + c_0 e'_1),
//               x_i = d'_i + x_0 e'_i.  Both right-hand sides share one
//               sweep (as the real/imaginary pair of the complex path) and
//               the correction is applied before the store, so neither a
//               scratch e-array nor a second pass is needed.
// --------------------------------------------------------------------------
template <bool CYC>
__global__ void __launch_bounds__(256) k_tdma_arr(const double* __restrict__ a, const double* __restrict__ b,
                                                  const double* __restrict__ c, double* __restrict__ d, int n_sys,
                                                  int n_row, int lgS, int* __restrict__ err)
{
    constexpr int M = TDMA_M;
    extern __shared__ double sh[];
    const int S = 1 << lgS;
    const int P = blockDim.x >> lgS;
    const int sl = threadIdx.x & (S - 1), p = threadIdx.x >> lgS;
    const long sysl = (long)blockIdx.x * S + sl;
    const bool valid = sysl < n_sys;
    const long sys = valid ? sysl : 0;

    CoefArr co;
    co.a = a; co.b = b; co.c = c; co.nsys = n_sys; co.sys = sys;
    co.row0 = CYC ? 1 : 0;
    co.nrow = CYC ? n_row - 1 : n_row;

    const int z0 = p * M;
    double dr[M], di[M], al[M], ga[M];
#pragma unroll
    for (int r = 0; r < M; ++r) {
        const int zr = z0 + r;
        dr[r] = 0.0; di[r] = 0.0;
        if (zr < co.nrow) {
            const long o = (long)(zr + co.row0) * n_sys + sys;
            dr[r] = d[o];
            if (CYC) {
                if (zr == 0) di[r] -= __ldg(a + o);
                if (zr == co.nrow - 1) di[r] -= __ldg(c + o);
            }
        }
    }
    double F[5], L[5];
    eliminate<double, M, CYC, CoefArr>(co, z0, dr, di, al, ga, F, L);
    double x0r, x0i, xLr, xLi;
    double* freebuf = reduced_solve(sh, p, sl, S, P, F, L, x0r, x0i, xLr, xLi);
    update_rows<M, CYC>(dr, di, al, ga, x0r, x0i, xLr, xLi);

    double xfirst = 0.0;
    if (CYC) {
        // d'_1, e'_1 live in partition 0 (local row 0); d'_{n-1}, e'_{n-1}
        // in partition (n-2)/M at local row (n-2)%M
        const int last = co.nrow - 1;
        const int pl = last / M, rl = last % M;
        if (p == 0) { freebuf[sl] = dr[0]; freebuf[S + sl] = di[0]; }
        if (p == pl) {
#pragma unroll
            for (int r = 0; r < M; ++r)
                if (r == rl) { freebuf[2 * S + sl] = dr[r]; freebuf[3 * S + sl] = di[r]; }
        }
        __syncthreads();
        if (valid) {
            const double d1 = freebuf[sl], e1 = freebuf[S + sl];
            const double dn = freebuf[2 * S + sl], en = freebuf[3 * S + sl];
            const double a0 = __ldg(a + sys), b0 = __ldg(b + sys), c0 = __ldg(c + sys), d0 = d[sys];
            xfirst = (d0 - a0 * dn - c0 * d1) / (b0 + a0 * en + c0 * e1);
        }
        __syncthreads();  // every thread has read d_0 before partition 0 stores x_0
    }
    bool bad = false;
    if (valid) {
#pragma unroll
        for (int r = 0; r < M; ++r) {
            const int zr = z0 + r;
            if (zr < co.nrow) {
                const double x = CYC ? dr[r] + xfirst * di[r] : dr[r];
                if (!isfinite(x)) bad = true;
                d[(long)(zr + co.row0) * n_sys + sys] = x;
            }
        }
        if (CYC && p == 0) d[sys] = xfirst;
    }
    if (bad && err) atomicOr(err, 1);
}

cudaError_t launch_tdma_many(const double* a, const double* b, const double* c, double* d, int n_sys, int n_row,
                             bool cyclic, int* err, cudaStream_t st)
{
    int P, S, lgS;
    if (!tdma_shape(cyclic ? n_row - 1 : n_row, P, S, lgS)) return cudaErrorInvalidConfiguration;
    const int threads = S * P;
    const size_t smem = (size_t)2 * 4 * (2 * P) * S * sizeof(double);
    dim3 grid((unsigned)(((long)n_sys + S - 1) / S));
    if (cyclic) {
        auto kern = k_tdma_arr<true>;
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
        }
        kern<<<grid, threads, smem, st>>>(a, b, c, d, n_sys, n_row, lgS, err);
    } else {
        auto kern = k_tdma_arr<false>;
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
        }
        kern<<<grid, threads, smem, st>>>(a, b, c, d, n_sys, n_row, lgS, err);
    }
    return cudaGetLastError();
}

// z coefficients of cuda_Poisson_TDMA_z_* (fft_3d_poisson.f90:1139-1142):
// am_k = 1/dx3_k/dmx3_k, ap_k = 1/dx3_k/dmx3_{k+1}, am_1 = ap_n3m = 0; plus
// max_k dx3_k^2 for the low-wavenumber precision switch.  One CTA.
__global__ void __launch_bounds__(256) k_zcoef(const double* __restrict__ dx3, const double* __restrict__ dmx3,
                                               int nz, double* __restrict__ am, double* __restrict__ ap,
                                               double* __restrict__ dzmax2)
{
    __shared__ double red[256];
    double mx = 0.0;
    for (int k = threadIdx.x; k < nz; k += blockDim.x) {
        const int kk = k + 1;
        double av = 1.0 / dx3[kk] / dmx3[kk];
        double cv = 1.0 / dx3[kk] / dmx3[kk + 1];
        if (k == 0) av = 0.0;
        if (k == nz - 1) cv = 0.0;
        am[k] = av;
        ap[k] = cv;
        mx = fmax(mx, dx3[kk] * dx3[kk]);
    }
    red[threadIdx.x] = mx;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *dzmax2 = red[0];
}

cudaError_t launch_zcoef(const double* dx3, const double* dmx3, int nz, double* am, double* ap, double* dzmax2,
                         cudaStream_t st)
{
    k_zcoef<<<1, 256, 0, st>>>(dx3, dmx3, nz, am, ap, dzmax2);
    return cudaGetLastError();
}

}  // namespace ppf
