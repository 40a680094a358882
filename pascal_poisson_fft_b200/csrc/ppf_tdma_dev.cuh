// ppf_tdma_dev.cuh -- device-side pieces of the Poisson z solve shared by
// the z kernels (ppf_tdma.cu) and the persistent batch kernel (ppf_batch.cu):
// element access, the arithmetic policies and the per-system Thomas sweeps
// (reference arithmetic: 01_Fortran/PaScaL_TDMA/src/tdmas.f90:114-213).
#pragma once
#include "ppf_kernels.cuh"

#include <math.h>

namespace ppf {
namespace zdev {

constexpr int CH = 16;  // rows per checkpoint chunk
constexpr int TPB = 128;

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

// Poisson coefficient sources of one system (see coef_row).
struct Coef {
    const double* am;
    const double* ap;
    double lx, ly;
    bool pin;
};

// Arithmetic policies: Exact reproduces the reference's rounding (FP64,
// explicitly rounded intrinsics, IEEE division); Fast is the FP32 path of
// the mixed-precision solve (its error is removed by the FP64 refinement),
// free to contract and to use the approximate reciprocal.
struct Exact {
    using T = double;
    static constexpr int CH = 8;    // rows per checkpoint chunk (register budget of FP64 complex rows)
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
    static __device__ __forceinline__ double rcp(double a) { return __drcp_rn(a); }   // == 1.0/a, correctly rounded
};
struct Fast {
    using T = float;
    static constexpr int CH = 8;
    static __device__ __forceinline__ float mul(float a, float b) { return a * b; }
    static __device__ __forceinline__ float sub(float a, float b) { return a - b; }
    static __device__ __forceinline__ float add(float a, float b) { return a + b; }
    static __device__ __forceinline__ float div(float a, float b) { return __fdividef(a, b); }
    static __device__ __forceinline__ float rcp(float a) { return __fdividef(1.0f, a); }
};

// b = ac - dxk2 - dyk2 with ac = -am - ap, left to right
template <typename A>
__device__ __forceinline__ void coef_row(const Coef& co, int zr, typename A::T& a, typename A::T& b,
                                         typename A::T& c)
{
    using CT = typename A::T;
    if (co.pin && zr == 0) {
        a = (CT)0; b = (CT)1; c = (CT)0;
        return;
    }
    // plain loads: in the persistent batch kernel these tables are written
    // earlier in the same launch, where the read-only cache is not coherent
    const double amv = co.am[zr], apv = co.ap[zr];
    a = (CT)amv;
    c = (CT)apv;
    b = A::sub(A::sub(A::sub((CT)(-amv), (CT)apv), (CT)co.lx), (CT)co.ly);
}

// One Thomas forward step on the row state (c', d'); the first row divides.
template <typename A, bool CPLX>
__device__ __forceinline__ void fwd_row(bool first, typename A::T a, typename A::T b, typename A::T c,
                                        typename A::T dr_in, typename A::T di_in, typename A::T& cp,
                                        typename A::T& dr, typename A::T& di)
{
    if (first) {
        dr = A::div(dr_in, b);
        if (CPLX) di = A::div(di_in, b);
        cp = A::div(c, b);
    } else {
        const typename A::T r = A::rcp(A::sub(b, A::mul(a, cp)));
        dr = A::mul(r, A::sub(dr_in, A::mul(a, dr)));
        if (CPLX) di = A::mul(r, A::sub(di_in, A::mul(a, di)));
        cp = A::mul(r, c);
    }
}

template <typename T, typename CT>
__device__ __forceinline__ void ld_cv(const cx<T>* p, CT& r, CT& i)
{
    const cx<T> v = *p;
    r = (CT)v.x;
    i = (CT)v.y;
}
template <typename T, typename CT>
__device__ __forceinline__ void ld_cv(const T* p, CT& r, CT& i)
{
    r = (CT)*p;
    i = (CT)0;
}

// The z-solve of one Poisson system.  Checkpoints (c', d'r, d'i) after
// every CH rows go to global memory, [chunk][component][system], so each
// warp's checkpoint traffic is coalesced and the shared memory stays free.
template <typename T, typename A, bool CPLX>
__device__ __forceinline__ void thomas_poisson(typename Elem<T, CPLX>::type* data, long sys, long plane, int nz,
                                               const Coef& co, double scale, double* ck, double& zsum, bool& bad)
{
    using CT = typename A::T;
    constexpr int CH = A::CH;
    const int nch = (nz + CH - 1) / CH;
    CT cp = 0, dr = 0, di = 0;
    for (int ch = 0; ch < nch; ++ch) {
        const int z0 = ch * CH;
        CT vr[CH], vi[CH];
#pragma unroll
        for (int r = 0; r < CH; ++r) {
            vr[r] = (CT)0; vi[r] = (CT)0;
            if (z0 + r < nz) ld_cv<T, CT>(data + (long)(z0 + r) * plane + sys, vr[r], vi[r]);
        }
#pragma unroll
        for (int r = 0; r < CH; ++r) {
            const int zr = z0 + r;
            if (zr < nz) {
                CT a, b, c;
                coef_row<A>(co, zr, a, b, c);
                const bool pinrow = co.pin && zr == 0;
                fwd_row<A, CPLX>(zr == 0, a, b, c, pinrow ? (CT)0 : vr[r], pinrow ? (CT)0 : vi[r], cp, dr, di);
            }
        }
        double* c3 = ck + (long)(3 * ch) * plane;
        c3[0] = (double)cp;
        c3[plane] = (double)dr;
        if (CPLX) c3[2 * plane] = (double)di;
    }
    CT xr = 0, xi = 0;
    for (int ch = nch - 1; ch >= 0; --ch) {
        const int z0 = ch * CH;
        CT vr[CH], vi[CH], c_[CH];
#pragma unroll
        for (int r = 0; r < CH; ++r) {
            vr[r] = (CT)0; vi[r] = (CT)0;
            if (z0 + r < nz) ld_cv<T, CT>(data + (long)(z0 + r) * plane + sys, vr[r], vi[r]);
        }
        CT pcp = 0, pdr = 0, pdi = 0;
        if (ch > 0) {
            const double* c3 = ck + (long)(3 * (ch - 1)) * plane;
            pcp = (CT)c3[0];
            pdr = (CT)c3[plane];
            if (CPLX) pdi = (CT)c3[2 * plane];
        }
#pragma unroll
        for (int r = 0; r < CH; ++r) {
            const int zr = z0 + r;
            if (zr < nz) {
                CT a, b, c;
                coef_row<A>(co, zr, a, b, c);
                const bool pinrow = co.pin && zr == 0;
                fwd_row<A, CPLX>(zr == 0, a, b, c, pinrow ? (CT)0 : vr[r], pinrow ? (CT)0 : vi[r], pcp, pdr, pdi);
            }
            c_[r] = pcp; vr[r] = pdr; vi[r] = pdi;
        }
#pragma unroll
        for (int r = CH - 1; r >= 0; --r) {
            const int zr = z0 + r;
            if (zr < nz) {
                if (zr == nz - 1) {
                    xr = vr[r];
                    xi = vi[r];
                } else {
                    xr = A::sub(vr[r], A::mul(c_[r], xr));
                    if (CPLX) xi = A::sub(vi[r], A::mul(c_[r], xi));
                }
                const double sr = (double)xr * scale, si = (double)xi * scale;
                zsum += sr;
                if (!isfinite(sr) || !isfinite(si)) bad = true;
                st_elem<T>(data + (long)zr * plane + sys, sr, si);
            }
        }
    }
}

// Periodic z: the reference routes the solve through the cyclic Thomas
// algorithm (cuda_ptdma_core, fft_3d_poisson.f90:898-913 ->
// tdma_cycl_many_cuda) even though its coefficients zero am at k=1 and ap at
// k=n3m.  Reproduced here operation for operation (tdmas.f90:160-213):
// rows 1..nz-1 are swept for d and e (e_1 = -a_1, e_{nz-1} = -c_{nz-1}),
// x_0 is formed from the back-substituted d_1, e_1, then x_i = d_i + x_0 e_i.
// The back substitution runs twice (first for d_1, e_1) instead of storing e.
template <typename T, typename A, bool CPLX>
__device__ __forceinline__ void thomas_poisson_cyc(typename Elem<T, CPLX>::type* data, long sys, long plane, int nz,
                                                   const Coef& co, double scale, double* ck, double& zsum, bool& bad)
{
    using CT = typename A::T;
    constexpr int CH = A::CH;
    const int m = nz - 1;
    const int nch = (m + CH - 1) / CH;
    CT a1, b1, c1, an, bn, cn;
    coef_row<A>(co, 1, a1, b1, c1);
    coef_row<A>(co, nz - 1, an, bn, cn);
    const CT e_first = -a1, e_last = -cn;
    auto e_in = [&](int q) -> CT { return (q == m - 1) ? e_last : ((q == 0) ? e_first : (CT)0); };
    CT cp = 0, dr = 0, di = 0, ep = 0, dum = 0;
    for (int ch = 0; ch < nch; ++ch) {
        const int q0 = ch * CH;
        CT vr[CH], vi[CH];
#pragma unroll
        for (int r = 0; r < CH; ++r) {
            vr[r] = (CT)0; vi[r] = (CT)0;
            if (q0 + r < m) ld_cv<T, CT>(data + (long)(q0 + r + 1) * plane + sys, vr[r], vi[r]);
        }
#pragma unroll
        for (int r = 0; r < CH; ++r) {
            const int q = q0 + r;
            if (q < m) {
                CT a, b, c;
                coef_row<A>(co, q + 1, a, b, c);
                CT cpe = cp;
                fwd_row<A, CPLX>(q == 0, a, b, c, vr[r], vi[r], cp, dr, di);
                fwd_row<A, false>(q == 0, a, b, c, e_in(q), (CT)0, cpe, ep, dum);
            }
        }
        double* c4 = ck + (long)(4 * ch) * plane;
        c4[0] = (double)cp;
        c4[plane] = (double)dr;
        c4[2 * plane] = (double)di;
        c4[3 * plane] = (double)ep;
    }
    const CT dtop_r = dr, dtop_i = di, etop = ep;
    CT d1r = 0, d1i = 0, e1 = 0;
    CT x0r = 0, x0i = 0;
    for (int pass = 0; pass < 2; ++pass) {
        if (pass == 1) {
            CT a0, b0, c0;
            coef_row<A>(co, 0, a0, b0, c0);
            CT v0r = 0, v0i = 0;
            if (!co.pin) ld_cv<T, CT>(data + sys, v0r, v0i);
            const CT den = A::add(A::add(b0, A::mul(a0, etop)), A::mul(c0, e1));
            x0r = A::div(A::sub(A::sub(v0r, A::mul(a0, dtop_r)), A::mul(c0, d1r)), den);
            x0i = A::div(A::sub(A::sub(v0i, A::mul(a0, dtop_i)), A::mul(c0, d1i)), den);
        }
        CT yr = 0, yi = 0, ye = 0;
        for (int ch = nch - 1; ch >= 0; --ch) {
            const int q0 = ch * CH;
            CT vr[CH], vi[CH], c_[CH], e_[CH];
#pragma unroll
            for (int r = 0; r < CH; ++r) {
                vr[r] = (CT)0; vi[r] = (CT)0;
                if (q0 + r < m) ld_cv<T, CT>(data + (long)(q0 + r + 1) * plane + sys, vr[r], vi[r]);
            }
            CT pc = 0, pr = 0, pi = 0, pe = 0;
            if (ch > 0) {
                const double* c4 = ck + (long)(4 * (ch - 1)) * plane;
                pc = (CT)c4[0]; pr = (CT)c4[plane]; pi = (CT)c4[2 * plane]; pe = (CT)c4[3 * plane];
            }
#pragma unroll
            for (int r = 0; r < CH; ++r) {
                const int q = q0 + r;
                if (q < m) {
                    CT a, b, c;
                    coef_row<A>(co, q + 1, a, b, c);
                    CT pce = pc;
                    fwd_row<A, CPLX>(q == 0, a, b, c, vr[r], vi[r], pc, pr, pi);
                    fwd_row<A, false>(q == 0, a, b, c, e_in(q), (CT)0, pce, pe, dum);
                }
                c_[r] = pc; vr[r] = pr; vi[r] = pi; e_[r] = pe;
            }
#pragma unroll
            for (int r = CH - 1; r >= 0; --r) {
                const int q = q0 + r;
                if (q < m) {
                    if (q == m - 1) { yr = vr[r]; yi = vi[r]; ye = e_[r]; }
                    else {
                        yr = A::sub(vr[r], A::mul(c_[r], yr));
                        if (CPLX) yi = A::sub(vi[r], A::mul(c_[r], yi));
                        ye = A::sub(e_[r], A::mul(c_[r], ye));
                    }
                    if (pass == 1) {
                        const CT xr = A::add(yr, A::mul(x0r, ye));
                        const CT xi = CPLX ? A::add(yi, A::mul(x0i, ye)) : (CT)0;
                        const double sr = (double)xr * scale, si = (double)xi * scale;
                        zsum += sr;
                        if (!isfinite(sr) || !isfinite(si)) bad = true;
                        st_elem<T>(data + (long)(q + 1) * plane + sys, sr, si);
                    }
                }
            }
        }
        if (pass == 0) { d1r = yr; d1i = yi; e1 = ye; }
    }
    const double sr = (double)x0r * scale, si = (double)x0i * scale;
    zsum += sr;
    if (!isfinite(sr) || !isfinite(si)) bad = true;
    st_elem<T>(data + sys, sr, si);
}

}  // namespace zdev
}  // namespace ppf
