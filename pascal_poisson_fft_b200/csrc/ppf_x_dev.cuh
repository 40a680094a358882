// ppf_x_dev.cuh -- device bodies of the x-direction transforms, shared by
// the x kernels (ppf_x.cu) and the persistent batch kernel (ppf_batch.cu).
// One call transforms tile `tile` of W consecutive x-lines (fixed y, z) in
// shared memory (ppf_fft.cuh): a real FFT through a half-length complex FFT
// and a split, or a DCT-II with Makhoul's reordering folded into the tile load
// and the post-twiddle folded into the store (the reference runs each as a
// cuFFT call bracketed by reorder, twiddle, copy and scale passes,
// 01_Fortran/src/fft_3d_poisson.f90:378-419, 561-616, 915-1033).
#pragma once
#include "ppf_xy_common.cuh"

#include <type_traits>

namespace ppf {

constexpr int ct_log2(int w) { return w <= 1 ? 0 : 1 + ct_log2(w / 2); }
constexpr int MAXW = 128;  // widest tile of any shape (FP32, n = 32)

// Per-line tables and reduction slots of the x tiles.  They live in
// non-template functions so that a kernel holding several instantiations of
// the tile bodies (the persistent batch kernel) has one copy of each, not one
// per instantiation (static shared memory is limited to 48 KB).
__device__ __forceinline__ long* x_line_longs()      // 3 x MAXW
{
    __shared__ long buf[3 * MAXW];
    return buf;
}
__device__ __forceinline__ double* x_line_doubles()  // 2 x MAXW
{
    __shared__ double buf[2 * MAXW];
    return buf;
}
__device__ __forceinline__ double* x_red_slots()     // 3 x 32
{
    __shared__ double buf[3 * 32];
    return buf;
}

// n elements at base + o into L2, in bulk: the 16-byte aligned part of the
// range (start rounded up, end rounded down), so the copy never leaves it
template <typename U>
__device__ __forceinline__ void prefetch_row(const U* base, long o, int n)
{
    const size_t a = (reinterpret_cast<size_t>(base + o) + 15) & ~(size_t)15;
    const size_t e = reinterpret_cast<size_t>(base + o + n) & ~(size_t)15;
    if (e > a) prefetch_l2(reinterpret_cast<const void*>(a), (unsigned)(e - a));
}

// the two values at p, p+1 (p 16-byte aligned for FP64, 8-byte for FP32);
// NC: through the read-only cache (only for data no earlier part of the
// same kernel launch wrote)
template <bool NC>
__device__ __forceinline__ void ld_pair_al(const double* p, double& a, double& b)
{
    const double2 v = NC ? __ldg(reinterpret_cast<const double2*>(p)) : *reinterpret_cast<const double2*>(p);
    a = v.x;
    b = v.y;
}
template <bool NC>
__device__ __forceinline__ void ld_pair_al(const float* p, double& a, double& b)
{
    const float2 v = NC ? __ldg(reinterpret_cast<const float2*>(p)) : *reinterpret_cast<const float2*>(p);
    a = (double)v.x;
    b = (double)v.y;
}

// --------------------------------------------------------------------------
// x forward: real lines (FP64 input, optionally f - L u) -> half spectrum
// (R2C, complex rows of nx/2+1) or DCT-II (real rows of nx).  RESID: 0 none,
// 1 the residual of the FP64 iterate rs.P, 2 of the FP32 iterate rs.U (same
// ghosted layout; its values are FP32 numbers, so f - L u is the same).
// --------------------------------------------------------------------------
template <typename T, bool DCT, int RESID, typename SH, bool NC = true>
__device__ __forceinline__ void xfwd(const double* __restrict__ f, const ResidIn& rs, const Geom& g,
                                     void* __restrict__ out_, long out_pitch, const FftSched& sch, int Wrt, int lgWrt,
                                     const cx<T>* __restrict__ tw_half, const cx<T>* __restrict__ tw_n,
                                     const cx<T>* __restrict__ tw_dct, const int* __restrict__ skip, long tile)
{
    if (skip && *skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* s = reinterpret_cast<cx<T>*>(smem_raw);
    constexpr bool CT = SH::CT;
    const int W = CT ? SH::W : Wrt;
    const int lgW = CT ? ct_log2(SH::W) : lgWrt;
    const int NTH = CT ? SH::NT : (int)blockDim.x;
    const int nc = CT ? SH::N : (g.nx >> 1);
    const int nx = 2 * nc;
    const long nlines = (long)g.ny * g.nz;
    const long line0 = tile * W;
    const int E = nc << lgW;
    // per line of the tile: offset of its first cell in the ghosted P and
    // the z coefficients of its level (no per-element division)
    long* const line_c = x_line_longs();
    double* const line_am = x_line_doubles();
    double* const line_ap = line_am + MAXW;
    if (RESID) {
        for (int l = threadIdx.x; l < W; l += NTH) {
            const long line = line0 + l;
            const long j = line % g.ny, k = line / g.ny;
            line_c[l] = 1 + (j + 1) * g.pstride_y + (k + 1) * g.pstride_z;
            line_am[l] = (k < g.nz) ? rs.am[k] : 0.0;
            line_ap[l] = (k < g.nz) ? rs.ap[k] : 0.0;
        }
        __syncthreads();
    }
    // this tile's rows of f (and the iterate's rows of its lines) into L2 in
    // bulk, so the loads below wait on L2, not on HBM: one warp issues few
    // loads at a time and the tile's 64 KB would otherwise trickle in
    if (threadIdx.x < W && line0 + threadIdx.x < nlines) {
        const long line = line0 + threadIdx.x;
        prefetch_row(f, line * nx, nx);
        if constexpr (RESID != 0) {
            const long o = (line % g.ny + 1) * g.pstride_y + (line / g.ny + 1) * g.pstride_z;
            if constexpr (RESID == 2) prefetch_row(rs.U, o, nx + 2);
            else prefetch_row(rs.P, o, nx + 2);
        }
    }
    // f and the iterate are 16-byte aligned (cudaMalloc'd arrays): pairs load
    // as one vector (the pair (2n-1, 2n) of a ghosted row starts at an even index)
    const bool vec = ((reinterpret_cast<size_t>(f) | reinterpret_cast<size_t>(rs.P) |
                       reinterpret_cast<size_t>(rs.U)) & 15) == 0;
    const long sy = g.pstride_y, sz = g.pstride_z;

    for (int e = threadIdx.x; e < E; e += NTH) {
        const int l = e / nc, n = e - l * nc;
        const long line = line0 + l;
        cx<T> z = mk<T>((T)0, (T)0);
        if (line < nlines) {
            const double* fl = f + line * nx + 2 * n;
            double a, b;
            if (vec) {
                const double2 fv = __ldg(reinterpret_cast<const double2*>(fl));
                a = fv.x;
                b = fv.y;
            } else {
                a = fl[0];
                b = fl[1];
            }
            if (RESID) {
                // f - L_h u at cells 2n and 2n+1.  The ghost cells hold the
                // stencil's neighbours (periodic copies or wall mirrors, written
                // by the previous x-inverse pass), so no index wraps here.
                using UT = typename std::conditional<RESID == 2, float, double>::type;
                const UT* ub;
                if constexpr (RESID == 2) ub = rs.U; else ub = rs.P;
                const UT* c = ub + line_c[l] + 2 * n;   // c[0] = u(2n), odd offset
                double xm, u0, u1, xp;
                if (vec) {
                    ld_pair_al<NC>(c - 1, xm, u0);
                    ld_pair_al<NC>(c + 1, u1, xp);
                } else {
                    xm = c[-1]; u0 = c[0]; u1 = c[1]; xp = c[2];
                }
                const double ym0 = c[-sy], ym1 = c[1 - sy], yp0 = c[sy], yp1 = c[1 + sy];
                const double zm0 = c[-sz], zm1 = c[1 - sz], zp0 = c[sz], zp1 = c[1 + sz];
                const double am = line_am[l], ap = line_ap[l];
                a -= (xm - 2.0 * u0 + u1) * rs.ix2 + (ym0 - 2.0 * u0 + yp0) * rs.iy2 + am * (zm0 - u0) +
                     ap * (zp0 - u0);
                b -= (u0 - 2.0 * u1 + xp) * rs.ix2 + (ym1 - 2.0 * u1 + yp1) * rs.iy2 + am * (zm1 - u1) +
                     ap * (zp1 - u1);
            }
            z = mk<T>((T)a, (T)b);
        }
        s[tidx<T, SH>(n, l, W)] = z;
    }
    __syncthreads();

    if (DCT) {
        // Makhoul order v = [x0, x2, .., x_{n-2}, x_{n-1}, .., x3, x1]
        // (cuda_Poisson_DCT_f_pre, fft_3d_poisson.f90:915-935), packed as
        // complex pairs (v_{2m}, v_{2m+1}) for the half-length FFT.
        constexpr int EPT = CT ? (SH::N * SH::W + SH::NT - 1) / SH::NT : 8;
        cx<T> tmp[EPT];
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
            const int e = threadIdx.x + i * NTH;
            if (e < E) {
                const int l = e / nc, m = e - l * nc;
                const int q0 = 2 * m, q1 = 2 * m + 1;
                const T v0 = (q0 < nc) ? s[tidx<T, SH>(q0, l, W)].x : s[tidx<T, SH>(nx - 1 - q0, l, W)].y;
                const T v1 = (q1 < nc) ? s[tidx<T, SH>(q1, l, W)].x : s[tidx<T, SH>(nx - 1 - q1, l, W)].y;
                tmp[i] = mk<T>(v0, v1);
            }
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
            const int e = threadIdx.x + i * NTH;
            if (e < E) {
                const int l = e / nc, m = e - l * nc;
                s[tidx<T, SH>(m, l, W)] = tmp[i];
            }
        }
        __syncthreads();
    }

    tile_fft<T, false, SH>(s, sch, W, lgW, tw_half);

    if (!DCT) {
        cx<T>* out = reinterpret_cast<cx<T>*>(out_);
        // R2C split, one pair (k, nc-k) per iteration from z_k and z_{nc-k}
        const int NP = nc / 2 + 1;
        for (int e = threadIdx.x; e < (NP << lgW); e += NTH) {
            const int l = e / NP, k = e - l * NP;
            const long line = line0 + l;
            if (line >= nlines) continue;
            const int kc = nc - k;
            const cx<T> a = s[tidx<T, SH>(k, l, W)];
            const cx<T> b = s[tidx<T, SH>(k == 0 ? 0 : kc, l, W)];
            cx<T>* orow = out + line * out_pitch;
            {
                const cx<T> zc = conj(b);
                const cx<T> Ev = (a + zc) * (T)0.5;
                const cx<T> D = a - zc;
                const cx<T> O = mk<T>(D.y * (T)0.5, -D.x * (T)0.5);
                orow[k] = Ev + cmul(ldg(tw_n + k), O);
            }
            if (kc != k) {
                const cx<T> zc = conj(a);
                const cx<T> Ev = (b + zc) * (T)0.5;
                const cx<T> D = b - zc;
                const cx<T> O = mk<T>(D.y * (T)0.5, -D.x * (T)0.5);
                orow[kc] = Ev + cmul(ldg(tw_n + kc), O);
            }
        }
    } else {
        // X_k = 2 Re(e^{-i pi k/(2n)} V_k), V_{n-k} = conj(V_k)
        // (cuda_Poisson_DCT_f_post, fft_3d_poisson.f90:937-969)
        T* out = reinterpret_cast<T*>(out_);
        const int Eo = nx * W;
        for (int e = threadIdx.x; e < Eo; e += NTH) {
            const int l = e / nx, k = e - l * nx;
            const long line = line0 + l;
            if (line >= nlines) continue;
            const int kap = (k <= nc) ? k : nx - k;
            const cx<T> zk = s[tidx<T, SH>(kap == nc ? 0 : kap, l, W)];
            const cx<T> zc = conj(s[tidx<T, SH>(kap == 0 ? 0 : nc - kap, l, W)]);
            const cx<T> Ev = (zk + zc) * (T)0.5;
            const cx<T> D = zk - zc;
            const cx<T> O = mk<T>(D.y * (T)0.5, -D.x * (T)0.5);
            cx<T> V = Ev + cmul(ldg(tw_n + kap), O);
            if (k > nc) V = conj(V);
            const cx<T> w = ldg(tw_dct + k);
            out[line * out_pitch + k] = (T)2 * (w.x * V.x - w.y * V.y);
        }
    }
}

template <int UK>
__device__ __forceinline__ void x_ghosts(double* __restrict__ P, float* __restrict__ U, const Geom& g, long line0,
                                         int W, long nlines, int nx)
{
    for (int t = threadIdx.x; t < 2 * W; t += blockDim.x) {
        const long line = line0 + (t >> 1);
        if (line >= nlines) continue;
        const long ob = 1 + (line % g.ny + 1) * g.pstride_y + (line / g.ny + 1) * g.pstride_z;
        const long from = (t & 1) ? ob + nx - 1 : ob;
        const long to = (t & 1) ? from + (g.px ? -nx : 1) : from + (g.px ? nx : -1);
        if constexpr (UK == U_WRITE) U[to] = U[from];
        else P[to] = P[from];
    }
}

// --------------------------------------------------------------------------
// x inverse: half spectrum (C2R) or DCT coefficients (inverse DCT) ->
// interior of the ghosted output.  ACC: u <- (u - mean_prev) + du.
// partials (optional): per-block [sum du^2, sum u^2, sum u].  UK (UKind):
// U_P reads and writes the FP64 P, U_WRITE writes the FP32 field U instead
// (values that are FP32 numbers already), U_ACC reads u from U and writes P.
// --------------------------------------------------------------------------
template <typename T, bool DCT, bool ACC, bool GHOST, typename SH, int UK = U_P>
__device__ __forceinline__ void xinv(const void* __restrict__ in_, long in_pitch, double* __restrict__ P,
                                     float* __restrict__ U, const Geom& g, double* __restrict__ partials,
                                     const double* __restrict__ mean_prev, const FftSched& sch, int Wrt, int lgWrt,
                                     const cx<T>* __restrict__ tw_half, const cx<T>* __restrict__ tw_n,
                                     const cx<T>* __restrict__ tw_dct, const int* __restrict__ skip, long tile)
{
    if (skip && *skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* s = reinterpret_cast<cx<T>*>(smem_raw);
    constexpr bool CT = SH::CT;
    const int W = CT ? SH::W : Wrt;
    const int lgW = CT ? ct_log2(SH::W) : lgWrt;
    const int NTH = CT ? SH::NT : (int)blockDim.x;
    const int nc = CT ? SH::N : (g.nx >> 1);
    const int nx = 2 * nc;
    const long nlines = (long)g.ny * g.nz;
    const long line0 = tile * W;
    const int E = nc << lgW;
    // the tile's spectral rows into L2 in bulk
    if (threadIdx.x < W && line0 + threadIdx.x < nlines) {
        const long line = line0 + threadIdx.x;
        if (DCT) prefetch_row(reinterpret_cast<const T*>(in_), line * in_pitch, nx);
        else prefetch_row(reinterpret_cast<const cx<T>*>(in_), line * in_pitch, nc + 1);
    }
    // the rows of u this tile updates are fetched into L2 in bulk now, so that
    // the read-modify-write after the transform finds them there
    if (ACC && threadIdx.x < W) {
        const long line = line0 + threadIdx.x;
        const long o = (line % g.ny + 1) * g.pstride_y + (line / g.ny + 1) * g.pstride_z;
        if (line < nlines) {
            if (UK == U_ACC) prefetch_row(U, o, nx + 2);
            else prefetch_row(P, o, nx + 2);
        }
    }
    // the iterate read by ACC and the one written
    auto src = [&](long o) -> double {
        if constexpr (UK == U_ACC) return (double)U[o];
        else return P[o];
    };
    auto put = [&](long o, double v) {
        if constexpr (UK == U_WRITE) U[o] = (float)v;
        else P[o] = v;
    };

    if constexpr (!DCT) {
        // C2R split, one pair (k, nc-k) per iteration: Z_k from (X_k, conj X_{nc-k}),
        // Z_{nc-k} from (X_{nc-k}, conj X_k)
        const int NP = nc / 2 + 1;
        for (int e = threadIdx.x; e < (NP << lgW); e += NTH) {
            const int l = e / NP, k = e - l * NP;
            const int kc = nc - k;
            const long line = line0 + l;
            cx<T> Zk = mk<T>((T)0, (T)0), Zc = Zk;
            if (line < nlines) {
                const cx<T>* row = reinterpret_cast<const cx<T>*>(in_) + line * in_pitch;
                cx<T> xa = row[k], xb = row[kc];
                if (k == 0) { xa.y = (T)0; xb.y = (T)0; }
                {
                    const cx<T> c = conj(xb);
                    const cx<T> Ev = xa + c, D = xa - c;
                    const cx<T> O = cmul(D, conj(ldg(tw_n + k)));
                    Zk = mk<T>(Ev.x - O.y, Ev.y + O.x);
                }
                {
                    const cx<T> c = conj(xa);
                    const cx<T> Ev = xb + c, D = xb - c;
                    const cx<T> O = cmul(D, conj(ldg(tw_n + kc)));
                    Zc = mk<T>(Ev.x - O.y, Ev.y + O.x);
                }
            }
            s[tidx<T, SH>(k, l, W)] = Zk;
            if (k != 0 && kc != k) s[tidx<T, SH>(kc, l, W)] = Zc;
        }
    } else
    for (int e = threadIdx.x; e < E; e += NTH) {
        const int l = e / nc, k = e - l * nc;
        const long line = line0 + l;
        cx<T> Z = mk<T>((T)0, (T)0);
        if (line < nlines) {
            cx<T> xk, xc;
            if (!DCT) {
                const cx<T>* row = reinterpret_cast<const cx<T>*>(in_) + line * in_pitch;
                xk = row[k];
                xc = conj(row[nc - k]);
                if (k == 0) { xk.y = (T)0; xc.y = (T)0; }
            } else {
                // b_pre: Zs_j = e^{i pi j/(2n)} (X_j - i X_{n-j}), X_n = 0
                const T* row = reinterpret_cast<const T*>(in_) + line * in_pitch;
                const int j0 = k, j1 = nc - k;
                const T a0 = row[j0], b0 = (j0 == 0) ? (T)0 : row[nx - j0];
                const T a1 = row[j1], b1 = (j1 == 0) ? (T)0 : row[nx - j1];
                const cx<T> w0 = ldg(tw_dct + j0), w1 = ldg(tw_dct + j1);
                const T c0 = w0.x, s0 = -w0.y, c1 = w1.x, s1 = -w1.y;
                xk = mk<T>(c0 * a0 + s0 * b0, s0 * a0 - c0 * b0);
                xc = mk<T>(c1 * a1 + s1 * b1, -(s1 * a1 - c1 * b1));
                if (k == 0) { xk.y = (T)0; xc.y = (T)0; }
            }
            const cx<T> Ev = xk + xc;
            const cx<T> D = xk - xc;
            const cx<T> O = cmul(D, conj(ldg(tw_n + k)));
            Z = mk<T>(Ev.x - O.y, Ev.y + O.x);
        }
        s[tidx<T, SH>(k, l, W)] = Z;
    }
    // ghosted-output offset of each line of the tile, and (GHOST) the offsets
    // of the ghost lines its values are copied to (0: none)
    long* const line_base = x_line_longs();
    long* const line_gy = line_base + MAXW;
    long* const line_gz = line_base + 2 * MAXW;
    bool has_yz = false;
    for (int l = threadIdx.x; l < W; l += NTH) {
        const long line = line0 + l;
        const long j = line % g.ny, k = line / g.ny;
        line_base[l] = 1 + (j + 1) * g.pstride_y + (k + 1) * g.pstride_z;
        if (GHOST) {
            // y: periodic copy to the opposite ghost row, or mirror at the wall
            long gy = 0;
            if (j == 0) gy = g.py ? (long)g.ny * g.pstride_y : -g.pstride_y;
            else if (j == g.ny - 1) gy = g.py ? -(long)g.ny * g.pstride_y : g.pstride_y;
            // z: any finite value (the wall coefficients am_1, ap_n3m are 0)
            long gz = 0;
            if (k == 0) gz = -g.pstride_z;
            else if (k == g.nz - 1) gz = g.pstride_z;
            line_gy[l] = gy;
            line_gz[l] = gz;
            has_yz |= (line < nlines) && (gy || gz);
        }
    }
    // whether any line of the tile has y or z ghosts (most tiles have none)
    const bool yz = __syncthreads_or(has_yz);
    tile_fft<T, true, SH>(s, sch, W, lgW, tw_half);

    double acc_du = 0.0, acc_u = 0.0, acc_s = 0.0;
    const double mprev = (ACC && mean_prev) ? *mean_prev : 0.0;
    const int Eo = nx << lgW;
    if constexpr (!DCT) {
        // periodic x: outputs x_2n, x_2n+1 are Re, Im of z_n -- two per iteration
        for (int e = threadIdx.x; e < E; e += NTH) {
            const int l = e / nc, n = e - l * nc;
            if (line0 + l >= nlines) continue;
            const cx<T> zv = s[tidx<T, SH>(n, l, W)];
            const double x0 = (double)zv.x, x1 = (double)zv.y;
            const long o = line_base[l] + 2 * n;
            // refinement: u <- u + du - mean(u), the FP64 mean of the previous
            // iterate (the residual cannot see constants, so the gauge is kept here)
            double u0 = x0, u1 = x1;
            if (ACC) {
                u0 = (src(o) - mprev) + x0;
                u1 = (src(o + 1) - mprev) + x1;
            }
            put(o, u0);
            put(o + 1, u1);
            if (GHOST && yz) {
                // y and z stencil ghosts for the next residual (the reference's
                // ghost update overwrites them after the last sweep)
                const long gy = line_gy[l], gz = line_gz[l];
                if (gy) { put(o + gy, u0); put(o + 1 + gy, u1); }
                if (gz) { put(o + gz, u0); put(o + 1 + gz, u1); }
            }
            if (partials) {
                // the norms feed the gate after a refinement sweep only
                if (ACC) {
                    acc_du += x0 * x0 + x1 * x1;
                    acc_u += u0 * u0 + u1 * u1;
                }
                acc_s += u0 + u1;
            }
        }
    } else {
        for (int e = threadIdx.x; e < Eo; e += NTH) {
            const int l = e / nx, i = e - l * nx;
            const long line = line0 + l;
            if (line >= nlines) continue;
            int n = i;
            // inverse Makhoul order (cuda_Poisson_DCT_b_post, :1013-1033)
            if (DCT) n = (i & 1) ? (nc + ((nx - 1 - i) >> 1)) : (i >> 1);
            const cx<T> zv = s[tidx<T, SH>(n >> 1, l, W)];
            const double x = (double)((n & 1) ? zv.y : zv.x);
            const long o = line_base[l] + i;
            // refinement: u <- u + du - mean(u), the FP64 mean of the previous
            // iterate (the residual cannot see constants, so the gauge is kept here)
            const double un = ACC ? (src(o) - mprev) + x : x;
            put(o, un);
            if (GHOST && yz) {
                // y and z stencil ghosts for the next residual (the reference's
                // ghost update overwrites them after the last sweep)
                const long gy = line_gy[l], gz = line_gz[l];
                if (gy) put(o + gy, un);
                if (gz) put(o + gz, un);
            }
            if (partials) {
                if (ACC) {
                    acc_du += x * x;
                    acc_u += un * un;
                }
                acc_s += un;
            }
        }
    }
    if (GHOST) {
        __syncthreads();
        x_ghosts<UK>(P, U, g, line0, W, nlines, nx);
    }
    if (partials) {
        // deterministic per-block partial sums (reduced in a fixed order by the gate)
        double(*red)[32] = reinterpret_cast<double(*)[32]>(x_red_slots());
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            acc_du += __shfl_down_sync(0xffffffffu, acc_du, off);
            acc_u += __shfl_down_sync(0xffffffffu, acc_u, off);
            acc_s += __shfl_down_sync(0xffffffffu, acc_s, off);
        }
        const int w = threadIdx.x >> 5, nw = (NTH + 31) >> 5;
        if ((threadIdx.x & 31) == 0) { red[0][w] = acc_du; red[1][w] = acc_u; red[2][w] = acc_s; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = 0, b = 0, c = 0;
            for (int q = 0; q < nw; ++q) { a += red[0][q]; b += red[1][q]; c += red[2][q]; }
            partials[3 * tile + 0] = a;
            partials[3 * tile + 1] = b;
            partials[3 * tile + 2] = c;
        }
    }
}

}  // namespace ppf
