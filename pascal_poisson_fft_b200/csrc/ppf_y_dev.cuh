// ppf_y_dev.cuh -- device bodies of the y-direction transforms, shared by
// the y kernels (ppf_y.cu) and the persistent batch kernel (ppf_batch.cu).
// One call transforms column block `cblk` (W consecutive spectral columns)
// of z-plane `z`, all ny rows, in shared memory (ppf_fft.cuh); the spectral
// rows stay in the [z][ky][kx] order the z solve reads, so no transpose pass
// exists (the reference transposes before and after every y transform,
// 01_Fortran/src/fft_3d_poisson.f90:421-559, 1035-1119).
//   Y_C2C  : complex FFT along y (periodic y on complex x-spectra)
//   Y_CDCT : DCT-II of real and imaginary parts at once (Neumann y; also the
//            real N-N case with adjacent kx columns packed as complex)
//   Y_RPAIR: real FFT of two packed real columns (DCT-x data, periodic y);
//            ny/2+1 rows of two complex columns per packed pair
#pragma once
#include "ppf_xy_common.cuh"

namespace ppf {

constexpr int ct_log2y(int w) { return w <= 1 ? 0 : 1 + ct_log2y(w / 2); }

template <typename T, int KIND, typename SH>
__device__ __forceinline__ void yfwd(const cx<T>* __restrict__ in, long in_pitch, cx<T>* __restrict__ out,
                                     long out_pitch, int ncols, const Geom& g, const FftSched& sch, int Wrt, int lgWrt,
                                     const cx<T>* __restrict__ tw_ny, const cx<T>* __restrict__ tw_dct,
                                     const int* __restrict__ skip, int cblk, int z)
{
    if (skip && *skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* s = reinterpret_cast<cx<T>*>(smem_raw);
    constexpr bool CT = SH::CT;
    const int W = CT ? SH::W : Wrt;
    const int lgW = CT ? ct_log2y(SH::W) : lgWrt;
    const int NTH = CT ? SH::NT : (int)blockDim.x;
    const int ny = CT ? SH::N : g.ny;
    const int col0 = cblk * W;
    const cx<T>* inp = in + (long)z * ny * in_pitch;
    const int E = ny << lgW;

    for (int e = threadIdx.x; e < E; e += NTH) {
        const int l = e & (W - 1), y = e >> lgW;
        const int col = col0 + l;
        cx<T> v = mk<T>((T)0, (T)0);
        if (col < ncols) v = inp[(long)y * in_pitch + col];
        int row = y;
        if (KIND == Y_CDCT) row = (y & 1) ? (ny - 1 - (y >> 1)) : (y >> 1);
        s[tidx<T, SH>(row, l, W)] = v;
    }
    __syncthreads();
    tile_fft<T, false, SH>(s, sch, W, lgW, tw_ny);

    if (KIND == Y_C2C) {
        cx<T>* outp = out + (long)z * ny * out_pitch;
        for (int e = threadIdx.x; e < E; e += NTH) {
            const int l = e & (W - 1), k = e >> lgW;
            const int col = col0 + l;
            if (col < ncols) outp[(long)k * out_pitch + col] = s[tidx<T, SH>(k, l, W)];
        }
    } else if (KIND == Y_CDCT) {
        cx<T>* outp = out + (long)z * ny * out_pitch;
        for (int e = threadIdx.x; e < E; e += NTH) {
            const int l = e & (W - 1), k = e >> lgW;
            const int col = col0 + l;
            if (col >= ncols) continue;
            const cx<T> V = s[tidx<T, SH>(k, l, W)];
            const cx<T> Vp = s[tidx<T, SH>(k == 0 ? 0 : ny - k, l, W)];
            const cx<T> w = ldg(tw_dct + k);
            cx<T> X;
            X.x = w.x * (V.x + Vp.x) - w.y * (V.y - Vp.y);
            X.y = w.x * (V.y + Vp.y) + w.y * (V.x - Vp.x);
            outp[(long)k * out_pitch + col] = X;
        }
    } else {
        const int my = ny / 2 + 1;
        cx<T>* outp = out + (long)z * my * out_pitch;
        const int Eo = my << lgW;
        for (int e = threadIdx.x; e < Eo; e += NTH) {
            const int l = e & (W - 1), k = e >> lgW;
            const int col = col0 + l;
            if (col >= ncols) continue;
            const cx<T> zk = s[tidx<T, SH>(k == ny ? 0 : k, l, W)];
            const cx<T> zc = conj(s[tidx<T, SH>(k == 0 ? 0 : ny - k, l, W)]);
            const cx<T> X1 = (zk + zc) * (T)0.5;
            const cx<T> D = zk - zc;
            const cx<T> X2 = mk<T>(D.y * (T)0.5, -D.x * (T)0.5);
            outp[(long)k * out_pitch + 2 * col] = X1;
            outp[(long)k * out_pitch + 2 * col + 1] = X2;
        }
    }
}

template <typename T, int KIND, typename SH>
__device__ __forceinline__ void yinv(const cx<T>* __restrict__ in, long in_pitch, cx<T>* __restrict__ out,
                                     long out_pitch, int ncols, const Geom& g, const FftSched& sch, int Wrt, int lgWrt,
                                     const cx<T>* __restrict__ tw_ny, const cx<T>* __restrict__ tw_dct,
                                     const double* __restrict__ dc_shift, const int* __restrict__ skip, int cblk,
                                     int z)
{
    if (skip && *skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* s = reinterpret_cast<cx<T>*>(smem_raw);
    constexpr bool CT = SH::CT;
    const int W = CT ? SH::W : Wrt;
    const int lgW = CT ? ct_log2y(SH::W) : lgWrt;
    const int NTH = CT ? SH::NT : (int)blockDim.x;
    const int ny = CT ? SH::N : g.ny;
    const int col0 = cblk * W;
    const int E = ny << lgW;
    // the zero mode's z-average, removed from the (kx,ky) = (0,0) coefficient
    const T shift = (col0 == 0 && dc_shift) ? (T)*dc_shift : (T)0;

    if (KIND == Y_C2C) {
        const cx<T>* inp = in + (long)z * ny * in_pitch;
        for (int e = threadIdx.x; e < E; e += NTH) {
            const int l = e & (W - 1), k = e >> lgW;
            const int col = col0 + l;
            cx<T> v = mk<T>((T)0, (T)0);
            if (col < ncols) v = inp[(long)k * in_pitch + col];
            if (k == 0 && col == 0) v.x -= shift;
            s[tidx<T, SH>(k, l, W)] = v;
        }
    } else if (KIND == Y_CDCT) {
        // Z_k = e^{i pi k/(2n)} (X_k - i X_{n-k}) per real component
        // (cuda_Poisson_DCT_b_pre, fft_3d_poisson.f90:971-1011), both
        // components packed into one complex inverse FFT.
        const cx<T>* inp = in + (long)z * ny * in_pitch;
        for (int e = threadIdx.x; e < E; e += NTH) {
            const int l = e & (W - 1), k = e >> lgW;
            const int col = col0 + l;
            cx<T> Z = mk<T>((T)0, (T)0);
            if (col < ncols) {
                cx<T> X = inp[(long)k * in_pitch + col];
                if (k == 0 && col == 0) X.x -= shift;
                const cx<T> Xp = (k == 0) ? mk<T>((T)0, (T)0) : inp[(long)(ny - k) * in_pitch + col];
                const cx<T> w = ldg(tw_dct + k);
                const T c = w.x, sn = -w.y;
                const T zax = c * X.x + sn * Xp.x, zay = sn * X.x - c * Xp.x;
                const T zbx = c * X.y + sn * Xp.y, zby = sn * X.y - c * Xp.y;
                Z = mk<T>(zax - zby, zay + zbx);
            }
            s[tidx<T, SH>(k, l, W)] = Z;
        }
    } else {
        const int my = ny / 2 + 1;
        const cx<T>* inp = in + (long)z * my * in_pitch;
        for (int e = threadIdx.x; e < E; e += NTH) {
            const int l = e & (W - 1), k = e >> lgW;
            const int col = col0 + l;
            cx<T> Z = mk<T>((T)0, (T)0);
            if (col < ncols) {
                const int kk = (k <= ny / 2) ? k : ny - k;
                cx<T> X1 = inp[(long)kk * in_pitch + 2 * col];
                cx<T> X2 = inp[(long)kk * in_pitch + 2 * col + 1];
                if (k > ny / 2) { X1 = conj(X1); X2 = conj(X2); }
                if (k == 0 || k == ny / 2) { X1.y = (T)0; X2.y = (T)0; }
                if (k == 0 && col == 0) X1.x -= shift;
                Z = mk<T>(X1.x - X2.y, X1.y + X2.x);
            }
            s[tidx<T, SH>(k, l, W)] = Z;
        }
    }
    __syncthreads();
    tile_fft<T, true, SH>(s, sch, W, lgW, tw_ny);

    cx<T>* outp = out + (long)z * ny * out_pitch;
    for (int e = threadIdx.x; e < E; e += NTH) {
        const int l = e & (W - 1), i = e >> lgW;
        const int col = col0 + l;
        if (col >= ncols) continue;
        int n = i;
        // inverse Makhoul order (cuda_Poisson_DCT_b_post, :1013-1033)
        if (KIND == Y_CDCT) n = (i & 1) ? (ny / 2 + ((ny - 1 - i) >> 1)) : (i >> 1);
        outp[(long)i * out_pitch + col] = s[tidx<T, SH>(n, l, W)];
    }
}

}  // namespace ppf
