// ppf_xy.cu -- x and y transform kernels of libppf (sm_100a).
//
// One CTA transforms a tile of W lines in shared memory (ppf_fft.cuh).
//   x pass: W consecutive x-lines (fixed y,z) -> real FFT via a half-length
//           complex FFT, or DCT-II via Makhoul's reordering folded into the
//           tile load and the post-twiddle folded into the store.
//   y pass: W consecutive spectral columns of one z-plane, all ny rows.
// The reference runs each of these as cuFFT calls bracketed by separate
// reorder / twiddle / transpose / dscal passes (01_Fortran/src/
// fft_3d_poisson.f90:378-616, 915-1119); here each is one read and one
// write of the field.
#include "ppf_fft.cuh"
#include "ppf_kernels.cuh"

namespace ppf {

namespace {

__device__ __forceinline__ double lap_at(const ResidIn& r, const Geom& g, int i, int j, int k)
{
    const double* P = r.P;
    const long base = (long)(i + 1) + (long)(j + 1) * g.pstride_y + (long)(k + 1) * g.pstride_z;
    const double u = P[base];
    double uxm, uxp, uym, uyp, uzm, uzp;
    if (g.px) {
        uxm = P[base + (i == 0 ? (g.nx - 1) : -1)];
        uxp = P[base + (i == g.nx - 1 ? -(g.nx - 1) : 1)];
    } else {
        uxm = (i == 0) ? u : P[base - 1];
        uxp = (i == g.nx - 1) ? u : P[base + 1];
    }
    if (g.py) {
        uym = P[base + (j == 0 ? (long)(g.ny - 1) * g.pstride_y : -g.pstride_y)];
        uyp = P[base + (j == g.ny - 1 ? -(long)(g.ny - 1) * g.pstride_y : g.pstride_y)];
    } else {
        uym = (j == 0) ? u : P[base - g.pstride_y];
        uyp = (j == g.ny - 1) ? u : P[base + g.pstride_y];
    }
    uzm = (k == 0) ? u : P[base - g.pstride_z];
    uzp = (k == g.nz - 1) ? u : P[base + g.pstride_z];
    const double am = r.am[k], ap = r.ap[k];
    return (uxm - 2.0 * u + uxp) * r.ix2 + (uym - 2.0 * u + uyp) * r.iy2 + am * (uzm - u) + ap * (uzp - u);
}

template <typename T> struct TileW { static constexpr int value = SwizzleG<T>::value; };

inline int ilog2(int w) { int l = 0; while ((1 << l) < w) ++l; return l; }

template <typename K>
cudaError_t set_smem(K kern, size_t bytes)
{
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

inline int threads_for(int n, int W)
{
    int t = (n * W + 7) / 8;
    t = (t + 31) & ~31;
    if (t < 64) t = 64;
    return t;
}

// Lines per tile: a full 128-byte bank row of each FFT element when the
// tile fits 512 threads, fewer lines otherwise.
template <typename T>
inline int pick_w(int n, int& threads)
{
    int W = TileW<T>::value;
    while (W > 1 && threads_for(n, W) > 512) W >>= 1;
    threads = threads_for(n, W);
    return W;
}

}  // namespace

// --------------------------------------------------------------------------
// x forward: real lines (FP64 input, optionally f - L u) -> half spectrum
// (R2C, complex rows of nx/2+1) or DCT-II (real rows of nx).
// --------------------------------------------------------------------------
template <typename T, bool DCT, bool RESID>
__global__ void __launch_bounds__(512) k_xfwd(const double* __restrict__ f, ResidIn rs, Geom g,
                                               void* __restrict__ out_, long out_pitch, FftSched sch,
                                               int W, int lgW, const cx<T>* __restrict__ tw_half,
                                               const cx<T>* __restrict__ tw_n,
                                               const cx<T>* __restrict__ tw_dct,
                                               const int* __restrict__ skip)
{
    if (skip && *skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* s = reinterpret_cast<cx<T>*>(smem_raw);
    const int nx = g.nx, nc = nx >> 1;
    const long nlines = (long)g.ny * g.nz;
    const long line0 = (long)blockIdx.x * W;
    const int E = nc << lgW;

    for (int e = threadIdx.x; e < E; e += blockDim.x) {
        const int l = e / nc, n = e - l * nc;
        const long line = line0 + l;
        cx<T> z = mk<T>((T)0, (T)0);
        if (line < nlines) {
            const double* fl = f + line * nx;
            double a = fl[2 * n], b = fl[2 * n + 1];
            if (RESID) {
                const int j = (int)(line % g.ny), k = (int)(line / g.ny);
                a -= lap_at(rs, g, 2 * n, j, k);
                b -= lap_at(rs, g, 2 * n + 1, j, k);
            }
            z = mk<T>((T)a, (T)b);
        }
        s[sidx<T>(n, l, W)] = z;
    }
    __syncthreads();

    if (DCT) {
        // Makhoul order v = [x0, x2, .., x_{n-2}, x_{n-1}, .., x3, x1]
        // (cuda_Poisson_DCT_f_pre, fft_3d_poisson.f90:915-935), packed as
        // complex pairs (v_{2m}, v_{2m+1}) for the half-length FFT.
        constexpr int EPT = 8;
        cx<T> tmp[EPT];
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
            const int e = threadIdx.x + i * blockDim.x;
            if (e < E) {
                const int l = e / nc, m = e - l * nc;
                const int q0 = 2 * m, q1 = 2 * m + 1;
                const T v0 = (q0 < nc) ? s[sidx<T>(q0, l, W)].x : s[sidx<T>(nx - 1 - q0, l, W)].y;
                const T v1 = (q1 < nc) ? s[sidx<T>(q1, l, W)].x : s[sidx<T>(nx - 1 - q1, l, W)].y;
                tmp[i] = mk<T>(v0, v1);
            }
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < EPT; ++i) {
            const int e = threadIdx.x + i * blockDim.x;
            if (e < E) {
                const int l = e / nc, m = e - l * nc;
                s[sidx<T>(m, l, W)] = tmp[i];
            }
        }
        __syncthreads();
    }

    fft_tile<T, false>(s, sch, W, lgW, tw_half);

    if (!DCT) {
        cx<T>* out = reinterpret_cast<cx<T>*>(out_);
        const int Eo = (nc + 1) * W;
        for (int e = threadIdx.x; e < Eo; e += blockDim.x) {
            const int l = e / (nc + 1), k = e - l * (nc + 1);
            const long line = line0 + l;
            if (line >= nlines) continue;
            const cx<T> zk = s[sidx<T>(k == nc ? 0 : k, l, W)];
            const cx<T> zc = conj(s[sidx<T>(k == 0 ? 0 : nc - k, l, W)]);
            const cx<T> Ev = (zk + zc) * (T)0.5;
            const cx<T> D = zk - zc;
            const cx<T> O = mk<T>(D.y * (T)0.5, -D.x * (T)0.5);
            out[line * out_pitch + k] = Ev + cmul(ldg(tw_n + k), O);
        }
    } else {
        // X_k = 2 Re(e^{-i pi k/(2n)} V_k), V_{n-k} = conj(V_k)
        // (cuda_Poisson_DCT_f_post, fft_3d_poisson.f90:937-969)
        T* out = reinterpret_cast<T*>(out_);
        const int Eo = nx * W;
        for (int e = threadIdx.x; e < Eo; e += blockDim.x) {
            const int l = e / nx, k = e - l * nx;
            const long line = line0 + l;
            if (line >= nlines) continue;
            const int kap = (k <= nc) ? k : nx - k;
            const cx<T> zk = s[sidx<T>(kap == nc ? 0 : kap, l, W)];
            const cx<T> zc = conj(s[sidx<T>(kap == 0 ? 0 : nc - kap, l, W)]);
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

// --------------------------------------------------------------------------
// y forward on complex columns of one z-plane.
//   Y_C2C  : complex FFT along y (periodic y on complex x-spectra)
//   Y_CDCT : DCT-II of real and imaginary parts at once (Neumann y; also the
//            real N-N case with adjacent kx columns packed as complex)
//   Y_RPAIR: real FFT of two packed real columns (DCT-x data, periodic y);
//            writes ny/2+1 rows of two complex columns per packed pair
// --------------------------------------------------------------------------
template <typename T, int KIND>
__global__ void __launch_bounds__(512) k_yfwd(const cx<T>* __restrict__ in, long in_pitch,
                                               cx<T>* __restrict__ out, long out_pitch, int ncols,
                                               Geom g, FftSched sch, int W, int lgW,
                                               const cx<T>* __restrict__ tw_ny,
                                               const cx<T>* __restrict__ tw_dct,
                                               const int* __restrict__ skip)
{
    if (skip && *skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* s = reinterpret_cast<cx<T>*>(smem_raw);
    const int ny = g.ny;
    const int z = blockIdx.y;
    const int col0 = blockIdx.x * W;
    const cx<T>* inp = in + (long)z * ny * in_pitch;
    const int E = ny << lgW;

    for (int e = threadIdx.x; e < E; e += blockDim.x) {
        const int l = e & (W - 1), y = e >> lgW;
        const int col = col0 + l;
        cx<T> v = mk<T>((T)0, (T)0);
        if (col < ncols) v = inp[(long)y * in_pitch + col];
        int row = y;
        if (KIND == Y_CDCT) row = (y & 1) ? (ny - 1 - (y >> 1)) : (y >> 1);
        s[sidx<T>(row, l, W)] = v;
    }
    __syncthreads();
    fft_tile<T, false>(s, sch, W, lgW, tw_ny);

    if (KIND == Y_C2C) {
        cx<T>* outp = out + (long)z * ny * out_pitch;
        for (int e = threadIdx.x; e < E; e += blockDim.x) {
            const int l = e & (W - 1), k = e >> lgW;
            const int col = col0 + l;
            if (col < ncols) outp[(long)k * out_pitch + col] = s[sidx<T>(k, l, W)];
        }
    } else if (KIND == Y_CDCT) {
        cx<T>* outp = out + (long)z * ny * out_pitch;
        for (int e = threadIdx.x; e < E; e += blockDim.x) {
            const int l = e & (W - 1), k = e >> lgW;
            const int col = col0 + l;
            if (col >= ncols) continue;
            const cx<T> V = s[sidx<T>(k, l, W)];
            const cx<T> Vp = s[sidx<T>(k == 0 ? 0 : ny - k, l, W)];
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
        for (int e = threadIdx.x; e < Eo; e += blockDim.x) {
            const int l = e & (W - 1), k = e >> lgW;
            const int col = col0 + l;
            if (col >= ncols) continue;
            const cx<T> zk = s[sidx<T>(k == ny ? 0 : k, l, W)];
            const cx<T> zc = conj(s[sidx<T>(k == 0 ? 0 : ny - k, l, W)]);
            const cx<T> X1 = (zk + zc) * (T)0.5;
            const cx<T> D = zk - zc;
            const cx<T> X2 = mk<T>(D.y * (T)0.5, -D.x * (T)0.5);
            outp[(long)k * out_pitch + 2 * col] = X1;
            outp[(long)k * out_pitch + 2 * col + 1] = X2;
        }
    }
}

// --------------------------------------------------------------------------
// y inverse (the three kinds above, unnormalised)
// --------------------------------------------------------------------------
template <typename T, int KIND>
__global__ void __launch_bounds__(512) k_yinv(const cx<T>* __restrict__ in, long in_pitch,
                                               cx<T>* __restrict__ out, long out_pitch, int ncols,
                                               Geom g, FftSched sch, int W, int lgW,
                                               const cx<T>* __restrict__ tw_ny,
                                               const cx<T>* __restrict__ tw_dct,
                                               const double* __restrict__ dc_shift,
                                               const int* __restrict__ skip)
{
    if (skip && *skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* s = reinterpret_cast<cx<T>*>(smem_raw);
    const int ny = g.ny;
    const int z = blockIdx.y;
    const int col0 = blockIdx.x * W;
    const int E = ny << lgW;
    // the zero mode's z-average, removed from the (kx,ky) = (0,0) coefficient
    const T shift = (col0 == 0 && dc_shift) ? (T)*dc_shift : (T)0;

    if (KIND == Y_C2C) {
        const cx<T>* inp = in + (long)z * ny * in_pitch;
        for (int e = threadIdx.x; e < E; e += blockDim.x) {
            const int l = e & (W - 1), k = e >> lgW;
            const int col = col0 + l;
            cx<T> v = mk<T>((T)0, (T)0);
            if (col < ncols) v = inp[(long)k * in_pitch + col];
            if (k == 0 && col == 0) v.x -= shift;
            s[sidx<T>(k, l, W)] = v;
        }
    } else if (KIND == Y_CDCT) {
        // Z_k = e^{i pi k/(2n)} (X_k - i X_{n-k}) per real component
        // (cuda_Poisson_DCT_b_pre, fft_3d_poisson.f90:971-1011), both
        // components packed into one complex inverse FFT.
        const cx<T>* inp = in + (long)z * ny * in_pitch;
        for (int e = threadIdx.x; e < E; e += blockDim.x) {
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
            s[sidx<T>(k, l, W)] = Z;
        }
    } else {
        const int my = ny / 2 + 1;
        const cx<T>* inp = in + (long)z * my * in_pitch;
        for (int e = threadIdx.x; e < E; e += blockDim.x) {
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
            s[sidx<T>(k, l, W)] = Z;
        }
    }
    __syncthreads();
    fft_tile<T, true>(s, sch, W, lgW, tw_ny);

    cx<T>* outp = out + (long)z * ny * out_pitch;
    for (int e = threadIdx.x; e < E; e += blockDim.x) {
        const int l = e & (W - 1), i = e >> lgW;
        const int col = col0 + l;
        if (col >= ncols) continue;
        int n = i;
        // inverse Makhoul order (cuda_Poisson_DCT_b_post, :1013-1033)
        if (KIND == Y_CDCT) n = (i & 1) ? (ny / 2 + ((ny - 1 - i) >> 1)) : (i >> 1);
        outp[(long)i * out_pitch + col] = s[sidx<T>(n, l, W)];
    }
}

// --------------------------------------------------------------------------
// x inverse: half spectrum (C2R) or DCT coefficients (inverse DCT) ->
// interior of the ghosted FP64 output (write or accumulate).
// --------------------------------------------------------------------------
template <typename T, bool DCT, bool ACC>
__global__ void __launch_bounds__(512) k_xinv(const void* __restrict__ in_, long in_pitch,
                                               double* __restrict__ P, Geom g, double* __restrict__ partials,
                                               const double* __restrict__ mean_prev,
                                               FftSched sch, int W, int lgW,
                                               const cx<T>* __restrict__ tw_half,
                                               const cx<T>* __restrict__ tw_n,
                                               const cx<T>* __restrict__ tw_dct,
                                               const int* __restrict__ skip)
{
    if (skip && *skip) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* s = reinterpret_cast<cx<T>*>(smem_raw);
    const int nx = g.nx, nc = nx >> 1;
    const long nlines = (long)g.ny * g.nz;
    const long line0 = (long)blockIdx.x * W;
    const int E = nc << lgW;

    for (int e = threadIdx.x; e < E; e += blockDim.x) {
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
        s[sidx<T>(k, l, W)] = Z;
    }
    __syncthreads();
    fft_tile<T, true>(s, sch, W, lgW, tw_half);

    double acc_du = 0.0, acc_u = 0.0, acc_s = 0.0;
    const double mprev = (ACC && mean_prev) ? *mean_prev : 0.0;
    const int Eo = nx << lgW;
    for (int e = threadIdx.x; e < Eo; e += blockDim.x) {
        const int l = e / nx, i = e - l * nx;
        const long line = line0 + l;
        if (line >= nlines) continue;
        int n = i;
        if (DCT) n = (i & 1) ? (nc + ((nx - 1 - i) >> 1)) : (i >> 1);
        const cx<T> zv = s[sidx<T>(n >> 1, l, W)];
        const double x = (double)((n & 1) ? zv.y : zv.x);
        const int j = (int)(line % g.ny), k = (int)(line / g.ny);
        const long o = (long)(i + 1) + (long)(j + 1) * g.pstride_y + (long)(k + 1) * g.pstride_z;
        // refinement: u <- u + du - mean(u), the FP64 mean of the previous
        // iterate (the residual cannot see constants, so the gauge is kept here)
        const double un = ACC ? (P[o] - mprev) + x : x;
        P[o] = un;
        if (partials) {
            acc_du += x * x;
            acc_u += un * un;
            acc_s += un;
        }
    }
    if (partials) {
        // deterministic per-block partial sums (reduced in a fixed order by the gate)
        __shared__ double red[3][32];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            acc_du += __shfl_down_sync(0xffffffffu, acc_du, off);
            acc_u += __shfl_down_sync(0xffffffffu, acc_u, off);
            acc_s += __shfl_down_sync(0xffffffffu, acc_s, off);
        }
        const int w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
        if ((threadIdx.x & 31) == 0) { red[0][w] = acc_du; red[1][w] = acc_u; red[2][w] = acc_s; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = 0, b = 0, c = 0;
            for (int i = 0; i < nw; ++i) { a += red[0][i]; b += red[1][i]; c += red[2][i]; }
            partials[3 * blockIdx.x + 0] = a;
            partials[3 * blockIdx.x + 1] = b;
            partials[3 * blockIdx.x + 2] = c;
        }
    }
}

// --------------------------------------------------------------------------
// launchers
// --------------------------------------------------------------------------
template <typename T>
cudaError_t launch_xfwd(bool dct, const double* f, const ResidIn* resid, const Geom& g, void* out,
                        long out_pitch, const FftSched& sch, const cx<T>* tw_half, const cx<T>* tw_n,
                        const cx<T>* tw_dct, const int* skip_flag, cudaStream_t st)
{
    const int nc = g.nx / 2;
    int threads;
    const int W = pick_w<T>(nc, threads), lgW = ilog2(W);
    if (threads > 512) return cudaErrorInvalidConfiguration;
    const size_t smem = (size_t)nc * W * sizeof(cx<T>);
    const long nlines = (long)g.ny * g.nz;
    dim3 grid((unsigned)((nlines + W - 1) / W));
    ResidIn rs{};
    if (resid) rs = *resid;
#define PPF_XF(D, R)                                                                             \
    {                                                                                            \
        auto kern = k_xfwd<T, D, R>;                                                             \
        cudaError_t e = set_smem(kern, smem);                                                    \
        if (e != cudaSuccess) return e;                                                          \
        kern<<<grid, threads, smem, st>>>(f, rs, g, out, out_pitch, sch, W, lgW, tw_half, tw_n,  \
                                         tw_dct, skip_flag);                                     \
    }
    if (dct) { if (resid) PPF_XF(true, true) else PPF_XF(true, false) }
    else     { if (resid) PPF_XF(false, true) else PPF_XF(false, false) }
#undef PPF_XF
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_yfwd(int kind, const cx<T>* in, long in_pitch, cx<T>* out, long out_pitch, int ncols,
                        const Geom& g, const FftSched& sch, const cx<T>* tw_ny, const cx<T>* tw_dct,
                        const int* skip_flag, cudaStream_t st)
{
    int threads;
    const int W = pick_w<T>(g.ny, threads), lgW = ilog2(W);
    if (threads > 512) return cudaErrorInvalidConfiguration;
    const size_t smem = (size_t)g.ny * W * sizeof(cx<T>);
    dim3 grid((unsigned)((ncols + W - 1) / W), (unsigned)g.nz);
#define PPF_YF(KD)                                                                               \
    {                                                                                            \
        auto kern = k_yfwd<T, KD>;                                                               \
        cudaError_t e = set_smem(kern, smem);                                                    \
        if (e != cudaSuccess) return e;                                                          \
        kern<<<grid, threads, smem, st>>>(in, in_pitch, out, out_pitch, ncols, g, sch, W, lgW,  \
                                         tw_ny, tw_dct, skip_flag);                              \
    }
    if (kind == Y_C2C) PPF_YF(Y_C2C)
    else if (kind == Y_CDCT) PPF_YF(Y_CDCT)
    else PPF_YF(Y_RPAIR)
#undef PPF_YF
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_yinv(int kind, const cx<T>* in, long in_pitch, cx<T>* out, long out_pitch, int ncols,
                        const Geom& g, const FftSched& sch, const cx<T>* tw_ny, const cx<T>* tw_dct,
                        const double* dc_shift, const int* skip_flag, cudaStream_t st)
{
    int threads;
    const int W = pick_w<T>(g.ny, threads), lgW = ilog2(W);
    if (threads > 512) return cudaErrorInvalidConfiguration;
    const size_t smem = (size_t)g.ny * W * sizeof(cx<T>);
    dim3 grid((unsigned)((ncols + W - 1) / W), (unsigned)g.nz);
#define PPF_YI(KD)                                                                               \
    {                                                                                            \
        auto kern = k_yinv<T, KD>;                                                               \
        cudaError_t e = set_smem(kern, smem);                                                    \
        if (e != cudaSuccess) return e;                                                          \
        kern<<<grid, threads, smem, st>>>(in, in_pitch, out, out_pitch, ncols, g, sch, W, lgW,  \
                                         tw_ny, tw_dct, dc_shift, skip_flag);                    \
    }
    if (kind == Y_C2C) PPF_YI(Y_C2C)
    else if (kind == Y_CDCT) PPF_YI(Y_CDCT)
    else PPF_YI(Y_RPAIR)
#undef PPF_YI
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_xinv(bool dct, const void* in, long in_pitch, double* P, const Geom& g, bool accumulate,
                        double* partials, const double* mean_prev, const FftSched& sch, const cx<T>* tw_half,
                        const cx<T>* tw_n, const cx<T>* tw_dct, const int* skip_flag, cudaStream_t st)
{
    const int nc = g.nx / 2;
    int threads;
    const int W = pick_w<T>(nc, threads), lgW = ilog2(W);
    if (threads > 512) return cudaErrorInvalidConfiguration;
    const size_t smem = (size_t)nc * W * sizeof(cx<T>);
    const long nlines = (long)g.ny * g.nz;
    dim3 grid((unsigned)((nlines + W - 1) / W));
#define PPF_XI(D, A)                                                                             \
    {                                                                                            \
        auto kern = k_xinv<T, D, A>;                                                             \
        cudaError_t e = set_smem(kern, smem);                                                    \
        if (e != cudaSuccess) return e;                                                          \
        kern<<<grid, threads, smem, st>>>(in, in_pitch, P, g, partials, mean_prev, sch, W, lgW,  \
                                         tw_half, tw_n, tw_dct, skip_flag);                      \
    }
    if (dct) { if (accumulate) PPF_XI(true, true) else PPF_XI(true, false) }
    else     { if (accumulate) PPF_XI(false, true) else PPF_XI(false, false) }
#undef PPF_XI
    return cudaGetLastError();
}

template <typename T>
long xinv_blocks(const Geom& g)
{
    int threads;
    const int W = pick_w<T>(g.nx / 2, threads);
    const long nlines = (long)g.ny * g.nz;
    return (nlines + W - 1) / W;
}
template long xinv_blocks<double>(const Geom&);
template long xinv_blocks<float>(const Geom&);

#define PPF_INST(T)                                                                                        \
    template cudaError_t launch_xfwd<T>(bool, const double*, const ResidIn*, const Geom&, void*, long,     \
                                        const FftSched&, const cx<T>*, const cx<T>*, const cx<T>*,         \
                                        const int*, cudaStream_t);                                         \
    template cudaError_t launch_yfwd<T>(int, const cx<T>*, long, cx<T>*, long, int, const Geom&,           \
                                        const FftSched&, const cx<T>*, const cx<T>*, const int*,           \
                                        cudaStream_t);                                                     \
    template cudaError_t launch_yinv<T>(int, const cx<T>*, long, cx<T>*, long, int, const Geom&,           \
                                        const FftSched&, const cx<T>*, const cx<T>*, const double*,        \
                                        const int*, cudaStream_t);                                         \
    template cudaError_t launch_xinv<T>(bool, const void*, long, double*, const Geom&, bool, double*,      \
                                        const double*, const FftSched&, const cx<T>*, const cx<T>*,        \
                                        const cx<T>*, const int*, cudaStream_t);
PPF_INST(double)
PPF_INST(float)
#undef PPF_INST

}  // namespace ppf
