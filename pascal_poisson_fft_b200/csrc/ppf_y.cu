// ppf_y.cu -- y-direction transform kernels of libppf (sm_100a).
//
// One CTA transforms W consecutive spectral columns of one z-plane, all ny
// rows, in shared memory (ppf_fft.cuh).  The spectral rows stay in the
// [z][ky][kx] order the z solve reads, so no transpose pass exists (the
// reference transposes before and after every y transform,
// 01_Fortran/src/fft_3d_poisson.f90:421-559, 1035-1119).
//   Y_C2C  : complex FFT along y (periodic y on complex x-spectra)
//   Y_CDCT : DCT-II of real and imaginary parts at once (Neumann y; also the
//            real N-N case with adjacent kx columns packed as complex)
//   Y_RPAIR: real FFT of two packed real columns (DCT-x data, periodic y);
//            ny/2+1 rows of two complex columns per packed pair
#include "ppf_tma.cuh"
#include "ppf_y_dev.cuh"

#ifndef PPF_Y_TMA
#define PPF_Y_TMA 1
#endif
// tile widths of the paired passes (16 columns: 512-point lines; 8: 768)
#ifndef PPF_Y_PAIR8
#define PPF_Y_PAIR8 1
#endif
// tile widths loaded by TMA
#ifndef PPF_Y_TMA_W
#define PPF_Y_TMA_W(w) ((w) == 16 || (PPF_Y_PAIR8 && (w) == 8))
#endif

namespace ppf {

template <typename T, int KIND, typename SH>
__global__ void __launch_bounds__(512) k_yfwd(const cx<T>* __restrict__ in, long in_pitch, cx<T>* __restrict__ out,
                                               long out_pitch, int ncols, Geom g, FftSched sch, int Wrt, int lgWrt,
                                               const cx<T>* __restrict__ tw_ny, const cx<T>* __restrict__ tw_dct,
                                               const int* __restrict__ skip)
{
    yfwd<T, KIND, SH>(in, in_pitch, out, out_pitch, ncols, g, sch, Wrt, lgWrt, tw_ny, tw_dct, skip, blockIdx.x,
                      blockIdx.y);
}

template <typename T, int KIND, typename SH>
__global__ void __launch_bounds__(512) k_yinv(const cx<T>* __restrict__ in, long in_pitch, cx<T>* __restrict__ out,
                                               long out_pitch, int ncols, Geom g, FftSched sch, int Wrt, int lgWrt,
                                               const cx<T>* __restrict__ tw_ny, const cx<T>* __restrict__ tw_dct,
                                               const double* __restrict__ dc_shift, const int* __restrict__ skip)
{
    yinv<T, KIND, SH>(in, in_pitch, out, out_pitch, ncols, g, sch, Wrt, lgWrt, tw_ny, tw_dct, dc_shift, skip,
                      blockIdx.x, blockIdx.y);
}

// Persistent, double-buffered complex y transform (forward, or inverse
// with the zero-mode shift) for the compile-time shapes: each CTA walks the
// (z, column block) tiles with a grid stride, and the next tile's columns
// are copied into the second buffer with cp.async while the current tile
// is transformed and stored, so the loads of one tile overlap the
// butterflies of the previous one.
//
// PAIR (FP32 tiles of 16 columns, 16-byte aligned rows): the tile is
// unswizzled, copied in 16-byte pairs of columns, and transformed by the
// paired passes (fft_pass_pair), which also store column pairs.
template <typename T, bool INV, typename SH, bool PAIR>
__device__ __forceinline__ void y_c2c_pipe(const cx<T>* __restrict__ in, long in_pitch, cx<T>* __restrict__ out,
                                           long out_pitch, int ncols, int nz, const cx<T>* __restrict__ tw,
                                           const double* __restrict__ dc_shift, const int* __restrict__ skip)
{
    if (skip && *skip) return;
    constexpr int N = SH::N, W = SH::W, NT = SH::NT;
    constexpr int LGW = ct_log2y(W);
    constexpr int EPT = (N * W) / NT;
    static_assert(EPT * NT == N * W, "tile elements must divide over the threads");
    static_assert(!PAIR || (sizeof(T) == 4 && W % 2 == 0 && EPT % 2 == 0), "paired tiles: FP32, an even width");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* cur = reinterpret_cast<cx<T>*>(smem_raw);
    cx<T>* nxt = cur + N * W;
    const int nblk = (ncols + W - 1) / W;
    const long ntiles = (long)nblk * nz;
    auto issue = [&](long t, cx<T>* b) {
        const int z = (int)(t / nblk), col0 = (int)(t - (long)z * nblk) * W;
        const cx<T>* inp = in + (long)z * N * in_pitch + col0;
        if constexpr (PAIR) {
            constexpr int P = W / 2;
#pragma unroll
            for (int i = 0; i < EPT / 2; ++i) {
                const int e = threadIdx.x + i * NT;
                const int p = e % P, y = e / P;
                cx<T>* d = b + y * W + 2 * p;
                const cx<T>* src = inp + (long)y * in_pitch + 2 * p;
                const int c = col0 + 2 * p;
                if (c + 1 < ncols) {
                    cp_async_16(d, src);
                } else {
                    if (c < ncols) cp_async_elem(d, src);
                    else d[0] = mk<T>((T)0, (T)0);
                    d[1] = mk<T>((T)0, (T)0);
                }
            }
        } else {
#pragma unroll
            for (int i = 0; i < EPT; ++i) {
                const int e = threadIdx.x + i * NT;
                const int l = e & (W - 1), y = e >> LGW;
                cx<T>* d = b + sidx_ct<T, W, SH::N>(y, l);
                if (col0 + l < ncols) cp_async_elem(d, inp + (long)y * in_pitch + l);
                else *d = mk<T>((T)0, (T)0);
            }
        }
        cp_async_commit();
    };
    long t = blockIdx.x;
    if (t < ntiles) issue(t, cur);
    for (; t < ntiles; t += gridDim.x) {
        const long tn = t + gridDim.x;
        if (tn < ntiles) issue(tn, nxt);
        else cp_async_commit();
        cp_async_wait<1>();  // this thread's copies of tile t have landed
        const int z = (int)(t / nblk), col0 = (int)(t - (long)z * nblk) * W;
        // the zero mode's z-average, removed from the (kx,ky) = (0,0) coefficient
        // (element (0,0) is copied by thread 0)
        if (INV && dc_shift && col0 == 0 && threadIdx.x == 0) cur[sidx_ct<T, W, SH::N>(0, 0)].x -= (T)*dc_shift;
        __syncthreads();
        // the last pass stores the tile's rows straight to the output (a warp
        // writes whole W-column row segments, as a copy-out loop would); the
        // tile is free for the refill two tiles on when the transform returns
        cx<T>* outp = out + (long)z * N * out_pitch + col0;
        if constexpr (PAIR) {
            auto yst2 = [&](int k, int p, cx<T> u, cx<T> v) {
                cx<T>* o = outp + (long)k * out_pitch + 2 * p;
                const int c = col0 + 2 * p;
                if (c + 1 < ncols) *reinterpret_cast<float4*>(o) = make_float4(u.x, u.y, v.x, v.y);
                else if (c < ncols) *o = u;
            };
            SH::template fft_pair_st<INV>(cur, tw, yst2);
        } else {
            auto yst = [&](int k, int l, cx<T> v) {
                if (col0 + l < ncols) outp[(long)k * out_pitch + l] = v;
            };
            SH::template fft_st<T, INV>(cur, tw, yst);
        }
        cx<T>* tmp = cur;
        cur = nxt;
        nxt = tmp;
    }
}

// The paired FP32 pipeline with its tiles loaded by TMA: thread 0 issues the
// boxes of the next tile (W columns x up to 256 rows each, one row of a
// box = one unswizzled tile row of 8W bytes; columns past ncols read as zero)
// onto that buffer's mbarrier, every thread waits on the current buffer's
// barrier (bounded: about 2 s of sleeping polls, then err bit 2 and the
// CTA stops), and the transform and stores are those of
// y_c2c_pipe<float, INV, SH, true>.  The tensor map covers this GPU's
// spectrum only (rows of 2 ncols FP32 values, in_pitch complex apart).
constexpr unsigned YT_POLL_NS = 20000;
constexpr long YT_WAIT_LIMIT = 100000;

template <int W> struct PairWidth { static constexpr bool value = W == 16 || (PPF_Y_PAIR8 && W == 8); };

template <bool INV, typename SH>
__global__ void __launch_bounds__(SH::NT, 1) k_y_c2c_tma(const __grid_constant__ CUtensorMap tmap,
                                                     cx<float>* __restrict__ out, long out_pitch, int ncols, int nz,
                                                     const cx<float>* __restrict__ tw,
                                                     const double* __restrict__ dc_shift,
                                                     const int* __restrict__ skip, int* __restrict__ err)
{
    if (skip && *skip) return;
    using T = float;
    constexpr int N = SH::N, W = SH::W;
    static_assert(W % 2 == 0, "paired tiles of an even width");
    constexpr int BR = N < 256 ? N : 256;   // rows per box
    static_assert(N % BR == 0, "whole boxes per tile");
    constexpr unsigned TILE_BYTES = (unsigned)(N * W * sizeof(cx<T>));
    extern __shared__ __align__(128) unsigned char smem_raw[];
    // TMA destinations start on 128-byte boundaries: the dynamic region is
    // rounded up (the launch adds 128 bytes for it)
    cx<T>* cur = reinterpret_cast<cx<T>*>(((uintptr_t)smem_raw + 127) & ~(uintptr_t)127);
    cx<T>* nxt = cur + N * W;
    __shared__ __align__(8) uint64_t ybar[2];
    __shared__ int yabort;
    if (threadIdx.x == 0) {
        mbar_init(&ybar[0], 1);
        mbar_init(&ybar[1], 1);
        mbar_init_fence();
        yabort = 0;
    }
    __syncthreads();
    const int nblk = (ncols + W - 1) / W;
    const long ntiles = (long)nblk * nz;
    const uint64_t pol = l2_policy_evict_first();   // every value is read once
    auto issue = [&](long t, cx<T>* b, int bi) {
        if (threadIdx.x == 0) {
            const int z = (int)(t / nblk), col0 = (int)(t - (long)z * nblk) * W;
            fence_proxy_async_smem();   // the previous tile's reads of b come first
            mbar_arrive_expect_tx(&ybar[bi], TILE_BYTES);
#pragma unroll
            for (int q = 0; q < N / BR; ++q)
                tma_load_2d(b + q * BR * W, &tmap, 2 * col0, z * N + q * BR, &ybar[bi], pol);
        }
    };
    int cb = 0;
    unsigned par = 0;
    long t = blockIdx.x;
    if (t < ntiles) issue(t, cur, 0);
    for (; t < ntiles; t += gridDim.x) {
        const long tn = t + gridDim.x;
        if (tn < ntiles) issue(tn, nxt, cb ^ 1);
        if (!mbar_wait_sleep_bounded(&ybar[cb], (par >> cb) & 1u, YT_POLL_NS, YT_WAIT_LIMIT)) yabort = 1;
        par ^= 1u << cb;
        const int z = (int)(t / nblk), col0 = (int)(t - (long)z * nblk) * W;
        // the zero mode's z-average, removed from the (kx,ky) = (0,0) coefficient
        if (INV && dc_shift && col0 == 0 && threadIdx.x == 0) cur[0].x -= (T)*dc_shift;
        __syncthreads();
        if (yabort) {
            if (threadIdx.x == 0) {
                if (err) atomicOr(err, 2);
                // the next tile's boxes may be in flight: wait for them (bounded)
                if (tn < ntiles)
                    mbar_wait_sleep_bounded(&ybar[cb ^ 1], (par >> (cb ^ 1)) & 1u, YT_POLL_NS, YT_WAIT_LIMIT);
            }
            break;
        }
        cx<T>* outp = out + (long)z * N * out_pitch + col0;
        auto yst2 = [&](int k, int p, cx<T> u, cx<T> v) {
            cx<T>* o = outp + (long)k * out_pitch + 2 * p;
            const int c = col0 + 2 * p;
            if (c + 1 < ncols) *reinterpret_cast<float4*>(o) = make_float4(u.x, u.y, v.x, v.y);
            else if (c < ncols) *o = u;
        };
        SH::template fft_pair_st<INV>(cur, tw, yst2);
        cx<T>* tmp = cur;
        cur = nxt;
        nxt = tmp;
        cb ^= 1;
    }
}

// FP32 tiles: one CTA per SM (two 64 KB buffers at 512 threads)
template <typename T, bool INV, typename SH, bool PAIR>
__global__ void __launch_bounds__(SH::NT) k_y_c2c_pipe(const cx<T>* __restrict__ in, long in_pitch,
                                                      cx<T>* __restrict__ out, long out_pitch, int ncols, int nz,
                                                      const cx<T>* __restrict__ tw,
                                                      const double* __restrict__ dc_shift,
                                                      const int* __restrict__ skip)
{
    y_c2c_pipe<T, INV, SH, PAIR>(in, in_pitch, out, out_pitch, ncols, nz, tw, dc_shift, skip);
}

// FP64 tiles (half width, 256 threads): three resident CTAs per SM, which
// bounds the registers to 85 a thread
template <bool INV, typename SH>
__global__ void __launch_bounds__(SH::NT, 3) k_y_c2c_pipe64(const cx<double>* __restrict__ in, long in_pitch,
                                                           cx<double>* __restrict__ out, long out_pitch, int ncols,
                                                           int nz, const cx<double>* __restrict__ tw,
                                                           const double* __restrict__ dc_shift,
                                                           const int* __restrict__ skip)
{
    y_c2c_pipe<double, INV, SH, false>(in, in_pitch, out, out_pitch, ncols, nz, tw, dc_shift, skip);
}

// Tile shape of the pipelined y kernel.  FP64 tiles of 512-thread shapes
// are halved (W/2 columns, 256 threads): two 32 KB buffers per CTA let three
// CTAs share an SM, with 8 complex values per thread.
template <typename T, typename SH>
struct PipeShape {
    using type = SH;
};
template <int N, int W, int... RS>
struct PipeShape<double, ShapeCT<N, W, 512, RS...>> {
    using type = ShapeCT<N, W / 2, 256, RS...>;
};

template <typename T, bool INV, typename SH>
cudaError_t launch_y_c2c_pipe(const cx<T>* in, long in_pitch, cx<T>* out, long out_pitch, int ncols, int nz,
                              const cx<T>* tw, const double* dc_shift, const int* skip_flag, cudaStream_t st,
                              int* err)
{
    if constexpr (sizeof(T) == 4 && PairWidth<SH::W>::value && PPF_Y_TMA_W(SH::W) &&
                  (SH::N <= 256 || SH::N % 256 == 0)) {
        // TMA-fed paired tiles where the map can describe the spectrum
        CUtensorMap map;
        const bool tma = PPF_Y_TMA && ((uintptr_t)in & 15) == 0 && ((uintptr_t)out & 15) == 0 && in_pitch % 2 == 0 &&
                         out_pitch % 2 == 0 &&
                         tma_map_2d_f32(&map, const_cast<cx<T>*>(in), 2ull * (unsigned long long)ncols,
                                        (unsigned long long)nz * SH::N, (unsigned long long)in_pitch * sizeof(cx<T>),
                                        2u * SH::W, (unsigned)(SH::N < 256 ? SH::N : 256));
        if (tma) {
            auto kern = k_y_c2c_tma<INV, SH>;
            const size_t smem = 2 * (size_t)SH::N * SH::W * sizeof(cx<T>) + 128;
            cudaError_t e = set_smem(kern, smem);
            if (e != cudaSuccess) return e;
            const long tiles = (long)((ncols + SH::W - 1) / SH::W) * nz;
            unsigned grid = 0;
            e = persistent_grid(kern, SH::NT, smem, tiles, &grid);
            if (e != cudaSuccess) return e;
            kern<<<grid, SH::NT, smem, st>>>(map, reinterpret_cast<cx<float>*>(out), out_pitch, ncols, nz,
                                            reinterpret_cast<const cx<float>*>(tw), dc_shift, skip_flag, err);
            return cudaGetLastError();
        }
    }
    // paired passes where the tile is 16 FP32 columns and every column pair
    // starts on a 16-byte boundary
    constexpr bool PAIRABLE = sizeof(T) == 4 && PairWidth<SH::W>::value;
    const bool pair = PAIRABLE && in_pitch % 2 == 0 && out_pitch % 2 == 0 && ((uintptr_t)in & 15) == 0 &&
                      ((uintptr_t)out & 15) == 0;
    auto kern = [&] {
        if constexpr (sizeof(T) == 8) return k_y_c2c_pipe64<INV, SH>;
        else if constexpr (PAIRABLE) return pair ? k_y_c2c_pipe<T, INV, SH, true> : k_y_c2c_pipe<T, INV, SH, false>;
        else return k_y_c2c_pipe<T, INV, SH, false>;
    }();
    const size_t smem = 2 * (size_t)SH::N * SH::W * sizeof(cx<T>);
    cudaError_t e = set_smem(kern, smem);
    if (e != cudaSuccess) return e;
    const long tiles = (long)((ncols + SH::W - 1) / SH::W) * nz;
    unsigned grid = 0;
    e = persistent_grid(kern, SH::NT, smem, tiles, &grid);
    if (e != cudaSuccess) return e;
    kern<<<grid, SH::NT, smem, st>>>(in, in_pitch, out, out_pitch, ncols, nz, tw, dc_shift, skip_flag);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_yfwd(int kind, const cx<T>* in, long in_pitch, cx<T>* out, long out_pitch, int ncols,
                        const Geom& g, const FftSched& sch, const cx<T>* tw_ny, const cx<T>* tw_dct,
                        const int* skip_flag, cudaStream_t st, int* err_bits)
{
    cudaError_t err = cudaSuccess;
    with_shape<T>(sch, [&](auto sh) {
        using SH = decltype(sh);
        int W, threads;
        shape_geom<T, SH>(sch, W, threads);
        if (threads > 512) { err = cudaErrorInvalidConfiguration; return; }
        const size_t smem = (size_t)g.ny * W * sizeof(cx<T>);
        dim3 grid((unsigned)((ncols + W - 1) / W), (unsigned)g.nz);
        auto go = [&](auto kern) {
            err = set_smem(kern, smem);
            if (err != cudaSuccess) return;
            kern<<<grid, threads, smem, st>>>(in, in_pitch, out, out_pitch, ncols, g, sch, W, ilog2i(W), tw_ny, tw_dct,
                                              skip_flag);
            err = cudaGetLastError();
        };
        if (kind == Y_C2C) {
            if constexpr (SH::CT)
                err = launch_y_c2c_pipe<T, false, typename PipeShape<T, SH>::type>(in, in_pitch, out, out_pitch,
                                                                                  ncols, g.nz, tw_ny, nullptr,
                                                                                  skip_flag, st, err_bits);
            else go(k_yfwd<T, Y_C2C, SH>);
        }
        else if (kind == Y_CDCT) go(k_yfwd<T, Y_CDCT, SH>);
        else go(k_yfwd<T, Y_RPAIR, SH>);
    });
    return err;
}

template <typename T>
cudaError_t launch_yinv(int kind, const cx<T>* in, long in_pitch, cx<T>* out, long out_pitch, int ncols,
                        const Geom& g, const FftSched& sch, const cx<T>* tw_ny, const cx<T>* tw_dct,
                        const double* dc_shift, const int* skip_flag, cudaStream_t st, int* err_bits)
{
    cudaError_t err = cudaSuccess;
    with_shape<T>(sch, [&](auto sh) {
        using SH = decltype(sh);
        int W, threads;
        shape_geom<T, SH>(sch, W, threads);
        if (threads > 512) { err = cudaErrorInvalidConfiguration; return; }
        const size_t smem = (size_t)g.ny * W * sizeof(cx<T>);
        dim3 grid((unsigned)((ncols + W - 1) / W), (unsigned)g.nz);
        auto go = [&](auto kern) {
            err = set_smem(kern, smem);
            if (err != cudaSuccess) return;
            kern<<<grid, threads, smem, st>>>(in, in_pitch, out, out_pitch, ncols, g, sch, W, ilog2i(W), tw_ny, tw_dct,
                                              dc_shift, skip_flag);
            err = cudaGetLastError();
        };
        if (kind == Y_C2C) {
            if constexpr (SH::CT)
                err = launch_y_c2c_pipe<T, true, typename PipeShape<T, SH>::type>(in, in_pitch, out, out_pitch,
                                                                                 ncols, g.nz, tw_ny, dc_shift,
                                                                                 skip_flag, st, err_bits);
            else go(k_yinv<T, Y_C2C, SH>);
        }
        else if (kind == Y_CDCT) go(k_yinv<T, Y_CDCT, SH>);
        else go(k_yinv<T, Y_RPAIR, SH>);
    });
    return err;
}

#define PPF_INST(T)                                                                                        \
    template cudaError_t launch_yfwd<T>(int, const cx<T>*, long, cx<T>*, long, int, const Geom&,           \
                                        const FftSched&, const cx<T>*, const cx<T>*, const int*,           \
                                        cudaStream_t, int*);                                               \
    template cudaError_t launch_yinv<T>(int, const cx<T>*, long, cx<T>*, long, int, const Geom&,           \
                                        const FftSched&, const cx<T>*, const cx<T>*, const double*,        \
                                        const int*, cudaStream_t, int*);
PPF_INST(double)
PPF_INST(float)
#undef PPF_INST

}  // namespace ppf
