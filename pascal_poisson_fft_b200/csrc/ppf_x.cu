// ppf_x.cu -- x-direction transform kernels of libppf (sm_100a).
//
// One CTA transforms W consecutive x-lines (fixed y, z) in shared memory
// (ppf_fft.cuh): a real FFT through a half-length complex FFT and a split,
// or a DCT-II with Makhoul's reordering folded into the tile load and the
// post-twiddle folded into the store.  The reference runs each of these as
// a cuFFT call bracketed by separate reorder, twiddle, copy and scale
// passes (01_Fortran/src/fft_3d_poisson.f90:378-419, 561-616, 915-1033);
// here each is one read and one write of the field.  SH selects the
// compile-time engine of a common length or the run-time engine.
#include "ppf_tma.cuh"
#include "ppf_x_dev.cuh"

#include <type_traits>

#ifndef PPF_XINV_BULK
#define PPF_XINV_BULK 1
#endif
// resident CTAs per SM asked of the 256-point x-inverse pipeline (a register bound)
#ifndef PPF_XINV_256_CTAS
#define PPF_XINV_256_CTAS 5
#endif

namespace ppf {

#define PPF_XFWD_PARAMS                                                                                      \
    const double* __restrict__ f, ResidIn rs, Geom g, void* __restrict__ out_, long out_pitch, FftSched sch,    \
        int Wrt, int lgWrt, const cx<T>* __restrict__ tw_half, const cx<T>* __restrict__ tw_n,                \
        const cx<T>* __restrict__ tw_dct, const int* __restrict__ skip
#define PPF_XFWD_ARGS f, rs, g, out_, out_pitch, sch, Wrt, lgWrt, tw_half, tw_n, tw_dct, skip, (long)blockIdx.x

// the plain periodic transform of 384-point tiles (768-point lines) is bounded
// to four resident CTAs of 384 threads: 32 registers, five CTAs fit an SM
template <typename T, bool DCT, int RESID, typename SH>
__global__ void __launch_bounds__(512, (SH::N == 384 && !DCT && RESID == 0) ? 4 : 0) k_xfwd(PPF_XFWD_PARAMS)
{
    xfwd<T, DCT, RESID, SH>(PPF_XFWD_ARGS);
}

// FP64 compile-time tiles: five resident CTAs of SH::NT threads per SM
template <bool DCT, typename SH, typename T = double>
__global__ void __launch_bounds__(SH::NT, 5) k_xfwd64(PPF_XFWD_PARAMS)
{
    xfwd<T, DCT, 0, SH>(PPF_XFWD_ARGS);
}

// The x stencil ghosts of a tile's lines (the periodic copy, or the wall
// mirror, of each line's first and last interior value), copied after the
// tile's interior values are written and visible to the block: the value a
// ghost receives is the one just stored, in every iterate kind.
#define PPF_XINV_PARAMS                                                                                      \
    const void* __restrict__ in_, long in_pitch, double* __restrict__ P, float* __restrict__ U, Geom g,        \
        double* __restrict__ partials,                                                                         \
        const double* __restrict__ mean_prev, FftSched sch, int Wrt, int lgWrt,                                \
        const cx<T>* __restrict__ tw_half, const cx<T>* __restrict__ tw_n, const cx<T>* __restrict__ tw_dct,   \
        const int* __restrict__ skip
#define PPF_XINV_ARGS in_, in_pitch, P, U, g, partials, mean_prev, sch, Wrt, lgWrt, tw_half, tw_n, tw_dct, skip, \
    (long)blockIdx.x

template <typename T, bool DCT, bool ACC, bool GHOST, typename SH, int UK = U_P>
__global__ void __launch_bounds__(512) k_xinv(PPF_XINV_PARAMS)
{
    xinv<T, DCT, ACC, GHOST, SH, UK>(PPF_XINV_ARGS);
}

// FP64 compile-time tiles: five resident CTAs of SH::NT threads per SM
template <bool DCT, typename SH, typename T = double>
__global__ void __launch_bounds__(SH::NT, 5) k_xinv64(PPF_XINV_PARAMS)
{
    xinv<T, DCT, false, false, SH>(PPF_XINV_ARGS);
}

// --------------------------------------------------------------------------
// x inverse of FP32 spectra, periodic x, compile-time shapes: persistent
// CTAs walk tiles of W lines; the next tile's half-spectrum rows are copied
// with cp.async into the second of two raw buffers ([k][line], nc+1 rows)
// while the current tile is transformed: the C2R split is formed as the
// first FFT pass loads its inputs, and the last pass hands its outputs to
// the accumulate and store -- the output semantics of
// k_xinv<T, false, ACC, GHOST, SH, UK>.  (FP64 tiles take the non-pipelined kernel:
// two 66 KB buffers at 128 registers leave too few resident CTAs.)  BULK:
// each line's spectral row arrives as one bulk copy (cp.async.bulk, one
// thread, completion on an mbarrier per buffer) into a raw buffer of rows
// XINV_RS(NC) values apart, instead of one cp.async per value: rows of
// NC + 2 values (16-byte multiples), which the row pitch must hold; the row
// stride is 4 mod 16 values, so the split's line-fastest reads spread over
// the banks.  A wait that gives up (about 2 s of sleeping polls) sets err
// bit 2 and ends the CTA's walk.
// --------------------------------------------------------------------------
constexpr int xinv_rs(int nc) { return ((nc + 2 + 11) / 16) * 16 + 4; }
constexpr unsigned XB_POLL_NS = 20000;
constexpr long XB_WAIT_LIMIT = 100000;

template <typename T, bool ACC, bool GHOST, typename SH, int UK = U_P, bool BULK = false>
__global__ void __launch_bounds__(SH::NT, (SH::N <= 128) ? 2 : SH::N == 384 ? 3 : (SH::N == 256 ? PPF_XINV_256_CTAS : 0)) k_xinv_pipe(const cx<T>* __restrict__ in, long in_pitch,
                                                     double* __restrict__ P, float* __restrict__ U, Geom g,
                                                     double* __restrict__ partials,
                                                     const double* __restrict__ mean_prev,
                                                     const cx<T>* __restrict__ tw_half,
                                                     const cx<T>* __restrict__ tw_n, const int* __restrict__ skip,
                                                     int* __restrict__ err)
{
    if (skip && *skip) return;
    constexpr int NC = SH::N, W = SH::W, NT = SH::NT;
    constexpr int NR = NC + 1;
    constexpr int RS = xinv_rs(NC);                       // BULK: raw row stride
    constexpr unsigned RB = (unsigned)((NC + 2) * sizeof(cx<T>));   // BULK: bytes per row copy
    static_assert(!BULK || (NC % 2 == 0 && RS >= NC + 2 && RS * W >= NC * W), "bulk rows");
    constexpr int ER = BULK ? RS * W : NR * W;
    constexpr int NX = 2 * NC;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cx<T>* cur = reinterpret_cast<cx<T>*>(smem_raw);
    cx<T>* nxt = cur + ER;
    __shared__ long line_base[W], line_gy[W], line_gz[W];
    __shared__ __align__(8) uint64_t xbar[2];
    __shared__ int xabort;
    const long nlines = (long)g.ny * g.nz;
    const long ntiles = (nlines + W - 1) / W;
    if (BULK) {
        if (threadIdx.x == 0) {
            mbar_init(&xbar[0], 1);
            mbar_init(&xbar[1], 1);
            mbar_init_fence();
            xabort = 0;
        }
        __syncthreads();
    }
    int cb = 0;            // BULK: the barrier of the current buffer
    unsigned xpar = 0;     // BULK: bit b, parity of buffer b's next completion
    auto src = [&](long o) -> double {
        if constexpr (UK == U_ACC) return (double)U[o];
        else return P[o];
    };
    auto put = [&](long o, double v) {
        if constexpr (UK == U_WRITE) U[o] = (float)v;
        else P[o] = v;
    };
    auto issue = [&](long t, cx<T>* b, int bi) {
        const long line0 = t * W;
        if constexpr (BULK) {
            if (threadIdx.x == 0) {
                const int nl = (int)(nlines - line0 < W ? nlines - line0 : W);
                fence_proxy_async_smem();   // the previous tile's reads of b come first
                mbar_arrive_expect_tx(&xbar[bi], (unsigned)nl * RB);
                for (int l = 0; l < nl; ++l) bulk_load(b + l * RS, in + (line0 + l) * in_pitch, RB, &xbar[bi]);
            }
        } else {
            for (int e = threadIdx.x; e < ER; e += NT) {
                const int l = e / NR, k = e - l * NR;
                cx<T>* d = b + sidx_ct<T, W, SH::N>(k, l);
                if (line0 + l < nlines) cp_async_elem(d, in + (line0 + l) * in_pitch + k);
                else *d = mk<T>((T)0, (T)0);
            }
            cp_async_commit();
        }
    };
    double acc_du = 0.0, acc_u = 0.0, acc_s = 0.0;
    const double mprev = (ACC && mean_prev) ? *mean_prev : 0.0;
    long t = blockIdx.x;
    if (t < ntiles) issue(t, cur, cb);
    for (; t < ntiles; t += gridDim.x) {
        const long line0 = t * W;
        const long tn = t + gridDim.x;
        if (tn < ntiles) issue(tn, nxt, cb ^ 1);
        else if (!BULK) cp_async_commit();
        // this tile's rows of u into L2 ahead of the read-modify-write
        if (ACC && threadIdx.x < W && line0 + threadIdx.x < nlines) {
            const long line = line0 + threadIdx.x;
            const long o = (line % g.ny + 1) * g.pstride_y + (line / g.ny + 1) * g.pstride_z;
            if (UK == U_ACC) prefetch_row(U, o, NX + 2);
            else prefetch_row(P, o, NX + 2);
        }
        bool has_yz = false;
        for (int l = threadIdx.x; l < W; l += NT) {
            const long line = line0 + l;
            const long j = line % g.ny, k = line / g.ny;
            line_base[l] = 1 + (j + 1) * g.pstride_y + (k + 1) * g.pstride_z;
            if (GHOST) {
                long gy = 0;
                if (j == 0) gy = g.py ? (long)g.ny * g.pstride_y : -g.pstride_y;
                else if (j == g.ny - 1) gy = g.py ? -(long)g.ny * g.pstride_y : g.pstride_y;
                long gz = 0;
                if (k == 0) gz = -g.pstride_z;
                else if (k == g.nz - 1) gz = g.pstride_z;
                line_gy[l] = gy;
                line_gz[l] = gz;
                has_yz |= (line < nlines) && (gy || gz);
            }
        }
        if constexpr (BULK) {
            // the rows of tile t have landed (every thread observes the barrier)
            if (!mbar_wait_sleep_bounded(&xbar[cb], (xpar >> cb) & 1u, XB_POLL_NS, XB_WAIT_LIMIT)) xabort = 1;
            xpar ^= 1u << cb;
        } else {
            cp_async_wait<1>();  // this thread's copies of tile t have landed
        }
        // whether any line of the tile has y or z ghosts (most tiles have none)
        const bool yz = __syncthreads_or(has_yz);
        if (BULK && xabort) {
            if (threadIdx.x == 0 && err) atomicOr(err, 2);
            // the next tile's rows may be in flight: wait for them (bounded)
            // before the CTA's shared memory is released
            if (threadIdx.x == 0 && tn < ntiles)
                mbar_wait_sleep_bounded(&xbar[cb ^ 1], (xpar >> (cb ^ 1)) & 1u, XB_POLL_NS, XB_WAIT_LIMIT);
            break;
        }
        // the C2R split, Z_m from (X_m, conj X_{nc-m}) with w_m, formed as the
        // first FFT pass loads its inputs (X_0 and X_nc enter with zero
        // imaginary parts)
        auto zsplit = [&](int m, int l) -> cx<T> {
            cx<T> a = BULK ? cur[l * RS + m] : cur[sidx_ct<T, W, SH::N>(m, l)];
            cx<T> xc = BULK ? cur[l * RS + NC - m] : cur[sidx_ct<T, W, SH::N>(NC - m, l)];
            if (m == 0) { a.y = (T)0; xc.y = (T)0; }
            const cx<T> b = conj(xc);
            const cx<T> Ev = a + b, D = a - b;
            const cx<T> O = cmul(D, conj(ldg(tw_n + m)));
            return mk<T>(Ev.x - O.y, Ev.y + O.x);
        };
        // the last pass hands z_n of line l to the output (x_2n, x_2n+1 are
        // its real and imaginary parts); a warp writes consecutive points of
        // one line
        auto zout = [&](int n, int l, cx<T> zv) {
            if (line0 + l >= nlines) return;
            const long o = line_base[l] + 2 * n;
            if constexpr (UK == U_WRITE && !ACC && sizeof(T) == 4) {
                // the FP32 first iterate: the values go out as they are, and
                // only their sum is kept (the initial gate after this pass
                // needs the mean, not the norms)
                U[o] = zv.x;
                U[o + 1] = zv.y;
                if (GHOST && yz) {
                    const long gy = line_gy[l], gz = line_gz[l];
                    if (gy) { U[o + gy] = zv.x; U[o + 1 + gy] = zv.y; }
                    if (gz) { U[o + gz] = zv.x; U[o + 1 + gz] = zv.y; }
                }
                if (partials) acc_s += (double)zv.x + (double)zv.y;
                return;
            }
            const double x0 = (double)zv.x, x1 = (double)zv.y;
            double u0 = x0, u1 = x1;
            if (ACC) {
                u0 = (src(o) - mprev) + x0;
                u1 = (src(o + 1) - mprev) + x1;
            }
            put(o, u0);
            put(o + 1, u1);
            if (GHOST && yz) {
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
        };
        SH::template fft_ld_st<T, true>(cur, tw_half, zsplit, zout);
        __syncthreads();  // cur and the line tables are refilled
        if (GHOST) x_ghosts<UK>(P, U, g, line0, W, nlines, NX);
        cx<T>* tmp = cur;
        cur = nxt;
        nxt = tmp;
        cb ^= 1;
    }
    if (partials) {
        __shared__ double red[3][32];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            acc_du += __shfl_down_sync(0xffffffffu, acc_du, off);
            acc_u += __shfl_down_sync(0xffffffffu, acc_u, off);
            acc_s += __shfl_down_sync(0xffffffffu, acc_s, off);
        }
        const int w = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0) { red[0][w] = acc_du; red[1][w] = acc_u; red[2][w] = acc_s; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = 0, b = 0, c = 0;
            for (int q = 0; q < NT / 32; ++q) { a += red[0][q]; b += red[1][q]; c += red[2][q]; }
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
cudaError_t launch_xfwd(bool dct, const double* f, const ResidIn* resid, const Geom& g, void* out, long out_pitch,
                        const FftSched& sch, const cx<T>* tw_half, const cx<T>* tw_n, const cx<T>* tw_dct,
                        const int* skip_flag, cudaStream_t st)
{
    const int nc = g.nx / 2;
    ResidIn rs{};
    if (resid) rs = *resid;
    cudaError_t err = cudaSuccess;
    with_shape<T>(sch, [&](auto sh) {
        using SH = decltype(sh);
        int W, threads;
        shape_geom<T, SH>(sch, W, threads);
        if (threads > 512) { err = cudaErrorInvalidConfiguration; return; }
        const size_t smem = (size_t)nc * W * sizeof(cx<T>);
        dim3 grid((unsigned)(((long)g.ny * g.nz + W - 1) / W));
        auto go = [&](auto kern) {
            err = set_smem(kern, smem);
            if (err != cudaSuccess) return;
            kern<<<grid, threads, smem, st>>>(f, rs, g, out, out_pitch, sch, W, ilog2i(W), tw_half, tw_n, tw_dct,
                                              skip_flag);
            err = cudaGetLastError();
        };
        if constexpr (SH::CT && sizeof(T) == 8) {
            if (!resid) {
                if (dct) go(k_xfwd64<true, SH>);
                else go(k_xfwd64<false, SH>);
                return;
            }
        }
        if constexpr (sizeof(T) == 4) {
            if (resid && rs.U) {
                if (dct) go(k_xfwd<T, true, 2, SH>);
                else go(k_xfwd<T, false, 2, SH>);
                return;
            }
        }
        if (dct) {
            if (resid) go(k_xfwd<T, true, 1, SH>);
            else go(k_xfwd<T, true, 0, SH>);
        } else {
            if (resid) go(k_xfwd<T, false, 1, SH>);
            else go(k_xfwd<T, false, 0, SH>);
        }
    });
    return err;
}

template <typename T>
cudaError_t launch_xinv(bool dct, const void* in, long in_pitch, double* P, float* U, int ukind, const Geom& g,
                        bool accumulate, bool stencil_ghosts, double* partials, const double* mean_prev,
                        const FftSched& sch, const cx<T>* tw_half, const cx<T>* tw_n, const cx<T>* tw_dct,
                        const int* skip_flag, cudaStream_t st, long* blocks_used, int* err_bits)
{
    const int nc = g.nx / 2;
    int* const ebits = err_bits;
    // the FP32 iterate belongs to the refinement of FP32 spectra: U_WRITE
    // with stencil ghosts and no accumulate, U_ACC with both
    if (ukind != U_P && (sizeof(T) != 4 || !U || !stencil_ghosts || accumulate != (ukind == U_ACC)))
        return cudaErrorInvalidValue;
    cudaError_t err = cudaSuccess;
    with_shape<T, true>(sch, [&](auto sh) {
        using SH = decltype(sh);
        int W, threads;
        shape_geom<T, SH>(sch, W, threads);
        if (threads > 512) { err = cudaErrorInvalidConfiguration; return; }
        const size_t smem = (size_t)nc * W * sizeof(cx<T>);
        dim3 grid((unsigned)(((long)g.ny * g.nz + W - 1) / W));
        if (blocks_used) *blocks_used = grid.x;
        auto go = [&](auto kern) {
            err = set_smem(kern, smem);
            if (err != cudaSuccess) return;
            kern<<<grid, threads, smem, st>>>(in, in_pitch, P, U, g, partials, mean_prev, sch, W, ilog2i(W), tw_half,
                                              tw_n, tw_dct, skip_flag);
            err = cudaGetLastError();
        };
        if constexpr (SH::CT && sizeof(T) == 4) {
            if (!dct) {  // pipelined FP32 tiles
                auto pipe = [&](auto kern, bool bulk) {
                    const size_t rows = bulk ? (size_t)xinv_rs(SH::N) : (size_t)(SH::N + 1);
                    const size_t psmem = 2 * rows * SH::W * sizeof(cx<T>);
                    err = set_smem(kern, psmem);
                    unsigned pgrid = 0;
                    if (err == cudaSuccess) err = persistent_grid(kern, SH::NT, psmem, (long)grid.x, &pgrid);
                    if (err != cudaSuccess) return;
                    if (blocks_used) *blocks_used = pgrid;
                    kern<<<pgrid, SH::NT, psmem, st>>>(reinterpret_cast<const cx<T>*>(in), in_pitch, P, U, g,
                                                      partials, mean_prev, tw_half, tw_n, skip_flag, ebits);
                    err = cudaGetLastError();
                };
                // bulk row copies where every row starts on a 16-byte boundary
                // and the pitch holds the NC + 2 values a copy reads
                const bool bulk = PPF_XINV_BULK && in_pitch >= SH::N + 2 && (in_pitch * sizeof(cx<T>)) % 16 == 0 &&
                                  ((uintptr_t)in & 15) == 0;
                auto pick = [&](auto k_bulk, auto k_elem) {
                    if (bulk) pipe(k_bulk, true);
                    else pipe(k_elem, false);
                };
                if (ukind == U_WRITE)
                    pick(k_xinv_pipe<T, false, true, SH, U_WRITE, true>, k_xinv_pipe<T, false, true, SH, U_WRITE, false>);
                else if (ukind == U_ACC)
                    pick(k_xinv_pipe<T, true, true, SH, U_ACC, true>, k_xinv_pipe<T, true, true, SH, U_ACC, false>);
                else if (!stencil_ghosts)
                    pick(k_xinv_pipe<T, false, false, SH, U_P, true>, k_xinv_pipe<T, false, false, SH, U_P, false>);
                else if (accumulate)
                    pick(k_xinv_pipe<T, true, true, SH, U_P, true>, k_xinv_pipe<T, true, true, SH, U_P, false>);
                else
                    pick(k_xinv_pipe<T, false, true, SH, U_P, true>, k_xinv_pipe<T, false, true, SH, U_P, false>);
                return;
            }
        }
        if constexpr (SH::CT && sizeof(T) == 8) {
            if (!stencil_ghosts && !accumulate) {
                if (dct) go(k_xinv64<true, SH>);
                else go(k_xinv64<false, SH>);
                return;
            }
        }
        if constexpr (sizeof(T) == 4) {
            if (ukind == U_WRITE) {
                if (dct) go(k_xinv<T, true, false, true, SH, U_WRITE>);
                else go(k_xinv<T, false, false, true, SH, U_WRITE>);
                return;
            }
            if (ukind == U_ACC) {
                if (dct) go(k_xinv<T, true, true, true, SH, U_ACC>);
                else go(k_xinv<T, false, true, true, SH, U_ACC>);
                return;
            }
        }
        if (stencil_ghosts) {
            if (dct) {
                if (accumulate) go(k_xinv<T, true, true, true, SH>);
                else go(k_xinv<T, true, false, true, SH>);
            } else {
                if (accumulate) go(k_xinv<T, false, true, true, SH>);
                else go(k_xinv<T, false, false, true, SH>);
            }
        } else if (dct) {
            go(k_xinv<T, true, false, false, SH>);
        } else {
            go(k_xinv<T, false, false, false, SH>);
        }
    });
    return err;
}

template <typename T>
long xinv_blocks(const Geom& g, const FftSched& sch)
{
    long blocks = 0;
    with_shape<T, true>(sch, [&](auto sh) {
        using SH = decltype(sh);
        int W, threads;
        shape_geom<T, SH>(sch, W, threads);
        blocks = ((long)g.ny * g.nz + W - 1) / W;
    });
    return blocks;
}

template long xinv_blocks<double>(const Geom&, const FftSched&);
template long xinv_blocks<float>(const Geom&, const FftSched&);

#define PPF_INST(T)                                                                                        \
    template cudaError_t launch_xfwd<T>(bool, const double*, const ResidIn*, const Geom&, void*, long,     \
                                        const FftSched&, const cx<T>*, const cx<T>*, const cx<T>*,         \
                                        const int*, cudaStream_t);                                         \
    template cudaError_t launch_xinv<T>(bool, const void*, long, double*, float*, int, const Geom&, bool,  \
                                        bool,                                                              \
                                        double*, const double*, const FftSched&, const cx<T>*,             \
                                        const cx<T>*, const cx<T>*, const int*, cudaStream_t, long*, int*);
PPF_INST(double)
PPF_INST(float)
#undef PPF_INST

}  // namespace ppf
