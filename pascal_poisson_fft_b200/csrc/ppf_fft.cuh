// ppf_fft.cuh -- shared-memory Stockham FFT engine of libppf (sm_100a).
//
// A CTA holds W interleaved complex lines of length n in shared memory
// (layout of sidx()).  Each pass of radix R computes all n/R butterflies of
// all W lines: every thread first loads the inputs of its butterflies into
// registers, the CTA synchronises, then the butterflies are applied and the
// outputs stored in Stockham autosort order, so the tile is transformed in
// place and ends in natural order.  Forward uses e^{-2 pi i jk/n}, inverse
// e^{+2 pi i jk/n}; neither normalises (the reference's cuFFT/FFTW
// convention, fft_3d_poisson.f90:195-286).
#pragma once
#include "ppf_common.cuh"

#include <type_traits>

namespace ppf {

template <typename T> struct K;
template <> struct K<double> {
    static constexpr double s3 = 0.86602540378443864676;   // sin(pi/3)
    static constexpr double r2 = 0.70710678118654752440;   // 1/sqrt(2)
    static constexpr double c1 = 0.30901699437494742410;   // cos(2pi/5)
    static constexpr double c2 = -0.80901699437494742410;  // cos(4pi/5)
    static constexpr double s1 = 0.95105651629515357212;   // sin(2pi/5)
    static constexpr double s2 = 0.58778525229247312917;   // sin(4pi/5)
    static constexpr double c16 = 0.92387953251128675613;  // cos(pi/8)
    static constexpr double s16 = 0.38268343236508977173;  // sin(pi/8)
};
template <> struct K<float> {
    static constexpr float s3 = 0.86602540378443864676f;
    static constexpr float r2 = 0.70710678118654752440f;
    static constexpr float c1 = 0.30901699437494742410f;
    static constexpr float c2 = -0.80901699437494742410f;
    static constexpr float s1 = 0.95105651629515357212f;
    static constexpr float s2 = 0.58778525229247312917f;
    static constexpr float c16 = 0.92387953251128675613f;
    static constexpr float s16 = 0.38268343236508977173f;
};

template <typename T, bool INV, int R> struct Dft;

template <typename T, bool INV> struct Dft<T, INV, 2> {
    static __device__ __forceinline__ void run(cx<T>* v)
    {
        cx<T> a = v[0], b = v[1];
        v[0] = a + b;
        v[1] = a - b;
    }
};

template <typename T, bool INV> struct Dft<T, INV, 4> {
    static __device__ __forceinline__ void run(cx<T>* v)
    {
        cx<T> a0 = v[0] + v[2], a1 = v[0] - v[2];
        cx<T> b0 = v[1] + v[3], b1 = mul_mi<T, INV>(v[1] - v[3]);
        v[0] = a0 + b0;
        v[2] = a0 - b0;
        v[1] = a1 + b1;
        v[3] = a1 - b1;
    }
};

template <typename T, bool INV> struct Dft<T, INV, 3> {
    static __device__ __forceinline__ void run(cx<T>* v)
    {
        cx<T> t1 = v[1] + v[2];
        cx<T> t2 = v[0] - t1 * (T)0.5;
        // forward: (-i sin(pi/3)) (x1 - x2); inverse: (+i sin(pi/3)) (x1 - x2)
        cx<T> t3 = mul_mi<T, INV>(v[1] - v[2]) * K<T>::s3;
        v[0] = v[0] + t1;
        v[1] = t2 + t3;
        v[2] = t2 - t3;
    }
};

template <typename T, bool INV> struct Dft<T, INV, 5> {
    static __device__ __forceinline__ void run(cx<T>* v)
    {
        cx<T> t1 = v[1] + v[4], t2 = v[2] + v[3];
        cx<T> t3 = v[1] - v[4], t4 = v[2] - v[3];
        cx<T> a1 = v[0] + t1 * K<T>::c1 + t2 * K<T>::c2;
        cx<T> a2 = v[0] + t1 * K<T>::c2 + t2 * K<T>::c1;
        cx<T> b1 = t3 * K<T>::s1 + t4 * K<T>::s2;
        cx<T> b2 = t3 * K<T>::s2 - t4 * K<T>::s1;
        // forward: y1 = a1 - i b1, y4 = a1 + i b1, y2 = a2 - i b2, y3 = a2 + i b2
        cx<T> mb1 = mul_mi<T, INV>(b1), mb2 = mul_mi<T, INV>(b2);
        v[0] = v[0] + t1 + t2;
        v[1] = a1 + mb1;
        v[4] = a1 - mb1;
        v[2] = a2 + mb2;
        v[3] = a2 - mb2;
    }
};

// w8^k multipliers for k = 1,2,3 (forward w8 = e^{-i pi/4})
template <typename T, bool INV>
__device__ __forceinline__ cx<T> w8(cx<T> a, int k)
{
    const T r = K<T>::r2;
    if (k == 1) return INV ? mk((a.x - a.y) * r, (a.x + a.y) * r) : mk((a.x + a.y) * r, (a.y - a.x) * r);
    if (k == 2) return mul_mi<T, INV>(a);
    return INV ? mk(-(a.x + a.y) * r, (a.x - a.y) * r) : mk((a.y - a.x) * r, -(a.x + a.y) * r);
}

template <typename T, bool INV> struct Dft<T, INV, 8> {
    static __device__ __forceinline__ void run(cx<T>* v)
    {
        cx<T> a[4], b[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            a[k] = v[k] + v[k + 4];
            b[k] = v[k] - v[k + 4];
        }
        b[1] = w8<T, INV>(b[1], 1);
        b[2] = w8<T, INV>(b[2], 2);
        b[3] = w8<T, INV>(b[3], 3);
        Dft<T, INV, 4>::run(a);
        Dft<T, INV, 4>::run(b);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            v[2 * m] = a[m];
            v[2 * m + 1] = b[m];
        }
    }
};

template <typename T, bool INV> struct Dft<T, INV, 16> {
    static __device__ __forceinline__ void run(cx<T>* v)
    {
        cx<T> a[8], b[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            a[k] = v[k] + v[k + 8];
            b[k] = v[k] - v[k + 8];
        }
        // b[k] *= w16^k, w16 = e^{-i pi/8} (forward)
        const T c = K<T>::c16, s = K<T>::s16, r = K<T>::r2;
        const T sg = INV ? (T)1 : (T)-1;
        const cx<T> w1 = mk(c, sg * s), w3 = mk(s, sg * c), w5 = mk(-s, sg * c), w7 = mk(-c, sg * s);
        b[1] = cmul(b[1], w1);
        b[2] = w8<T, INV>(b[2], 1);
        b[3] = cmul(b[3], w3);
        b[4] = mul_mi<T, INV>(b[4]);
        b[5] = cmul(b[5], w5);
        b[6] = w8<T, INV>(b[6], 3);
        b[7] = cmul(b[7], w7);
        (void)r;
        Dft<T, INV, 8>::run(a);
        Dft<T, INV, 8>::run(b);
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            v[2 * m] = a[m];
            v[2 * m + 1] = b[m];
        }
    }
};

// The twiddles w^r (r = 1..R-1, w = tw[k ts]) of one butterfly applied to
// its inputs v[1..R-1].  FP64 reads every power from the table.  FP32 reads
// w and forms w^2 = w w, w^3 = w w^2, w^4 = w^2 w^2, w^5 = w^4 w,
// w^6 = w^4 w^2, w^7 = w^4 w^3 (at most three products deep, a few ulp of
// FP32, which the FP64 refinement absorbs): one load instead of R-1 in the
// passes the FP32 y kernels are bound by.
template <typename T, bool INV, int R>
__device__ __forceinline__ void twiddle_powers(cx<T>* w, const cx<T>* __restrict__ tw, int k, int ts)
{
    static_assert(sizeof(T) == 4 && (R == 4 || R == 5 || R == 8), "FP32 radix 4, 5 or 8");
    w[1] = ldg(tw + k * ts);
    if (INV) w[1].y = -w[1].y;
    w[2] = cmul(w[1], w[1]);
    w[3] = cmul(w[1], w[2]);
    if constexpr (R >= 5) w[4] = cmul(w[2], w[2]);
    if constexpr (R == 8) {
        w[5] = cmul(w[4], w[1]);
        w[6] = cmul(w[4], w[2]);
        w[7] = cmul(w[4], w[3]);
    }
}

template <typename T, bool INV, int R>
__device__ __forceinline__ void twiddle_mul(cx<T>* v, const cx<T>* __restrict__ tw, int k, int ts)
{
    if constexpr (sizeof(T) == 4 && (R == 4 || R == 5 || R == 8)) {
        cx<T> w[R];
        twiddle_powers<T, INV, R>(w, tw, k, ts);
#pragma unroll
        for (int r = 1; r < R; ++r) v[r] = cmul(v[r], w[r]);
    } else {
#pragma unroll
        for (int r = 1; r < R; ++r) {
            cx<T> w = ldg(tw + r * k * ts);
            if (INV) w.y = -w.y;
            v[r] = cmul(v[r], w);
        }
    }
}

// One Stockham pass of radix R over the W-line tile.  tw[k] = e^{-2 pi i k/n}.
// v is the caller's register buffer (VMAX complex), shared by every radix so
// that all passes reuse the same registers.
constexpr int VMAX = 10;

template <typename T, bool INV, int R>
__device__ __forceinline__ void fft_pass(cx<T>* s, int n, int W, int lgW, int Ns, const cx<T>* __restrict__ tw,
                                         cx<T> (&v)[VMAX])
{
    constexpr int Q = (8 + R - 1) / R;  // butterflies per thread: tiles launch >= n*W/8 threads
    static_assert(Q * R <= VMAX, "register buffer too small");
    const int nb = n / R;
    const int items = nb << lgW;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int t = threadIdx.x + q * blockDim.x;
        if (t < items) {
            const int l = t & (W - 1), j = t >> lgW;
#pragma unroll
            for (int r = 0; r < R; ++r) v[q * R + r] = s[sidx<T>(j + r * nb, l, W)];
        }
    }
    __syncthreads();
    const int tstride = n / (Ns * R);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int t = threadIdx.x + q * blockDim.x;
        if (t < items) {
            const int l = t & (W - 1), j = t >> lgW;
            const int k = j % Ns;
            if (Ns > 1) twiddle_mul<T, INV, R>(v + q * R, tw, k, tstride);
            Dft<T, INV, R>::run(v + q * R);
            const int base = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) s[sidx<T>(base + r * Ns, l, W)] = v[q * R + r];
        }
    }
    __syncthreads();
}

// Full transform of the tile.  Caller synchronises before (tile loaded);
// the tile is complete and visible to all threads on return.
template <typename T, bool INV>
__device__ __forceinline__ void fft_tile(cx<T>* s, const FftSched& sch, int W, int lgW,
                                         const cx<T>* __restrict__ tw)
{
    cx<T> v[VMAX];
    int Ns = 1;
    for (int p = 0; p < sch.npass; ++p) {
        const int R = sch.radix[p];
        switch (R) {
            case 2: fft_pass<T, INV, 2>(s, sch.n, W, lgW, Ns, tw, v); break;
            case 3: fft_pass<T, INV, 3>(s, sch.n, W, lgW, Ns, tw, v); break;
            case 4: fft_pass<T, INV, 4>(s, sch.n, W, lgW, Ns, tw, v); break;
            case 5: fft_pass<T, INV, 5>(s, sch.n, W, lgW, Ns, tw, v); break;
            default: fft_pass<T, INV, 8>(s, sch.n, W, lgW, Ns, tw, v); break;
        }
        Ns *= R;
    }
}

// ---------------------------------------------------------------------------
// Compile-time engine: length N, W lines, NT threads and the radix sequence
// are template parameters, so every index, division and loop bound is a
// constant.  Same layout and pass structure as fft_tile.
// ---------------------------------------------------------------------------
// Tiles of length N whose rows are half a 128-byte bank row (W complex
// values of 64 bytes) and whose first pass is radix 8: that pass stores
// rows 8 apart and the position-fastest last pass reads 32 consecutive
// rows, which in the plain layout fall on one half of the bank rows; row n
// trades places with row n ^ 1 when bit 3 of n is set, which spreads both
// over the two halves.  (N is a multiple of 16, so every row has its
// partner; a row N past the end, the pipelines' extra Nyquist row, has
// bit 3 clear.)  Used where shared-memory throughput bounds the kernel, the
// FP64 512-point y pipeline (y passes 0.462 -> 0.450 ms per FP64 solve);
// the FP32 256-point x tiles, issue-bound, lose more to the three integer
// instructions per access than they gain (x passes +5-8 %).
template <typename T, int W, int N>
struct HalfRowSwap {
    static constexpr bool value = W * (int)sizeof(cx<T>) == 64 && sizeof(T) == 8 && N == 512;
};

template <typename T, int W, int N = 0>
__device__ __forceinline__ int sidx_ct(int n, int l)
{
    constexpr int G = SwizzleG<T>::value;
    constexpr int MASK = (W < G ? W : G) - 1;
    const int m = HalfRowSwap<T, W, N>::value ? (n ^ ((n >> 3) & 1)) : n;
    return m * W + (l ^ (n & MASK));
}

// Marker loader and storer of fft_pass_ct: the pass reads its inputs from
// and writes its outputs to the tile.
struct TileLd {};
struct TileSt {};

// LD: the inputs of the pass come from ld(n, l) instead of the tile (the
// first pass of a transform whose input is formed on the fly).  ST: the
// outputs go to st(n, l, value) instead of the tile (the last pass of a
// transform whose output is stored straight to global memory).  JF: the
// butterflies are assigned position-fastest (consecutive threads take
// consecutive j of one line) instead of line-fastest; in a last pass that
// makes a warp's outputs consecutive points of one line.
template <typename T, bool INV, int N, int W, int NT, int R, int NS, typename LD = TileLd, typename ST = TileSt,
          bool JF = false>
__device__ __forceinline__ void fft_pass_ct(cx<T>* s, const cx<T>* __restrict__ tw, LD ld = LD{}, ST st = ST{})
{
    constexpr int NB = N / R;
    constexpr int ITEMS = NB * W;
    constexpr int Q = (ITEMS + NT - 1) / NT;
    constexpr int TS = N / (NS * R);
    cx<T> v[Q * R];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int t = threadIdx.x + q * NT;
        if (ITEMS % NT == 0 || t < ITEMS) {
            const int l = JF ? t / NB : t % W, j = JF ? t % NB : t / W;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if constexpr (std::is_same<LD, TileLd>::value) v[q * R + r] = s[sidx_ct<T, W, N>(j + r * NB, l)];
                else v[q * R + r] = ld(j + r * NB, l);
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int t = threadIdx.x + q * NT;
        if (ITEMS % NT == 0 || t < ITEMS) {
            const int l = JF ? t / NB : t % W, j = JF ? t % NB : t / W;
            const int k = j % NS;
            if (NS > 1) twiddle_mul<T, INV, R>(v + q * R, tw, k, TS);
            Dft<T, INV, R>::run(v + q * R);
            const int base = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if constexpr (std::is_same<ST, TileSt>::value) s[sidx_ct<T, W, N>(base + r * NS, l)] = v[q * R + r];
                else st(base + r * NS, l, v[q * R + r]);
            }
        }
    }
    __syncthreads();
}

template <typename T, bool INV, int N, int W, int NT, int NS>
__device__ __forceinline__ void fft_ct_passes(cx<T>*, const cx<T>* __restrict__) {}

template <typename T, bool INV, int N, int W, int NT, int NS, int R0, int... RS>
__device__ __forceinline__ void fft_ct_passes(cx<T>* s, const cx<T>* __restrict__ tw)
{
    fft_pass_ct<T, INV, N, W, NT, R0, NS>(s, tw);
    fft_ct_passes<T, INV, N, W, NT, NS * R0, RS...>(s, tw);
}

// The passes of a radix sequence with a loader on the first and a storer
// on the last (position-fastest, so a warp stores consecutive points of one
// line)
template <typename T, bool INV, int N, int W, int NT, int NS, bool FIRST, typename LD, typename ST, int R0,
          int... RS>
__device__ __forceinline__ void fft_ct_chain(cx<T>* s, const cx<T>* __restrict__ tw, LD ld, ST st)
{
    constexpr bool LAST = sizeof...(RS) == 0;
    if constexpr (FIRST && LAST) fft_pass_ct<T, INV, N, W, NT, R0, NS, LD, ST, true>(s, tw, ld, st);
    else if constexpr (FIRST) fft_pass_ct<T, INV, N, W, NT, R0, NS, LD, TileSt>(s, tw, ld, TileSt{});
    else if constexpr (LAST) fft_pass_ct<T, INV, N, W, NT, R0, NS, TileLd, ST, true>(s, tw, TileLd{}, st);
    else fft_pass_ct<T, INV, N, W, NT, R0, NS>(s, tw);
    if constexpr (!LAST) fft_ct_chain<T, INV, N, W, NT, NS * R0, false, LD, ST, RS...>(s, tw, ld, st);
}

// Every pass of a radix sequence, the last one handing its outputs to st
template <typename T, bool INV, int N, int W, int NT, int NS, typename ST, int R0, int... RS>
__device__ __forceinline__ void fft_ct_last_st(cx<T>* s, const cx<T>* __restrict__ tw, ST st)
{
    if constexpr (sizeof...(RS) == 0) {
        fft_pass_ct<T, INV, N, W, NT, R0, NS, TileLd, ST>(s, tw, TileLd{}, st);
    } else {
        fft_pass_ct<T, INV, N, W, NT, R0, NS>(s, tw);
        fft_ct_last_st<T, INV, N, W, NT, NS * R0, ST, RS...>(s, tw, st);
    }
}

// ---------------------------------------------------------------------------
// Paired passes: FP32 tiles of W lines (W even; 16 or 8: rows of one or
// half a 128-byte bank row).  A thread takes the butterflies of lines 2p and
// 2p + 1 at one position, so one 16-byte shared access moves the values of
// both lines and one set of twiddle powers serves both (the same operations
// per line as fft_pass_ct).  Element (n, l) sits at n * W + l, unswizzled: a
// warp's accesses cover whole consecutive rows, or rows R apart in a first
// pass of odd radix R, which is free of bank conflicts.
// ---------------------------------------------------------------------------
template <bool INV, int N, int W, int NT, int R, int NS, typename ST = TileSt>
__device__ __forceinline__ void fft_pass_pair(cx<float>* s, const cx<float>* __restrict__ tw, ST st = ST{})
{
    static_assert(W % 2 == 0, "paired tiles hold an even number of lines");
    constexpr int P = W / 2;
    constexpr int NB = N / R;
    constexpr int ITEMS = NB * P;
    constexpr int Q = (ITEMS + NT - 1) / NT;
    constexpr int TS = N / (NS * R);
    float4* s4 = reinterpret_cast<float4*>(s);
    cx<float> a[Q * R], b[Q * R];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int t = threadIdx.x + q * NT;
        if (ITEMS % NT == 0 || t < ITEMS) {
            const int p = t % P, j = t / P;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const float4 f = s4[(j + r * NB) * P + p];
                a[q * R + r] = mk(f.x, f.y);
                b[q * R + r] = mk(f.z, f.w);
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int t = threadIdx.x + q * NT;
        if (ITEMS % NT == 0 || t < ITEMS) {
            const int p = t % P, j = t / P;
            const int k = j % NS;
            if constexpr (NS > 1) {
                cx<float> w[R];
                if constexpr (R == 4 || R == 5 || R == 8) {
                    twiddle_powers<float, INV, R>(w, tw, k, TS);
                } else {
#pragma unroll
                    for (int r = 1; r < R; ++r) {
                        w[r] = ldg(tw + r * k * TS);
                        if (INV) w[r].y = -w[r].y;
                    }
                }
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    a[q * R + r] = cmul(a[q * R + r], w[r]);
                    b[q * R + r] = cmul(b[q * R + r], w[r]);
                }
            }
            Dft<float, INV, R>::run(a + q * R);
            Dft<float, INV, R>::run(b + q * R);
            const int base = (j - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const cx<float> u = a[q * R + r], v = b[q * R + r];
                if constexpr (std::is_same<ST, TileSt>::value) s4[(base + r * NS) * P + p] = make_float4(u.x, u.y, v.x, v.y);
                else st(base + r * NS, p, u, v);
            }
        }
    }
    __syncthreads();
}

// Every paired pass of a radix sequence, the last one handing outputs n of
// lines 2p and 2p + 1 to st(n, p, u, v) instead of the tile
template <bool INV, int N, int W, int NT, int NS, typename ST, int R0, int... RS>
__device__ __forceinline__ void fft_pair_last_st(cx<float>* s, const cx<float>* __restrict__ tw, ST st)
{
    if constexpr (sizeof...(RS) == 0) {
        fft_pass_pair<INV, N, W, NT, R0, NS, ST>(s, tw, st);
    } else {
        fft_pass_pair<INV, N, W, NT, R0, NS>(s, tw);
        fft_pair_last_st<INV, N, W, NT, NS * R0, ST, RS...>(s, tw, st);
    }
}

// Tile shapes.  ShapeRT: everything at run time (fft_tile).  ShapeCT: a
// fixed length N = product of RS, W lines, NT threads per CTA.
struct ShapeRT {
    static constexpr bool CT = false;
    static constexpr int N = 0, W = 0, NT = 0;
};
template <int N_, int W_, int NT_, int... RS>
struct ShapeCT {
    static constexpr bool CT = true;
    static constexpr int N = N_, W = W_, NT = NT_;
    template <typename T, bool INV>
    static __device__ __forceinline__ void fft(cx<T>* s, const cx<T>* __restrict__ tw)
    {
        fft_ct_passes<T, INV, N_, W_, NT_, 1, RS...>(s, tw);
    }
    // the same transform with the last pass handing output n of line l to
    // st(n, l, value) instead of the tile; every read of the tile is done
    // when it returns (the last pass ends with a barrier)
    template <typename T, bool INV, typename ST>
    static __device__ __forceinline__ void fft_st(cx<T>* s, const cx<T>* __restrict__ tw, ST st)
    {
        fft_ct_last_st<T, INV, N_, W_, NT_, 1, ST, RS...>(s, tw, st);
    }
    // the same transform with the first pass reading ld(n, l) and the last
    // one handing output n of line l to st(n, l, value); the caller
    // synchronises before (ld's sources ready), the first pass's barrier
    // separates every ld from the in-place stores, and every read of the tile
    // is done when it returns
    template <typename T, bool INV, typename LD, typename ST>
    static __device__ __forceinline__ void fft_ld_st(cx<T>* s, const cx<T>* __restrict__ tw, LD ld, ST st)
    {
        fft_ct_chain<T, INV, N_, W_, NT_, 1, true, LD, ST, RS...>(s, tw, ld, st);
    }
    // fft_st in paired passes (FP32, W even): st(n, p, u, v) receives
    // outputs n of lines 2p and 2p + 1
    template <bool INV, typename ST>
    static __device__ __forceinline__ void fft_pair_st(cx<float>* s, const cx<float>* __restrict__ tw, ST st)
    {
        fft_pair_last_st<INV, N_, W_, NT_, 1, ST, RS...>(s, tw, st);
    }
};

// The element (n, l) of a tile of shape SH: the compile-time layout of a
// compile-time shape (the one its FFT passes use), else sidx.
template <typename T, typename SH>
__device__ __forceinline__ int tidx(int n, int l, int W)
{
    if constexpr (SH::CT) return sidx_ct<T, SH::W, SH::N>(n, l);
    else return sidx<T>(n, l, W);
}

}  // namespace ppf
