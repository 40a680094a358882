// ppf_xy_common.cuh -- shared pieces of the x and y transform kernels.
#pragma once
#include "ppf_fft.cuh"
#include "ppf_kernels.cuh"

#include <algorithm>
#include <mutex>

namespace ppf {

inline int ilog2i(int w)
{
    int l = 0;
    while ((1 << l) < w) ++l;
    return l;
}

// Opt a kernel into `bytes` of dynamic shared memory.  The 48 KB default
// covers static plus dynamic memory, and the transform kernels hold up to
// 4 KB of static arrays (line tables, reduction slots), so the attribute
// is set from 40 KB of dynamic memory on.
template <typename K>
cudaError_t set_smem(K kern, size_t bytes)
{
    if (bytes <= 40 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// run-time tile shape: W lines (a 128-byte bank row of elements when it
// fits) and >= n*W/8 threads, at most 512
inline int threads_for(int n, int W)
{
    int t = (n * W + 7) / 8;
    t = (t + 31) & ~31;
    if (t < 64) t = 64;
    return t;
}
template <typename T>
inline int pick_w(int n, int& threads)
{
    int W = SwizzleG<T>::value;
    while (W > 1 && threads_for(n, W) > 512) W >>= 1;
    threads = threads_for(n, W);
    return W;
}

// Compile-time shapes of the common lengths: W lines, NT threads (16 FP32
// or 8 FP64 elements per thread), radix sequence.  Other lengths use the
// run-time engine.  XINV: the shape of the x inverse, whose FP32 384-point
// lines run faster with the radix-3 pass last (the other transforms with it
// first); the tile width is the same either way.
template <typename T, bool XINV = false, typename F>
void with_shape(const FftSched& sch, F&& f)
{
    const int n = sch.n;
    if (sch.rt) { f(ShapeRT{}); return; }
    if constexpr (sizeof(T) == 8) {
        switch (n) {
            case 32:  f(ShapeCT<32, 64, 256, 8, 4>{}); return;
            case 64:  f(ShapeCT<64, 32, 256, 8, 8>{}); return;
            case 128: f(ShapeCT<128, 16, 256, 8, 4, 4>{}); return;
            case 256: f(ShapeCT<256, 8, 256, 8, 8, 4>{}); return;
            case 384: f(ShapeCT<384, 8, 384, 8, 4, 4, 3>{}); return;
            case 512: f(ShapeCT<512, 8, 512, 8, 8, 8>{}); return;
            case 768: f(ShapeCT<768, 4, 384, 8, 8, 4, 3>{}); return;
            default: break;
        }
    } else {
        switch (n) {
            case 32:  f(ShapeCT<32, 128, 256, 8, 4>{}); return;
            case 64:  f(ShapeCT<64, 64, 256, 8, 8>{}); return;
            case 128: f(ShapeCT<128, 32, 256, 8, 4, 4>{}); return;
            case 256: f(ShapeCT<256, 8, 256, 8, 8, 4>{}); return;
            case 384:
                if constexpr (XINV) f(ShapeCT<384, 8, 384, 8, 4, 4, 3>{});
                else f(ShapeCT<384, 8, 384, 3, 8, 4, 4>{});
                return;
            case 512: f(ShapeCT<512, 16, 512, 8, 8, 8>{}); return;
            case 768: f(ShapeCT<768, 8, 384, 3, 8, 8, 4>{}); return;
            default: break;
        }
    }
    f(ShapeRT{});
}

// launch geometry of a shape (run-time shapes: the schedule's width, else pick_w)
template <typename T, typename SH>
inline void shape_geom(const FftSched& sch, int& W, int& threads)
{
    if constexpr (SH::CT) {
        W = SH::W;
        threads = SH::NT;
    } else if (sch.w > 0) {
        W = sch.w;
        threads = threads_for(sch.n, W);
    } else {
        W = pick_w<T>(sch.n, threads);
    }
}

// a run-time width is usable: power of two, at most 128 lines, 512 threads
// and 200 KB of shared memory
template <typename T>
inline bool width_ok(int n, int W)
{
    if (W < 1 || W > 128 || (W & (W - 1))) return false;
    return threads_for(n, W) <= 512 && (size_t)n * W * sizeof(cx<T>) <= 200u * 1024u;
}

// FFT of the tile with the shape's engine
template <typename T, bool INV, typename SH>
__device__ __forceinline__ void tile_fft(cx<T>* s, const FftSched& sch, int W, int lgW, const cx<T>* __restrict__ tw)
{
    if constexpr (SH::CT) SH::template fft<T, INV>(s, tw);
    else fft_tile<T, INV>(s, sch, W, lgW, tw);
}

// grid of a persistent kernel: resident CTAs on every SM, at most one per
// tile.  Resident CTAs are computed once per kernel and device.
template <typename K>
cudaError_t persistent_grid(K kern, int threads, size_t smem, long tiles, unsigned* grid)
{
    struct Slot { const void* fn; int dev; int slots; };
    static Slot cache[256];
    static int used = 0;
    static std::mutex mu;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const void* fn = reinterpret_cast<const void*>(kern);
    int slots = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        for (int i = 0; i < used; ++i)
            if (cache[i].fn == fn && cache[i].dev == dev) { slots = cache[i].slots; break; }
    }
    if (slots == 0) {
        int sms = 0, per = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, threads, smem);
        if (e != cudaSuccess) return e;
        if (per < 1) return cudaErrorInvalidConfiguration;
        slots = sms * per;
        std::lock_guard<std::mutex> lk(mu);
        if (used < 256) cache[used++] = Slot{ fn, dev, slots };
    }
    const long g = std::min<long>(tiles, (long)slots);
    *grid = (unsigned)std::max<long>(g, 1);
    return cudaSuccess;
}

}  // namespace ppf
