// ppf_common.cuh -- shared device helpers of libppf (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ppf {

template <typename T>
struct __align__(2 * sizeof(T)) cx {
    T x, y;
};

template <typename T> __device__ __forceinline__ cx<T> mk(T a, T b) { cx<T> r; r.x = a; r.y = b; return r; }
template <typename T> __device__ __forceinline__ cx<T> operator+(cx<T> a, cx<T> b) { return mk(a.x + b.x, a.y + b.y); }
template <typename T> __device__ __forceinline__ cx<T> operator-(cx<T> a, cx<T> b) { return mk(a.x - b.x, a.y - b.y); }
template <typename T> __device__ __forceinline__ cx<T> operator*(cx<T> a, T s) { return mk(a.x * s, a.y * s); }
template <typename T> __device__ __forceinline__ cx<T> cmul(cx<T> a, cx<T> b)
{
    return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T> __device__ __forceinline__ cx<T> conj(cx<T> a) { return mk(a.x, -a.y); }
// multiply by -i (forward) or +i (inverse)
template <typename T, bool INV> __device__ __forceinline__ cx<T> mul_mi(cx<T> a)
{
    return INV ? mk(-a.y, a.x) : mk(a.y, -a.x);
}

template <typename T> __device__ __forceinline__ cx<T> ldg(const cx<T>* p) { return *p; }
template <> __device__ __forceinline__ cx<double> ldg(const cx<double>* p)
{
    double2 v = __ldg(reinterpret_cast<const double2*>(p));
    return mk(v.x, v.y);
}
template <> __device__ __forceinline__ cx<float> ldg(const cx<float>* p)
{
    float2 v = __ldg(reinterpret_cast<const float2*>(p));
    return mk(v.x, v.y);
}

// Shared-memory tile layout: element (n, l) of W interleaved lines, row n
// holds the W lines' n-th elements.  The low bits of the line index are
// XOR-swizzled with the row so that column-wise writes (one line, many n)
// and row-wise accesses are both free of bank conflicts.  G = elements per
// 128-byte bank row; W is a power of two (rows narrower than a bank row
// are swizzled over W).
template <typename T> struct SwizzleG { static constexpr int value = 128 / (int)sizeof(cx<T>); };

template <typename T>
__device__ __forceinline__ int sidx(int n, int l, int W)
{
    constexpr int G = SwizzleG<T>::value;
    return n * W + (l ^ (n & (W - 1) & (G - 1)));
}

// Asynchronous global -> shared copies (cp.async): one element per call,
// completion tracked per thread by commit groups.
__device__ __forceinline__ void cp_async_elem(float* dst, const float* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_elem(cx<float>* dst, const cx<float>* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_f64(double* dst, const double* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_elem(cx<double>* dst, const cx<double>* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
// 16 bytes, both addresses 16-byte aligned
__device__ __forceinline__ void cp_async_16(void* dst, const void* src)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most N of this thread's most recent groups are pending
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Bulk prefetch of `bytes` (a multiple of 16) at a 16-byte aligned global
// address into L2.
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;\n" ::"l"(p), "r"(bytes) : "memory");
}

// Per-axis FFT schedule: complex length n = prod(radix[0..npass)).
struct FftSched {
    int n;
    int npass;
    int radix[12];
    int w;    // lines per tile of the run-time engine (0: default width)
    int rt;   // 1: run-time engine even where a compile-time shape exists
};

}  // namespace ppf
