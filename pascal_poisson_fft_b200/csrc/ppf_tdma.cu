// ppf_tdma.cu -- batched tridiagonal solves by the Thomas algorithm (sm_100a).
//
// One thread per system; consecutive threads own consecutive systems, so
// every row access of a warp is one contiguous segment.  The arithmetic of
// each row is the reference's, operation for operation
// (01_Fortran/PaScaL_TDMA/src/tdmas.f90:114-147 tdma_many, :160-213
// tdma_cycl_many; tdmas_cuda.f90:35-217): the first row divides by b, every
// later row forms r = 1/(b - a c'), d' = r (d - a d'), c' = r c, and the
// back substitution is d = d' - c' d_next.  Products and sums use explicitly
// rounded intrinsics so the compiler cannot contract them into FMAs: the
// solve reproduces the reference's rounding, which matters because the low
// wavenumber systems are ill-conditioned (a different elimination order
// changes their solution at the cond * eps level).
//
// The reference writes c' and d' of every row back to global memory and
// reads them again in the back substitution.  Here the forward sweep keeps
// only a checkpoint (c', d') every CH rows in global memory; the backward
// sweep re-reads the CH right-hand sides of a chunk, recomputes its c', d'
// from the checkpoint (the same operations, so the same bits) and
// substitutes.  Per row the field is read twice and written once.
//
// k_thomas_z is the Poisson z-solve: the coefficients of
// cuda_Poisson_TDMA_z_{real,complex} (01_Fortran/src/fft_3d_poisson.f90:
// 1121-1344) -- am = 1/dx3_k/dmx3_k, ap = 1/dx3_k/dmx3_{k+1},
// b = (-am - ap) - dxk2 - dyk2, the pin (a,b,c,d) = (0,1,0,0) at
// (kx,ky,k) = (0,0,1) -- are generated in registers rather than stored as
// six N-sized arrays, and real and imaginary parts share one sweep (they
// are separate sweeps with identical coefficients in the reference).  The
// thread of the (0,0) system also reports the z-average of its solution,
// which the y-inverse pass subtracts (the arithmetic-mean removal of
// cuda_Poisson_average_elimination, :628-664, done in spectral space).
// k_thomas_arr / k_thomas_cycl solve systems given as coefficient arrays
// (PaScaL_TDMA_many_solve[_cycle] replacements).
#include "ppf_kernels.cuh"
#include "ppf_tdma_dev.cuh"
#include "ppf_misc_dev.cuh"
#include "ppf_tma.cuh"

#include <math.h>
#include <mutex>

namespace ppf {

using namespace zdev;

namespace {
// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// dependency on libcuda)
using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encode_tiled()
{
    static EncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiled>(p);
    });
    return fn;
}
}  // namespace

bool tma_map_2d_f32(CUtensorMap* map, void* base, unsigned long long inner, unsigned long long rows,
                    unsigned long long row_bytes, unsigned box_inner, unsigned box_rows)
{
    const EncodeTiled enc = encode_tiled();
    if (!enc) return false;
    const cuuint64_t dims[2] = { inner, rows };
    const cuuint64_t strides[1] = { row_bytes };
    const cuuint32_t box[2] = { box_inner, box_rows };
    const cuuint32_t estr[2] = { 1, 1 };
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// MODE 0: every system, arithmetic A.  MODE 1: only systems above the
// low-wavenumber threshold (FP32 path).  MODE 2: only systems below it.
template <typename T, typename A, bool CPLX, int MODE, bool CYC>
__global__ void __launch_bounds__(TPB) k_thomas_z(void* __restrict__ data_, ZSys z, const int* __restrict__ skip,
                                                  int* __restrict__ err)
{
    if (skip && *skip) return;
    using E = typename Elem<T, CPLX>::type;
    E* data = reinterpret_cast<E*>(data_);
    const long sys = (long)blockIdx.x * TPB + threadIdx.x;
    const int kx = (int)(sys % z.pitch), ky = (int)(sys / z.pitch);
    if (kx >= z.mx || ky >= z.my) return;

    Coef co;
    co.am = z.am; co.ap = z.ap;
    co.lx = z.lamx[kx];
    co.ly = z.lamy[ky];
    co.pin = (kx == 0 && ky == 0);
    if (MODE != 0) {
        const bool low = (co.lx + co.ly) * __ldg(z.dzmin2) < z.lowk;
        if ((MODE == 1) == low) return;
    }
    double zsum = 0.0;
    bool bad = false;
    double* ck = z.ckpt + sys;
    if (CYC) thomas_poisson_cyc<T, A, CPLX>(data, sys, z.plane, z.nz, co, z.scale, ck, zsum, bad);
    else     thomas_poisson<T, A, CPLX>(data, sys, z.plane, z.nz, co, z.scale, ck, zsum, bad);
    if (co.pin && z.dc_shift) *z.dc_shift = zsum / (double)z.nz;
    if (bad && err) atomicOr(err, 1);
}

long tdma_z_ckpt_doubles(int nz, long plane, int cyclic, bool fp32)
{
    const int m = cyclic ? nz - 1 : nz;
    const int ch = Exact::CH < Fast::CH ? Exact::CH : Fast::CH;   // the finer chunking of the two paths
    const long nch = (m + ch - 1) / ch;
    const long dbl = nch * (cyclic ? 4 : 3) * plane;
    // FP32 storage: FP32 checkpoints of the bulk kernel follow the FP64 ones,
    // then the low-|k| list (at most plane system indices)
    return fp32 ? dbl + (dbl + 1) / 2 + (plane + 2) / 2 + 1 : dbl;
}

float* tdma_z_ckpt_f32(double* ckpt, int nz, long plane, int cyclic)
{
    return reinterpret_cast<float*>(ckpt + tdma_z_ckpt_doubles(nz, plane, cyclic, false));
}

int* tdma_z_lowk_list(double* ckpt, int nz, long plane, int cyclic)
{
    const long dbl = tdma_z_ckpt_doubles(nz, plane, cyclic, false);
    return reinterpret_cast<int*>(ckpt + dbl + (dbl + 1) / 2);
}

namespace {
// One chunk of C rows from z0 of the FP32 bulk sweep: the forward
// elimination from the state (cp, dr, di) ending the previous chunk, c' and
// d' of every row kept in cs, vr, vi (vr, vi enter as the right-hand
// sides).  zlev[k] = (am, ap, -am - ap) of level k; rows from nz on are
// skipped.
template <bool CPLX, int C>
__device__ __forceinline__ void fast_chunk_elim(const float4* zlev, float lamf, int nz, int z0, float* vr, float* vi,
                                                float* cs, float& cp, float& dr, float& di)
{
    if (z0 == 0) {
        const float4 l0 = zlev[0];
        fwd_row<Fast, CPLX>(true, l0.x, l0.z - lamf, l0.y, vr[0], vi[0], cp, dr, di);
        cs[0] = cp; vr[0] = dr; vi[0] = di;
#pragma unroll
        for (int q = 1; q < C; ++q) {
            if (q < nz) {
                const float4 lv = zlev[q];
                fwd_row<Fast, CPLX>(false, lv.x, lv.z - lamf, lv.y, vr[q], vi[q], cp, dr, di);
            }
            cs[q] = cp; vr[q] = dr; vi[q] = di;
        }
    } else if (z0 + C <= nz) {
#pragma unroll
        for (int q = 0; q < C; ++q) {
            const float4 lv = zlev[z0 + q];
            fwd_row<Fast, CPLX>(false, lv.x, lv.z - lamf, lv.y, vr[q], vi[q], cp, dr, di);
            cs[q] = cp; vr[q] = dr; vi[q] = di;
        }
    } else {
#pragma unroll
        for (int q = 0; q < C; ++q) {
            if (z0 + q < nz) {
                const float4 lv = zlev[z0 + q];
                fwd_row<Fast, CPLX>(false, lv.x, lv.z - lamf, lv.y, vr[q], vi[q], cp, dr, di);
            }
            cs[q] = cp; vr[q] = dr; vi[q] = di;
        }
    }
}

// The back substitution of that chunk, top row first, from x of the row
// above (xr, xi); each solution row is scaled and stored at col + row * pl,
// and added to fsum (the non-finite check).
template <bool CPLX, int C, typename E>
__device__ __forceinline__ void fast_chunk_subst(E* col, unsigned pl, int nz, int z0, const float* vr,
                                                 const float* vi, const float* cs, float sc, float& xr, float& xi,
                                                 float& fsum)
{
    auto put = [&](int q) {
        xr = vr[q] - cs[q] * xr;
        if (CPLX) xi = vi[q] - cs[q] * xi;
        fsum += xr + xi;
        E* o = col + (size_t)(unsigned)(z0 + q) * pl;
        if constexpr (CPLX) *o = mk<float>(xr * sc, xi * sc);
        else *o = xr * sc;
    };
    if (z0 + C <= nz) {
#pragma unroll
        for (int q = C - 1; q >= 0; --q) put(q);
    } else {
#pragma unroll
        for (int q = C - 1; q >= 0; --q)
            if (z0 + q < nz) put(q);
    }
}

// FP32 bulk of the mixed-precision z solve (systems with lam dz_min^2 >=
// lowk, non-periodic z).  The same Thomas sweep as thomas_poisson<Fast>,
// with the level coefficients (am, ap, -am-ap) staged once per CTA in shared
// memory (b = -am-ap - lam, a single rounding more than the FP64 order,
// which the refinement absorbs) and FP32 checkpoints in their own region.
// Kept lean because the kernel is close to issue-bound: the next chunk's
// rows (and, backward, the next checkpoint) are loaded while the current
// chunk is eliminated; full chunks run without per-row bounds tests, the
// first row is peeled; row addresses are 32-bit row x plane products on the
// column pointer; the back substitution starts from x = 0 above the top row
// (x_top = d'_top - c'_top * 0 = d'_top exactly), and non-finite results
// are detected once, on a running sum of the outputs.
template <bool CPLX>
__global__ void __launch_bounds__(TPB, CPLX ? 7 : 6) k_thomas_fast(void* __restrict__ data_, ZSys z, const int* __restrict__ skip,
                                                     int* __restrict__ err)
{
    if (skip && *skip) return;
    extern __shared__ float4 zlev[];
    for (int k = threadIdx.x; k < z.nz; k += TPB) {
        const double am = z.am[k], ap = z.ap[k];
        zlev[k] = make_float4((float)am, (float)ap, (float)(-am - ap), 0.f);
    }
    __syncthreads();
    using E = typename Elem<float, CPLX>::type;
    const long sys = (long)blockIdx.x * TPB + threadIdx.x;
    const int kx = (int)(sys % z.pitch), ky = (int)(sys / z.pitch);
    if (kx >= z.mx || ky >= z.my) return;
    const double lam = z.lamx[kx] + z.lamy[ky];
    if (lam * __ldg(z.dzmin2) < z.lowk) return;  // solved in FP64 (includes the pinned zero mode)
    const float lamf = (float)lam, sc = (float)z.scale;
    const int nz = z.nz;
    const unsigned pl = (unsigned)z.plane;
    constexpr int C = Fast::CH;
    const int nch = (nz + C - 1) / C;
    E* col = reinterpret_cast<E*>(data_) + sys;
    const float* ckr = z.ckpt_f + sys;
    float* ckw = z.ckpt_f + sys;
    auto row = [&](int zr) { return col + (size_t)(unsigned)zr * pl; };
    float nr[C], ni[C];
    auto load = [&](int z0) {
        if (z0 + C <= nz) {
#pragma unroll
            for (int q = 0; q < C; ++q) ld_cv<float, float>(row(z0 + q), nr[q], ni[q]);
        } else {
#pragma unroll
            for (int q = 0; q < C; ++q) {
                nr[q] = 0.f;
                ni[q] = 0.f;
                if (z0 + q < nz) ld_cv<float, float>(row(z0 + q), nr[q], ni[q]);
            }
        }
    };
    load(0);
    float cp = 0.f, dr = 0.f, di = 0.f;
    for (int ch = 0; ch < nch; ++ch) {
        float vr[C], vi[C], cs[C];
#pragma unroll
        for (int q = 0; q < C; ++q) { vr[q] = nr[q]; vi[q] = ni[q]; }
        if (ch + 1 < nch) load((ch + 1) * C);
        fast_chunk_elim<CPLX, C>(zlev, lamf, nz, ch * C, vr, vi, cs, cp, dr, di);
        float* c3 = ckw + (size_t)(unsigned)(3 * ch) * pl;
        c3[0] = cp;
        c3[pl] = dr;
        if (CPLX) c3[(size_t)2 * pl] = di;
    }
    float xr = 0.f, xi = 0.f, fsum = 0.f;
    load((nch - 1) * C);
    float kc = 0.f, kr = 0.f, ki = 0.f;           // checkpoint ending chunk ch - 1
    if (nch > 1) {
        const float* c3 = ckr + (size_t)(unsigned)(3 * (nch - 2)) * pl;
        kc = c3[0];
        kr = c3[pl];
        if (CPLX) ki = c3[(size_t)2 * pl];
    }
    for (int ch = nch - 1; ch >= 0; --ch) {
        float vr[C], vi[C], cs[C];
#pragma unroll
        for (int q = 0; q < C; ++q) { vr[q] = nr[q]; vi[q] = ni[q]; }
        float pcp = kc, pdr = kr, pdi = ki;
        if (ch > 0) {
            load((ch - 1) * C);
            if (ch > 1) {
                const float* c3 = ckr + (size_t)(unsigned)(3 * (ch - 2)) * pl;
                kc = c3[0];
                kr = c3[pl];
                if (CPLX) ki = c3[(size_t)2 * pl];
            } else {
                kc = 0.f; kr = 0.f; ki = 0.f;
            }
        }
        fast_chunk_elim<CPLX, C>(zlev, lamf, nz, ch * C, vr, vi, cs, pcp, pdr, pdi);
        fast_chunk_subst<CPLX, C>(col, pl, nz, ch * C, vr, vi, cs, sc, xr, xi, fsum);
    }
    if (!isfinite(fsum) && err) atomicOr(err, 1);
}

// The FP32 bulk sweep with the field streamed through shared memory.  One
// persistent CTA per SM walks blocks of W consecutive FP32 values of a z
// row; each value's column is one tridiagonal system (the real and the
// imaginary part of a complex system are two columns with the same
// coefficients).  Each column is solved by a twisted factorisation with two
// threads: one eliminates the lower half top-down (Thomas: r = 1/(b - a c'),
// c' = r c, d' = r (d - a d')), the other the upper half bottom-up
// (r = 1/(b - c a''), a'' = r a, d'' = r (d - c d'')), the two halves meet
// in a 2 x 2 solve for the middle rows, and each thread then substitutes
// outwards through its half (x = d' - c' x_above, x = d'' - a'' x_below).
// Rows arrive as TMA boxes (R rows x W values, one box of each half per
// step) through a ring of `stages` buffers, several steps ahead; the
// elimination keeps chunk checkpoints in shared memory and the
// substitution loads its chunks again and recomputes their c', d' (a'', d'')
// from the checkpoints.  With one block per SM in flight, the columns
// between a first read and their re-read (SMs x W x nz values: 78 MB at 512
// levels) fit in the L2 cache, which serves the re-read (first reads with
// the evict_last priority, re-reads with evict_first), so each value
// crosses the HBM interface once each way.  The FFT normalisation is folded
// into the staged coefficients (A/s solves for s x) and the reciprocals are
// the approximate ones: the FP64 refinement absorbs this path's rounding.
__device__ __forceinline__ float rcp_approx(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

struct ZStream {
    static constexpr int W = 256;        // columns per block and box row (a TMA box holds at most 256)
    static constexpr int NC = 2 * W;     // consumer threads: lower half, upper half of each column
    static constexpr int NT = NC + 32;   // + the producer warp
    static constexpr int R = 16;         // rows per box and checkpoint chunk
    static constexpr int MAX_STAGES = 8;
    static constexpr unsigned BOX = (unsigned)(R * W * sizeof(float));
    static constexpr unsigned STAGE = 2 * BOX;   // one box of each half
    static __host__ __device__ int nch(int nz) { return (nz + R - 1) / R; }
    static __host__ __device__ size_t ck_bytes(int nz) { return (size_t)nch(nz) * 2 * W * sizeof(float); }
    // + the middle exchange, 4 values per column, for two blocks
    static size_t smem(int nz, int stages)
    {
        return 128 + (size_t)stages * STAGE + ck_bytes(nz) + sizeof(float4) * (size_t)nz + 8 * W * sizeof(float);
    }
};
// Bound of a wait for one step's boxes: polls that each sleep up to
// ZS_POLL_NS while the boxes are in flight (about 2 s in all): far above any
// load time, so it only ends a kernel whose copies never complete, with err
// bit 2 set.
constexpr unsigned ZS_POLL_NS = 20000;
constexpr long ZS_WAIT_LIMIT = 100000;

// The level coefficients are staged over the FFT normalisation n:
// zlev[k] = (am_k, ap_k, -am_k - ap_k) / n, and lam / n with them, so the
// sweeps solve (A / n) y = rhs for y = n x.

// Rows z0 .. z0+R-1 of the lower half, eliminated top-down from the state
// (e, d) = (c', d') of the row below z0 (r = 1/(b - a e), c' = r c,
// d' = r (d - a d')); the sweep starts from (0, 0), for which the general
// step is the first row's.  KEEP: c', d' of every row into g, v (v enters
// as the right-hand sides).
template <bool KEEP>
__device__ __forceinline__ void zs_down(const float4* zlev, float lam, int z0, float* v, float* g, float& e, float& d)
{
#pragma unroll
    for (int q = 0; q < ZStream::R; ++q) {
        const float4 zl = zlev[z0 + q];
        const float r = rcp_approx((zl.z - lam) - zl.x * e);
        d = r * (v[q] - zl.x * d);
        e = r * zl.y;
        if (KEEP) { g[q] = e; v[q] = d; }
    }
}
// Rows z0+R-1 .. z0 of the upper half, eliminated bottom-up from the state
// (e, d) = (a'', d'') of the row above (r = 1/(b - c e), a'' = r a,
// d'' = r (d - c d'')); TOP: the chunk holds the top row nz-1, rows from nz
// on are skipped.
template <bool TOP, bool KEEP>
__device__ __forceinline__ void zs_up(const float4* zlev, float lam, int z0, int nz, float* v, float* g, float& e,
                                      float& d)
{
#pragma unroll
    for (int q = ZStream::R - 1; q >= 0; --q) {
        if (!TOP || z0 + q < nz) {
            const float4 zl = zlev[z0 + q];
            const float r = rcp_approx((zl.z - lam) - zl.y * e);
            d = r * (v[q] - zl.y * d);
            e = r * zl.x;
        }
        if (KEEP) { g[q] = e; v[q] = d; }
    }
}

// OR of `pred` over the `n` threads of named barrier `id` (a warp-multiple
// subset of the CTA), which all wait there
__device__ __forceinline__ bool bar_or(int id, int n, bool pred)
{
    unsigned r;
    asm volatile("{\n .reg .pred p, q;\n setp.ne.u32 p, %1, 0;\n bar.red.or.pred q, %2, %3, p;\n"
                 " selp.u32 %0, 1, 0, q;\n}\n"
                 : "=r"(r)
                 : "r"((unsigned)pred), "r"(id), "r"(n)
                 : "memory");
    return r != 0;
}

// CPLX: complex systems, value u of a row is part (u & 1) of system u >> 1.
// The ring is a producer/consumer pipeline: full[b] completes when the
// boxes of the step in buffer b have landed, empty[b] when every consumer
// warp has finished reading them, and a producer warp refills each buffer
// as soon as its empty phase completes, so the loads run ahead of the
// slowest warp by the ring's depth.  The consumers meet once per block (the
// middle exchange, double-buffered by block) at a named barrier, which
// also carries the vote on a wait that gave up.
template <bool CPLX>
__global__ void __launch_bounds__(ZStream::NT, 1)
    k_thomas_stream(const __grid_constant__ CUtensorMap tmap, void* __restrict__ data_, ZSys z, int stages,
                    const int* __restrict__ skip, int* __restrict__ err)
{
    if (skip && *skip) return;
    using S = ZStream;
    constexpr int W = S::W, R = S::R, SH = CPLX ? 1 : 0, NC = S::NC;
    extern __shared__ __align__(128) unsigned char zs_raw[];
    __shared__ __align__(8) uint64_t full[S::MAX_STAGES];
    __shared__ __align__(8) uint64_t empty[S::MAX_STAGES];
    __shared__ int abort_flag;
    unsigned char* const base = reinterpret_cast<unsigned char*>(((uintptr_t)zs_raw + 127) & ~(uintptr_t)127);
    float* const ring = reinterpret_cast<float*>(base);
    const int nz = z.nz, nch = S::nch(nz);
    const int hl = nch / 2, hu = nch - hl;   // chunks of the lower and the upper half (hu >= 1)
    float* const ck = reinterpret_cast<float*>(base + (size_t)stages * S::STAGE);
    float4* const zlev = reinterpret_cast<float4*>(base + (size_t)stages * S::STAGE + S::ck_bytes(nz));
    float* const xch = reinterpret_cast<float*>(zlev + nz);
    const int tid = threadIdx.x, lane = tid & 31;
    const long nval = z.plane << SH;     // values per z row
    const long nblk = (nval + W - 1) / W;
    const long mine = (long)blockIdx.x < nblk ? (nblk - 1 - blockIdx.x) / gridDim.x + 1 : 0;
    const long total = mine * 2 * hu;    // steps of this CTA, in order
    volatile int* const abort_v = &abort_flag;
    if (tid == 0) {
        for (int q = 0; q < stages; ++q) {
            mbar_init(&full[q], 1);
            mbar_init(&empty[q], NC / 32);
        }
        mbar_init_fence();
        abort_flag = 0;
    }
    const double isc = 1.0 / z.scale;
    for (int k = tid; k < nz; k += S::NT) {
        const double am = z.am[k], ap = z.ap[k];
        zlev[k] = make_float4((float)(am * isc), (float)(ap * isc), (float)((-am - ap) * isc), 0.f);
    }
    __syncthreads();

    if (tid >= NC) {
        // ---- producer warp (one thread): step p of block iteration p_it is
        // elimination step j = p_pos (< hu) or substitution step j = p_pos - hu
        if (tid != NC) return;
        const uint64_t pol_keep = l2_policy_evict_last(), pol_drop = l2_policy_evict_first();
        long issued = 0, p_it = 0, p_round = 0;
        int p_pos = 0, p_buf = 0;
        bool ok = true;
        while (issued < total) {
            if (p_round > 0) {   // the buffer's previous step has been read by every consumer warp
                ok = false;
                for (long q = 0; q < ZS_WAIT_LIMIT && !ok; ++q) {
                    ok = mbar_try_wait_sleep(&empty[p_buf], (unsigned)((p_round - 1) & 1), ZS_POLL_NS);
                    if (!ok && *abort_v) break;
                }
                if (!ok) break;
            }
            const bool elim = p_pos < hu;
            const int j = elim ? p_pos : p_pos - hu;
            const int cl = elim ? j : hl - 1 - j;            // lower chunk (if j < hl)
            const int cu = elim ? nch - 1 - j : hl + j;      // upper chunk
            const bool has_l = j < hl;
            const long blk = blockIdx.x + p_it * gridDim.x;
            float* dst = ring + (size_t)p_buf * 2 * R * W;
            const uint64_t pol = elim ? pol_keep : pol_drop;
            fence_proxy_async_smem();   // the consumers' reads of the buffer come before its refill
            mbar_arrive_expect_tx(&full[p_buf], has_l ? S::STAGE : S::BOX);
            if (has_l) tma_load_2d(dst, &tmap, (int)(blk * W), cl * R, &full[p_buf], pol);
            tma_load_2d(dst + R * W, &tmap, (int)(blk * W), cu * R, &full[p_buf], pol);
            ++issued;
            if (++p_pos == 2 * hu) { p_pos = 0; ++p_it; }
            if (++p_buf == stages) { p_buf = 0; ++p_round; }
        }
        if (!ok) {
            *abort_v = 1;
            if (err) atomicOr(err, 2);
        }
        // the last load into every buffer has landed before the CTA's shared
        // memory can be released
        for (int b = 0; b < stages; ++b) {
            const long nb = issued > b ? (issued - 1 - b) / stages + 1 : 0;   // loads into buffer b
            if (nb > 0) mbar_wait_sleep_bounded(&full[b], (unsigned)((nb - 1) & 1), ZS_POLL_NS, ZS_WAIT_LIMIT);
        }
        return;
    }

    // ---- consumers
    const bool upper = tid >= W;
    const int col_i = upper ? tid - W : tid;
    const double dzmin2 = __ldg(z.dzmin2);
    int c_buf = 0;
    unsigned c_par = 0;
    // the boxes of the next step have landed; false: a wait gave up, here
    // or elsewhere (the abort flag)
    auto ready = [&]() -> bool {
        for (long q = 0; q < ZS_WAIT_LIMIT; ++q) {
            if (mbar_try_wait_sleep(&full[c_buf], c_par, ZS_POLL_NS)) return true;
            if (*abort_v) return false;
        }
        *abort_v = 1;
        if (err) atomicOr(err, 2);
        return false;
    };
    // this warp is done with the boxes of the step
    auto release = [&]() {
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[c_buf]);
        if (++c_buf == stages) { c_buf = 0; c_par ^= 1u; }
    };
    const unsigned pl = (unsigned)nval;
    float fsum = 0.f;
    bool failed = false;
    for (long i = 0; i < mine; ++i) {
        const long u = (blockIdx.x + i * gridDim.x) * W + col_i;
        const long sys = u >> SH;
        const int kx = (int)(sys % z.pitch), ky = (int)(sys / z.pitch);
        bool act = u < nval && kx < z.mx && ky < z.my;
        float lam = 0.f;
        if (act) {
            const double l = z.lamx[kx] + z.lamy[ky];
            act = !(l * dzmin2 < z.lowk);   // else solved in FP64 (the pinned zero mode among them)
            lam = (float)(l * isc);
        }
        // ---- elimination: the lower half top-down over chunks 0 .. hl-1,
        // the upper half bottom-up over chunks nch-1 .. hl
        float e = 0.f, d = 0.f;   // lower: c', d'; upper: a'', d''
        for (int j = 0; j < hu && !failed; ++j) {
            if (!ready()) { failed = true; break; }
            if (act && (upper || j < hl)) {
                const float* t = ring + (size_t)c_buf * 2 * R * W + (upper ? R * W : 0) + col_i;
                float v[R];
#pragma unroll
                for (int q = 0; q < R; ++q) v[q] = t[q * W];
                float* k2;
                if (!upper) {
                    zs_down<false>(zlev, lam, j * R, v, nullptr, e, d);   // lower chunks are full
                    k2 = ck + (size_t)j * 2 * W + col_i;
                } else {
                    const int c = nch - 1 - j;
                    if (j == 0) zs_up<true, false>(zlev, lam, c * R, nz, v, nullptr, e, d);
                    else zs_up<false, false>(zlev, lam, c * R, nz, v, nullptr, e, d);
                    k2 = ck + (size_t)c * 2 * W + col_i;
                }
                k2[0] = e;
                k2[W] = d;
            }
            release();
        }
        // ---- the middle rows m-1 (lower) and m (upper): x_{m-1} + c' x_m = d',
        // a'' x_{m-1} + x_m = d''
        float* const xb = xch + (i & 1) * 4 * W;
        if (upper) { xb[2 * W + col_i] = e; xb[3 * W + col_i] = d; }
        else { xb[col_i] = e; xb[W + col_i] = d; }
        if (bar_or(1, NC, failed)) { failed = true; break; }
        float x = 0.f;   // lower: x of the row above; upper: x of the row below
        {
            const float cl = hl ? xb[col_i] : 0.f, dl = hl ? xb[W + col_i] : 0.f;
            const float au = xb[2 * W + col_i], du = xb[3 * W + col_i];
            const float xm = (du - au * dl) / (1.f - au * cl);
            x = upper ? dl - cl * xm : xm;
        }
        // ---- substitution: the lower half chunks hl-1 .. 0, the upper half
        // chunks hl .. nch-1, each recomputed from its checkpoint
        float* colp = reinterpret_cast<float*>(data_) + u;
        for (int j = 0; j < hu && !failed; ++j) {
            if (!ready()) { failed = true; break; }
            if (act && (upper || j < hl)) {
                const float* t = ring + (size_t)c_buf * 2 * R * W + (upper ? R * W : 0) + col_i;
                float v[R], g[R];
#pragma unroll
                for (int q = 0; q < R; ++q) v[q] = t[q * W];
                if (!upper) {
                    const int c = hl - 1 - j, z0 = c * R;
                    float ee = 0.f, dd = 0.f;
                    if (c > 0) { const float* k2 = ck + (size_t)(c - 1) * 2 * W + col_i; ee = k2[0]; dd = k2[W]; }
                    zs_down<true>(zlev, lam, z0, v, g, ee, dd);
                    float* o = colp + (size_t)(unsigned)(z0 + R - 1) * pl;
#pragma unroll
                    for (int q = R - 1; q >= 0; --q) {
                        x = v[q] - g[q] * x;
                        *o = x;
                        o -= pl;
                    }
                } else {
                    const int c = hl + j, z0 = c * R;
                    float ee = 0.f, dd = 0.f;
                    float* o = colp + (size_t)(unsigned)z0 * pl;
                    if (c < nch - 1) {
                        const float* k2 = ck + (size_t)(c + 1) * 2 * W + col_i;
                        ee = k2[0];
                        dd = k2[W];
                        zs_up<false, true>(zlev, lam, z0, nz, v, g, ee, dd);
#pragma unroll
                        for (int q = 0; q < R; ++q) {
                            x = v[q] - g[q] * x;
                            *o = x;
                            o += pl;
                        }
                    } else {
                        zs_up<true, true>(zlev, lam, z0, nz, v, g, ee, dd);
#pragma unroll
                        for (int q = 0; q < R; ++q) {
                            if (z0 + q < nz) {
                                x = v[q] - g[q] * x;
                                *o = x;
                                o += pl;
                            }
                        }
                    }
                }
                fsum += x;
            }
            release();
        }
    }
    // every consumer arrives here: the loop's named barrier is taken by all
    // of them or left by all together
    if (bar_or(1, NC, failed)) {
        *abort_v = 1;   // the producer stops issuing and waits for its loads
        return;
    }
    if (!isfinite(fsum) && err) atomicOr(err, 1);
}

// The streamed bulk kernel where it applies (non-periodic z, a field whose
// rows the tensor map can describe, shared memory for at least three
// boxes); *used false: the caller takes k_thomas_fast.
template <bool CPLX>
cudaError_t launch_stream(void* data, const ZSys& z, const int* skip, int* err, cudaStream_t st, bool* used)
{
    using S = ZStream;
    constexpr int EC = CPLX ? 2 : 1;
    *used = false;
    if (z.cyclic || z.shared_gpu || (uintptr_t)data % 16 || (z.plane * EC * sizeof(float)) % 16 ||
        z.plane * EC >= (1L << 31))
        return cudaSuccess;
    int dev = 0, sms = 0, optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    const size_t fixed = S::smem(z.nz, 0) + 2 * sizeof(uint64_t) * S::MAX_STAGES + 16;
    if ((size_t)optin <= fixed) return cudaSuccess;
    long stages = (long)(((size_t)optin - fixed) / S::STAGE);
    if (stages > 6) stages = 6;
    if (stages < 3) return cudaSuccess;
    CUtensorMap map;
    if (!tma_map_2d_f32(&map, data, (unsigned long long)z.plane * EC, (unsigned long long)z.nz,
                        (unsigned long long)z.plane * EC * sizeof(float), (unsigned)S::W, (unsigned)S::R))
        return cudaSuccess;
    const size_t smem = S::smem(z.nz, (int)stages);
    e = cudaFuncSetAttribute(k_thomas_stream<CPLX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    // a plane of fewer blocks than SMs leaves most SMs idle behind a few long
    // chains and fences the others off from concurrent work (batched
    // problems) with its shared memory: the one-thread-per-system kernel
    // serves it better
    const long nblk = (z.plane * EC + S::W - 1) / S::W;
    if (nblk < sms) return cudaSuccess;
    const long grid = sms;
    k_thomas_stream<CPLX><<<(unsigned)grid, S::NT, smem, st>>>(map, data, z, (int)stages, skip, err);
    *used = true;
    return cudaGetLastError();
}

// FP64 z solve of all systems (non-periodic z): thomas_poisson<Exact> with
// the level coefficients staged once per CTA in shared memory (the same
// rounded operations: b = ((-am - ap) - lx) - ly with -am - ap kept per
// level) and, with PREF, the next chunk's rows loaded while the current one
// is eliminated.
template <bool CPLX, bool PREF>
__global__ void __launch_bounds__(TPB) k_thomas_exact(void* __restrict__ data_, ZSys z, const int* __restrict__ skip,
                                                      int* __restrict__ err)
{
    if (skip && *skip) return;
    extern __shared__ double zl[];     // am[nz], ap[nz], s[nz] = -am - ap
    const int nz = z.nz;
    for (int k = threadIdx.x; k < nz; k += TPB) {
        const double am = z.am[k], ap = z.ap[k];
        zl[k] = am;
        zl[nz + k] = ap;
        zl[2 * nz + k] = __dsub_rn(-am, ap);
    }
    __syncthreads();
    using E = typename Elem<double, CPLX>::type;
    using X = Exact;
    const long sys = (long)blockIdx.x * TPB + threadIdx.x;
    const int kx = (int)(sys % z.pitch), ky = (int)(sys / z.pitch);
    if (kx >= z.mx || ky >= z.my) return;
    const double lx = z.lamx[kx], ly = z.lamy[ky];
    const bool pin = (kx == 0 && ky == 0);
    const long plane = z.plane;
    constexpr int C = Exact::CH;
    const int nch = (nz + C - 1) / C;
    E* col = reinterpret_cast<E*>(data_) + sys;
    double* ck = z.ckpt + sys;
    auto coef = [&](int zr, double& a, double& b, double& c) {
        if (pin && zr == 0) { a = 0.0; b = 1.0; c = 0.0; return; }
        a = zl[zr];
        c = zl[nz + zr];
        b = X::sub(X::sub(zl[2 * nz + zr], lx), ly);
    };
    double nr[C], ni[C];
    auto load = [&](int z0) {
#pragma unroll
        for (int q = 0; q < C; ++q) {
            nr[q] = 0.0; ni[q] = 0.0;
            if (z0 + q < nz) ld_cv<double, double>(col + (long)(z0 + q) * plane, nr[q], ni[q]);
        }
    };
    if (PREF) load(0);
    double cp = 0, dr = 0, di = 0;
    for (int ch = 0; ch < nch; ++ch) {
        const int z0 = ch * C;
        double vr[C], vi[C];
        if (PREF) {
#pragma unroll
            for (int q = 0; q < C; ++q) { vr[q] = nr[q]; vi[q] = ni[q]; }
            if (ch + 1 < nch) load((ch + 1) * C);
        } else {
            load(z0);
#pragma unroll
            for (int q = 0; q < C; ++q) { vr[q] = nr[q]; vi[q] = ni[q]; }
        }
#pragma unroll
        for (int q = 0; q < C; ++q) {
            const int zr = z0 + q;
            if (zr < nz) {
                double a, b, c;
                coef(zr, a, b, c);
                const bool pr = pin && zr == 0;
                fwd_row<Exact, CPLX>(zr == 0, a, b, c, pr ? 0.0 : vr[q], pr ? 0.0 : vi[q], cp, dr, di);
            }
        }
        double* c3 = ck + (long)(3 * ch) * plane;
        c3[0] = cp;
        c3[plane] = dr;
        if (CPLX) c3[2 * plane] = di;
    }
    double xr = 0, xi = 0, zsum = 0.0;
    bool bad = false;
    if (PREF) load((nch - 1) * C);
    for (int ch = nch - 1; ch >= 0; --ch) {
        const int z0 = ch * C;
        double vr[C], vi[C], c_[C];
        double pcp = 0, pdr = 0, pdi = 0;
        if (PREF) {
#pragma unroll
            for (int q = 0; q < C; ++q) { vr[q] = nr[q]; vi[q] = ni[q]; }
        } else {
            load(z0);
#pragma unroll
            for (int q = 0; q < C; ++q) { vr[q] = nr[q]; vi[q] = ni[q]; }
        }
        if (ch > 0) {
            const double* c3 = ck + (long)(3 * (ch - 1)) * plane;
            pcp = c3[0];
            pdr = c3[plane];
            if (CPLX) pdi = c3[2 * plane];
            if (PREF) load((ch - 1) * C);
        }
#pragma unroll
        for (int q = 0; q < C; ++q) {
            const int zr = z0 + q;
            if (zr < nz) {
                double a, b, c;
                coef(zr, a, b, c);
                const bool pr = pin && zr == 0;
                fwd_row<Exact, CPLX>(zr == 0, a, b, c, pr ? 0.0 : vr[q], pr ? 0.0 : vi[q], pcp, pdr, pdi);
            }
            c_[q] = pcp; vr[q] = pdr; vi[q] = pdi;
        }
#pragma unroll
        for (int q = C - 1; q >= 0; --q) {
            const int zr = z0 + q;
            if (zr < nz) {
                if (zr == nz - 1) {
                    xr = vr[q];
                    xi = vi[q];
                } else {
                    xr = X::sub(vr[q], X::mul(c_[q], xr));
                    if (CPLX) xi = X::sub(vi[q], X::mul(c_[q], xi));
                }
                const double sr = xr * z.scale, si = xi * z.scale;
                zsum += sr;
                if (!isfinite(sr) || !isfinite(si)) bad = true;
                st_elem<double>(col + (long)zr * plane, sr, si);
            }
        }
    }
    if (pin && z.dc_shift) *z.dc_shift = zsum / (double)nz;
    if (bad && err) atomicOr(err, 1);
}

// Low-|k| systems of the mixed-precision z solve (lam * dz_min^2 < lowk, the
// complement of k_thomas_fast's set): one thread per system, a warp ballot
// and one atomic per warp append them to the list.  The order of the list
// does not matter for the results (every system is solved on its own), so
// no scan is needed.  Runs once per solve, after the z-coefficient kernel
// (dz_min) and with the count zeroed.
__global__ void __launch_bounds__(256) k_lowk_list(ZSys z)
{
    const long s = (long)blockIdx.x * 256 + threadIdx.x;
    bool low = false;
    if (s < z.plane) {
        const int kx = (int)s % (int)z.pitch, ky = (int)s / (int)z.pitch;
        low = kx < z.mx && ky < z.my && (z.lamx[kx] + z.lamy[ky]) * __ldg(z.dzmin2) < z.lowk;
    }
    const unsigned m = __ballot_sync(0xffffffffu, low);
    if (!m) return;
    const int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == 0) base = atomicAdd(z.lowk_count, __popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (low) z.lowk_list[base + __popc(m & ((1u << lane) - 1))] = (int)s;
}

// the list exists for FP32 storage with non-periodic z and 32-bit indices
bool lowk_listed(const ZSys& z)
{
    return z.lowk_list && z.lowk_count && !z.cyclic && z.lowk > 0.0 && z.plane < (1L << 30);
}

constexpr int LK_NS = 8;   // ring slots of the low-|k| kernel, Exact::CH rows each

template <bool CPLX>
size_t lowk_smem(int nz)
{
    const size_t nch = (size_t)(nz + Exact::CH - 1) / Exact::CH;
    return sizeof(double) * (3 * (size_t)nz + 96 * nch + 96 * Exact::CH) +
           (sizeof(typename Elem<float, CPLX>::type) + sizeof(double)) * LK_NS * Exact::CH * 32;
}

// the level coefficients am, ap, -am - ap of the z operator into shared memory
__device__ __forceinline__ void stage_levels(const ZSys& z, double* zl)
{
    const int nz = z.nz;
    for (int k = threadIdx.x; k < nz; k += blockDim.x) {
        const double am = z.am[k], ap = z.ap[k];
        zl[k] = am;
        zl[nz + k] = ap;
        zl[2 * nz + k] = __dsub_rn(-am, ap);
    }
}

// The coefficient half of the low-|k| Thomas sweep, which does not depend on
// the right-hand side: c'_1 = c_1 / b_1 and, below the first row,
// r_k = 1 / (b_k - a_k c'_{k-1}), c'_k = r_k c_k, with thomas_poisson<Exact>'s
// operations.  Table entry k of a system holds r_k (c'_1 for the first row),
// [group][row][lane], for the groups of 32 listed systems that fit in `cap`
// doubles.  Once per solve: every pass of the solve has the same operator.
__global__ void __launch_bounds__(32) k_lowk_table(ZSys z, const int* __restrict__ skip)
{
    if (skip && *skip) return;
    using X = Exact;
    extern __shared__ double zl[];
    stage_levels(z, zl);
    __syncwarp();
    const int nz = z.nz, lane = threadIdx.x;
    const int count = *z.lowk_count;
    for (int g = blockIdx.x; g * 32 < count && (long)(g + 1) * 32 * nz <= z.lowk_cap; g += gridDim.x) {
        const int idx = g * 32 + lane;
        if (idx >= count) continue;
        const int sys = z.lowk_list[idx];
        const int kx = sys % (int)z.pitch, ky = sys / (int)z.pitch;
        const double lx = z.lamx[kx], ly = z.lamy[ky];
        const bool pin = (kx == 0 && ky == 0);
        double* tab = z.lowk_tab + (size_t)g * nz * 32 + lane;
        double cp = pin ? X::div(0.0, 1.0) : X::div(zl[nz], X::sub(X::sub(zl[2 * nz], lx), ly));
        tab[0] = cp;
#pragma unroll 4
        for (int zr = 1; zr < nz; ++zr) {
            const double b = X::sub(X::sub(zl[2 * nz + zr], lx), ly);
            const double r = X::rcp(X::sub(b, X::mul(zl[zr], cp)));
            cp = X::mul(r, zl[nz + zr]);
            tab[(size_t)zr * 32] = r;
        }
    }
}

// One group of 32 listed systems (one per lane) of k_thomas_lowk.  TAB: r_k
// and c'_1 come from the k_lowk_table entries, streamed through the ring
// beside the rows, so the sweeps are multiply-subtract chains; otherwise the
// reciprocals are formed here.  Either way the operations and their order
// are thomas_poisson<float, Exact>'s.
template <bool CPLX, bool TAB>
__device__ __forceinline__ void lowk_group(void* data_, const ZSys& z, int g, int sys, const double* zl, double* ckp,
                                           double* scr, typename Elem<float, CPLX>::type* ring, double* rring,
                                           int* err)
{
    using E = typename Elem<float, CPLX>::type;
    using X = Exact;
    constexpr int C = Exact::CH;
    const int nz = z.nz, nch = (nz + C - 1) / C, lane = threadIdx.x;
    const long plane = z.plane;
    const int kx = sys % (int)z.pitch, ky = sys / (int)z.pitch;
    const double lx = z.lamx[kx], ly = z.lamy[ky];
    const bool pin = (kx == 0 && ky == 0);
    E* col = reinterpret_cast<E*>(data_) + sys;
    const double* tab = TAB ? z.lowk_tab + (size_t)g * nz * 32 + lane : nullptr;
    // chunk ch into its slot; one commit group per call, empty out of range
    auto issue = [&](int ch) {
        if (ch >= 0 && ch < nch) {
            const size_t so = (size_t)(ch % LK_NS) * C * 32 + lane;
            const int nq = min(C, nz - ch * C);
            for (int q = 0; q < nq; ++q) {
                cp_async_elem(ring + so + q * 32, col + (long)(ch * C + q) * plane);
                if (TAB) cp_async_f64(rring + so + q * 32, tab + (size_t)(ch * C + q) * 32);
            }
        }
        cp_async_commit();
    };
    const double b0 = pin ? 1.0 : X::sub(X::sub(zl[2 * nz], lx), ly);
    // the first row: d'_1 = d_1 / b_1 (pinned: a, b, c, d = 0, 1, 0, 0)
    auto first = [&](const E* v, const double* rv, double& cp, double& dr, double& di) {
        double vr, vi;
        ld_cv<float, double>(v, vr, vi);
        if (pin) { vr = 0.0; vi = 0.0; }
        if (TAB) {
            dr = X::div(vr, b0);
            if (CPLX) di = X::div(vi, b0);
            cp = *rv;
        } else {
            fwd_row<Exact, CPLX>(true, 0.0, b0, pin ? 0.0 : zl[nz], vr, vi, cp, dr, di);
        }
    };
    // a row below the first, b = ((-am - ap) - lx) - ly
    auto step = [&](int zr, const E* v, const double* rv, double& cp, double& dr, double& di) {
        double vr, vi;
        ld_cv<float, double>(v, vr, vi);
        const double a = zl[zr];
        if (TAB) {
            const double r = *rv;
            dr = X::mul(r, X::sub(vr, X::mul(a, dr)));
            if (CPLX) di = X::mul(r, X::sub(vi, X::mul(a, di)));
            cp = X::mul(r, zl[nz + zr]);
        } else {
            const double b = X::sub(X::sub(zl[2 * nz + zr], lx), ly);
            fwd_row<Exact, CPLX>(false, a, b, zl[nz + zr], vr, vi, cp, dr, di);
        }
    };
    for (int c = 0; c < LK_NS - 1; ++c) issue(c);
    double cp = 0, dr = 0, di = 0;
    for (int ch = 0; ch < nch; ++ch) {
        cp_async_wait<LK_NS - 2>();          // chunk ch has landed
        issue(ch + LK_NS - 1);               // into the slot chunk ch - 1 left
        const size_t so = (size_t)(ch % LK_NS) * C * 32 + lane;
        const int z0 = ch * C, nq = min(C, nz - z0);
        if (TAB && ch > 0 && nq == C) {
            // a full chunk: the rows and table entries into registers, then
            // the chain (multiply, subtract, multiply per row)
            double vr[C], vi[C], rr[C];
#pragma unroll
            for (int q = 0; q < C; ++q) {
                ld_cv<float, double>(ring + so + q * 32, vr[q], vi[q]);
                rr[q] = rring[so + q * 32];
            }
#pragma unroll
            for (int q = 0; q < C; ++q) {
                const double a = zl[z0 + q];
                dr = X::mul(rr[q], X::sub(vr[q], X::mul(a, dr)));
                if (CPLX) di = X::mul(rr[q], X::sub(vi[q], X::mul(a, di)));
            }
        } else {
            int q = 0;
            if (ch == 0) { first(ring + so, rring + so, cp, dr, di); q = 1; }
#pragma unroll 1
            for (; q < nq; ++q) step(z0 + q, ring + so + q * 32, rring + so + q * 32, cp, dr, di);
        }
        double* c3 = ckp + (size_t)ch * 96 + lane;
        c3[0] = cp;
        c3[32] = dr;
        c3[64] = di;
    }
    double xr = 0, xi = 0, zsum = 0.0;
    bool bad = false;
    for (int ch = nch - 1; ch >= 0; --ch) {
        cp_async_wait<LK_NS - 1>();          // the top LK_NS chunks are resident since the forward sweep
        const size_t so = (size_t)(ch % LK_NS) * C * 32 + lane;
        const int z0 = ch * C, nq = min(C, nz - z0);
        if (TAB && ch > 0 && nq == C) {
            // a full chunk in registers: recompute d' from the checkpoint,
            // c' = r c, then substitute
            double vr[C], vi[C], rr[C];
#pragma unroll
            for (int q = 0; q < C; ++q) {
                ld_cv<float, double>(ring + so + q * 32, vr[q], vi[q]);
                rr[q] = rring[so + q * 32];
            }
            const double* c3 = ckp + (size_t)(ch - 1) * 96 + lane;
            double pdr = c3[32], pdi = c3[64];
#pragma unroll
            for (int q = 0; q < C; ++q) {
                const double a = zl[z0 + q];
                pdr = X::mul(rr[q], X::sub(vr[q], X::mul(a, pdr)));
                if (CPLX) pdi = X::mul(rr[q], X::sub(vi[q], X::mul(a, pdi)));
                vr[q] = pdr;
                vi[q] = pdi;
                rr[q] = X::mul(rr[q], zl[nz + z0 + q]);
            }
            issue(ch - LK_NS);               // the slot just consumed
#pragma unroll
            for (int q = C - 1; q >= 0; --q) {
                const int zr = z0 + q;
                if (zr == nz - 1) {
                    xr = vr[q];
                    xi = vi[q];
                } else {
                    xr = X::sub(vr[q], X::mul(rr[q], xr));
                    if (CPLX) xi = X::sub(vi[q], X::mul(rr[q], xi));
                }
                const double sr = xr * z.scale, si = xi * z.scale;
                zsum += sr;
                if (!isfinite(sr) || !isfinite(si)) bad = true;
                st_elem<float>(col + (long)zr * plane, sr, si);
            }
            continue;
        }
        double pcp = 0, pdr = 0, pdi = 0;
        int q = 0;
        if (ch > 0) {
            const double* c3 = ckp + (size_t)(ch - 1) * 96 + lane;
            pcp = c3[0];
            pdr = c3[32];
            pdi = c3[64];
        } else {
            first(ring + so, rring + so, pcp, pdr, pdi);
            scr[lane] = pcp; scr[32 + lane] = pdr; scr[64 + lane] = pdi;
            q = 1;
        }
#pragma unroll 1
        for (; q < nq; ++q) {
            step(z0 + q, ring + so + q * 32, rring + so + q * 32, pcp, pdr, pdi);
            double* r3 = scr + q * 96 + lane;
            r3[0] = pcp; r3[32] = pdr; r3[64] = pdi;
        }
        issue(ch - LK_NS);                   // the slot just consumed
        for (q = nq - 1; q >= 0; --q) {
            const int zr = z0 + q;
            const double* r3 = scr + q * 96 + lane;
            if (zr == nz - 1) {
                xr = r3[32];
                xi = r3[64];
            } else {
                xr = X::sub(r3[32], X::mul(r3[0], xr));
                if (CPLX) xi = X::sub(r3[64], X::mul(r3[0], xi));
            }
            const double sr = xr * z.scale, si = xi * z.scale;
            zsum += sr;
            if (!isfinite(sr) || !isfinite(si)) bad = true;
            st_elem<float>(col + (long)zr * plane, sr, si);
        }
    }
    cp_async_wait<0>();
    if (pin && z.dc_shift) *z.dc_shift = zsum / (double)nz;
    if (bad && err) atomicOr(err, 1);
}

// FP64 z solve of the listed low-|k| systems with FP32 spectral storage:
// thomas_poisson<float, Exact> operation for operation (same results, bit
// for bit), organised for latency.  Persistent one-warp blocks take 32
// systems of the list at a time, one lane per system.  Every lane streams
// its column (and the group's table entries) through its own ring of LK_NS
// chunks in shared memory with cp.async, so up to LK_NS - 1 chunks of rows
// are in flight while it eliminates: the sweeps are bound by their FP64
// dependency chains, not by one HBM round trip per chunk under the
// concurrent bulk kernel's load.  The first row (the only division) is
// peeled and the row loops are not unrolled, so one warp per SM runs a short
// instruction stream.  The forward checkpoints, the level coefficients and
// the recomputed chunk of the backward sweep stay in shared memory; the
// backward sweep finds the top LK_NS chunks still in the ring and refills
// every slot it empties with the chunk LK_NS below.  A lane only reads what
// it wrote or copied itself, so no barrier is needed after the staging.
template <bool CPLX>
__global__ void __launch_bounds__(32) k_thomas_lowk(void* __restrict__ data_, ZSys z, const int* __restrict__ skip,
                                                    int* __restrict__ err)
{
    if (skip && *skip) return;
    using E = typename Elem<float, CPLX>::type;
    constexpr int C = Exact::CH;
    const int nz = z.nz, nch = (nz + C - 1) / C;
    extern __shared__ double lk[];
    double* zl = lk;                                              // am[nz], ap[nz], -am - ap[nz]
    double* ckp = zl + 3 * nz;                                    // [chunk][3][32]
    double* scr = ckp + (size_t)nch * 96;                         // [C][3][32] recomputed chunk
    double* rring = scr + 96 * C;                                 // [LK_NS][C][32] table entries
    E* ring = reinterpret_cast<E*>(rring + LK_NS * C * 32);       // [LK_NS][C][32] rows
    stage_levels(z, zl);
    __syncwarp();
    const int count = *z.lowk_count;
    for (int g = blockIdx.x; g * 32 < count; g += gridDim.x) {
        const int idx = g * 32 + threadIdx.x;
        if (idx >= count) continue;
        const int sys = z.lowk_list[idx];
        if (z.lowk_tab && (long)(g + 1) * 32 * nz <= z.lowk_cap)
            lowk_group<CPLX, true>(data_, z, g, sys, zl, ckp, scr, ring, rring, err);
        else
            lowk_group<CPLX, false>(data_, z, g, sys, zl, ckp, scr, ring, rring, err);
    }
}

template <bool CPLX, bool CYC>
cudaError_t launch_z(double*, const ZSys& z, void* data, const int* skip, int* err, const ZStreams& zs)
{
    dim3 grid((unsigned)((z.plane + TPB - 1) / TPB));  // pitch * my systems incl. padding columns
    if (CYC) k_thomas_z<double, Exact, CPLX, 0, CYC><<<grid, TPB, 0, zs.st>>>(data, z, skip, err);
    else k_thomas_exact<CPLX, true><<<grid, TPB, 3 * sizeof(double) * z.nz, zs.st>>>(data, z, skip, err);
    return cudaGetLastError();
}
// FP32 data: the bulk in FP32 and, concurrently on the auxiliary stream when
// one is given, the few low-|k| systems in FP64 (a short grid-wide launch
// whose duration is the latency of its long FP64 Thomas chains)
template <bool CPLX, bool CYC>
cudaError_t launch_z(float*, const ZSys& z, void* data, const int* skip, int* err, const ZStreams& zs)
{
    dim3 grid((unsigned)((z.plane + TPB - 1) / TPB));
    cudaStream_t lo = zs.st;
    if (zs.aux) {
        cudaError_t e = cudaEventRecord(zs.fork, zs.st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(zs.aux, zs.fork, 0);
        if (e != cudaSuccess) return e;
        lo = zs.aux;
    }
    const size_t lsm = lowk_smem<CPLX>(z.nz);
    if (!CYC && lowk_listed(z) && lsm <= 160 * 1024) {
        // persistent one-warp blocks (one per SM) over the list; the first
        // pass of a solve fills the coefficient table before
        int dev = 0, sms = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess) e = cudaFuncSetAttribute(k_thomas_lowk<CPLX>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lsm);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_lowk_table, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(3 * sizeof(double) * z.nz));
        if (e != cudaSuccess) return e;
        const long groups = (z.plane + 31) / 32;
        const unsigned lg = (unsigned)(groups < sms ? groups : sms);
        if (z.lowk_tab && z.lowk_build)
            k_lowk_table<<<lg, 32, 3 * sizeof(double) * z.nz, lo>>>(z, skip);
        k_thomas_lowk<CPLX><<<lg, 32, lsm, lo>>>(data, z, skip, err);
    } else {
        k_thomas_z<float, Exact, CPLX, 2, CYC><<<grid, TPB, 0, lo>>>(data, z, skip, err);
    }
    bool streamed = false;
    if (!CYC && z.ckpt_f) {
        const cudaError_t e = launch_stream<CPLX>(data, z, skip, err, zs.st, &streamed);
        if (e != cudaSuccess) return e;
    }
    if (!streamed) {
        if (CYC || !z.ckpt_f || z.plane >= (1L << 31) / 4)
            k_thomas_z<float, Fast, CPLX, 1, CYC><<<grid, TPB, 0, zs.st>>>(data, z, skip, err);
        else
            k_thomas_fast<CPLX><<<grid, TPB, sizeof(float4) * z.nz, zs.st>>>(data, z, skip, err);
    }
    if (zs.aux) {
        cudaError_t e = cudaEventRecord(zs.join, zs.aux);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(zs.st, zs.join, 0);
        if (e != cudaSuccess) return e;
    }
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_lowk_list(const ZSys& z, cudaStream_t st)
{
    if (!lowk_listed(z)) return cudaSuccess;
    k_lowk_list<<<(unsigned)((z.plane + 255) / 256), 256, 0, st>>>(z);
    return cudaGetLastError();
}

template <typename T, bool CPLX>
cudaError_t launch_tdma_z(void* data, const ZSys& z, const int* skip_flag, int* err_flag, const ZStreams& zs)
{
    if (z.cyclic) return launch_z<CPLX, true>((T*)nullptr, z, data, skip_flag, err_flag, zs);
    return launch_z<CPLX, false>((T*)nullptr, z, data, skip_flag, err_flag, zs);
}

template cudaError_t launch_tdma_z<double, true>(void*, const ZSys&, const int*, int*, const ZStreams&);
template cudaError_t launch_tdma_z<double, false>(void*, const ZSys&, const int*, int*, const ZStreams&);
template cudaError_t launch_tdma_z<float, true>(void*, const ZSys&, const int*, int*, const ZStreams&);
template cudaError_t launch_tdma_z<float, false>(void*, const ZSys&, const int*, int*, const ZStreams&);

// --------------------------------------------------------------------------
// Coefficient-array solves, element (sys, row) at [row * n_sys + sys].
// --------------------------------------------------------------------------
namespace {

struct ArrIn {
    const double* a;
    const double* b;
    const double* c;
    double* d;
    long ns, sys;
};

// loads CH rows [z0, z0+CH) of a, b, c, d (rows >= n are zero)
__device__ __forceinline__ void ld_chunk(const ArrIn& A, int z0, int n, double* a, double* b, double* c, double* d)
{
#pragma unroll
    for (int r = 0; r < CH; ++r) {
        a[r] = 0.0; b[r] = 1.0; c[r] = 0.0; d[r] = 0.0;
        if (z0 + r < n) {
            const long o = (long)(z0 + r) * A.ns + A.sys;
            a[r] = __ldg(A.a + o); b[r] = __ldg(A.b + o); c[r] = __ldg(A.c + o); d[r] = A.d[o];
        }
    }
}

}  // namespace

// tdma_many (tdmas.f90:114-147)
__global__ void __launch_bounds__(TPB) k_thomas_arr(const double* __restrict__ a, const double* __restrict__ b,
                                                    const double* __restrict__ c, double* __restrict__ d, int n_sys,
                                                    int n)
{
    extern __shared__ double ck[];
    const long sys = (long)blockIdx.x * TPB + threadIdx.x;
    if (sys >= n_sys) return;
    double* my = ck + threadIdx.x;
    ArrIn A{ a, b, c, d, n_sys, sys };
    const int nch = (n + CH - 1) / CH;
    double cp = 0, dp = 0, dum = 0;
    double av[CH], bv[CH], cv[CH], dv[CH];
    for (int ch = 0; ch < nch; ++ch) {
        const int z0 = ch * CH;
        ld_chunk(A, z0, n, av, bv, cv, dv);
#pragma unroll
        for (int r = 0; r < CH; ++r)
            if (z0 + r < n) fwd_row<Exact, false>(z0 + r == 0, av[r], bv[r], cv[r], dv[r], 0.0, cp, dp, dum);
        my[(2 * ch) * TPB] = cp;
        my[(2 * ch + 1) * TPB] = dp;
    }
    double x = 0;
    for (int ch = nch - 1; ch >= 0; --ch) {
        const int z0 = ch * CH;
        ld_chunk(A, z0, n, av, bv, cv, dv);
        double pc = 0, pd = 0;
        if (ch > 0) { pc = my[(2 * ch - 2) * TPB]; pd = my[(2 * ch - 1) * TPB]; }
        double c_[CH], d_[CH];
#pragma unroll
        for (int r = 0; r < CH; ++r) {
            if (z0 + r < n) fwd_row<Exact, false>(z0 + r == 0, av[r], bv[r], cv[r], dv[r], 0.0, pc, pd, dum);
            c_[r] = pc; d_[r] = pd;
        }
#pragma unroll
        for (int r = CH - 1; r >= 0; --r) {
            const int zr = z0 + r;
            if (zr < n) {
                x = (zr == n - 1) ? d_[r] : __dsub_rn(d_[r], __dmul_rn(c_[r], x));
                d[(long)zr * n_sys + sys] = x;
            }
        }
    }
}

// tdma_cycl_many (tdmas.f90:160-213): rows 1..n-1 are swept for the
// right-hand sides d and e (e_1 = -a_1, e_{n-1} = -c_{n-1}); x_0 needs the
// back-substituted d_1, e_1, so the back substitution runs twice (first to
// obtain them, then to write x_i = d_i + x_0 e_i) instead of storing e.
__global__ void __launch_bounds__(TPB) k_thomas_cycl(const double* __restrict__ a, const double* __restrict__ b,
                                                     const double* __restrict__ c, double* __restrict__ d,
                                                     int n_sys, int n)
{
    extern __shared__ double ck[];
    const long sys = (long)blockIdx.x * TPB + threadIdx.x;
    if (sys >= n_sys) return;
    double* my = ck + threadIdx.x;
    // view of rows 1..n-1 as a system of m = n-1 rows
    ArrIn A{ a + n_sys, b + n_sys, c + n_sys, d + n_sys, n_sys, sys };
    const int m = n - 1;
    const int nch = (m + CH - 1) / CH;
    double av[CH], bv[CH], cv[CH], dv[CH];
    const double e_first = -__ldg(a + n_sys + sys);                // -a(2)
    const double e_last = -__ldg(c + (long)(n - 1) * n_sys + sys);  // -c(n2)
    auto e_in = [&](int zr) -> double {
        // e(2) = -a(2) is set before e(n2) = -c(n2) (tdmas.f90:172-174)
        if (zr == m - 1) return e_last;
        if (zr == 0) return e_first;
        return 0.0;
    };
    double cp = 0, dp = 0, ep = 0;
    for (int ch = 0; ch < nch; ++ch) {
        const int z0 = ch * CH;
        ld_chunk(A, z0, m, av, bv, cv, dv);
#pragma unroll
        for (int r = 0; r < CH; ++r)
            if (z0 + r < m) fwd_row<Exact, true>(z0 + r == 0, av[r], bv[r], cv[r], dv[r], e_in(z0 + r), cp, dp, ep);
        my[(3 * ch) * TPB] = cp;
        my[(3 * ch + 1) * TPB] = dp;
        my[(3 * ch + 2) * TPB] = ep;
    }
    // pass 1: d_1, e_1 after back substitution (d_{n-1}, e_{n-1} are d', e' of the top row)
    const double d_top = dp, e_top = ep;
    double xd = 0, xe = 0;
    for (int pass = 0; pass < 2; ++pass) {
        double x0 = 0.0;
        if (pass == 1) {
            const double a0 = __ldg(a + sys), b0 = __ldg(b + sys), c0 = __ldg(c + sys), d0 = d[sys];
            // d(1) = (d(1) - a(1) d(n2) - c(1) d(2)) / (b(1) + a(1) e(n2) + c(1) e(2))
            x0 = __ddiv_rn(__dsub_rn(__dsub_rn(d0, __dmul_rn(a0, d_top)), __dmul_rn(c0, xd)),
                           __dadd_rn(__dadd_rn(b0, __dmul_rn(a0, e_top)), __dmul_rn(c0, xe)));
        }
        double yd = 0, ye = 0;
        for (int ch = nch - 1; ch >= 0; --ch) {
            const int z0 = ch * CH;
            ld_chunk(A, z0, m, av, bv, cv, dv);
            double pc = 0, pd = 0, pe = 0;
            if (ch > 0) { pc = my[(3 * ch - 3) * TPB]; pd = my[(3 * ch - 2) * TPB]; pe = my[(3 * ch - 1) * TPB]; }
            double c_[CH], d_[CH], e_[CH];
#pragma unroll
            for (int r = 0; r < CH; ++r) {
                if (z0 + r < m) fwd_row<Exact, true>(z0 + r == 0, av[r], bv[r], cv[r], dv[r], e_in(z0 + r), pc, pd, pe);
                c_[r] = pc; d_[r] = pd; e_[r] = pe;
            }
#pragma unroll
            for (int r = CH - 1; r >= 0; --r) {
                const int zr = z0 + r;
                if (zr < m) {
                    if (zr == m - 1) { yd = d_[r]; ye = e_[r]; }
                    else {
                        yd = __dsub_rn(d_[r], __dmul_rn(c_[r], yd));
                        ye = __dsub_rn(e_[r], __dmul_rn(c_[r], ye));
                    }
                    if (pass == 1) d[(long)(zr + 1) * n_sys + sys] = __dadd_rn(yd, __dmul_rn(x0, ye));
                }
            }
        }
        if (pass == 0) { xd = yd; xe = ye; }
        else d[sys] = x0;
    }
}

cudaError_t launch_tdma_many(const double* a, const double* b, const double* c, double* d, int n_sys, int n_row,
                             bool cyclic, int* err, cudaStream_t st)
{
    (void)err;
    const int m = cyclic ? n_row - 1 : n_row;
    const int nch = (m + CH - 1) / CH;
    const size_t smem = (size_t)(cyclic ? 3 : 2) * nch * TPB * sizeof(double);
    if (smem > 200 * 1024) return cudaErrorInvalidConfiguration;
    dim3 grid((unsigned)(((long)n_sys + TPB - 1) / TPB));
    if (cyclic) {
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(k_thomas_cycl, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
        }
        k_thomas_cycl<<<grid, TPB, smem, st>>>(a, b, c, d, n_sys, n_row);
    } else {
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(k_thomas_arr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
        }
        k_thomas_arr<<<grid, TPB, smem, st>>>(a, b, c, d, n_sys, n_row);
    }
    return cudaGetLastError();
}

// --------------------------------------------------------------------------
// Rows of the systems split over ranks (z slabs): PaScaL's modified Thomas
// algorithm (01_Fortran/PaScaL_TDMA/src/pascal_tdma_cuda.f90:332-473).  Each
// rank eliminates its local rows so that every row depends only on its own
// unknown and on the unknowns of the rank's first and last rows; those two
// rows form the rank's part of a reduced system of 2 * nranks rows per
// system (b = 1), which the caller gathers, solves and scatters back, and
// k_tdma_update finishes the local rows (:483-520).  The arithmetic follows
// the reference operation for operation (rounding-explicit, as in the
// single-rank kernels).  Layout: element (sys, row) at [row * n_sys + sys];
// reduced rows (sys, r) at [r * n_sys + sys], r = 0 (first row), 1 (last).
// --------------------------------------------------------------------------
__global__ void __launch_bounds__(TPB) k_tdma_modified(double* __restrict__ a, const double* __restrict__ b,
                                                       double* __restrict__ c, double* __restrict__ d,
                                                       double* __restrict__ a_rd, double* __restrict__ c_rd,
                                                       double* __restrict__ d_rd, long ns, int n)
{
    const long s = (long)blockIdx.x * TPB + threadIdx.x;
    if (s >= ns) return;
    using X = Exact;
    auto at = [&](int i) { return (long)i * ns + s; };
    // rows 1 and 2 are normalised by their diagonal
    double a0 = X::div(a[at(0)], b[at(0)]), c0 = X::div(c[at(0)], b[at(0)]), d0 = X::div(d[at(0)], b[at(0)]);
    a[at(0)] = a0; c[at(0)] = c0; d[at(0)] = d0;
    double a1 = X::div(a[at(1)], b[at(1)]), c1 = X::div(c[at(1)], b[at(1)]), d1 = X::div(d[at(1)], b[at(1)]);
    a[at(1)] = a1; c[at(1)] = c1; d[at(1)] = d1;
    // elimination of the lower diagonal, rows 3..n
    for (int i = 2; i < n; ++i) {
        a0 = a1; c0 = c1; d0 = d1;
        const double ai = a[at(i)], bi = b[at(i)], ci = c[at(i)], di = d[at(i)];
        const double r = X::div(1.0, X::sub(bi, X::mul(ai, c0)));
        d1 = X::mul(r, X::sub(di, X::mul(ai, d0)));
        c1 = X::mul(r, ci);
        a1 = X::mul(X::mul(-r, ai), a0);
        a[at(i)] = a1; c[at(i)] = c1; d[at(i)] = d1;
    }
    a_rd[ns + s] = a1;
    c_rd[ns + s] = c1;
    d_rd[ns + s] = d1;
    // elimination of the upper diagonal, rows n-2..2, from row n-1
    a1 = a0; c1 = c0; d1 = d0;
    for (int i = n - 3; i >= 1; --i) {
        double ai = a[at(i)], ci = c[at(i)], di = d[at(i)];
        di = X::sub(di, X::mul(ci, d1));
        ai = X::sub(ai, X::mul(ci, a1));
        ci = X::mul(-ci, c1);
        a1 = ai; c1 = ci; d1 = di;
        a[at(i)] = ai; c[at(i)] = ci; d[at(i)] = di;
    }
    {
        double ai = a[at(0)], ci = c[at(0)], di = d[at(0)];
        const double r = X::div(1.0, X::sub(1.0, X::mul(a1, ci)));
        di = X::mul(r, X::sub(di, X::mul(ci, d1)));
        ai = X::mul(r, ai);
        ci = X::mul(X::mul(-r, ci), c1);
        a[at(0)] = ai; c[at(0)] = ci; d[at(0)] = di;
        a_rd[s] = ai;
        c_rd[s] = ci;
        d_rd[s] = di;
    }
}

__global__ void __launch_bounds__(TPB) k_tdma_update(const double* __restrict__ a, const double* __restrict__ c,
                                                     double* __restrict__ d, const double* __restrict__ x_rd, long ns,
                                                     int n)
{
    const long s = (long)blockIdx.x * TPB + threadIdx.x;
    if (s >= ns) return;
    const double xs = x_rd[s], xe = x_rd[ns + s];
    d[s] = xs;
    d[(long)(n - 1) * ns + s] = xe;
    for (int i = 1; i < n - 1; ++i) {
        const long o = (long)i * ns + s;
        d[o] = __dsub_rn(__dsub_rn(d[o], __dmul_rn(a[o], xs)), __dmul_rn(c[o], xe));
    }
}

cudaError_t launch_tdma_modified(double* a, const double* b, double* c, double* d, double* a_rd, double* c_rd,
                                 double* d_rd, long n_sys, int n_row, cudaStream_t st)
{
    dim3 grid((unsigned)((n_sys + TPB - 1) / TPB));
    k_tdma_modified<<<grid, TPB, 0, st>>>(a, b, c, d, a_rd, c_rd, d_rd, n_sys, n_row);
    return cudaGetLastError();
}

cudaError_t launch_tdma_update(const double* a, const double* c, double* d, const double* x_rd, long n_sys, int n_row,
                               cudaStream_t st)
{
    dim3 grid((unsigned)((n_sys + TPB - 1) / TPB));
    k_tdma_update<<<grid, TPB, 0, st>>>(a, c, d, x_rd, n_sys, n_row);
    return cudaGetLastError();
}

__global__ void __launch_bounds__(256) k_zcoef(const double* __restrict__ dx3, const double* __restrict__ dmx3,
                                               int nz, double* __restrict__ am, double* __restrict__ ap,
                                               double* __restrict__ dzmin2)
{
    zcoef(dx3, dmx3, nz, am, ap, dzmin2);
}

cudaError_t launch_zcoef(const double* dx3, const double* dmx3, int nz, double* am, double* ap, double* dzmin2,
                         cudaStream_t st)
{
    k_zcoef<<<1, 256, 0, st>>>(dx3, dmx3, nz, am, ap, dzmin2);
    return cudaGetLastError();
}

}  // namespace ppf
