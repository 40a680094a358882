// ppf_batch.cu -- the persistent work-queue kernel of a batch of independent
// solves (sm_100a).
//
// One launch runs every stage of every problem of the batch.  The host lays
// the stages out as tasks (ppf_batch.cuh: one per stage and problem, in
// stage-major order across the problems, each split into tiles of work); a
// fixed grid of CTAs, resident on every SM, takes tiles from a global
// counter in queue order.  A tile's task may start once every tile of the
// problem's previous stage is done: the CTA that took it polls that stage's
// done count (acquire loads with a backoff, bounded: after about 0.1 s it
// records error bit 4 and goes on).  Tiles are handed out in queue order
// and a task only depends on an earlier one, so the earliest unfinished tile
// never waits on an unfinished one and the queue always progresses.
//
// The tiles run the same device bodies as the separate kernels (ppf_x_dev,
// ppf_y_dev, ppf_tdma_dev, ppf_misc_dev): x and y transforms with the
// run-time engine at tile widths sized for BATCH_THREADS threads, the z
// systems one per thread (the reference's Thomas arithmetic; FP32 spectra:
// the low-|k| systems, lambda dz_min^2 below the plan's threshold, in FP64
// as in the separate path), the refinement gate, the ghost cells.  Loads of
// fields written earlier in the launch avoid the read-only cache, and every
// stage's writes are released (fence + done count) before its dependants
// read them.
#include "ppf_batch.cuh"
#include "ppf_misc_dev.cuh"
#include "ppf_tdma_dev.cuh"
#include "ppf_x_dev.cuh"
#include "ppf_y_dev.cuh"

namespace ppf {

namespace {

// polls of a dependency's done count before giving up (each after a
// nanosleep backoff: about 0.1 s in all, some hundred times the longest
// tile); once one wait has given up, later ones are not attempted, so a
// broken queue drains at once with error bit 4 set
constexpr long BATCH_WAIT_LIMIT = 1L << 20;

__device__ __forceinline__ int ld_acquire(const int* p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Each stage body below is its own (not inlined) function, so that the
// registers of one stage's code are allocated apart from the others'.

// the z system `sys` of the problem (one thread each)
template <typename T, bool CPLX, bool CYC>
__device__ __noinline__ void z_system(const BProb& pb, long sys, int* err)
{
    using namespace zdev;
    const ZSys& z = pb.z;
    if (sys >= z.plane) return;
    const int kx = (int)(sys % z.pitch), ky = (int)(sys / z.pitch);
    if (kx >= z.mx || ky >= z.my) return;
    Coef co;
    co.am = z.am;
    co.ap = z.ap;
    co.lx = z.lamx[kx];
    co.ly = z.lamy[ky];
    co.pin = (kx == 0 && ky == 0);
    using E = typename Elem<T, CPLX>::type;
    E* data = reinterpret_cast<E*>(pb.B);
    double* ck = z.ckpt + sys;
    double zsum = 0.0;
    bool bad = false;
    bool exact = true;
    if constexpr (sizeof(T) == 4) exact = (co.lx + co.ly) * (*z.dzmin2) < z.lowk;
    if (exact) {
        if (CYC) thomas_poisson_cyc<T, Exact, CPLX>(data, sys, z.plane, z.nz, co, z.scale, ck, zsum, bad);
        else thomas_poisson<T, Exact, CPLX>(data, sys, z.plane, z.nz, co, z.scale, ck, zsum, bad);
    } else {
        if constexpr (sizeof(T) == 4) {
            if (CYC) thomas_poisson_cyc<T, Fast, CPLX>(data, sys, z.plane, z.nz, co, z.scale, ck, zsum, bad);
            else thomas_poisson<T, Fast, CPLX>(data, sys, z.plane, z.nz, co, z.scale, ck, zsum, bad);
        }
    }
    if (co.pin && z.dc_shift) *z.dc_shift = zsum / (double)z.nz;
    if (bad && err) atomicOr(err, 1);
}

template <typename T, bool DCT>
__device__ __noinline__ void x_forward(const BProb& pb, int resid, const int* skip, long tile)
{
    const cx<T>* tw = reinterpret_cast<const cx<T>*>(pb.tw);
    ResidIn rs{};
    rs.P = pb.P;
    rs.U = (resid == 2) ? pb.U : nullptr;
    rs.am = pb.z.am;
    rs.ap = pb.z.ap;
    rs.ix2 = pb.ix2;
    rs.iy2 = pb.iy2;
#define PPF_BX(R)                                                                                                \
    xfwd<T, DCT, R, ShapeRT, false>(pb.f, rs, pb.g, pb.A, pb.a_pitch, pb.sx, pb.wx, pb.lgwx, tw + pb.tw_off[0],   \
                                    tw + pb.tw_off[1], tw + pb.tw_off[2], skip, tile)
    if constexpr (sizeof(T) == 4) {
        if (resid == 1) { PPF_BX(1); return; }
        if (resid == 2) { PPF_BX(2); return; }
    }
    PPF_BX(0);
#undef PPF_BX
}

template <typename T, bool DCT>
__device__ __noinline__ void x_inverse(const BProb& pb, int arg, const int* skip, long tile)
{
    const cx<T>* tw = reinterpret_cast<const cx<T>*>(pb.tw);
    double* part = pb.mixed ? pb.partials : nullptr;
#define PPF_BI(ACC, GHOST, UK)                                                                                   \
    xinv<T, DCT, ACC, GHOST, ShapeRT, UK>(pb.A, pb.a_pitch, pb.P, pb.U, pb.g, part, pb.scal + 5, pb.sx, pb.wx,   \
                                          pb.lgwx, tw + pb.tw_off[0], tw + pb.tw_off[1], tw + pb.tw_off[2], skip,   \
                                          tile)
    if constexpr (sizeof(T) == 4) {
        switch (arg) {
            case 0 | 2 | (U_P << 2): PPF_BI(false, true, U_P); return;
            case 0 | 2 | (U_WRITE << 2): PPF_BI(false, true, U_WRITE); return;
            case 1 | 2 | (U_ACC << 2): PPF_BI(true, true, U_ACC); return;
            case 1 | 2 | (U_P << 2): PPF_BI(true, true, U_P); return;
            default: break;
        }
    }
    PPF_BI(false, false, U_P);
#undef PPF_BI
}

template <typename T, bool INV>
__device__ __noinline__ void y_pass(const BProb& pb, const int* skip, long tile)
{
    const cx<T>* tw = reinterpret_cast<const cx<T>*>(pb.tw);
    const cx<T>* A = reinterpret_cast<const cx<T>*>(pb.A);
    const cx<T>* B = reinterpret_cast<const cx<T>*>(pb.B);
    const int cblk = (int)(tile % pb.y_cblk), zz = (int)(tile / pb.y_cblk);
    const cx<T>* tyn = tw + pb.tw_off[3];
    const cx<T>* tyd = tw + pb.tw_off[4];
#define PPF_BY(K)                                                                                                  \
    if (INV)                                                                                                       \
        yinv<T, K, ShapeRT>(B, pb.b_cp, const_cast<cx<T>*>(A), pb.a_cp, pb.ycols, pb.g, pb.sy, pb.wy, pb.lgwy, tyn, \
                            tyd, pb.scal + 4, skip, cblk, zz);                                                     \
    else                                                                                                           \
        yfwd<T, K, ShapeRT>(A, pb.a_cp, const_cast<cx<T>*>(B), pb.b_cp, pb.ycols, pb.g, pb.sy, pb.wy, pb.lgwy, tyn, \
                            tyd, skip, cblk, zz)
    if (pb.ykind == Y_C2C) { PPF_BY(Y_C2C); }
    else if (pb.ykind == Y_CDCT) { PPF_BY(Y_CDCT); }
    else { PPF_BY(Y_RPAIR); }
#undef PPF_BY
}

template <typename T>
__device__ __forceinline__ void run_tile(const BProb& pb, const BTask& tk, long tile, int* err)
{
    const int* skip = tk.skip ? pb.flags : nullptr;
    switch (tk.kind) {
        case BK_ZCOEF:
            // the per-solve resets of the plan's flags and scalars, then the z
            // coefficients and min dz^2 (one tile)
            if (threadIdx.x < 4) pb.flags[threadIdx.x] = 0;
            if (threadIdx.x >= 1 && threadIdx.x < 8) pb.scal[threadIdx.x] = 0.0;
            __syncthreads();
            zcoef(pb.dx3, pb.dmx3, pb.g.nz, const_cast<double*>(pb.z.am), const_cast<double*>(pb.z.ap), pb.scal);
            break;
        case BK_XFWD:
            if (pb.xdct) x_forward<T, true>(pb, tk.arg, skip, tile);
            else x_forward<T, false>(pb, tk.arg, skip, tile);
            break;
        case BK_YFWD: y_pass<T, false>(pb, skip, tile); break;
        case BK_Z: {
            if (skip && *skip) break;
            const long sys = tile * blockDim.x + threadIdx.x;
            if (pb.cplx) {
                if (pb.z.cyclic) z_system<T, true, true>(pb, sys, pb.flags + 2);
                else z_system<T, true, false>(pb, sys, pb.flags + 2);
            } else {
                if (pb.z.cyclic) z_system<T, false, true>(pb, sys, pb.flags + 2);
                else z_system<T, false, false>(pb, sys, pb.flags + 2);
            }
            break;
        }
        case BK_YINV: y_pass<T, true>(pb, skip, tile); break;
        case BK_XINV:
            if (pb.xdct) x_inverse<T, true>(pb, tk.arg, skip, tile);
            else x_inverse<T, false>(pb, tk.arg, skip, tile);
            break;
        case BK_GATE:
            sweep_gate(pb.partials, pb.x_tiles, pb.ncell, pb.scal + 5, pb.flags, pb.flags + 1, pb.scal + 3,
                       pb.sweep_tol, tk.arg);
            break;
        case BK_GHOST: {
            const int d = tk.arg & 3, neumann = tk.arg >> 2;
            const double* dmx = d == 0 ? pb.dmx1 : (d == 1 ? pb.dmx2 : pb.dmx3);
            ghost_axis(pb.P, d, neumann, pb.g.nx, pb.g.ny, pb.g.nz, pb.g.pstride_y, pb.g.pstride_z, dmx, 3,
                       tile * blockDim.x + threadIdx.x, (long)tk.tiles * blockDim.x);
            break;
        }
        default: break;
    }
    (void)err;
}

__global__ void __launch_bounds__(BATCH_THREADS, 1)
    k_batch(const BProb* __restrict__ probs, const BTask* __restrict__ tasks, int ntasks, long total,
            int* __restrict__ counters)
{
    __shared__ long s_tile;
    __shared__ int s_task, s_ok;
    unsigned long long* next = reinterpret_cast<unsigned long long*>(counters);
    int* err = counters + 2;
    int* done = counters + 4;
    for (;;) {
        if (threadIdx.x == 0) {
            const long t = (long)atomicAdd(next, 1ull);
            int k = -1, ok = 1;
            if (t < total) {
                int lo = 0, hi = ntasks - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (tasks[mid].first <= t) lo = mid;
                    else hi = mid - 1;
                }
                k = lo;
                const int dep = tasks[k].dep;
                if (dep >= 0 && (ld_acquire(err) & 4)) ok = 0;
                if (dep >= 0 && ok) {
                    const int need = tasks[dep].tiles;
                    long it = 0;
                    while (ld_acquire(done + dep) < need) {
                        if (++it > BATCH_WAIT_LIMIT) {
                            atomicOr(err, 4);
                            ok = 0;
                            break;
                        }
                        __nanosleep(100);
                    }
                }
            }
            s_tile = t;
            s_task = k;
            s_ok = ok;
        }
        __syncthreads();
        const long t = s_tile;
        if (t >= total) break;
        const int k = s_task;
        if (s_ok) {
            const BTask tk = tasks[k];
            const BProb& pb = probs[tk.prob];
            if (pb.elem == 8) run_tile<double>(pb, tk, t - tk.first, err);
            else run_tile<float>(pb, tk, t - tk.first, err);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();   // this tile's writes before its done count
            atomicAdd(done + k, 1);
        }
    }
}

}  // namespace

size_t batch_smem(const BProb* probs, int count)
{
    size_t m = 0;
    for (int i = 0; i < count; ++i) {
        const BProb& p = probs[i];
        const size_t ce = 2 * (size_t)p.elem;
        m = std::max(m, (size_t)(p.g.nx / 2) * p.wx * ce);
        m = std::max(m, (size_t)p.g.ny * p.wy * ce);
    }
    return m;
}

cudaError_t batch_persistent_grid(size_t smem, int* grid)
{
    int dev = 0, sms = 0, per = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch, BATCH_THREADS, smem);
    if (e != cudaSuccess) return e;
    if (per < 1) return cudaErrorInvalidConfiguration;
    *grid = sms * per;
    return cudaSuccess;
}

cudaError_t launch_batch_persistent(const BProb* probs_d, const BTask* tasks_d, int ntasks, long total_tiles,
                                    int* counters_d, size_t smem, int grid, cudaStream_t st)
{
    cudaError_t e = cudaFuncSetAttribute(k_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_batch<<<grid, BATCH_THREADS, smem, st>>>(probs_d, tasks_d, ntasks, total_tiles, counters_d);
    return cudaGetLastError();
}

}  // namespace ppf
