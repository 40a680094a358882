// ppf_api.cu -- plans, solve orchestration and the C ABI of libppf.
#include "../../include/ppf.h"
#include "ppf_kernels.cuh"
#include "ppf_xy_common.cuh"
#include "ppf_batch.cuh"

#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <array>
#include <map>
#include <mutex>
#include <tuple>
#include <new>
#include <vector>

using namespace ppf;

namespace {

thread_local char g_err[512] = "";

int fail(int code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int cuda_fail(cudaError_t e, const char* where)
{
    return fail(PPF_ERR_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

#define PPF_CK(call)                                          \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);   \
    } while (0)

const long double PI_L = 3.141592653589793238462643383279502884L;

// e^{-2 pi i k num/den} accurately (long double argument reduction)
void cexp_tab(int count, long double num, long double den, std::vector<double>& out)
{
    out.resize(2 * (size_t)count);
    for (int k = 0; k < count; ++k) {
        long double a = -2.0L * PI_L * (long double)k * num / den;
        out[2 * k] = (double)cosl(a);
        out[2 * k + 1] = (double)sinl(a);
    }
}

// Radix schedule of a length-n transform.  order 0: radix 8 first, then 4,
// 2, 3, 5 (fewest passes); 1: no radix 8; 2: radices 3 and 5 first.
bool factor(int n, FftSched& s, int order_id = 0)
{
    static const int orders[3][5] = { { 8, 4, 2, 3, 5 }, { 4, 2, 3, 5, 0 }, { 3, 5, 8, 4, 2 } };
    s = FftSched{};
    s.n = n;
    if (n < 1 || order_id < 0 || order_id > 2) return false;
    int m = n;
    for (int r : orders[order_id]) {
        while (r > 0 && m % r == 0 && m > 1) {
            if (s.npass >= 12) return false;
            s.radix[s.npass++] = r;
            m /= r;
        }
    }
    if (n == 1) { s.radix[0] = 2; s.npass = 0; }
    return m == 1;
}

// modified wavenumbers, fft_3d_poisson.f90:288-351
double wn_dct(int m, int n, double h)
{
    const double PI = 3.141592653589793238462643383279502884;
    double s = std::sin(0.5 * (double)m * PI / (double)n);
    return 4.0 * (s * s) / (h * h);
}
double wn_fft(int m, int n, double h)
{
    const double PI = 3.141592653589793238462643383279502884;
    return 2.0 * (1.0 - std::cos(2.0 * (double)m * PI / (double)n)) / (h * h);
}

}  // namespace

struct ppf_plan {
    ppf_desc d{};
    int dev = 0;
    bool batch_member = false;   // solved beside other problems (ppf_batch): z solve without the streamed kernel
    Geom g{};
    bool xdct = false, ydct = false, cplx = true;
    int ykind = Y_C2C;
    // spectral buffers: A after the x pass, B after the y pass
    long a_pitch = 0;      // elements of A's row type (complex for periodic x, real for DCT x)
    long b_pitch = 0;      // elements of B's row type
    int ycols = 0;         // complex columns the y pass walks
    int mx = 0, my = 0;    // system grid
    size_t elem = 8;       // sizeof(T) of the spectral data
    void* A = nullptr;
    void* B = nullptr;
    size_t a_bytes = 0, b_bytes = 0;
    double* lamx = nullptr;
    double* lamy = nullptr;
    double* am = nullptr;
    double* ap = nullptr;
    double* scal = nullptr;    // [0] min dz^2, [3] last ||du||/||u||, [4] zero-mode shift, [5] mean of the iterate
    int* flags = nullptr;      // [0] skip, [1] sweeps_done, [2] err, [3] FP64 low-|k| systems of a mixed solve
    double* partials = nullptr;  // per-block sums of the x-inverse pass (mixed precision)
    long xinv_nblk = 0;
    double* ckpt = nullptr;      // Thomas checkpoints of the z solve
    long ckpt_doubles = 0;
    float* U = nullptr;          // FP32 first iterate of a refining mixed solve (ghosted layout)
    bool own_work = true;        // A, B, ckpt, partials, U belong to the plan (not to a batch)
    // auxiliary stream of the FP64 low-|k| z solves of the mixed and FP32 paths
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    void* tw = nullptr;        // twiddle tables (type T)
    size_t tw_off[5] = {};     // element offsets: x half, x n, x dct, y n, y dct
    FftSched sx{}, sy{};
    double scale = 1.0;
    // device staging of ppf_solve_host (allocated on first use)
    double* f_dev = nullptr;
    double* p_dev = nullptr;
    double* m_dev = nullptr;
    // work memory of ppf_solve_adjoint (allocated on first use)
    double* adj_W = nullptr;       // ghosted solution of the scaled right-hand side
    double* adj_red = nullptr;     // plane partial sums (5 * nz * nchunk), correction (nz), scratch (4 * nz)
    long adj_chunk = 0;
    int adj_nchunk = 0;
    double* slab_part = nullptr;   // interior partial sums of ppf_slab_sum (allocated on first use)
    // per-stage timing (ppf_stage_timing)
    bool timing = false;
    std::vector<std::pair<int, cudaEvent_t>> marks;   // stage id (-1 = start), event
};

namespace {

template <typename T>
int upload_twiddles(ppf_plan* p)
{
    const int nx = p->g.nx, ny = p->g.ny;
    std::vector<double> xh, xn, xd, yn, yd;
    cexp_tab(nx / 2, 1, nx / 2, xh);
    cexp_tab(nx, 1, nx, xn);
    cexp_tab(nx, 1, 4.0L * nx, xd);   // e^{-i pi k/(2 nx)}
    cexp_tab(ny, 1, ny, yn);
    cexp_tab(ny, 1, 4.0L * ny, yd);   // e^{-i pi k/(2 ny)}
    std::vector<T> all;
    const std::vector<double>* parts[5] = { &xh, &xn, &xd, &yn, &yd };
    size_t off = 0;
    for (int i = 0; i < 5; ++i) {
        p->tw_off[i] = off / 2;
        for (double v : *parts[i]) all.push_back((T)v);
        off += parts[i]->size();
        while (off % 4) { all.push_back((T)0); ++off; }  // keep 16-byte alignment of every table
    }
    PPF_CK(cudaMalloc(&p->tw, all.size() * sizeof(T)));
    PPF_CK(cudaMemcpy(p->tw, all.data(), all.size() * sizeof(T), cudaMemcpyHostToDevice));
    return PPF_OK;
}

void drop_marks(ppf_plan* p)
{
    for (auto& m : p->marks) cudaEventDestroy(m.second);
    p->marks.clear();
}

// records an event after a stage's launch when timing is enabled
void mark(ppf_plan* p, int stage, cudaStream_t st)
{
    if (!p->timing) return;
    cudaEvent_t ev;
    if (cudaEventCreate(&ev) != cudaSuccess) return;
    cudaEventRecord(ev, st);
    p->marks.emplace_back(stage, ev);
}

void free_plan(ppf_plan* p)
{
    if (!p) return;
    drop_marks(p);
    void* ptrs[] = { p->lamx, p->lamy, p->am, p->ap, p->scal, p->flags, p->tw,
                     p->f_dev, p->p_dev, p->m_dev, p->adj_W, p->adj_red, p->slab_part };
    for (void* q : ptrs)
        if (q) cudaFree(q);
    if (p->aux) cudaStreamDestroy(p->aux);
    if (p->ev_fork) cudaEventDestroy(p->ev_fork);
    if (p->ev_join) cudaEventDestroy(p->ev_join);
    if (p->own_work) {
        void* work[] = { p->A, p->B, p->partials, p->ckpt, p->U };
        for (void* q : work)
            if (q) cudaFree(q);
    }
    delete p;
}

int validate(const ppf_desc* d)
{
    if (!d) return fail(PPF_ERR_INVALID, "null descriptor");
    if (d->n1m < 2 || d->n2m < 2 || d->n3m < 3)
        return fail(PPF_ERR_INVALID, "grid %dx%dx%d too small (need n1m,n2m >= 2, n3m >= 3)", d->n1m, d->n2m, d->n3m);
    if ((d->n1m & 1) || (d->n2m & 1))
        return fail(PPF_ERR_INVALID, "n1m and n2m must be even (got %d, %d)", d->n1m, d->n2m);
    if (!(d->L1 > 0.0) || !(d->L2 > 0.0)) return fail(PPF_ERR_INVALID, "L1, L2 must be positive");
    if (d->precision < PPF_FP64 || d->precision > PPF_FP32)
        return fail(PPF_ERR_INVALID, "unknown precision %d", d->precision);
    if (d->max_sweeps > 8) return fail(PPF_ERR_INVALID, "max_sweeps %d > 8", d->max_sweeps);
    if (d->n3m > 1024) return fail(PPF_ERR_UNSUPPORTED, "n3m %d > 1024", d->n3m);
    FftSched s;
    if (!factor(d->n1m / 2, s)) return fail(PPF_ERR_UNSUPPORTED, "n1m/2 = %d is not a product of 2, 3, 5", d->n1m / 2);
    if (!factor(d->n2m, s)) return fail(PPF_ERR_UNSUPPORTED, "n2m = %d is not a product of 2, 3, 5", d->n2m);
    const int limx = (d->precision == PPF_FP64) ? 2048 : 1024;
    if (d->n1m > limx || d->n2m > 2048)
        return fail(PPF_ERR_UNSUPPORTED, "n1m %d / n2m %d beyond the transform tile limits", d->n1m, d->n2m);
    return PPF_OK;
}

long round_up(long v, long m) { return (v + m - 1) / m * m; }

int plan_init(ppf_plan* p, const ppf_desc* d)
{
    p->d = *d;
    if (p->d.max_sweeps < 0) p->d.max_sweeps = 2;
    if (!(p->d.lowk_threshold > 0.0)) p->d.lowk_threshold = 1e-3;
    PPF_CK(cudaGetDevice(&p->dev));
    const int nx = d->n1m, ny = d->n2m, nz = d->n3m;
    p->g.nx = nx; p->g.ny = ny; p->g.nz = nz;
    p->g.px = d->pbc1 ? 1 : 0; p->g.py = d->pbc2 ? 1 : 0; p->g.pz = d->pbc3 ? 1 : 0;
    p->g.pstride_y = nx + 2;
    p->g.pstride_z = (long)(nx + 2) * (ny + 2);
    p->xdct = !d->pbc1;
    p->ydct = !d->pbc2;
    p->elem = (d->precision == PPF_FP64) ? 8 : 4;
    const size_t ce = 2 * p->elem;  // complex element bytes
    factor(nx / 2, p->sx);
    factor(ny, p->sy);

    const int nh = nx / 2 + 1;
    if (!p->xdct) {
        // A: complex rows of nx/2+1
        p->a_pitch = round_up(nh, 16);
        p->a_bytes = (size_t)p->a_pitch * ny * nz * ce;
        p->ycols = nh;
        p->b_pitch = p->a_pitch;
        p->ykind = p->ydct ? Y_CDCT : Y_C2C;
        p->mx = nh; p->my = ny;
        p->b_bytes = (size_t)p->b_pitch * ny * nz * ce;
        p->cplx = true;
    } else {
        // A: real rows of nx (packed as nx/2 complex pairs in the y pass)
        p->a_pitch = round_up(nx, 32);
        p->a_bytes = (size_t)p->a_pitch * ny * nz * p->elem;
        p->ycols = nx / 2;
        if (p->ydct) {
            p->ykind = Y_CDCT;
            p->b_pitch = p->a_pitch;  // real
            p->mx = nx; p->my = ny;
            p->b_bytes = (size_t)p->b_pitch * ny * nz * p->elem;
            p->cplx = false;
        } else {
            p->ykind = Y_RPAIR;
            p->b_pitch = round_up(nx, 16);  // complex, ny/2+1 rows
            p->mx = nx; p->my = ny / 2 + 1;
            p->b_bytes = (size_t)p->b_pitch * (ny / 2 + 1) * nz * ce;
            p->cplx = true;
        }
    }
    // normalisation of the unnormalised inverse transforms: 1/n (FFT), 1/(2n) (DCT)
    p->scale = 1.0 / ((p->xdct ? 2.0 * nx : (double)nx) * (p->ydct ? 2.0 * ny : (double)ny));

    // eigenvalue tables (host FP64, the reference's formulas)
    const double hx = d->L1 / nx, hy = d->L2 / ny;
    std::vector<double> lx(p->mx), ly(p->my);
    for (int i = 0; i < p->mx; ++i) lx[i] = p->xdct ? wn_dct(i, nx, hx) : wn_fft(i, nx, hx);
    for (int j = 0; j < p->my; ++j) {
        if (p->ydct) { ly[j] = wn_dct(j, ny, hy); continue; }
        int jm = j;
        if (!p->xdct && j + 1 > ny / 2 + 1) jm = ny - j;   // periodic-periodic fold (:339-346)
        ly[j] = wn_fft(jm, ny, hy);
    }
    PPF_CK(cudaMalloc(&p->lamx, sizeof(double) * p->mx));
    PPF_CK(cudaMalloc(&p->lamy, sizeof(double) * p->my));
    PPF_CK(cudaMalloc(&p->am, sizeof(double) * nz));
    PPF_CK(cudaMalloc(&p->ap, sizeof(double) * nz));
    PPF_CK(cudaMalloc(&p->scal, sizeof(double) * 8));
    PPF_CK(cudaMalloc(&p->flags, sizeof(int) * 4));
    PPF_CK(cudaMemset(p->scal, 0, sizeof(double) * 8));
    PPF_CK(cudaMemset(p->flags, 0, sizeof(int) * 4));
    p->ckpt_doubles = tdma_z_ckpt_doubles(nz, p->b_pitch * (long)p->my, p->g.pz, p->elem == 4);
    if (p->elem == 4) {
        PPF_CK(cudaStreamCreateWithFlags(&p->aux, cudaStreamNonBlocking));
        PPF_CK(cudaEventCreateWithFlags(&p->ev_fork, cudaEventDisableTiming));
        PPF_CK(cudaEventCreateWithFlags(&p->ev_join, cudaEventDisableTiming));
    }
    PPF_CK(cudaMemcpy(p->lamx, lx.data(), sizeof(double) * p->mx, cudaMemcpyHostToDevice));
    PPF_CK(cudaMemcpy(p->lamy, ly.data(), sizeof(double) * p->my, cudaMemcpyHostToDevice));
    int rc = (p->elem == 8) ? upload_twiddles<double>(p) : upload_twiddles<float>(p);
    return rc;
}

// blocks of the x-inverse pass with the plan's current x schedule (mixed
// precision keeps 3 partial sums per block)
long partials_doubles(const ppf_plan* p)
{
    return (p->d.precision == PPF_MIXED) ? 3 * xinv_blocks<float>(p->g, p->sx) : 0;
}

// the FP32 first iterate of a mixed solve that refines: ghosted, like P
size_t u_bytes(const ppf_plan* p)
{
    if (p->d.precision != PPF_MIXED || p->d.max_sweeps == 0) return 0;
    return sizeof(float) * (size_t)(p->g.nx + 2) * (p->g.ny + 2) * (p->g.nz + 2);
}

// the plan's own work memory: spectral buffers, Thomas checkpoints,
// partials, the FP32 first iterate
int plan_alloc_work(ppf_plan* p)
{
    p->own_work = true;
    if (cudaMalloc(&p->A, p->a_bytes) != cudaSuccess || cudaMalloc(&p->B, p->b_bytes) != cudaSuccess) {
        cudaGetLastError();
        return fail(PPF_ERR_NOMEM, "cannot allocate %.1f MB of spectral work memory",
                    (p->a_bytes + p->b_bytes) / 1048576.0);
    }
    PPF_CK(cudaMalloc(&p->ckpt, sizeof(double) * p->ckpt_doubles));
    const long np = partials_doubles(p);
    if (np > 0) {
        p->xinv_nblk = np / 3;
        PPF_CK(cudaMalloc(&p->partials, sizeof(double) * np));
    }
    const size_t ub = u_bytes(p);
    if (ub && cudaMalloc(&p->U, ub) != cudaSuccess) {
        cudaGetLastError();
        p->U = nullptr;
        return fail(PPF_ERR_NOMEM, "cannot allocate %.1f MB for the FP32 first iterate", ub / 1048576.0);
    }
    return PPF_OK;
}

// One pass of transforms and z solves.  uk (UKind): where the x inverse
// puts the iterate (U_WRITE: the FP32 field p->U) and, with resid, where the
// residual and the accumulate read it (U_ACC: from p->U).
template <typename T>
int run_pass(ppf_plan* p, const double* f, double* P, bool resid, bool accumulate, const int* skip,
             cudaStream_t st, int uk = U_P)
{
    const cx<T>* tw = reinterpret_cast<const cx<T>*>(p->tw);
    const cx<T>* txh = tw + p->tw_off[0];
    const cx<T>* txn = tw + p->tw_off[1];
    const cx<T>* txd = tw + p->tw_off[2];
    const cx<T>* tyn = tw + p->tw_off[3];
    const cx<T>* tyd = tw + p->tw_off[4];
    ResidIn rs{};
    if (resid) {
        rs.P = P;
        rs.U = (uk == U_ACC) ? p->U : nullptr;
        rs.am = p->am;
        rs.ap = p->ap;
        const double hx = p->d.L1 / p->g.nx, hy = p->d.L2 / p->g.ny;
        rs.ix2 = 1.0 / (hx * hx);
        rs.iy2 = 1.0 / (hy * hy);
    }
    ZSys z{};
    z.mx = p->mx; z.my = p->my; z.pitch = p->b_pitch; z.plane = p->b_pitch * (long)p->my; z.nz = p->g.nz;
    z.lamx = p->lamx; z.lamy = p->lamy; z.am = p->am; z.ap = p->ap; z.scale = p->scale;
    z.lowk = (p->d.precision == PPF_FP64) ? 0.0 : p->d.lowk_threshold;
    z.dzmin2 = p->scal;
    z.dc_shift = p->scal + 4;
    z.cyclic = p->g.pz;
    z.shared_gpu = p->batch_member ? 1 : 0;
    z.ckpt = p->ckpt;
    z.ckpt_f = (sizeof(T) == 4) ? tdma_z_ckpt_f32(p->ckpt, z.nz, z.plane, z.cyclic) : nullptr;
    if (sizeof(T) == 4 && !z.cyclic) {
        // the FP64 low-|k| systems: their list, and the table of their
        // coefficient sweeps in the FP64 checkpoint region (unused here)
        z.lowk_count = p->flags + 3;
        z.lowk_list = tdma_z_lowk_list(p->ckpt, z.nz, z.plane, z.cyclic);
        z.lowk_tab = p->ckpt;
        z.lowk_cap = tdma_z_ckpt_doubles(z.nz, z.plane, z.cyclic, false);
        z.lowk_build = !resid;
    }
    cudaError_t e;
    if (!resid && z.lowk_list) {
        // the FP64 low-|k| set of this solve (flags[3], zeroed with the
        // flags, counts it); the z solve of every pass uses it
        e = launch_lowk_list(z, st);
        if (e != cudaSuccess) return cuda_fail(e, "low-|k| list");
    }
    e = launch_xfwd<T>(p->xdct, f, resid ? &rs : nullptr, p->g, p->A, p->a_pitch, p->sx, txh, txn, txd, skip, st);
    if (e != cudaSuccess) return cuda_fail(e, "x forward");
    mark(p, 1, st);
    // complex views of A and B for the y pass
    const long a_cp = p->xdct ? p->a_pitch / 2 : p->a_pitch;
    const long b_cp = (p->xdct && p->ydct) ? p->b_pitch / 2 : p->b_pitch;
    e = launch_yfwd<T>(p->ykind, reinterpret_cast<const cx<T>*>(p->A), a_cp, reinterpret_cast<cx<T>*>(p->B), b_cp,
                       p->ycols, p->g, p->sy, tyn, tyd, skip, st, p->flags + 2);
    if (e != cudaSuccess) return cuda_fail(e, "y forward");
    mark(p, 2, st);
    const ZStreams zs{ st, p->aux, p->ev_fork, p->ev_join };
    e = p->cplx ? launch_tdma_z<T, true>(p->B, z, skip, p->flags + 2, zs)
                : launch_tdma_z<T, false>(p->B, z, skip, p->flags + 2, zs);
    if (e != cudaSuccess) return cuda_fail(e, "z tridiagonal");
    mark(p, 3, st);
    e = launch_yinv<T>(p->ykind, reinterpret_cast<const cx<T>*>(p->B), b_cp, reinterpret_cast<cx<T>*>(p->A), a_cp,
                       p->ycols, p->g, p->sy, tyn, tyd, p->scal + 4, skip, st, p->flags + 2);
    if (e != cudaSuccess) return cuda_fail(e, "y inverse");
    mark(p, 4, st);
    // the mixed path keeps the stencil's ghost cells current for its residual
    long nblk = 0;
    e = launch_xinv<T>(p->xdct, p->A, p->a_pitch, P, p->U, uk, p->g, accumulate, p->d.precision == PPF_MIXED,
                       p->partials, p->scal + 5, p->sx, txh, txn, txd, skip, st, &nblk, p->flags + 2);
    if (p->partials) p->xinv_nblk = nblk;  // the refinement gate reduces these blocks' partial sums
    if (e != cudaSuccess) return cuda_fail(e, "x inverse");
    mark(p, 5, st);
    return PPF_OK;
}

int solve_impl(ppf_plan* p, const double* f, double* P, const double* dmx1, const double* dmx2,
               const double* dmx3, const double* dx3, cudaStream_t st)
{
    if (!p) return fail(PPF_ERR_INVALID, "null plan");
    if (!f || !P || !dmx1 || !dmx2 || !dmx3 || !dx3) return fail(PPF_ERR_INVALID, "null array argument");
    int cur = -1;
    PPF_CK(cudaGetDevice(&cur));
    if (cur != p->dev) return fail(PPF_ERR_STATE, "plan was created on device %d, current device is %d", p->dev, cur);
    mark(p, -1, st);
    PPF_CK(cudaMemsetAsync(p->flags, 0, sizeof(int) * 4, st));
    PPF_CK(cudaMemsetAsync(p->scal + 1, 0, sizeof(double) * 7, st));
    cudaError_t e = launch_zcoef(dx3, dmx3, p->g.nz, p->am, p->ap, p->scal, st);
    if (e != cudaSuccess) return cuda_fail(e, "z coefficients");
    mark(p, 0, st);
    int rc;
    if (p->elem == 8) {
        rc = run_pass<double>(p, f, P, false, false, nullptr, st);
    } else {
        // a refining mixed solve keeps its first iterate (FP32 values) in U;
        // the first sweep reads it from there and writes P
        const bool u32 = p->d.precision == PPF_MIXED && p->d.max_sweeps > 0 && p->U;
        rc = run_pass<float>(p, f, P, false, false, nullptr, st, u32 ? U_WRITE : U_P);
        if (rc == PPF_OK && p->d.precision == PPF_MIXED) {
            const double ncell = (double)p->g.nx * p->g.ny * p->g.nz;
            e = launch_sweep_gate(p->partials, p->xinv_nblk, ncell, p->scal + 5, p->flags, p->flags + 1,
                                  p->scal + 3, p->d.sweep_tol, 1, st);
            if (e != cudaSuccess) return cuda_fail(e, "sweep gate");
            mark(p, 6, st);
            for (int s = 0; s < p->d.max_sweeps && rc == PPF_OK; ++s) {
                rc = run_pass<float>(p, f, P, true, true, p->flags, st, (u32 && s == 0) ? U_ACC : U_P);
                if (rc != PPF_OK) break;
                e = launch_sweep_gate(p->partials, p->xinv_nblk, ncell, p->scal + 5, p->flags, p->flags + 1,
                                      p->scal + 3, p->d.sweep_tol, 0, st);
                if (e != cudaSuccess) return cuda_fail(e, "sweep gate");
                mark(p, 6, st);
            }
        }
    }
    if (rc != PPF_OK) return rc;
    e = launch_ghosts(P, p->g, dmx1, dmx2, dmx3, st);
    if (e != cudaSuccess) return cuda_fail(e, "ghost cells");
    mark(p, 7, st);
    return PPF_OK;
}

// Transpose of the solve (ppf_adjoint.cu has the derivation): df = M^T g,
// and with u the z-metric gradient of <g, u>.
int adjoint_impl(ppf_plan* p, const double* g, double* df, const double* u, double* ddx3, double* ddmx3,
                 const double* dmx1, const double* dmx2, const double* dmx3, const double* dx3, cudaStream_t st)
{
    if (!p) return fail(PPF_ERR_INVALID, "null plan");
    if (!g || !df || !dmx1 || !dmx2 || !dmx3 || !dx3) return fail(PPF_ERR_INVALID, "null array argument");
    if ((ddx3 || ddmx3) && !u) return fail(PPF_ERR_INVALID, "metric gradients need the forward solution u");
    int cur = -1;
    PPF_CK(cudaGetDevice(&cur));
    if (cur != p->dev) return fail(PPF_ERR_STATE, "plan was created on device %d, current device is %d", p->dev, cur);
    const Geom& gm = p->g;
    const int nz = gm.nz;
    if (!p->adj_W) {
        p->adj_nchunk = adjoint_chunks((long)gm.nx * gm.ny, &p->adj_chunk);
        const size_t wb = sizeof(double) * (size_t)(gm.nx + 2) * (gm.ny + 2) * (nz + 2);
        const size_t rb = sizeof(double) * ((size_t)5 * nz * p->adj_nchunk + 5 * (size_t)nz);
        if (cudaMalloc(&p->adj_W, wb) != cudaSuccess) {
            cudaGetLastError();
            p->adj_W = nullptr;
            return fail(PPF_ERR_NOMEM, "cannot allocate %.1f MB of adjoint work memory", wb / 1048576.0);
        }
        PPF_CK(cudaMalloc(&p->adj_red, rb));
    }
    const int nch = p->adj_nchunk;
    double* colpart = p->adj_red;
    double* mpart = colpart + (size_t)nz * nch;
    double* corr = mpart + (size_t)4 * nz * nch;
    double* wk = corr + nz;
    // h = (g - plane means) / dx3 into df (aliasing g is allowed), plane sums of g
    cudaError_t e = launch_adj_rhs(g, df, dx3, gm, p->adj_chunk, nch, colpart, st);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint right-hand side");
    // W = M h with the plan's precision (refinement included); this also
    // computes the z coefficients am, ap used below
    int rc = solve_impl(p, df, p->adj_W, dmx1, dmx2, dmx3, dx3, st);
    if (rc != PPF_OK) return rc;
    e = launch_adj_corr(colpart, nch, gm, p->am, p->ap, corr, wk, st);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint zero mode");
    e = launch_adj_out(p->adj_W, df, dx3, corr, (ddx3 || ddmx3) ? u : nullptr, gm, p->adj_chunk, nch, mpart, st);
    if (e != cudaSuccess) return cuda_fail(e, "adjoint output");
    if (ddx3 || ddmx3) {
        e = launch_adj_metric(mpart, nch, gm, p->am, p->ap, dx3, dmx3, ddx3, ddmx3, wk, st);
        if (e != cudaSuccess) return cuda_fail(e, "adjoint metric gradient");
    }
    return PPF_OK;
}

// host arrays: copy in on `st`, solve, copy out; `sync` waits for the stream
int host_impl(ppf_plan* plan, const double* f_h, double* p_h, const double* dmx1_h, const double* dmx2_h,
              const double* dmx3_h, const double* dx3_h, cudaStream_t st, bool sync)
{
    g_err[0] = 0;
    if (!plan) return fail(PPF_ERR_INVALID, "null plan");
    if (!f_h || !p_h || !dmx1_h || !dmx2_h || !dmx3_h || !dx3_h) return fail(PPF_ERR_INVALID, "null array argument");
    const Geom& g = plan->g;
    const size_t nf = (size_t)g.nx * g.ny * g.nz, np = (size_t)(g.nx + 2) * (g.ny + 2) * (g.nz + 2);
    const size_t nm = (size_t)(g.nx + 2) + (g.ny + 2) + 2 * (g.nz + 2);
    if (!plan->f_dev) {
        if (cudaMalloc((void**)&plan->f_dev, nf * sizeof(double)) != cudaSuccess ||
            cudaMalloc((void**)&plan->p_dev, np * sizeof(double)) != cudaSuccess ||
            cudaMalloc((void**)&plan->m_dev, nm * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            return fail(PPF_ERR_NOMEM, "cannot allocate device staging for host arrays");
        }
    }
    double *fd = plan->f_dev, *pd = plan->p_dev;
    double* d1 = plan->m_dev;
    double* d2 = d1 + (g.nx + 2);
    double* d3 = d2 + (g.ny + 2);
    double* x3 = d3 + (g.nz + 2);
    PPF_CK(cudaMemcpyAsync(fd, f_h, nf * sizeof(double), cudaMemcpyHostToDevice, st));
    PPF_CK(cudaMemcpyAsync(d1, dmx1_h, (g.nx + 2) * sizeof(double), cudaMemcpyHostToDevice, st));
    PPF_CK(cudaMemcpyAsync(d2, dmx2_h, (g.ny + 2) * sizeof(double), cudaMemcpyHostToDevice, st));
    PPF_CK(cudaMemcpyAsync(d3, dmx3_h, (g.nz + 2) * sizeof(double), cudaMemcpyHostToDevice, st));
    PPF_CK(cudaMemcpyAsync(x3, dx3_h, (g.nz + 2) * sizeof(double), cudaMemcpyHostToDevice, st));
    int rc = solve_impl(plan, fd, pd, d1, d2, d3, x3, st);
    if (rc == PPF_OK) {
        cudaError_t e = cudaMemcpyAsync(p_h, pd, np * sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) rc = cuda_fail(e, "copy out");
    }
    if (sync) {
        cudaError_t e = cudaStreamSynchronize(st);
        if (rc == PPF_OK && e != cudaSuccess) rc = cuda_fail(e, "synchronise");
    }
    return rc;
}

// one module-global plan for the reference-shaped API (p_poi, fft_3d_poisson.f90:43-59)
std::mutex g_mod_mu;
ppf_desc g_mod_desc{};
bool g_mod_desc_set = false;
ppf_plan* g_mod_plan = nullptr;
int g_mod_prec = PPF_FP64, g_mod_sweeps = -1;

}  // namespace

extern "C" {

const char* ppf_last_error(void) { return g_err; }

const char* ppf_version(void) { return "ppf 0.1.0 (sm_100a)"; }

int ppf_plan_create(const ppf_desc* desc, ppf_plan** plan)
{
    g_err[0] = 0;
    if (!plan) return fail(PPF_ERR_INVALID, "null plan pointer");
    *plan = nullptr;
    int rc = validate(desc);
    if (rc != PPF_OK) return rc;
    ppf_plan* p = new (std::nothrow) ppf_plan();
    if (!p) return fail(PPF_ERR_NOMEM, "host allocation failed");
    rc = plan_init(p, desc);
    if (rc == PPF_OK) rc = plan_alloc_work(p);
    if (rc != PPF_OK) {
        free_plan(p);
        return rc;
    }
    *plan = p;
    return PPF_OK;
}

int ppf_plan_destroy(ppf_plan* plan)
{
    free_plan(plan);
    return PPF_OK;
}

int ppf_stage_timing(ppf_plan* plan, int enable)
{
    if (!plan) return fail(PPF_ERR_INVALID, "null plan");
    plan->timing = enable != 0;
    if (!plan->timing) drop_marks(plan);
    return PPF_OK;
}

int ppf_stage_times(ppf_plan* plan, double* ms, int* launches)
{
    if (!plan || !ms || !launches) return fail(PPF_ERR_INVALID, "null argument");
    for (int i = 0; i < PPF_NSTAGES; ++i) { ms[i] = 0.0; launches[i] = 0; }
    cudaEvent_t prev = nullptr;
    for (auto& m : plan->marks) {
        cudaError_t e = cudaEventSynchronize(m.second);
        if (e != cudaSuccess) { drop_marks(plan); return cuda_fail(e, "event synchronise"); }
        if (m.first >= 0 && prev) {
            float t = 0.f;
            cudaEventElapsedTime(&t, prev, m.second);
            ms[m.first] += t;
            // ghosts launch one kernel per axis; every other stage one kernel
            launches[m.first] += (m.first == 7) ? 3 : 1;
        }
        prev = m.second;
    }
    drop_marks(plan);
    return PPF_OK;
}

int ppf_plan_workspace_bytes(const ppf_plan* plan, long long* bytes)
{
    if (!plan || !bytes) return fail(PPF_ERR_INVALID, "null argument");
    // spectral buffers, z-solve checkpoints (and low-|k| list), partial sums,
    // the FP32 first iterate of a refining mixed solve
    *bytes = (long long)(plan->a_bytes + plan->b_bytes + sizeof(double) * plan->ckpt_doubles +
                         sizeof(double) * partials_doubles(plan) + u_bytes(plan));
    return PPF_OK;
}

int ppf_solve(ppf_plan* plan, const double* f_d, double* p_d, const double* dmx1_d, const double* dmx2_d,
              const double* dmx3_d, const double* dx3_d, void* stream)
{
    g_err[0] = 0;
    return solve_impl(plan, f_d, p_d, dmx1_d, dmx2_d, dmx3_d, dx3_d, (cudaStream_t)stream);
}

int ppf_solve_adjoint(ppf_plan* plan, const double* g_d, double* df_d, const double* u_d, double* ddx3_d,
                      double* ddmx3_d, const double* dmx1_d, const double* dmx2_d, const double* dmx3_d,
                      const double* dx3_d, void* stream)
{
    return adjoint_impl(plan, g_d, df_d, u_d, ddx3_d, ddmx3_d, dmx1_d, dmx2_d, dmx3_d, dx3_d, (cudaStream_t)stream);
}

int ppf_solve_host(ppf_plan* plan, const double* f_h, double* p_h, const double* dmx1_h, const double* dmx2_h,
                   const double* dmx3_h, const double* dx3_h, void* stream)
{
    return host_impl(plan, f_h, p_h, dmx1_h, dmx2_h, dmx3_h, dx3_h, (cudaStream_t)stream, true);
}

int ppf_solve_host_async(ppf_plan* plan, const double* f_h, double* p_h, const double* dmx1_h, const double* dmx2_h,
                         const double* dmx3_h, const double* dx3_h, void* stream)
{
    return host_impl(plan, f_h, p_h, dmx1_h, dmx2_h, dmx3_h, dx3_h, (cudaStream_t)stream, false);
}

int ppf_last_sweeps(ppf_plan* plan, int* sweeps, double* last_rel_update, void* stream)
{
    if (!plan) return fail(PPF_ERR_INVALID, "null plan");
    int fl[4];
    double sc[4];
    cudaStream_t st = (cudaStream_t)stream;
    PPF_CK(cudaMemcpyAsync(fl, plan->flags, sizeof(fl), cudaMemcpyDeviceToHost, st));
    PPF_CK(cudaMemcpyAsync(sc, plan->scal, sizeof(sc), cudaMemcpyDeviceToHost, st));
    PPF_CK(cudaStreamSynchronize(st));
    if (sweeps) *sweeps = fl[1];
    if (last_rel_update) *last_rel_update = sc[3];
    if (fl[2]) return fail(PPF_ERR_NUMERIC, "a tridiagonal solve produced a non-finite value");
    return PPF_OK;
}

// ---- reference-shaped API -------------------------------------------------

int ppf_fft_poisson_plan_cuda_create(int n1, int n2, int n3, double L1, double L2, double L3, int pbc1, int pbc2,
                                     int pbc3)
{
    g_err[0] = 0;
    (void)L3;
    std::lock_guard<std::mutex> lk(g_mod_mu);
    ppf_desc d{};
    d.n1m = n1 - 1; d.n2m = n2 - 1; d.n3m = n3 - 1;     // n*m = n* - 1 (:103-104)
    d.L1 = L1; d.L2 = L2;
    d.pbc1 = pbc1 ? 1 : 0; d.pbc2 = pbc2 ? 1 : 0; d.pbc3 = pbc3 ? 1 : 0;
    d.precision = g_mod_prec;
    d.max_sweeps = g_mod_sweeps;
    int rc = validate(&d);
    if (rc != PPF_OK) return rc;
    g_mod_desc = d;
    g_mod_desc_set = true;
    return PPF_OK;
}

int ppf_cuda_poisson_fft_set_precision(int precision, int max_sweeps)
{
    std::lock_guard<std::mutex> lk(g_mod_mu);
    if (precision < PPF_FP64 || precision > PPF_FP32) return fail(PPF_ERR_INVALID, "unknown precision %d", precision);
    g_mod_prec = precision;
    g_mod_sweeps = max_sweeps;
    return PPF_OK;
}

int ppf_cuda_poisson_fft_initial(void)
{
    g_err[0] = 0;
    std::lock_guard<std::mutex> lk(g_mod_mu);
    if (!g_mod_desc_set) return fail(PPF_ERR_STATE, "ppf_fft_poisson_plan_cuda_create was not called");
    if (g_mod_plan) { free_plan(g_mod_plan); g_mod_plan = nullptr; }
    ppf_desc d = g_mod_desc;
    d.precision = g_mod_prec;
    d.max_sweeps = g_mod_sweeps;
    return ppf_plan_create(&d, &g_mod_plan);
}

int ppf_cuda_poisson_fft_1d(double* PRHS_d, double* P_d, const double* dmx1_d, const double* dmx2_d,
                            const double* dmx3_d, const double* dx3_d)
{
    g_err[0] = 0;
    std::lock_guard<std::mutex> lk(g_mod_mu);
    if (!g_mod_plan) return fail(PPF_ERR_STATE, "ppf_cuda_poisson_fft_initial was not called");
    int rc = solve_impl(g_mod_plan, PRHS_d, P_d, dmx1_d, dmx2_d, dmx3_d, dx3_d, (cudaStream_t)0);
    if (rc != PPF_OK) return rc;
    // the reference call is synchronous on the default stream
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)0);
    if (e != cudaSuccess) return cuda_fail(e, "synchronise");
    return PPF_OK;
}

int ppf_cuda_poisson_fft_clean(void)
{
    std::lock_guard<std::mutex> lk(g_mod_mu);
    free_plan(g_mod_plan);
    g_mod_plan = nullptr;
    g_mod_desc_set = false;
    return PPF_OK;
}

// ---- batched tridiagonal solves on coefficient arrays ----------------------

int ppf_tdma_many(const double* a, const double* b, const double* c, double* d, int n_sys, int n_row, void* stream)
{
    g_err[0] = 0;
    if (!a || !b || !c || !d) return fail(PPF_ERR_INVALID, "null array argument");
    if (n_sys < 1 || n_row < 1) return fail(PPF_ERR_INVALID, "n_sys %d, n_row %d must be positive", n_sys, n_row);
    if (n_row > 1024) return fail(PPF_ERR_UNSUPPORTED, "n_row %d > 1024", n_row);
    cudaError_t e = launch_tdma_many(a, b, c, d, n_sys, n_row, false, nullptr, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "tdma_many");
    return PPF_OK;
}

int ppf_tdma_cycl_many(const double* a, const double* b, const double* c, double* d, int n_sys, int n_row,
                       void* stream)
{
    g_err[0] = 0;
    if (!a || !b || !c || !d) return fail(PPF_ERR_INVALID, "null array argument");
    if (n_sys < 1 || n_row < 3) return fail(PPF_ERR_INVALID, "n_sys %d must be >= 1 and n_row %d >= 3", n_sys, n_row);
    if (n_row > 1025) return fail(PPF_ERR_UNSUPPORTED, "n_row %d > 1025", n_row);
    cudaError_t e = launch_tdma_many(a, b, c, d, n_sys, n_row, true, nullptr, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "tdma_cycl_many");
    return PPF_OK;
}

int ppf_tdma_many_modified(double* a, const double* b, double* c, double* d, double* a_rd, double* c_rd,
                           double* d_rd, int n_sys, int n_row, void* stream)
{
    g_err[0] = 0;
    if (!a || !b || !c || !d || !a_rd || !c_rd || !d_rd) return fail(PPF_ERR_INVALID, "null array argument");
    if (n_sys < 1 || n_row < 3) return fail(PPF_ERR_INVALID, "n_sys %d must be >= 1 and n_row %d >= 3", n_sys, n_row);
    cudaError_t e = launch_tdma_modified(a, b, c, d, a_rd, c_rd, d_rd, n_sys, n_row, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "tdma_many_modified");
    return PPF_OK;
}

int ppf_tdma_many_update(const double* a, const double* c, double* d, const double* x_rd, int n_sys, int n_row,
                         void* stream)
{
    g_err[0] = 0;
    if (!a || !c || !d || !x_rd) return fail(PPF_ERR_INVALID, "null array argument");
    if (n_sys < 1 || n_row < 3) return fail(PPF_ERR_INVALID, "n_sys %d must be >= 1 and n_row %d >= 3", n_sys, n_row);
    cudaError_t e = launch_tdma_update(a, c, d, x_rd, n_sys, n_row, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "tdma_many_update");
    return PPF_OK;
}

// ---- z-slab pieces of a multi-rank solve (the plan is this rank's slab) ----
static int slab_plan(ppf_plan* p)
{
    g_err[0] = 0;
    if (!p) return fail(PPF_ERR_INVALID, "null plan");
    if (p->elem != 8) return fail(PPF_ERR_UNSUPPORTED, "z-slab solves run in FP64 (the reference's precision)");
    int cur = -1;
    PPF_CK(cudaGetDevice(&cur));
    if (cur != p->dev) return fail(PPF_ERR_STATE, "plan was created on device %d, current device is %d", p->dev, cur);
    return PPF_OK;
}

int ppf_slab_systems(const ppf_plan* plan, int* n_sys)
{
    if (!plan || !n_sys) return fail(PPF_ERR_INVALID, "null argument");
    *n_sys = (int)((plan->cplx ? 2 : 1) * plan->b_pitch * (long)plan->my);
    return PPF_OK;
}

int ppf_slab_forward(ppf_plan* plan, const double* f_d, double* spec_d, void* stream)
{
    int rc = slab_plan(plan);
    if (rc != PPF_OK) return rc;
    if (!f_d || !spec_d) return fail(PPF_ERR_INVALID, "null array argument");
    ppf_plan* p = plan;
    cudaStream_t st = (cudaStream_t)stream;
    const cx<double>* tw = reinterpret_cast<const cx<double>*>(p->tw);
    cudaError_t e = launch_xfwd<double>(p->xdct, f_d, nullptr, p->g, p->A, p->a_pitch, p->sx, tw + p->tw_off[0],
                                        tw + p->tw_off[1], tw + p->tw_off[2], nullptr, st);
    if (e != cudaSuccess) return cuda_fail(e, "slab x forward");
    const long a_cp = p->xdct ? p->a_pitch / 2 : p->a_pitch;
    const long b_cp = (p->xdct && p->ydct) ? p->b_pitch / 2 : p->b_pitch;
    e = launch_yfwd<double>(p->ykind, reinterpret_cast<const cx<double>*>(p->A), a_cp,
                            reinterpret_cast<cx<double>*>(spec_d), b_cp, p->ycols, p->g, p->sy, tw + p->tw_off[3],
                            tw + p->tw_off[4], nullptr, st);
    if (e != cudaSuccess) return cuda_fail(e, "slab y forward");
    return PPF_OK;
}

int ppf_slab_coefficients(ppf_plan* plan, double* a_d, double* b_d, double* c_d, double* spec_d,
                          const double* dx3_g, const double* dmx3_g, int z0, int n3m_g, void* stream)
{
    int rc = slab_plan(plan);
    if (rc != PPF_OK) return rc;
    if (!a_d || !b_d || !c_d || !spec_d || !dx3_g || !dmx3_g) return fail(PPF_ERR_INVALID, "null array argument");
    if (z0 < 0 || z0 + plan->g.nz > n3m_g) return fail(PPF_ERR_INVALID, "slab rows %d..%d outside 0..%d", z0,
                                                       z0 + plan->g.nz, n3m_g);
    int ns = 0;
    ppf_slab_systems(plan, &ns);
    cudaError_t e = launch_slab_coef(a_d, b_d, c_d, spec_d, ns, plan->g.nz, plan->cplx ? 1 : 0, plan->b_pitch,
                                     plan->mx, plan->lamx, plan->lamy, dx3_g, dmx3_g, z0, n3m_g, plan->scale,
                                     (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "slab coefficients");
    return PPF_OK;
}

int ppf_slab_inverse(ppf_plan* plan, const double* spec_d, double* p_d, void* stream)
{
    int rc = slab_plan(plan);
    if (rc != PPF_OK) return rc;
    if (!spec_d || !p_d) return fail(PPF_ERR_INVALID, "null array argument");
    ppf_plan* p = plan;
    cudaStream_t st = (cudaStream_t)stream;
    const cx<double>* tw = reinterpret_cast<const cx<double>*>(p->tw);
    const long a_cp = p->xdct ? p->a_pitch / 2 : p->a_pitch;
    const long b_cp = (p->xdct && p->ydct) ? p->b_pitch / 2 : p->b_pitch;
    cudaError_t e = launch_yinv<double>(p->ykind, reinterpret_cast<const cx<double>*>(spec_d), b_cp,
                                        reinterpret_cast<cx<double>*>(p->A), a_cp, p->ycols, p->g, p->sy,
                                        tw + p->tw_off[3], tw + p->tw_off[4], nullptr, nullptr, st);
    if (e != cudaSuccess) return cuda_fail(e, "slab y inverse");
    e = launch_xinv<double>(p->xdct, p->A, p->a_pitch, p_d, nullptr, U_P, p->g, false, false, nullptr, nullptr, p->sx,
                            tw + p->tw_off[0], tw + p->tw_off[1], tw + p->tw_off[2], nullptr, st);
    if (e != cudaSuccess) return cuda_fail(e, "slab x inverse");
    return PPF_OK;
}

int ppf_slab_sum(ppf_plan* plan, const double* p_d, double* sum_d, void* stream)
{
    int rc = slab_plan(plan);
    if (rc != PPF_OK) return rc;
    if (!p_d || !sum_d) return fail(PPF_ERR_INVALID, "null array argument");
    if (!plan->slab_part) {
        if (cudaMalloc(&plan->slab_part, sizeof(double) * slab_sum_parts(plan->g)) != cudaSuccess) {
            cudaGetLastError();
            plan->slab_part = nullptr;
            return fail(PPF_ERR_NOMEM, "cannot allocate the slab reduction");
        }
    }
    cudaError_t e = launch_slab_sum(p_d, plan->g, plan->slab_part, sum_d, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "slab sum");
    return PPF_OK;
}

int ppf_slab_shift(ppf_plan* plan, double* p_d, const double* shift_d, void* stream)
{
    int rc = slab_plan(plan);
    if (rc != PPF_OK) return rc;
    if (!p_d || !shift_d) return fail(PPF_ERR_INVALID, "null array argument");
    cudaError_t e = launch_slab_shift(p_d, plan->g, shift_d, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "slab shift");
    return PPF_OK;
}

int ppf_slab_ghosts(ppf_plan* plan, double* p_d, const double* dmx1_d, const double* dmx2_d, const double* dmx3_d,
                    int z_lo_wall, int z_hi_wall, void* stream)
{
    int rc = slab_plan(plan);
    if (rc != PPF_OK) return rc;
    if (!p_d || !dmx1_d || !dmx2_d || !dmx3_d) return fail(PPF_ERR_INVALID, "null array argument");
    const int zf = plan->g.pz ? 0 : ((z_lo_wall ? 1 : 0) | (z_hi_wall ? 2 : 0));
    cudaError_t e = launch_ghosts(p_d, plan->g, dmx1_d, dmx2_d, dmx3_d, (cudaStream_t)stream, zf);
    if (e != cudaSuccess) return cuda_fail(e, "slab ghost cells");
    return PPF_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free FP64 solve.  All work memory (spectral buffers, tables,
// flags) lives in one file-scope device array of PPF_NOALLOC_SCRATCH_BYTES,
// so the call never allocates device memory.  The array is a per-device
// global of this library: every call on a device shares it and it keeps the
// last call's contents; calls whose kernels overlap on the GPU race on it.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_noalloc_scratch[PPF_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int NA_MAXDEV = 64;
constexpr size_t NA_STAGE = 32768;  // host staging of the tables (doubles)

struct NoallocDev {
    unsigned char* base = nullptr;  // device address of g_noalloc_scratch in context `ctx`
    unsigned long long ctx = 0;     // id of the CUDA context `base` and the tables belong to
    bool tables = false;            // tables of `last` are in the array
    ppf_desc last{};
};

// Unique id of the calling thread's current CUDA context (0 if the driver
// cannot tell).  A device reset or a new primary context gets a new id, and
// the static array is then a new allocation whose contents (the cached
// tables) are gone and whose address may differ, so the cache is keyed on it.
unsigned long long current_context_id()
{
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        looked_up = true;
        cudaDriverEntryPointQueryResult q;
        void* fn = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(fn);
        fn = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(fn);
    }
    if (!get_current || !get_id) return 0;
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (get_current(&c) != CUDA_SUCCESS || !c) return 0;
    if (get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

std::mutex g_na_mu;
NoallocDev g_na[NA_MAXDEV];
double g_na_stage[NA_STAGE];

size_t na_align(size_t v) { return (v + 255) & ~(size_t)255; }

bool same_desc(const ppf_desc& a, const ppf_desc& b)
{
    return a.n1m == b.n1m && a.n2m == b.n2m && a.n3m == b.n3m && a.L1 == b.L1 && a.L2 == b.L2 &&
           a.pbc1 == b.pbc1 && a.pbc2 == b.pbc2 && a.pbc3 == b.pbc3;
}

void na_cexp(int count, long double den, double* out)
{
    for (int k = 0; k < count; ++k) {
        long double a = -2.0L * PI_L * (long double)k / den;
        out[2 * k] = (double)cosl(a);
        out[2 * k + 1] = (double)sinl(a);
    }
}

}  // namespace

extern "C" int ppf_solve_noalloc(const ppf_desc* desc, const double* f_d, double* p_d, const double* dmx1_d,
                                 const double* dmx2_d, const double* dmx3_d, const double* dx3_d, void* stream)
{
    g_err[0] = 0;
    std::lock_guard<std::mutex> lk(g_na_mu);
    int rc = validate(desc);
    if (rc != PPF_OK) return rc;
    if (desc->precision != PPF_FP64) return fail(PPF_ERR_UNSUPPORTED, "ppf_solve_noalloc solves in FP64 only");
    if (!f_d || !p_d || !dmx1_d || !dmx2_d || !dmx3_d || !dx3_d) return fail(PPF_ERR_INVALID, "null array argument");
    int dev = -1;
    PPF_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NA_MAXDEV) return fail(PPF_ERR_UNSUPPORTED, "device index %d out of range", dev);
    NoallocDev& nd = g_na[dev];
    const unsigned long long ctx = current_context_id();   // 0 while no context is current yet
    if (!nd.base || ctx == 0 || ctx != nd.ctx) {
        // first call on this device, or in a new context after a device
        // reset: the device address of the array (the host-side symbol is
        // not a device address; the lookup also creates the device's primary
        // context if none is current) and the tables must be uploaded again
        void* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        nd.base = static_cast<unsigned char*>(ptr);
        nd.ctx = current_context_id();
        nd.tables = false;
    }

    // layout (the same as plan_init's for FP64), carved out of the array
    ppf_plan p;
    p.d = *desc;
    p.d.max_sweeps = 0;
    p.dev = dev;
    const int nx = desc->n1m, ny = desc->n2m, nz = desc->n3m;
    p.g.nx = nx; p.g.ny = ny; p.g.nz = nz;
    p.g.px = desc->pbc1 ? 1 : 0; p.g.py = desc->pbc2 ? 1 : 0; p.g.pz = desc->pbc3 ? 1 : 0;
    p.g.pstride_y = nx + 2;
    p.g.pstride_z = (long)(nx + 2) * (ny + 2);
    p.xdct = !desc->pbc1;
    p.ydct = !desc->pbc2;
    p.elem = 8;
    factor(nx / 2, p.sx);
    factor(ny, p.sy);
    const size_t ce = 16;
    const int nh = nx / 2 + 1;
    if (!p.xdct) {
        p.a_pitch = round_up(nh, 16);
        p.a_bytes = (size_t)p.a_pitch * ny * nz * ce;
        p.ycols = nh;
        p.b_pitch = p.a_pitch;
        p.ykind = p.ydct ? Y_CDCT : Y_C2C;
        p.mx = nh; p.my = ny;
        p.b_bytes = (size_t)p.b_pitch * ny * nz * ce;
        p.cplx = true;
    } else {
        p.a_pitch = round_up(nx, 32);
        p.a_bytes = (size_t)p.a_pitch * ny * nz * 8;
        p.ycols = nx / 2;
        if (p.ydct) {
            p.ykind = Y_CDCT; p.b_pitch = p.a_pitch; p.mx = nx; p.my = ny;
            p.b_bytes = (size_t)p.b_pitch * ny * nz * 8;
            p.cplx = false;
        } else {
            p.ykind = Y_RPAIR; p.b_pitch = round_up(nx, 16); p.mx = nx; p.my = ny / 2 + 1;
            p.b_bytes = (size_t)p.b_pitch * (ny / 2 + 1) * nz * ce;
            p.cplx = true;
        }
    }
    p.scale = 1.0 / ((p.xdct ? 2.0 * nx : (double)nx) * (p.ydct ? 2.0 * ny : (double)ny));
    // twiddle parts as upload_twiddles<double> lays them out
    const int tw_cnt[5] = { nx / 2, nx, nx, ny, ny };
    size_t tw_doubles = 0;
    for (int i = 0; i < 5; ++i) {
        p.tw_off[i] = tw_doubles / 2;
        tw_doubles += 2 * (size_t)tw_cnt[i];
        while (tw_doubles % 4) ++tw_doubles;
    }
    size_t off = 0;
    const size_t oA = off; off = na_align(off + p.a_bytes);
    const size_t oB = off; off = na_align(off + p.b_bytes);
    const size_t oLx = off; off = na_align(off + sizeof(double) * p.mx);
    const size_t oLy = off; off = na_align(off + sizeof(double) * p.my);
    const size_t oAm = off; off = na_align(off + sizeof(double) * nz);
    const size_t oAp = off; off = na_align(off + sizeof(double) * nz);
    const size_t oSc = off; off = na_align(off + sizeof(double) * 8);
    const size_t oFl = off; off = na_align(off + sizeof(int) * 4);
    const size_t oTw = off; off = na_align(off + sizeof(double) * tw_doubles);
    const size_t oCk = off; off = na_align(off + sizeof(double) * tdma_z_ckpt_doubles(nz, p.b_pitch * (long)p.my, p.g.pz, false));
    if (off > (size_t)PPF_NOALLOC_SCRATCH_BYTES)
        return fail(PPF_ERR_UNSUPPORTED,
                    "grid %dx%dx%d needs %zu bytes of work memory; ppf_solve_noalloc holds %zu (use ppf_plan_create)",
                    nx, ny, nz, off, (size_t)PPF_NOALLOC_SCRATCH_BYTES);
    if ((size_t)(p.mx + p.my) + tw_doubles > NA_STAGE)
        return fail(PPF_ERR_UNSUPPORTED, "table staging for %dx%d exceeds %zu values", nx, ny, NA_STAGE);
    unsigned char* b = nd.base;
    p.A = b + oA; p.B = b + oB;
    p.lamx = reinterpret_cast<double*>(b + oLx);
    p.lamy = reinterpret_cast<double*>(b + oLy);
    p.am = reinterpret_cast<double*>(b + oAm);
    p.ap = reinterpret_cast<double*>(b + oAp);
    p.scal = reinterpret_cast<double*>(b + oSc);
    p.flags = reinterpret_cast<int*>(b + oFl);
    p.tw = b + oTw;
    p.ckpt = reinterpret_cast<double*>(b + oCk);

    cudaStream_t st = (cudaStream_t)stream;
    if (!nd.tables || !same_desc(nd.last, *desc)) {
        // wavenumbers and twiddles, computed as plan_init does, staged in a
        // static host array (pageable copies return once the data is staged)
        double* lx = g_na_stage;
        double* ly = lx + p.mx;
        const double hx = desc->L1 / nx, hy = desc->L2 / ny;
        for (int i = 0; i < p.mx; ++i) lx[i] = p.xdct ? wn_dct(i, nx, hx) : wn_fft(i, nx, hx);
        for (int j = 0; j < p.my; ++j) {
            if (p.ydct) { ly[j] = wn_dct(j, ny, hy); continue; }
            int jm = j;
            if (!p.xdct && j + 1 > ny / 2 + 1) jm = ny - j;
            ly[j] = wn_fft(jm, ny, hy);
        }
        double* tw = ly + p.my;
        for (size_t q = 0; q < tw_doubles; ++q) tw[q] = 0.0;
        const long double den[5] = { (long double)(nx / 2), (long double)nx, 4.0L * nx, (long double)ny, 4.0L * ny };
        for (int i = 0; i < 5; ++i) na_cexp(tw_cnt[i], den[i], tw + 2 * p.tw_off[i]);
        nd.tables = false;
        PPF_CK(cudaMemcpyAsync(p.lamx, lx, sizeof(double) * p.mx, cudaMemcpyHostToDevice, st));
        PPF_CK(cudaMemcpyAsync(p.lamy, ly, sizeof(double) * p.my, cudaMemcpyHostToDevice, st));
        PPF_CK(cudaMemcpyAsync(p.tw, tw, sizeof(double) * tw_doubles, cudaMemcpyHostToDevice, st));
        nd.last = *desc;
        nd.tables = true;
    }
    PPF_CK(cudaMemsetAsync(p.scal, 0, sizeof(double) * 8, st));
    rc = solve_impl(&p, f_d, p_d, dmx1_d, dmx2_d, dmx3_d, dx3_d, st);
    p.ckpt = nullptr;
    return rc;
}

// ===========================================================================
// Batched solves of independent problems of uneven shape (ppf_batch_*).
//
// Each problem keeps a plan (tables, twiddles, schedules); the problems are
// spread over a few concurrent branches by estimated cost (longest first,
// each to the least-loaded branch), and every branch owns one set of work
// buffers sized for its largest problem, which its problems use in turn.
// The whole batch -- every problem's launches on its branch, branches
// forked from and joined to one origin -- is captured once into a CUDA
// graph and replayed with a single graph launch per ppf_batch_solve.
// With PPF_BATCH_AUTOTUNE, the tile width and radix order of every
// distinct x and y transform are picked by timing the candidates on the
// device before the capture.
// ===========================================================================
struct ppf_batch {
    std::vector<ppf_plan*> plans;
    std::vector<std::vector<int>> order;     // problems of each branch, in launch order
    std::vector<std::array<int, 8>> info;    // per problem: branch, x (w, rt, order), y (w, rt, order), 0
    std::vector<void*> work;                 // owned work buffers
    std::vector<cudaStream_t> streams;       // [0] capture origin, [1..] branches
    std::vector<cudaEvent_t> events;         // [0] fork, [1..] joins
    cudaGraphExec_t exec = nullptr;
    std::vector<const void*> key;            // pointers the graph was captured with
    int dev = 0;
    // the persistent work-queue form (PPF_BATCH_PERSISTENT): per-problem
    // descriptors and the task queue on the device, one kernel launch
    bool persistent = false;
    std::vector<BProb> probs;
    std::vector<BTask> tasks;
    BProb* probs_d = nullptr;
    BTask* tasks_d = nullptr;
    int* counters_d = nullptr;                // next tile, error bits, done tiles per task
    long total_tiles = 0;
    size_t pers_smem = 0;
    int pers_grid = 0;
};

namespace {

void free_batch(ppf_batch* b)
{
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    for (auto* p : b->plans) free_plan(p);
    for (void* w : b->work)
        if (w) cudaFree(w);
    for (auto s : b->streams)
        if (s) cudaStreamDestroy(s);
    for (auto e : b->events)
        if (e) cudaEventDestroy(e);
    for (void* q : { (void*)b->probs_d, (void*)b->tasks_d, (void*)b->counters_d })
        if (q) cudaFree(q);
    delete b;
}

// ---- persistent work-queue form ----------------------------------------

// widest power-of-two tile of the run-time engine for n-point lines at
// BATCH_THREADS threads (n * W <= 8 threads) and the x tiles' line tables
int batch_width(int n)
{
    int W = 1;
    while (2 * W <= 128 && (long)n * 2 * W <= 8L * BATCH_THREADS) W *= 2;
    return W;
}

// The stages of problem i, as solve_impl runs them, with tile counts.
void batch_stages(const ppf_plan* p, const BProb& q, int i, std::vector<BTask>& out)
{
    auto add = [&](int kind, long tiles, int arg, int skip) {
        BTask t{};
        t.kind = kind;
        t.prob = i;
        t.arg = arg;
        t.skip = skip;
        t.tiles = (int)std::max<long>(tiles, 1);
        t.dep = -1;
        out.push_back(t);
    };
    const long ztiles = (q.z.plane + BATCH_THREADS - 1) / BATCH_THREADS;
    auto pass = [&](int resid, int xinv_arg, int skip) {
        add(BK_XFWD, q.x_tiles, resid, skip);
        add(BK_YFWD, q.y_cblk * q.g.nz, 0, skip);
        add(BK_Z, ztiles, 0, skip);
        add(BK_YINV, q.y_cblk * q.g.nz, 0, skip);
        add(BK_XINV, q.x_tiles, xinv_arg, skip);
    };
    add(BK_ZCOEF, 1, 0, 0);
    if (p->elem == 8) {
        pass(0, 0 | 0 | (U_P << 2), 0);
    } else {
        const bool mixed = p->d.precision == PPF_MIXED;
        const bool u32 = mixed && p->d.max_sweeps > 0 && q.U;
        pass(0, (mixed ? 2 : 0) | ((u32 ? U_WRITE : U_P) << 2), 0);
        if (mixed) {
            add(BK_GATE, 1, 1, 0);
            for (int s = 0; s < p->d.max_sweeps; ++s) {
                const bool first = u32 && s == 0;
                pass(first ? 2 : 1, 1 | 2 | ((first ? U_ACC : U_P) << 2), 1);
                add(BK_GATE, 1, 0, 0);
            }
        }
    }
    // ghost cells: Neumann axes first, then periodic axes (launch_ghosts' order)
    const int per[3] = { p->g.px, p->g.py, p->g.pz };
    const long face[3] = { (long)(p->g.ny + 2) * (p->g.nz + 2), (long)(p->g.nx + 2) * (p->g.nz + 2),
                           (long)(p->g.nx + 2) * (p->g.ny + 2) };
    for (int pass_ = 0; pass_ < 2; ++pass_)
        for (int d = 0; d < 3; ++d) {
            const bool neumann = !per[d];
            if ((pass_ == 0) != neumann) continue;
            add(BK_GHOST, (face[d] + BATCH_THREADS - 1) / BATCH_THREADS, d | ((neumann ? 1 : 0) << 2), 0);
        }
}

// Per-problem work memory (every problem runs at once), descriptors and the
// task queue in stage-major order across the problems.
int batch_init_persistent(ppf_batch* b)
{
    const int count = (int)b->plans.size();
    b->persistent = true;
    b->probs.assign(count, BProb{});
    std::vector<std::vector<BTask>> lists(count);
    for (int i = 0; i < count; ++i) {
        ppf_plan* p = b->plans[i];
        BProb& q = b->probs[i];
        p->sx.rt = 1;
        p->sy.rt = 1;
        q.wx = batch_width(p->g.nx / 2);
        q.wy = batch_width(p->g.ny);
        q.lgwx = ilog2i(q.wx);
        q.lgwy = ilog2i(q.wy);
        p->sx.w = q.wx;
        p->sy.w = q.wy;
        q.x_tiles = ((long)p->g.ny * p->g.nz + q.wx - 1) / q.wx;
        q.y_cblk = (p->ycols + q.wy - 1) / q.wy;
        const bool mixed = p->d.precision == PPF_MIXED;
        const size_t ub = u_bytes(p);
        void *A = nullptr, *B = nullptr, *C = nullptr, *Pt = nullptr, *Uf = nullptr;
        if (cudaMalloc(&A, p->a_bytes) != cudaSuccess || cudaMalloc(&B, p->b_bytes) != cudaSuccess ||
            cudaMalloc(&C, sizeof(double) * std::max<long>(p->ckpt_doubles, 1)) != cudaSuccess ||
            (mixed && cudaMalloc(&Pt, sizeof(double) * 3 * q.x_tiles) != cudaSuccess) ||
            (ub && cudaMalloc(&Uf, ub) != cudaSuccess)) {
            cudaGetLastError();
            for (void* w : { A, B, C, Pt, Uf })
                if (w) cudaFree(w);
            return fail(PPF_ERR_NOMEM, "cannot allocate the work memory of problem %d", i);
        }
        for (void* w : { A, B, C, Pt, Uf })
            if (w) b->work.push_back(w);
        p->A = A; p->B = B; p->ckpt = (double*)C; p->partials = (double*)Pt; p->U = (float*)Uf;
        q.elem = (int)p->elem;
        q.mixed = mixed ? 1 : 0;
        q.xdct = p->xdct ? 1 : 0;
        q.ykind = p->ykind;
        q.cplx = p->cplx ? 1 : 0;
        q.g = p->g;
        ZSys& z = q.z;
        z.mx = p->mx; z.my = p->my; z.pitch = p->b_pitch; z.plane = p->b_pitch * (long)p->my; z.nz = p->g.nz;
        z.lamx = p->lamx; z.lamy = p->lamy; z.am = p->am; z.ap = p->ap; z.scale = p->scale;
        z.lowk = (p->d.precision == PPF_FP64) ? 0.0 : p->d.lowk_threshold;
        z.dzmin2 = p->scal;
        z.dc_shift = p->scal + 4;
        z.cyclic = p->g.pz;
        z.ckpt = p->ckpt;
        q.a_pitch = p->a_pitch;
        q.a_cp = p->xdct ? p->a_pitch / 2 : p->a_pitch;
        q.b_cp = (p->xdct && p->ydct) ? p->b_pitch / 2 : p->b_pitch;
        q.ycols = p->ycols;
        q.sx = p->sx;
        q.sy = p->sy;
        q.tw = p->tw;
        for (int k = 0; k < 5; ++k) q.tw_off[k] = (long)p->tw_off[k];
        q.A = A; q.B = B; q.U = (float*)Uf; q.partials = (double*)Pt;
        q.scal = p->scal;
        q.flags = p->flags;
        const double hx = p->d.L1 / p->g.nx, hy = p->d.L2 / p->g.ny;
        q.ix2 = 1.0 / (hx * hx);
        q.iy2 = 1.0 / (hy * hy);
        q.ncell = (double)p->g.nx * p->g.ny * p->g.nz;
        q.sweep_tol = p->d.sweep_tol;
        batch_stages(p, q, i, lists[i]);
        b->info[i][0] = 0;
        b->info[i][1] = q.wx; b->info[i][2] = 1; b->info[i][3] = 0;
        b->info[i][4] = q.wy; b->info[i][5] = 1; b->info[i][6] = 0;
    }
    // stage-major queue: every problem's first stage, then every second one, ...
    std::vector<int> at(count, 0);
    std::vector<int> last(count, -1);
    long first = 0;
    for (bool more = true; more;) {
        more = false;
        for (int i = 0; i < count; ++i) {
            if (at[i] >= (int)lists[i].size()) continue;
            more = true;
            BTask t = lists[i][at[i]++];
            t.dep = last[i];
            t.first = first;
            first += t.tiles;
            last[i] = (int)b->tasks.size();
            b->tasks.push_back(t);
        }
    }
    b->total_tiles = first;
    const int nt = (int)b->tasks.size();
    PPF_CK(cudaMalloc(&b->probs_d, sizeof(BProb) * count));
    PPF_CK(cudaMalloc(&b->tasks_d, sizeof(BTask) * nt));
    PPF_CK(cudaMalloc(&b->counters_d, sizeof(int) * (4 + (size_t)nt)));
    PPF_CK(cudaMemcpy(b->tasks_d, b->tasks.data(), sizeof(BTask) * nt, cudaMemcpyHostToDevice));
    b->pers_smem = batch_smem(b->probs.data(), count);
    cudaError_t e = batch_persistent_grid(b->pers_smem, &b->pers_grid);
    if (e != cudaSuccess) return cuda_fail(e, "persistent batch kernel occupancy");
    b->streams.assign(1, nullptr);
    PPF_CK(cudaStreamCreateWithFlags(&b->streams[0], cudaStreamNonBlocking));
    return PPF_OK;
}

// One graph: the queue counters reset and the persistent kernel.
int batch_capture_persistent(ppf_batch* b, const double* const* f, double* const* P, const double* const* m1,
                             const double* const* m2, const double* const* m3, const double* const* x3)
{
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    const int count = (int)b->probs.size();
    for (int i = 0; i < count; ++i) {
        BProb& q = b->probs[i];
        q.f = f[i]; q.P = P[i]; q.dmx1 = m1[i]; q.dmx2 = m2[i]; q.dmx3 = m3[i]; q.dx3 = x3[i];
    }
    // a launch still in flight reads the descriptors being replaced
    PPF_CK(cudaDeviceSynchronize());
    PPF_CK(cudaMemcpy(b->probs_d, b->probs.data(), sizeof(BProb) * count, cudaMemcpyHostToDevice));
    cudaStream_t o = b->streams[0];
    PPF_CK(cudaStreamBeginCapture(o, cudaStreamCaptureModeRelaxed));
    cudaError_t e = cudaMemsetAsync(b->counters_d, 0, sizeof(int) * (4 + b->tasks.size()), o);
    if (e == cudaSuccess)
        e = launch_batch_persistent(b->probs_d, b->tasks_d, (int)b->tasks.size(), b->total_tiles, b->counters_d,
                                    b->pers_smem, b->pers_grid, o);
    cudaGraph_t graph = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(o, &graph);
    int rc = PPF_OK;
    if (e != cudaSuccess) rc = cuda_fail(e, "persistent batch capture");
    else if (e2 != cudaSuccess) rc = cuda_fail(e2, "cudaStreamEndCapture");
    if (rc == PPF_OK) {
        e = cudaGraphInstantiate(&b->exec, graph, 0);
        if (e != cudaSuccess) {
            b->exec = nullptr;
            rc = cuda_fail(e, "cudaGraphInstantiate");
        }
    }
    if (graph) cudaGraphDestroy(graph);
    return rc;
}

struct TuneKey {
    int axis, n, kind, elem;
    bool operator<(const TuneKey& o) const
    {
        return std::tie(axis, n, kind, elem) < std::tie(o.axis, o.n, o.kind, o.elem);
    }
};
struct TuneChoice {
    FftSched s;
    int order;
};

// candidate schedules of one transform length: the compile-time shape when
// one exists, and run-time shapes over radix orders and tile widths
template <typename T>
std::vector<TuneChoice> tune_candidates(int n)
{
    std::vector<TuneChoice> out;
    TuneChoice base{};
    factor(n, base.s, 0);
    out.push_back(base);  // default (compile-time shape where one exists)
    int thr = 0;
    const int w0 = pick_w<T>(n, thr);
    for (int o = 0; o < 3; ++o) {
        TuneChoice c{};
        if (!factor(n, c.s, o)) continue;
        bool dup = false;
        for (int q = 0; q < o && !dup; ++q) {
            FftSched t{};
            factor(n, t, q);
            dup = (t.npass == c.s.npass) && std::equal(t.radix, t.radix + t.npass, c.s.radix);
        }
        if (dup) continue;
        for (int w : { w0 / 2, w0, 2 * w0, 4 * w0 }) {
            if (!width_ok<T>(n, w)) continue;
            TuneChoice r = c;
            r.s.rt = 1;
            r.s.w = w;
            r.order = o;
            out.push_back(r);
        }
    }
    return out;
}

template <typename T>
int time_axis(ppf_plan* p, int axis, const FftSched& s, const double* f, double* P, cudaStream_t st,
              cudaEvent_t e0, cudaEvent_t e1, float* ms)
{
    const cx<T>* tw = reinterpret_cast<const cx<T>*>(p->tw);
    const cx<T>* txh = tw + p->tw_off[0];
    const cx<T>* txn = tw + p->tw_off[1];
    const cx<T>* txd = tw + p->tw_off[2];
    const cx<T>* tyn = tw + p->tw_off[3];
    const cx<T>* tyd = tw + p->tw_off[4];
    const long a_cp = p->xdct ? p->a_pitch / 2 : p->a_pitch;
    const long b_cp = (p->xdct && p->ydct) ? p->b_pitch / 2 : p->b_pitch;
    auto run = [&]() -> cudaError_t {
        cudaError_t e;
        if (axis == 0) {
            e = launch_xfwd<T>(p->xdct, f, nullptr, p->g, p->A, p->a_pitch, s, txh, txn, txd, nullptr, st);
            if (e == cudaSuccess)
                e = launch_xinv<T>(p->xdct, p->A, p->a_pitch, P, nullptr, U_P, p->g, false, false, nullptr, nullptr, s, txh,
                                   txn, txd, nullptr, st);
        } else {
            e = launch_yfwd<T>(p->ykind, reinterpret_cast<const cx<T>*>(p->A), a_cp, reinterpret_cast<cx<T>*>(p->B),
                               b_cp, p->ycols, p->g, s, tyn, tyd, nullptr, st);
            if (e == cudaSuccess)
                e = launch_yinv<T>(p->ykind, reinterpret_cast<const cx<T>*>(p->B), b_cp,
                                   reinterpret_cast<cx<T>*>(p->A), a_cp, p->ycols, p->g, s, tyn, tyd, nullptr,
                                   nullptr, st);
        }
        return e;
    };
    cudaError_t e = run();  // warm-up (also sets the shared-memory attribute)
    if (e != cudaSuccess) return cuda_fail(e, "autotune");
    PPF_CK(cudaEventRecord(e0, st));
    for (int r = 0; r < 3; ++r) {
        e = run();
        if (e != cudaSuccess) return cuda_fail(e, "autotune");
    }
    PPF_CK(cudaEventRecord(e1, st));
    PPF_CK(cudaEventSynchronize(e1));
    PPF_CK(cudaEventElapsedTime(ms, e0, e1));
    return PPF_OK;
}

template <typename T>
int tune_plan(ppf_plan* p, std::map<TuneKey, TuneChoice>& cache, const double* f, double* P, cudaStream_t st,
              cudaEvent_t e0, cudaEvent_t e1, std::array<int, 8>& info)
{
    for (int axis = 0; axis < 2; ++axis) {
        const int n = axis == 0 ? p->g.nx / 2 : p->g.ny;
        const TuneKey key{ axis, n, axis == 0 ? (int)p->xdct : p->ykind, (int)p->elem };
        auto it = cache.find(key);
        if (it == cache.end()) {
            float best = 1e30f;
            TuneChoice pick{};
            for (const TuneChoice& c : tune_candidates<T>(n)) {
                float ms = 0.f;
                int rc = time_axis<T>(p, axis, c.s, f, P, st, e0, e1, &ms);
                if (rc != PPF_OK) return rc;
                if (ms < best) { best = ms; pick = c; }
            }
            it = cache.emplace(key, pick).first;
        }
        const TuneChoice& c = it->second;
        (axis == 0 ? p->sx : p->sy) = c.s;
        info[1 + 3 * axis] = c.s.w;
        info[2 + 3 * axis] = c.s.rt;
        info[3 + 3 * axis] = c.order;
    }
    return PPF_OK;
}

double est_cost(const ppf_plan* p)
{
    const double cells = (double)p->g.nx * p->g.ny * p->g.nz;
    const double passes = (p->d.precision == PPF_MIXED) ? 0.6 * (1 + p->d.max_sweeps * 1.4) : 1.0;
    return cells * passes;
}

int batch_init(ppf_batch* b, const ppf_desc* descs, int count, int flags, int branches)
{
    PPF_CK(cudaGetDevice(&b->dev));
    b->plans.assign(count, nullptr);
    b->info.assign(count, std::array<int, 8>{});
    for (int i = 0; i < count; ++i) {
        int rc = validate(&descs[i]);
        if (rc != PPF_OK) {
            char why[sizeof(g_err)];
            std::memcpy(why, g_err, sizeof(why));
            return fail(rc, "problem %d: %s", i, why);
        }
        ppf_plan* p = new (std::nothrow) ppf_plan();
        if (!p) return fail(PPF_ERR_NOMEM, "host allocation failed");
        b->plans[i] = p;
        p->own_work = false;
        p->batch_member = true;
        rc = plan_init(p, &descs[i]);
        if (rc != PPF_OK) return rc;
    }
    if (flags & PPF_BATCH_PERSISTENT) return batch_init_persistent(b);
    // autotune on temporary buffers sized for the largest problem
    if (flags & PPF_BATCH_AUTOTUNE) {
        size_t fa = 0, pa = 0, aa = 0, ba = 0;
        for (auto* p : b->plans) {
            fa = std::max(fa, sizeof(double) * (size_t)p->g.nx * p->g.ny * p->g.nz);
            pa = std::max(pa, sizeof(double) * (size_t)(p->g.nx + 2) * (p->g.ny + 2) * (p->g.nz + 2));
            aa = std::max(aa, p->a_bytes);
            ba = std::max(ba, p->b_bytes);
        }
        void *tf = nullptr, *tp = nullptr, *ta = nullptr, *tb = nullptr;
        cudaStream_t st = nullptr;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        int rc = PPF_OK;
        if (cudaMalloc(&tf, fa) != cudaSuccess || cudaMalloc(&tp, pa) != cudaSuccess ||
            cudaMalloc(&ta, aa) != cudaSuccess || cudaMalloc(&tb, ba) != cudaSuccess) {
            cudaGetLastError();
            rc = fail(PPF_ERR_NOMEM, "cannot allocate autotuning buffers");
        }
        if (rc == PPF_OK && (cudaMemset(tf, 0, fa) != cudaSuccess ||
                             cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess ||
                             cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess))
            rc = cuda_fail(cudaGetLastError(), "autotune setup");
        std::map<TuneKey, TuneChoice> cache;
        for (int i = 0; i < count && rc == PPF_OK; ++i) {
            ppf_plan* p = b->plans[i];
            p->A = ta;
            p->B = tb;
            rc = (p->elem == 8) ? tune_plan<double>(p, cache, (const double*)tf, (double*)tp, st, e0, e1, b->info[i])
                                : tune_plan<float>(p, cache, (const double*)tf, (double*)tp, st, e0, e1, b->info[i]);
            p->A = p->B = nullptr;
        }
        if (st) cudaStreamSynchronize(st);
        for (void* q : { tf, tp, ta, tb })
            if (q) cudaFree(q);
        if (st) cudaStreamDestroy(st);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (rc != PPF_OK) return rc;
    }
    // longest-first assignment to the least-loaded branch
    int nb = branches > 0 ? branches : 8;
    nb = std::max(1, std::min(nb, count));
    std::vector<int> idx(count);
    for (int i = 0; i < count; ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(),
                     [&](int x, int y) { return est_cost(b->plans[x]) > est_cost(b->plans[y]); });
    std::vector<double> load(nb, 0.0);
    b->order.assign(nb, {});
    for (int i : idx) {
        const int br = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        load[br] += est_cost(b->plans[i]);
        b->order[br].push_back(i);
        b->info[i][0] = br;
    }
    // one set of work buffers per branch, sized for its largest problem
    for (int br = 0; br < nb; ++br) {
        size_t aa = 0, ba = 0, ck = 0, pt = 0, ub = 0;
        for (int i : b->order[br]) {
            const ppf_plan* p = b->plans[i];
            ub = std::max(ub, u_bytes(p));
            aa = std::max(aa, p->a_bytes);
            ba = std::max(ba, p->b_bytes);
            ck = std::max(ck, (size_t)p->ckpt_doubles);
            pt = std::max(pt, (size_t)partials_doubles(p));
        }
        void *A = nullptr, *B = nullptr, *C = nullptr, *Pt = nullptr, *Uf = nullptr;
        if (cudaMalloc(&A, aa) != cudaSuccess || cudaMalloc(&B, ba) != cudaSuccess ||
            cudaMalloc(&C, sizeof(double) * std::max<size_t>(ck, 1)) != cudaSuccess ||
            (pt && cudaMalloc(&Pt, sizeof(double) * pt) != cudaSuccess) ||
            (ub && cudaMalloc(&Uf, ub) != cudaSuccess)) {
            cudaGetLastError();
            for (void* q : { A, B, C, Pt, Uf })
                if (q) cudaFree(q);
            return fail(PPF_ERR_NOMEM, "cannot allocate batch work memory for branch %d", br);
        }
        for (void* q : { A, B, C, Pt, Uf })
            if (q) b->work.push_back(q);
        for (int i : b->order[br]) {
            ppf_plan* p = b->plans[i];
            p->A = A;
            p->B = B;
            p->ckpt = (double*)C;
            p->U = u_bytes(p) ? (float*)Uf : nullptr;
            const long np = partials_doubles(p);
            p->partials = np ? (double*)Pt : nullptr;
            p->xinv_nblk = np / 3;
        }
    }
    b->streams.assign(nb + 1, nullptr);
    b->events.assign(nb + 1, nullptr);
    for (int s = 0; s <= nb; ++s) {
        PPF_CK(cudaStreamCreateWithFlags(&b->streams[s], cudaStreamNonBlocking));
        PPF_CK(cudaEventCreateWithFlags(&b->events[s], cudaEventDisableTiming));
    }
    return PPF_OK;
}

int batch_capture(ppf_batch* b, const double* const* f, double* const* P, const double* const* m1,
                  const double* const* m2, const double* const* m3, const double* const* x3)
{
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    cudaStream_t o = b->streams[0];
    PPF_CK(cudaStreamBeginCapture(o, cudaStreamCaptureModeRelaxed));
    int rc = PPF_OK;
    cudaError_t e = cudaEventRecord(b->events[0], o);
    const int nb = (int)b->order.size();
    for (int br = 0; br < nb && e == cudaSuccess; ++br) e = cudaStreamWaitEvent(b->streams[1 + br], b->events[0], 0);
    if (e != cudaSuccess) rc = cuda_fail(e, "batch capture");
    for (int br = 0; br < nb && rc == PPF_OK; ++br)
        for (int i : b->order[br]) {
            rc = solve_impl(b->plans[i], f[i], P[i], m1[i], m2[i], m3[i], x3[i], b->streams[1 + br]);
            if (rc != PPF_OK) break;
        }
    for (int br = 0; br < nb && rc == PPF_OK; ++br) {
        e = cudaEventRecord(b->events[1 + br], b->streams[1 + br]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(o, b->events[1 + br], 0);
        if (e != cudaSuccess) rc = cuda_fail(e, "batch capture");
    }
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(o, &graph);
    if (rc == PPF_OK && e != cudaSuccess) rc = cuda_fail(e, "cudaStreamEndCapture");
    if (rc == PPF_OK) {
        e = cudaGraphInstantiate(&b->exec, graph, 0);
        if (e != cudaSuccess) {
            b->exec = nullptr;
            rc = cuda_fail(e, "cudaGraphInstantiate");
        }
    }
    if (graph) cudaGraphDestroy(graph);
    return rc;
}

}  // namespace

extern "C" {

int ppf_batch_create(const ppf_desc* descs, int count, int flags, int branches, ppf_batch** batch)
{
    g_err[0] = 0;
    if (!batch) return fail(PPF_ERR_INVALID, "null batch pointer");
    *batch = nullptr;
    if (!descs || count < 1) return fail(PPF_ERR_INVALID, "empty batch");
    if (flags & ~(PPF_BATCH_AUTOTUNE | PPF_BATCH_PERSISTENT)) return fail(PPF_ERR_INVALID, "unknown batch flags 0x%x", flags);
    ppf_batch* b = new (std::nothrow) ppf_batch();
    if (!b) return fail(PPF_ERR_NOMEM, "host allocation failed");
    int rc = batch_init(b, descs, count, flags, branches);
    if (rc != PPF_OK) {
        free_batch(b);
        return rc;
    }
    *batch = b;
    return PPF_OK;
}

int ppf_batch_destroy(ppf_batch* batch)
{
    if (batch) cudaDeviceSynchronize();
    free_batch(batch);
    return PPF_OK;
}

int ppf_batch_solve(ppf_batch* batch, const double* const* f_d, double* const* p_d, const double* const* dmx1_d,
                    const double* const* dmx2_d, const double* const* dmx3_d, const double* const* dx3_d,
                    void* stream)
{
    if (!batch) return fail(PPF_ERR_INVALID, "null batch");
    if (!f_d || !p_d || !dmx1_d || !dmx2_d || !dmx3_d || !dx3_d) return fail(PPF_ERR_INVALID, "null pointer array");
    int cur = -1;
    PPF_CK(cudaGetDevice(&cur));
    if (cur != batch->dev) return fail(PPF_ERR_STATE, "batch was created on device %d, current is %d", batch->dev, cur);
    const int n = (int)batch->plans.size();
    std::vector<const void*> key;
    key.reserve(6 * (size_t)n);
    for (int i = 0; i < n; ++i) {
        if (!f_d[i] || !p_d[i] || !dmx1_d[i] || !dmx2_d[i] || !dmx3_d[i] || !dx3_d[i])
            return fail(PPF_ERR_INVALID, "null array argument of problem %d", i);
        key.insert(key.end(), { f_d[i], p_d[i], dmx1_d[i], dmx2_d[i], dmx3_d[i], dx3_d[i] });
    }
    if (!batch->exec || key != batch->key) {
        int rc = batch->persistent ? batch_capture_persistent(batch, f_d, p_d, dmx1_d, dmx2_d, dmx3_d, dx3_d)
                                   : batch_capture(batch, f_d, p_d, dmx1_d, dmx2_d, dmx3_d, dx3_d);
        if (rc != PPF_OK) {
            batch->key.clear();
            return rc;
        }
        batch->key = key;
    }
    PPF_CK(cudaGraphLaunch(batch->exec, (cudaStream_t)stream));
    return PPF_OK;
}

int ppf_ghost_update(double* P_d, int n1m, int n2m, int n3m, int pbc1, int pbc2, int pbc3, const double* dmx1_d,
                     const double* dmx2_d, const double* dmx3_d, int walls, void* stream)
{
    g_err[0] = 0;
    if (!P_d) return fail(PPF_ERR_INVALID, "ppf_ghost_update: null field");
    if (n1m < 1 || n2m < 1 || n3m < 1) return fail(PPF_ERR_INVALID, "ppf_ghost_update: empty grid");
    const int per[3] = { pbc1 ? 1 : 0, pbc2 ? 1 : 0, pbc3 ? 1 : 0 };
    const double* dmx[3] = { dmx1_d, dmx2_d, dmx3_d };
    if (walls)
        for (int d = 0; d < 3; ++d)
            if (!per[d] && !dmx[d]) return fail(PPF_ERR_INVALID, "ppf_ghost_update: wall axis %d needs its dmx", d + 1);
    const cudaError_t e = launch_ghost_update(P_d, n1m, n2m, n3m, per, dmx, walls, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "ppf_ghost_update");
    return PPF_OK;
}

int ppf_cell_to_node(const double* P_d, int n1m, int n2m, int n3m, const double* dx1_d, const double* dx2_d,
                     const double* dx3_d, double* G_d, void* stream)
{
    g_err[0] = 0;
    if (!P_d || !dx1_d || !dx2_d || !dx3_d || !G_d) return fail(PPF_ERR_INVALID, "ppf_cell_to_node: null array");
    if (n1m < 1 || n2m < 1 || n3m < 1) return fail(PPF_ERR_INVALID, "ppf_cell_to_node: empty grid");
    const cudaError_t e = launch_cell_to_node(P_d, n1m, n2m, n3m, dx1_d, dx2_d, dx3_d, G_d, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "ppf_cell_to_node");
    return PPF_OK;
}

int ppf_batch_info(const ppf_batch* batch, int index, int* info)
{
    if (!batch || !info) return fail(PPF_ERR_INVALID, "null argument");
    if (index < 0 || index >= (int)batch->plans.size()) return fail(PPF_ERR_INVALID, "index %d out of range", index);
    for (int k = 0; k < 8; ++k) info[k] = batch->info[index][k];
    info[7] = batch->persistent ? 0 : (int)batch->order.size();
    return PPF_OK;
}

}  // extern "C"
