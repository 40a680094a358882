// ppf_batch.cuh -- the persistent work-queue form of a batch of independent
// solves (ppf_batch_create with PPF_BATCH_PERSISTENT): problem and task
// descriptors shared by the host side (ppf_api.cu) and the kernel
// (ppf_batch.cu).
#pragma once
#include "ppf_kernels.cuh"

namespace ppf {

// Everything one problem's stages need, resolved on the host: geometry,
// transform schedules and tile widths of the run-time engine, the z system,
// and the problem's own work and output memory.
struct BProb {
    int elem;             // 8: FP64 spectra; 4: FP32 spectra
    int mixed;            // PPF_MIXED: refinement partial sums, stencil ghosts
    int xdct, ykind, cplx;
    Geom g;
    ZSys z;
    long a_pitch, a_cp, b_cp;
    int ycols;
    FftSched sx, sy;      // run-time schedules (rt = 1)
    int wx, lgwx, wy, lgwy;
    long x_tiles, y_cblk;  // x tiles (W lines), y column blocks per plane
    const void* tw;       // twiddle tables (elem type), offsets as the plan's
    long tw_off[5];
    void* A;
    void* B;
    float* U;             // FP32 first iterate of a refining mixed solve, or null
    double* partials;     // 3 doubles per x-inverse tile (mixed), or null
    double* scal;         // the plan's scalars: [0] min dz^2, [3] ||du||/||u||, [4] zero-mode shift, [5] mean
    int* flags;           // [0] skip, [1] sweeps done, [2] error
    const double* f;
    double* P;
    const double* dmx1;
    const double* dmx2;
    const double* dmx3;
    const double* dx3;
    double ix2, iy2;      // 1/dx^2, 1/dy^2 of the residual
    double ncell;
    double sweep_tol;
};

// Stage kinds of a solve, in the order solve_impl runs them.
enum BKind { BK_ZCOEF = 0, BK_XFWD, BK_YFWD, BK_Z, BK_YINV, BK_XINV, BK_GATE, BK_GHOST };

// One stage of one problem: `tiles` work items, all of which may start once
// every tile of task `dep` (the problem's previous stage, -1: none) is done.
// Tasks are stored in queue order; `first` is the global index of the first
// tile.  arg: XFWD residual input (0 none, 1 P, 2 U); XINV (ACC, GHOST, UKind)
// as ACC | GHOST << 1 | UKind << 2, partial sums when the problem is mixed;
// GATE 1 = initial; GHOST axis | neumann << 2; `skip` 1: the stage belongs
// to a refinement sweep and honours the problem's gate.
struct BTask {
    int kind, prob, arg, skip;
    int tiles, dep;
    long first;
};

// Threads of every CTA of the persistent kernel (the run-time transform
// tiles are sized for it: n * W <= 8 * BATCH_THREADS).
constexpr int BATCH_THREADS = 512;

// Dynamic shared memory the kernel needs for the problems (the largest x or
// y tile), and the launch of one pass over the whole queue.  counters:
// [0..1] next tile (64 bit), [2] error bits (1 non-finite, 4 a dependency
// wait gave up), [4 ..] done tiles per task; zeroed before every launch.
size_t batch_smem(const BProb* probs, int count);
cudaError_t launch_batch_persistent(const BProb* probs_d, const BTask* tasks_d, int ntasks, long total_tiles,
                                    int* counters_d, size_t smem, int grid, cudaStream_t st);
// CTAs of the kernel resident on the device (the persistent grid)
cudaError_t batch_persistent_grid(size_t smem, int* grid);

}  // namespace ppf
