// ppf_kernels.cuh -- launch interfaces of the libppf kernels.
#pragma once
#include <cuda_runtime.h>
#include "ppf_common.cuh"

namespace ppf {

// Geometry of a solve, as the kernels see it.
struct Geom {
    int nx, ny, nz;       // cells
    int px, py, pz;       // periodic flags
    long pstride_y;       // ghosted P strides (elements): (nx+2)
    long pstride_z;       // (nx+2)*(ny+2)
};

// Residual-input options of the x-forward pass (FP64 residual refinement).
struct ResidIn {
    const double* P;      // current iterate, ghosted layout (interior read)
    const float* U;       // or, when set, the FP32 first iterate (same ghosted layout)
    const double* am;     // z coefficient tables (nz)
    const double* ap;
    double ix2, iy2;      // 1/dx^2, 1/dy^2 (uniform x, y)
};

enum YKind { Y_C2C = 0, Y_CDCT = 1, Y_RPAIR = 2 };

// ---- transform launchers (ppf_x.cu, ppf_y.cu) ----
template <typename T>
cudaError_t launch_xfwd(bool dct, const double* f, const ResidIn* resid, const Geom& g,
                        void* out, long out_pitch, const FftSched& sch,
                        const cx<T>* tw_half, const cx<T>* tw_n, const cx<T>* tw_dct,
                        const int* skip_flag, cudaStream_t st);

template <typename T>
cudaError_t launch_yfwd(int kind, const cx<T>* in, long in_pitch, cx<T>* out, long out_pitch,
                        int ncols, const Geom& g, const FftSched& sch,
                        const cx<T>* tw_ny, const cx<T>* tw_dct, const int* skip_flag, cudaStream_t st,
                        int* err = nullptr);

template <typename T>
cudaError_t launch_yinv(int kind, const cx<T>* in, long in_pitch, cx<T>* out, long out_pitch,
                        int ncols, const Geom& g, const FftSched& sch,
                        const cx<T>* tw_ny, const cx<T>* tw_dct, const double* dc_shift,
                        const int* skip_flag, cudaStream_t st, int* err = nullptr);

// Where the x inverse reads and writes the iterate of a mixed solve.  The
// first iterate is made of FP32 values, so when a refinement sweep follows it
// is kept in an FP32 ghosted field U (half the bytes, the same values):
// U_P      accumulate reads P, the output goes to P (every other pass)
// U_WRITE  the output goes to U (first pass of a refining mixed solve)
// U_ACC    accumulate reads U, the output goes to P (its first sweep)
enum UKind { U_P = 0, U_WRITE = 1, U_ACC = 2 };

// x inverse into the ghosted output.  accumulate: u <- (u - *mean_prev) + du.
// partials (optional): per-block [sum du^2, sum u^2, sum u], 3 doubles per block.
template <typename T>
cudaError_t launch_xinv(bool dct, const void* in, long in_pitch, double* P, float* U, int ukind, const Geom& g,
                        bool accumulate, bool stencil_ghosts, double* partials, const double* mean_prev,
                        const FftSched& sch, const cx<T>* tw_half, const cx<T>* tw_n, const cx<T>* tw_dct,
                        const int* skip_flag, cudaStream_t st, long* blocks_used = nullptr, int* err = nullptr);

// upper bound of the blocks launch_xinv uses for geometry g (one per tile;
// size of the partials array / 3); the launch reports the blocks it used
template <typename T>
long xinv_blocks(const Geom& g, const FftSched& sch);

// ---- Poisson TDMA along z (ppf_tdma.cu) ----
struct ZSys {
    int mx, my;           // system grid (kx < mx, ky < my)
    long pitch;           // elements per spectral row (>= mx)
    long plane;           // elements per z plane (pitch * my)
    int nz;
    const double* lamx;   // eigenvalue tables (mx), (my)
    const double* lamy;
    const double* am;     // z coefficient tables (nz)
    const double* ap;
    double scale;         // normalisation folded into the solution
    double lowk;          // FP32 storage: systems with lam*dz_min^2 < lowk solve in FP64
    const double* dzmin2; // device scalar: min_k dx3_k^2 (written by the z-coefficient kernel)
    double* dc_shift;     // device scalar: z-average of the (0,0) solution (subtracted by the y inverse)
    int cyclic;           // periodic z: the reference's cyclic Thomas sequence
    int shared_gpu;       // other solves run beside this one (a batch): no whole-GPU streamed kernel
    double* ckpt;         // Thomas checkpoints, tdma_z_ckpt_doubles(nz, plane, cyclic, fp32) doubles
    float* ckpt_f;        // FP32 checkpoints of the FP32 bulk kernel (tdma_z_ckpt_f32), or null
    // FP32 storage, non-periodic z: the FP64 low-|k| systems
    int* lowk_count;      // device count (zeroed before the list is built)
    int* lowk_list;       // their indices (tdma_z_lowk_list), or null
    double* lowk_tab;     // coefficient table of the first groups (lowk_cap doubles), or null
    long lowk_cap;
    int lowk_build;       // first pass of a solve: fill the table before the z solve
};

// doubles of checkpoint memory the z solve needs (fp32: FP32 spectral storage)
long tdma_z_ckpt_doubles(int nz, long plane, int cyclic, bool fp32);
// start of the FP32 checkpoint region inside a checkpoint buffer of FP32 storage
float* tdma_z_ckpt_f32(double* ckpt, int nz, long plane, int cyclic);
// the low-|k| system list inside a checkpoint buffer of FP32 storage
int* tdma_z_lowk_list(double* ckpt, int nz, long plane, int cyclic);

// streams of the z solve: the FP32 bulk runs on st; the FP64 low-|k|
// systems run on aux (forked from and joined back to st through the two
// events) when aux is given, else on st after the bulk
struct ZStreams {
    cudaStream_t st;
    cudaStream_t aux;
    cudaEvent_t fork, join;
};

template <typename T, bool CPLX>
cudaError_t launch_tdma_z(void* data, const ZSys& z, const int* skip_flag, int* err_flag, const ZStreams& zs);

// the low-|k| system list of a mixed or FP32 solve (z.lowk_list), once per
// solve before its first z solve; a no-op where the list is not used
cudaError_t launch_lowk_list(const ZSys& z, cudaStream_t st);

cudaError_t launch_zcoef(const double* dx3, const double* dmx3, int nz, double* am, double* ap,
                         double* dzmin2, cudaStream_t st);

// ---- ghost cells (ppf_ghost.cu) ----
// zfaces: z faces to fill (1 lower, 2 upper; 3 for a whole domain, the
// ends of a z slab that are global walls for a slab)
cudaError_t launch_ghosts(double* P, const Geom& g, const double* dmx1, const double* dmx2,
                          const double* dmx3, cudaStream_t st, int zfaces = 3);

// ---- field IO of the example drivers (ppf_post.cu) ----
// ghost update of a ghosted field: walls != 0, the solve's (Neumann
// extrapolation on non-periodic axes with dmx[d], then periodic copies);
// walls == 0, only the periodic copies (the one-rank halo update)
cudaError_t launch_ghost_update(double* P, int n1m, int n2m, int n3m, const int* per, const double* const* dmx,
                                int walls, cudaStream_t st);
// node values (n1m, n2m, n3m) of a ghosted cell field for the 3-D instant field
cudaError_t launch_cell_to_node(const double* P, int n1m, int n2m, int n3m, const double* dx1, const double* dx2,
                                const double* dx3, double* G, cudaStream_t st);

// ---- z-slab pieces of the multi-rank solve (ppf_slab.cu) ----
cudaError_t launch_slab_coef(double* a, double* b, double* c, double* d, long ns, int nzl, int cplx, long pitch,
                             int mx, const double* lamx, const double* lamy, const double* dx3, const double* dmx3,
                             int z0, int nzg, double scale, cudaStream_t st);
long slab_sum_parts(const Geom& g);
cudaError_t launch_slab_sum(const double* P, const Geom& g, double* part, double* sum, cudaStream_t st);
cudaError_t launch_slab_shift(double* P, const Geom& g, const double* shift, cudaStream_t st);

// ---- generic batched TDMA on coefficient arrays (ppf_tdma.cu) ----
cudaError_t launch_tdma_many(const double* a, const double* b, const double* c, double* d,
                             int n_sys, int n_row, bool cyclic, int* err, cudaStream_t st);

// ---- rows split over ranks: PaScaL modified Thomas and update (ppf_tdma.cu) ----
cudaError_t launch_tdma_modified(double* a, const double* b, double* c, double* d, double* a_rd, double* c_rd,
                                 double* d_rd, long n_sys, int n_row, cudaStream_t st);
cudaError_t launch_tdma_update(const double* a, const double* c, double* d, const double* x_rd, long n_sys, int n_row,
                               cudaStream_t st);

// Refinement bookkeeping after an x-inverse pass with partials: reduces the
// partials in a fixed order, stores mean(u) for the next accumulate pass,
// and unless `initial`: counts the sweep, records ||du||/||u|| and closes
// the gate (skip_flag) below tol.
cudaError_t launch_sweep_gate(const double* partials, long nblocks, double ncell, double* mean_prev,
                              int* skip_flag, int* sweeps_done, double* last_rel, double tol, int initial,
                              cudaStream_t st);

// ---- transpose of the solve and z-metric gradient (ppf_adjoint.cu) ----
// per-level reductions run over nchunk blocks of `chunk` cells of a plane
int adjoint_chunks(long plane, long* chunk);
cudaError_t launch_adj_rhs(const double* g, double* h, const double* dx3, const Geom& gm, long chunk, int nchunk,
                           double* colpart, cudaStream_t st);
cudaError_t launch_adj_corr(const double* colpart, int nchunk, const Geom& gm, const double* am, const double* ap,
                            double* corr, double* wk, cudaStream_t st);
cudaError_t launch_adj_out(const double* W, double* df, const double* dx3, const double* corr, const double* u,
                           const Geom& gm, long chunk, int nchunk, double* mpart, cudaStream_t st);
cudaError_t launch_adj_metric(const double* mpart, int nchunk, const Geom& gm, const double* am, const double* ap,
                              const double* dx3, const double* dmx3, double* ddx3, double* ddmx3, double* wk,
                              cudaStream_t st);

}  // namespace ppf
