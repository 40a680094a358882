"""pascal_poisson_fft_b200 -- host-side mirror of the PaScaL_POISSON_FFT solve API.

The compute path is libppf.so (hand-written sm_100a CUDA kernels behind the
C ABI declared in include/ppf.h), loaded here with ctypes.  This module adds
nothing to the arithmetic: it marshals pointers, mirrors the reference's
call sequence and names, and builds the reference's mesh metrics on the
host.  There is no CPU fallback: if libppf.so is missing or no CUDA device
is present, every call raises.

Reference-shaped API (01_Fortran/src/fft_3d_poisson.f90):
    fft_poisson_plan_cuda_create(n1, n2, n3, L1, L2, L3, pbc1, pbc2, pbc3)   :70-108
    cuda_Poisson_FFT_initial()                                               :110-121
    cuda_Poisson_FFT_1D(PRHS_d, P_d, dmx1_d, dmx2_d, dmx3_d, dx3_d)           :353-626
    cuda_Poisson_FFT_clean()                                                  :123-130
PaScaL_TDMA (01_Fortran/PaScaL_TDMA/src/pascal_tdma_cuda.f90:230-318):
    PaScaL_TDMA_many_solve_cuda(a, b, c, d), PaScaL_TDMA_many_solve_cycle_cuda(...)
Handle API: Plan(...).solve(f, P, dmx1, dmx2, dmx3, dx3)

Device arrays are torch CUDA tensors (float64, contiguous) laid out as the
reference's Fortran arrays with the axes reversed: PRHS(1:n1m,1:n2m,1:n3m)
is a tensor of shape (n3m, n2m, n1m); the ghosted P(0:n1m+1,0:n2m+1,0:n3m+1)
has shape (n3m+2, n2m+2, n1m+2).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

__all__ = [
    "PPF_FP64", "PPF_MIXED", "PPF_FP32", "PPF_BATCH_AUTOTUNE", "PPFError", "lib", "Plan", "Batch", "mesh",
    "fft_poisson_plan_cuda_create", "cuda_Poisson_FFT_initial", "cuda_Poisson_FFT_1D",
    "cuda_Poisson_FFT_clean", "PaScaL_TDMA_many_solve_cuda", "PaScaL_TDMA_many_solve_cycle_cuda",
    "tdma_many", "tdma_cycl_many", "EXPORTED_SYMBOLS",
]

PPF_FP64, PPF_MIXED, PPF_FP32 = 0, 1, 2
_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libppf.so")

# every symbol include/ppf.h declares
EXPORTED_SYMBOLS = (
    "ppf_plan_create", "ppf_plan_destroy", "ppf_solve", "ppf_solve_host", "ppf_last_sweeps",
    "ppf_plan_workspace_bytes", "ppf_tdma_many", "ppf_tdma_cycl_many", "ppf_last_error", "ppf_version",
    "ppf_fft_poisson_plan_cuda_create", "ppf_cuda_poisson_fft_initial", "ppf_cuda_poisson_fft_1d",
    "ppf_cuda_poisson_fft_clean", "ppf_cuda_poisson_fft_set_precision", "ppf_stage_timing",
    "ppf_stage_times", "ppf_solve_noalloc", "ppf_solve_adjoint", "ppf_batch_create", "ppf_batch_destroy",
    "ppf_batch_solve", "ppf_batch_info", "ppf_solve_host_async", "ppf_tdma_many_modified",
    "ppf_tdma_many_update", "ppf_slab_systems", "ppf_slab_forward", "ppf_slab_coefficients",
    "ppf_slab_inverse", "ppf_slab_sum", "ppf_slab_shift", "ppf_slab_ghosts", "ppf_ghost_update",
    "ppf_cell_to_node",
)
PPF_BATCH_AUTOTUNE = 1
PPF_BATCH_PERSISTENT = 2
STAGES = ("z-coefficients", "x-forward", "y-forward", "tdma-z", "y-inverse", "x-inverse",
          "refine-gate", "ghost-cells")


class PPFError(RuntimeError):
    """A libppf entry point returned a non-zero status."""

    def __init__(self, func: str, code: int, msg: str):
        super().__init__(f"{func} failed ({code}): {msg}")
        self.code = code


class _Desc(ctypes.Structure):
    _fields_ = [("n1m", ctypes.c_int), ("n2m", ctypes.c_int), ("n3m", ctypes.c_int),
                ("L1", ctypes.c_double), ("L2", ctypes.c_double),
                ("pbc1", ctypes.c_int), ("pbc2", ctypes.c_int), ("pbc3", ctypes.c_int),
                ("precision", ctypes.c_int), ("max_sweeps", ctypes.c_int),
                ("sweep_tol", ctypes.c_double), ("lowk_threshold", ctypes.c_double)]


_LIB = None
_vp = ctypes.c_void_p


def lib() -> ctypes.CDLL:
    """Load libppf.so (built in-tree by pascal_poisson_fft_b200/build.py)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise PPFError("load", -1, f"{LIB_PATH} is missing; run pascal_poisson_fft_b200/build.py")
    L = ctypes.CDLL(LIB_PATH)
    L.ppf_last_error.restype = ctypes.c_char_p
    L.ppf_version.restype = ctypes.c_char_p
    L.ppf_plan_create.argtypes = [ctypes.POINTER(_Desc), ctypes.POINTER(_vp)]
    L.ppf_plan_destroy.argtypes = [_vp]
    L.ppf_solve.argtypes = [_vp] + [_vp] * 6 + [_vp]
    L.ppf_solve_host.argtypes = [_vp] + [_vp] * 6 + [_vp]
    L.ppf_solve_host_async.argtypes = [_vp] + [_vp] * 6 + [_vp]
    L.ppf_last_sweeps.argtypes = [_vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double), _vp]
    L.ppf_plan_workspace_bytes.argtypes = [_vp, ctypes.POINTER(ctypes.c_longlong)]
    L.ppf_tdma_many.argtypes = [_vp] * 4 + [ctypes.c_int, ctypes.c_int, _vp]
    L.ppf_tdma_cycl_many.argtypes = [_vp] * 4 + [ctypes.c_int, ctypes.c_int, _vp]
    L.ppf_tdma_many_modified.argtypes = [_vp] * 7 + [ctypes.c_int, ctypes.c_int, _vp]
    L.ppf_tdma_many_update.argtypes = [_vp] * 4 + [ctypes.c_int, ctypes.c_int, _vp]
    L.ppf_slab_systems.argtypes = [_vp, ctypes.POINTER(ctypes.c_int)]
    L.ppf_slab_forward.argtypes = [_vp] * 3 + [_vp]
    L.ppf_slab_coefficients.argtypes = [_vp] * 7 + [ctypes.c_int, ctypes.c_int, _vp]
    L.ppf_slab_inverse.argtypes = [_vp] * 3 + [_vp]
    L.ppf_slab_sum.argtypes = [_vp] * 3 + [_vp]
    L.ppf_slab_shift.argtypes = [_vp] * 3 + [_vp]
    L.ppf_slab_ghosts.argtypes = [_vp] * 5 + [ctypes.c_int, ctypes.c_int, _vp]
    L.ppf_fft_poisson_plan_cuda_create.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 3 + [ctypes.c_int] * 3
    L.ppf_cuda_poisson_fft_1d.argtypes = [_vp] * 6
    L.ppf_cuda_poisson_fft_set_precision.argtypes = [ctypes.c_int, ctypes.c_int]
    L.ppf_stage_timing.argtypes = [_vp, ctypes.c_int]
    L.ppf_solve_noalloc.argtypes = [ctypes.POINTER(_Desc)] + [_vp] * 6 + [_vp]
    L.ppf_stage_times.argtypes = [_vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)]
    L.ppf_solve_adjoint.argtypes = [_vp] * 10 + [_vp]
    L.ppf_batch_create.argtypes = [ctypes.POINTER(_Desc), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   ctypes.POINTER(_vp)]
    L.ppf_batch_destroy.argtypes = [_vp]
    L.ppf_batch_solve.argtypes = [_vp] + [ctypes.POINTER(_vp)] * 6 + [_vp]
    L.ppf_batch_info.argtypes = [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.ppf_ghost_update.argtypes = [_vp] + [ctypes.c_int] * 6 + [_vp] * 3 + [ctypes.c_int, _vp]
    L.ppf_cell_to_node.argtypes = [_vp] + [ctypes.c_int] * 3 + [_vp] * 5
    for name in ("ppf_last_error", "ppf_version", "ppf_cuda_poisson_fft_initial", "ppf_cuda_poisson_fft_clean"):
        getattr(L, name).argtypes = []
    for name in EXPORTED_SYMBOLS:
        if name not in ("ppf_last_error", "ppf_version"):
            getattr(L, name).restype = ctypes.c_int
    _LIB = L
    return L


def _check(func: str, rc: int) -> None:
    if rc != 0:
        msg = lib().ppf_last_error().decode(errors="replace")
        raise PPFError(func, rc, msg)


def _dptr(t, name: str, numel: int | None = None) -> int:
    """Device pointer of a contiguous float64 CUDA tensor (validated)."""
    import torch
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch CUDA tensor")
    if not t.is_cuda or t.dtype != torch.float64 or not t.is_contiguous():
        raise TypeError(f"{name} must be a contiguous float64 CUDA tensor")
    if numel is not None and t.numel() != numel:
        raise ValueError(f"{name} has {t.numel()} elements, expected {numel}")
    return t.data_ptr()


def _stream_ptr(stream) -> int | None:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


def mesh(nm: int, L: float, uniform: bool = True, gamma: float = 0.0, pbc: bool = True):
    """Faces x(0:nm+1), widths dx(0:nm+1), centre spacings dmx(0:nm+1) of one
    axis at one rank, as 01_Fortran/examples/mpi_subdomain.f90:397-472 builds
    them (uniform, or tanh-stretched with parameter gamma; a stretch
    beta in z_k = (1 + tanh(beta (2k/N - 1))/tanh(beta))/2 is gamma = 2 beta)."""
    idx = np.arange(0, nm + 2, dtype=np.float64)
    if uniform:
        x = (idx - 1) * L / nm
    else:
        x = L * 0.5 * (1.0 + np.tanh(0.5 * gamma * (2.0 * (idx - 1) / nm - 1.0)) / np.tanh(gamma * 0.5))
    if not pbc:
        x[0] = x[1]
    n = nm + 1
    dx = np.zeros(nm + 2)
    dmx = np.zeros(nm + 2)
    dx[1:nm + 1] = x[2:nm + 2] - x[1:nm + 1]
    if pbc:
        dx[0], dx[n] = dx[nm], dx[1]
    dmx[1:nm + 1] = 0.5 * (dx[0:nm] + dx[1:nm + 1])
    if pbc:
        dmx[0], dmx[n] = dmx[nm], dmx[1]
    else:
        dmx[n] = 0.5 * (dx[nm] + dx[n])
    return x, dx, dmx


@dataclass
class Metrics:
    """Device copies of the four metric arrays cuda_Poisson_FFT_1D takes."""
    dmx1: object
    dmx2: object
    dmx3: object
    dx3: object


class Plan:
    """A libppf plan (handle API).  precision: PPF_FP64 (the reference's),
    PPF_MIXED (FP32 transforms + FP64 residual refinement) or PPF_FP32."""

    def __init__(self, n1m, n2m, n3m, L1, L2, pbc1=True, pbc2=True, pbc3=False,
                 precision=PPF_FP64, max_sweeps=-1, sweep_tol=0.0, lowk_threshold=0.0):
        d = _Desc(n1m, n2m, n3m, float(L1), float(L2), int(bool(pbc1)), int(bool(pbc2)), int(bool(pbc3)),
                  int(precision), int(max_sweeps), float(sweep_tol), float(lowk_threshold))
        self.desc = d
        self.shape = (n3m, n2m, n1m)
        self.gshape = (n3m + 2, n2m + 2, n1m + 2)
        self._h = _vp()
        _check("ppf_plan_create", lib().ppf_plan_create(ctypes.byref(d), ctypes.byref(self._h)))

    def close(self) -> None:
        if self._h:
            lib().ppf_plan_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def workspace_bytes(self) -> int:
        b = ctypes.c_longlong()
        _check("ppf_plan_workspace_bytes", lib().ppf_plan_workspace_bytes(self._h, ctypes.byref(b)))
        return b.value

    def solve(self, f, P, dmx1, dmx2, dmx3, dx3, stream=None) -> None:
        """Asynchronous device solve: f (n3m,n2m,n1m) -> ghosted P."""
        n3m, n2m, n1m = self.shape
        args = [_dptr(f, "f", n1m * n2m * n3m), _dptr(P, "P", (n1m + 2) * (n2m + 2) * (n3m + 2)),
                _dptr(dmx1, "dmx1", n1m + 2), _dptr(dmx2, "dmx2", n2m + 2),
                _dptr(dmx3, "dmx3", n3m + 2), _dptr(dx3, "dx3", n3m + 2)]
        _check("ppf_solve", lib().ppf_solve(self._h, *args, _stream_ptr(stream)))

    def solve_adjoint(self, g, df, dmx1, dmx2, dmx3, dx3, u=None, ddx3=None, ddmx3=None,
                      stream=None) -> None:
        """Asynchronous transpose solve: df = M^T g (both (n3m,n2m,n1m)); with
        the forward solution u (ghosted) also d<g,u>/d dx3 and d<g,u>/d dmx3
        into ddx3, ddmx3 (n3m+2 each)."""
        n3m, n2m, n1m = self.shape
        cells = n1m * n2m * n3m
        up = _dptr(u, "u", (n1m + 2) * (n2m + 2) * (n3m + 2)) if u is not None else None
        gx = _dptr(ddx3, "ddx3", n3m + 2) if ddx3 is not None else None
        gm = _dptr(ddmx3, "ddmx3", n3m + 2) if ddmx3 is not None else None
        args = [_dptr(g, "g", cells), _dptr(df, "df", cells), up, gx, gm,
                _dptr(dmx1, "dmx1", n1m + 2), _dptr(dmx2, "dmx2", n2m + 2),
                _dptr(dmx3, "dmx3", n3m + 2), _dptr(dx3, "dx3", n3m + 2)]
        _check("ppf_solve_adjoint", lib().ppf_solve_adjoint(self._h, *args, _stream_ptr(stream)))

    def solve_host(self, f: np.ndarray, dmx1, dmx2, dmx3, dx3, P: np.ndarray | None = None,
                   stream=None) -> np.ndarray:
        """Host-array solve (copies in and out, synchronous)."""
        n3m, n2m, n1m = self.shape
        f = np.ascontiguousarray(f, dtype=np.float64)
        if f.shape != self.shape:
            raise ValueError(f"f has shape {f.shape}, expected {self.shape}")
        if P is None:
            P = np.empty(self.gshape)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (dmx1, dmx2, dmx3, dx3)]
        _check("ppf_solve_host", lib().ppf_solve_host(
            self._h, f.ctypes.data, P.ctypes.data, *[a.ctypes.data for a in arrs],
            _stream_ptr(stream) if stream is not None else None))
        return P

    def solve_host_async(self, f, P, dmx1, dmx2, dmx3, dx3, stream) -> None:
        """Enqueue copy-in, solve and copy-out of host arrays on `stream`
        (page-locked torch CPU tensors for asynchronous copies); returns at once."""
        n3m, n2m, n1m = self.shape
        cells, ghosted = n1m * n2m * n3m, (n1m + 2) * (n2m + 2) * (n3m + 2)
        ptrs = []
        for name, t, numel in (("f", f, cells), ("P", P, ghosted), ("dmx1", dmx1, n1m + 2),
                               ("dmx2", dmx2, n2m + 2), ("dmx3", dmx3, n3m + 2), ("dx3", dx3, n3m + 2)):
            if t.device.type != "cpu" or t.dtype.itemsize != 8 or not t.is_contiguous() or t.numel() != numel:
                raise TypeError(f"{name} must be a contiguous float64 host tensor of {numel} elements")
            ptrs.append(t.data_ptr())
        _check("ppf_solve_host_async", lib().ppf_solve_host_async(self._h, *ptrs, _stream_ptr(stream)))

    def stage_timing(self, enable: bool) -> None:
        _check("ppf_stage_timing", lib().ppf_stage_timing(self._h, int(bool(enable))))

    def stage_times(self):
        """{stage: (ms, launches)} accumulated since the last call."""
        ms = (ctypes.c_double * len(STAGES))()
        n = (ctypes.c_int * len(STAGES))()
        _check("ppf_stage_times", lib().ppf_stage_times(self._h, ms, n))
        return {s: (ms[k], n[k]) for k, s in enumerate(STAGES)}

    def last_sweeps(self, stream=None):
        s = ctypes.c_int()
        r = ctypes.c_double()
        _check("ppf_last_sweeps", lib().ppf_last_sweeps(self._h, ctypes.byref(s), ctypes.byref(r),
                                                        _stream_ptr(stream)))
        return s.value, r.value


class Batch:
    """Independent problems of uneven shape solved by one graph launch.

    problems: sequence of dicts with keys n1m, n2m, n3m, L1, L2, pbc (3-tuple),
    and optionally precision, max_sweeps, sweep_tol, lowk_threshold.
    persistent: run the batch as one persistent work-queue kernel instead of
    per-problem kernels on concurrent branches (autotune then has no effect)."""

    def __init__(self, problems, autotune=True, branches=0, persistent=False):
        descs = (_Desc * len(problems))()
        self.shapes = []
        for k, q in enumerate(problems):
            pbc = q.get("pbc", (1, 1, 0))
            descs[k] = _Desc(q["n1m"], q["n2m"], q["n3m"], float(q["L1"]), float(q["L2"]),
                             int(bool(pbc[0])), int(bool(pbc[1])), int(bool(pbc[2])),
                             int(q.get("precision", PPF_FP64)), int(q.get("max_sweeps", -1)),
                             float(q.get("sweep_tol", 0.0)), float(q.get("lowk_threshold", 0.0)))
            self.shapes.append((q["n3m"], q["n2m"], q["n1m"]))
        self._h = _vp()
        flags = (PPF_BATCH_AUTOTUNE if autotune else 0) | (PPF_BATCH_PERSISTENT if persistent else 0)
        _check("ppf_batch_create", lib().ppf_batch_create(descs, len(problems), flags, int(branches),
                                                          ctypes.byref(self._h)))

    def __len__(self):
        return len(self.shapes)

    def close(self) -> None:
        if self._h:
            lib().ppf_batch_destroy(self._h)
            self._h = _vp()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, fs, Ps, dmx1s, dmx2s, dmx3s, dx3s, stream=None) -> None:
        """Asynchronous: every problem k solves fs[k] -> Ps[k] (torch CUDA float64)."""
        n = len(self.shapes)
        arrs = []
        for name, ts, extra in (("f", fs, 0), ("P", Ps, 2), ("dmx1", dmx1s, -1), ("dmx2", dmx2s, -2),
                                ("dmx3", dmx3s, -3), ("dx3", dx3s, -3)):
            if len(ts) != n:
                raise ValueError(f"{name}: {len(ts)} arrays for {n} problems")
            a = (_vp * n)()
            for k, t in enumerate(ts):
                n3m, n2m, n1m = self.shapes[k]
                numel = {0: n1m * n2m * n3m, 2: (n1m + 2) * (n2m + 2) * (n3m + 2),
                         -1: n1m + 2, -2: n2m + 2, -3: n3m + 2}[extra]
                a[k] = _dptr(t, f"{name}[{k}]", numel)
            arrs.append(a)
        _check("ppf_batch_solve", lib().ppf_batch_solve(self._h, *arrs, _stream_ptr(stream)))

    def info(self, k: int) -> dict:
        v = (ctypes.c_int * 8)()
        _check("ppf_batch_info", lib().ppf_batch_info(self._h, int(k), v))
        return dict(branch=v[0], x_width=v[1], x_runtime=v[2], x_order=v[3],
                    y_width=v[4], y_runtime=v[5], y_order=v[6], branches=v[7])


# ---- reference-shaped module API ------------------------------------------

def fft_poisson_plan_cuda_create(n1, n2, n3, L1, L2, L3, pbc1, pbc2, pbc3,
                                 precision=PPF_FP64, max_sweeps=-1) -> None:
    """fft_poisson_plan_cuda_create at one rank (n1, n2, n3 are face counts)."""
    _check("ppf_cuda_poisson_fft_set_precision", lib().ppf_cuda_poisson_fft_set_precision(precision, max_sweeps))
    _check("ppf_fft_poisson_plan_cuda_create", lib().ppf_fft_poisson_plan_cuda_create(
        n1, n2, n3, float(L1), float(L2), float(L3), int(bool(pbc1)), int(bool(pbc2)), int(bool(pbc3))))


def cuda_Poisson_FFT_initial() -> None:
    _check("ppf_cuda_poisson_fft_initial", lib().ppf_cuda_poisson_fft_initial())


def cuda_Poisson_FFT_1D(PRHS_d, P_d, dmx1_d, dmx2_d, dmx3_d, dx3_d) -> None:
    """Synchronous solve on the legacy default stream, like the reference."""
    ptrs = [_dptr(t, n) for t, n in ((PRHS_d, "PRHS_d"), (P_d, "P_d"), (dmx1_d, "dmx1_d"),
                                     (dmx2_d, "dmx2_d"), (dmx3_d, "dmx3_d"), (dx3_d, "dx3_d"))]
    _check("ppf_cuda_poisson_fft_1d", lib().ppf_cuda_poisson_fft_1d(*ptrs))


def cuda_Poisson_FFT_clean() -> None:
    _check("ppf_cuda_poisson_fft_clean", lib().ppf_cuda_poisson_fft_clean())


# ---- batched tridiagonal solves -------------------------------------------

def tdma_many(a, b, c, d, stream=None) -> None:
    """In-place batched Thomas on (n_row, n_sys) float64 CUDA tensors (system
    index fastest): d <- x; a, b, c unchanged."""
    n_row, n_sys = d.shape
    ptrs = [_dptr(t, n, n_row * n_sys) for t, n in ((a, "a"), (b, "b"), (c, "c"), (d, "d"))]
    _check("ppf_tdma_many", lib().ppf_tdma_many(*ptrs, n_sys, n_row, _stream_ptr(stream)))


def tdma_cycl_many(a, b, c, d, stream=None) -> None:
    """Cyclic variant of tdma_many."""
    n_row, n_sys = d.shape
    ptrs = [_dptr(t, n, n_row * n_sys) for t, n in ((a, "a"), (b, "b"), (c, "c"), (d, "d"))]
    _check("ppf_tdma_cycl_many", lib().ppf_tdma_cycl_many(*ptrs, n_sys, n_row, _stream_ptr(stream)))


def PaScaL_TDMA_many_solve_cuda(a_d, b_d, c_d, d_d) -> None:
    """PaScaL_TDMA_many_solve_cuda at nprocs=1 on arrays (nx_sys, ny_sys, nz_row)
    in Fortran order, i.e. tensors of shape (nz_row, ny_sys, nx_sys)."""
    nz = d_d.shape[0]
    tdma_many(*(t.view(nz, -1) for t in (a_d, b_d, c_d, d_d)))


def PaScaL_TDMA_many_solve_cycle_cuda(a_d, b_d, c_d, d_d) -> None:
    nz = d_d.shape[0]
    tdma_cycl_many(*(t.view(nz, -1) for t in (a_d, b_d, c_d, d_d)))
