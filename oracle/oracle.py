"""ctypes front end of the CPU oracle (test infrastructure only).

Loads ``oracle/_build/libppf_oracle.so`` (built by ``oracle/Makefile``) and
exposes numpy-level helpers.  Only tests/, ``__graft_entry__.smoke()`` and
bench.py's CPU-baseline leg import this module; the product path never does.

Array conventions follow the reference (Fortran column-major, first index
fastest).  numpy arrays here are C-ordered with the axes reversed, i.e. a
field f(1:n1m,1:n2m,1:n3m) is an ndarray of shape (n3m, n2m, n1m).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

_dp = ctypes.POINTER(ctypes.c_double)


def build() -> None:
    """Compile the oracle (and the reference TDMA when its tree is present)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "_build", "libppf_oracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.ora_mesh.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                               ctypes.c_int, _dp, _dp, _dp]
        L.ora_wavenumbers.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.ora_tdma_many.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int]
        L.ora_tdma_cycl_many.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int]
        L.ora_fft_c2c.argtypes = [_dp, ctypes.c_int, ctypes.c_int]
        L.ora_fft_c2c.restype = ctypes.c_int
        L.ora_poisson_solve.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 2 + [ctypes.c_int] * 3 + \
            [_dp, _dp, _dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int]
        L.ora_poisson_solve.restype = ctypes.c_int
        L.ora_fill_ghosts.argtypes = [ctypes.c_int] * 6 + [_dp, _dp, _dp, _dp]
        L.ora_last_stage_seconds.argtypes = [_dp]
        L.ora_last_stage_seconds.restype = ctypes.c_int
        L.ora_residual.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 2 + [ctypes.c_int] * 2 + \
            [_dp, _dp, _dp, _dp, _dp]
        _LIB = L
    return _LIB


def ref_tdmas():
    """The reference's own 00_C/PaScaL_TDMA/src/tdmas.cpp, compiled by
    oracle/Makefile into oracle/_ref/libref_tdmas.so.  None when absent."""
    global _REF
    if _REF is None:
        path = os.path.join(_HERE, "_ref", "libref_tdmas.so")
        if not os.path.exists(path):
            return None
        L = ctypes.CDLL(path)
        for name in ("tdma_many", "tdma_cycl_many"):
            getattr(L, name).argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int, ctypes.c_int]
        L.tdma_single.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int]
        L.tdma_cycl_single.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_int]
        _REF = L
    return _REF


def mesh(nm: int, L: float, uniform: bool, gamma: float, pbc: bool):
    """Faces x(0:nm+1), widths dx(0:nm+1), spacings dmx(0:nm+1)."""
    x = np.zeros(nm + 2)
    dx = np.zeros(nm + 2)
    dmx = np.zeros(nm + 2)
    lib().ora_mesh(nm, L, int(uniform), gamma, int(pbc), _ptr(x), _ptr(dx), _ptr(dmx))
    return x, dx, dmx


def wavenumbers(n1m, n2m, L1, L2, pbc1, pbc2):
    kx = np.zeros(n1m)
    ky = np.zeros(n2m)
    lib().ora_wavenumbers(n1m, n2m, L1, L2, int(pbc1), int(pbc2), _ptr(kx), _ptr(ky))
    return kx, ky


def tdma_many(a, b, c, d, cyclic=False):
    """In-place batched Thomas, arrays shaped (n_row, n_sys) (system fastest)."""
    n_row, n_sys = d.shape
    fn = lib().ora_tdma_cycl_many if cyclic else lib().ora_tdma_many
    fn(_ptr(a), _ptr(b), _ptr(c), _ptr(d), n_sys, n_row)


def fft_c2c(x: np.ndarray, sign: int) -> np.ndarray:
    y = np.ascontiguousarray(x, dtype=np.complex128).copy()
    lib().ora_fft_c2c(y.view(np.float64).ctypes.data_as(_dp), y.size, sign)
    return y


def poisson_solve(f: np.ndarray, L1: float, L2: float, pbc, dmx1, dmx2, dmx3, dx3,
                  cpu_fft1_imag_zero: bool = True, nthreads: int = 0) -> np.ndarray:
    """One-rank restatement of cuda_Poisson_FFT_1D.  f has shape (n3m, n2m, n1m);
    returns the ghosted P of shape (n3m+2, n2m+2, n1m+2)."""
    n3m, n2m, n1m = f.shape
    f = np.ascontiguousarray(f, dtype=np.float64)
    P = np.zeros((n3m + 2, n2m + 2, n1m + 2))
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (dmx1, dmx2, dmx3, dx3)]
    rc = lib().ora_poisson_solve(n1m, n2m, n3m, L1, L2, int(pbc[0]), int(pbc[1]), int(pbc[2]),
                                 _ptr(f), _ptr(P), *[_ptr(a) for a in arrs],
                                 int(cpu_fft1_imag_zero), int(nthreads))
    if rc != 0:
        raise ValueError(f"ora_poisson_solve rejected the problem (rc={rc})")
    return P


def last_stage_seconds():
    """Per-stage seconds of the last poisson_solve: setup, forward transforms,
    z solves, inverse transforms, mean removal + ghosts (None if incomplete)."""
    out = np.zeros(5)
    n = lib().ora_last_stage_seconds(_ptr(out))
    if n != 6:
        return None
    return dict(zip(("setup", "fft-forward", "tdma-z", "fft-inverse", "update-solution"), out.tolist()))


def fill_ghosts(P: np.ndarray, pbc, dmx1, dmx2, dmx3) -> None:
    n3, n2, n1 = P.shape
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (dmx1, dmx2, dmx3)]
    lib().ora_fill_ghosts(n1 - 2, n2 - 2, n3 - 2, int(pbc[0]), int(pbc[1]), int(pbc[2]),
                          _ptr(P), *[_ptr(a) for a in arrs])


def residual(f, P, L1, L2, pbc, dmx3, dx3) -> np.ndarray:
    n3m, n2m, n1m = f.shape
    r = np.zeros_like(f)
    lib().ora_residual(n1m, n2m, n3m, L1, L2, int(pbc[0]), int(pbc[1]),
                       _ptr(np.ascontiguousarray(f)), _ptr(np.ascontiguousarray(P)),
                       _ptr(np.ascontiguousarray(dmx3)), _ptr(np.ascontiguousarray(dx3)), _ptr(r))
    return r


def zcoef(dmx3, dx3, n3m):
    """am_k = 1/dx3_k/dmx3_k, ap_k = 1/dx3_k/dmx3_{k+1} with the wall entries
    zeroed (fft_3d_poisson.f90:1143-1144); index k = 0..n3m-1 is cell k+1."""
    k = np.arange(1, n3m + 1)
    am = 1.0 / dx3[k] / dmx3[k]
    ap = 1.0 / dx3[k] / dmx3[k + 1]
    am[0] = 0.0
    ap[-1] = 0.0
    return am, ap


def _zero_mode_matrix(am, ap):
    """Dense z operator of the (kx, ky) = (0, 0) system with its first row
    replaced by the pin u_1 = 0 (fft_3d_poisson.f90:1240-1249)."""
    nz = am.size
    T = np.zeros((nz, nz))
    for k in range(nz):
        T[k, k] = -am[k] - ap[k]
        if k > 0:
            T[k, k - 1] = am[k]
        if k < nz - 1:
            T[k, k + 1] = ap[k]
    T[0, :] = 0.0
    T[0, 0] = 1.0
    return T


def poisson_adjoint(g, L1, L2, pbc, dmx1, dmx2, dmx3, dx3, u=None):
    """Transpose of the solve map f -> u (interior cells), and optionally the
    gradient of <g, u> with respect to the z metric arrays.

    The solve is u = P0 M' f: transforms in x and y, one z system per
    (kx, ky), inverse transforms, arithmetic-mean removal P0.  The x and y
    operators are symmetric; the z operator is T = V^-1 S with V = diag(dx3)
    and S symmetric, so T^-T = V T^-1 V^-1 for every system except the
    pinned zero mode.  Hence M^T g = V M (V^-1 g) + c(z), where c is a
    per-level constant that swaps the zero mode of V M V^-1 for the exact
    transposed pinned system (dense solves here).

    With u = M f given (ghosted, as returned by poisson_solve), returns also
    d<g,u>/d dx3 and d<g,u>/d dmx3 (arrays of n3m+2, Fortran indices 0..n3m+1):
    dJ/dtheta = -<M^T g, (dL/dtheta) u> with the pinned row excluded.
    """
    g = np.ascontiguousarray(g, dtype=np.float64)
    n3m, n2m, n1m = g.shape
    nxy = float(n1m * n2m)
    d3 = np.asarray(dx3, dtype=np.float64)[1:n3m + 1]
    W = poisson_solve(g / d3[:, None, None], L1, L2, pbc, dmx1, dmx2, dmx3, dx3)[1:-1, 1:-1, 1:-1]
    am, ap = zcoef(np.asarray(dmx3, dtype=np.float64), np.asarray(dx3, dtype=np.float64), n3m)
    T = _zero_mode_matrix(am, ap)
    cs_g = g.sum(axis=(1, 2))
    rhs = cs_g / d3
    rhs[0] = 0.0
    cp = np.linalg.solve(T, rhs) / nxy
    B = d3 * (cp - cp.mean())
    cA = np.linalg.solve(T.T, cs_g - cs_g.sum() / n3m) / nxy
    df = d3[:, None, None] * W + (cA - B)[:, None, None]
    if u is None:
        return df
    ui = np.asarray(u)[1:-1, 1:-1, 1:-1]
    Sm = np.zeros(n3m)
    Sp = np.zeros(n3m)
    Sm[1:] = (df[1:] * (ui[:-1] - ui[1:])).sum(axis=(1, 2))
    Sp[:-1] = (df[:-1] * (ui[1:] - ui[:-1])).sum(axis=(1, 2))
    dam, dap = -Sm, -Sp
    dap[0] += df[0].sum() * (ui[1].sum() - ui[0].sum()) / nxy
    dam[0] = 0.0
    dap[-1] = 0.0
    dmx3 = np.asarray(dmx3, dtype=np.float64)
    ddx3 = np.zeros(n3m + 2)
    ddmx3 = np.zeros(n3m + 2)
    ddx3[1:n3m + 1] = -(dam * am + dap * ap) / d3
    ddmx3[1:n3m + 1] += -dam * am / dmx3[1:n3m + 1]
    ddmx3[2:n3m + 2] += -dap * ap / dmx3[2:n3m + 2]
    return df, ddx3, ddmx3


def tdma_modified(a, b, c, d):
    """This rank's part of PaScaL_TDMA_many_solve at nprocs > 1
    (01_Fortran/PaScaL_TDMA/src/pascal_tdma.f90:522-566): the modified Thomas
    sweep on arrays of shape (n_row, n_sys), in place on a, c, d; returns the
    reduced rows (a_rd, c_rd, d_rd), each (2, n_sys) (b_rd = 1)."""
    n = d.shape[0]
    for j in (0, 1):
        a[j] /= b[j]
        d[j] /= b[j]
        c[j] /= b[j]
    for j in range(2, n):
        r = 1.0 / (b[j] - a[j] * c[j - 1])
        d[j] = r * (d[j] - a[j] * d[j - 1])
        c[j] = r * c[j]
        a[j] = -r * a[j] * a[j - 1]
    for j in range(n - 3, 0, -1):
        d[j] = d[j] - c[j] * d[j + 1]
        a[j] = a[j] - c[j] * a[j + 1]
        c[j] = -c[j] * c[j + 1]
    r = 1.0 / (1.0 - a[1] * c[0])
    d[0] = r * (d[0] - c[0] * d[1])
    a[0] = r * a[0]
    c[0] = -r * c[0] * c[1]
    return (np.stack([a[0], a[n - 1]]), np.stack([c[0], c[n - 1]]), np.stack([d[0], d[n - 1]]))


def tdma_update(a, c, d, x_rd):
    """pascal_tdma.f90:595-605: the local rows from the reduced solution."""
    n = d.shape[0]
    d[0] = x_rd[0]
    d[n - 1] = x_rd[1]
    for j in range(1, n - 1):
        d[j] = d[j] - a[j] * d[0] - c[j] * d[n - 1]
