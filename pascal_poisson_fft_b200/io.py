"""Field files of the reference's example drivers, for end-to-end runs
(01_Fortran/examples/module_post.f90).  Host-side numpy; arrays use this
package's convention (a Fortran P(0:n1m+1, 0:n2m+1, 0:n3m+1) is an ndarray
of shape (n3m+2, n2m+2, n1m+2), C order), which is byte-for-byte the
Fortran column-major layout.

- Restart, one file per rank (mpi_Post_FileOut/FileIn_Continue_Single_Process_IO,
  :374-411): `cont_P_<rank tag>.bin`, one direct-access unformatted record =
  the whole ghosted array, native float64.  The rank tag is the reference's
  17-character `xyzrank` (written '(I2.2,A1,I2.2,A1,I2.2)', blank-padded, and
  used untrimmed in the name).
- Restart, one shared file (mpi_Post_FileOut/FileIn_Continue_MPI_IO, :505-559):
  `cont_P.bin` = the global interior (n1m, n2m, n3m) in Fortran order; each
  rank writes and reads its block (a z slab is one contiguous range).  The
  ghost cells are refilled after reading (the reference calls its ghost
  update; here the caller runs the solve's ghost update or a solve).
- Instant field (mpi_Post_FileOut_InstanField, :127-186): Tecplot ASCII
  `Output_instantfield_XY<rank tag>.plt` with the x-y plane k = (n3sub-1)/2.
- RMS error against an exact solution (mpi_Post_error, :79-117).

The GPU example driver's field IO (01_Fortran/examples/cuda_post.f90,
main.f90), with the field in device memory (torch CUDA tensors):
- Restart load into the device field (main.f90:136-139:
  cuda_Post_FileIn_Continue_Post_Reassembly_IO, :224-258, then the copy to
  the device): `cont_P.bin` holds the global interior (n1m, n2m, n3m); the
  rank's block goes into the interior of P on the device and the ghost cells
  get the driver's subdomain halo update, which at one rank is the periodic
  copies along the periodic axes (ppf_ghost_update with walls = 0).
- 3-D instant field (cuda_Post_Fileout_InstantField_3D, :294-331): Tecplot
  ASCII `P_<rank>.PLT` of the node values, interpolated from the cells on the
  device (ppf_cell_to_node, calc_C2g :338-353), one line
  `(4(E11.4,1x))` per node with its face coordinates.
"""
from __future__ import annotations

import os

import numpy as np


def rank_tag(r1: int = 0, r2: int = 0, r3: int = 0) -> str:
    """The reference's xyzrank: 'ii_jj_kk' padded with blanks to 17 characters."""
    return f"{r1:02d}_{r2:02d}_{r3:02d}".ljust(17)


def restart_path(directory: str, ranks=(0, 0, 0)) -> str:
    return os.path.join(directory, "cont_P_" + rank_tag(*ranks) + ".bin")


def write_restart(directory: str, P: np.ndarray, ranks=(0, 0, 0)) -> str:
    path = restart_path(directory, ranks)
    np.ascontiguousarray(P, dtype=np.float64).tofile(path)
    return path


def read_restart(directory: str, shape, ranks=(0, 0, 0)) -> np.ndarray:
    """shape: (n3m+2, n2m+2, n1m+2) of this rank's ghosted array."""
    path = restart_path(directory, ranks)
    a = np.fromfile(path, dtype=np.float64)
    if a.size != int(np.prod(shape)):
        raise ValueError(f"{path}: {a.size} values, expected {int(np.prod(shape))}")
    return a.reshape(shape)


def write_restart_shared(directory: str, P: np.ndarray, n3m_global: int, z0: int = 0) -> str:
    """This rank's interior block (z rows z0 .. z0+rows-1) into the shared cont_P.bin."""
    path = os.path.join(directory, "cont_P.bin")
    inner = np.ascontiguousarray(P[1:-1, 1:-1, 1:-1], dtype=np.float64)
    rows, n2m, n1m = inner.shape
    total = n1m * n2m * n3m_global * 8
    mode = "r+b" if os.path.exists(path) else "w+b"
    with open(path, mode) as fh:
        fh.seek(0, os.SEEK_END)
        if fh.tell() < total:
            fh.truncate(total)
        fh.seek(z0 * n1m * n2m * 8)
        fh.write(inner.tobytes())
    return path


def read_restart_shared(directory: str, shape, n3m_global: int, z0: int = 0) -> np.ndarray:
    """This rank's ghosted array from the shared cont_P.bin; ghost cells are 0
    until the ghost update runs."""
    path = os.path.join(directory, "cont_P.bin")
    rows, n2m, n1m = shape[0] - 2, shape[1] - 2, shape[2] - 2
    if os.path.getsize(path) != n1m * n2m * n3m_global * 8:
        raise ValueError(f"{path}: size does not match a {n1m}x{n2m}x{n3m_global} interior")
    P = np.zeros(shape)
    with open(path, "rb") as fh:
        fh.seek(z0 * n1m * n2m * 8)
        P[1:-1, 1:-1, 1:-1] = np.frombuffer(fh.read(rows * n1m * n2m * 8), dtype=np.float64).reshape(rows, n2m, n1m)
    return P


def _fortran_d(v: float, w: int, d: int) -> str:
    """Fortran Dw.d: 0.ddddD+ee, right-justified in w columns."""
    if v == 0.0:
        m, e = 0.0, 0
    else:
        e = int(np.floor(np.log10(abs(v)))) + 1
        m = v / 10.0 ** e
        if round(abs(m), d) >= 1.0:
            m /= 10.0
            e += 1
    return f"{m:.{d}f}D{e:+03d}".rjust(w)


def write_instant_xy(directory: str, P: np.ndarray, x1, x2, x3, ranks=(0, 0, 0)) -> str:
    """Tecplot ASCII x-y plane k = (n3sub-1)/2 of this rank's ghosted field,
    appended to Output_instantfield_XY<rank tag>.plt as the reference does."""
    n3, n2, n1 = P.shape           # n*sub + 1 points each, indices 0..n*sub
    k = (n3 - 2) // 2              # (n3sub - 1) / 2 with n3sub = n3 - 1
    path = os.path.join(directory, "Output_instantfield_XY" + rank_tag(*ranks).rstrip() + ".plt")
    with open(path, "a") as fh:
        fh.write(' VARIABLES="X","Y","Z","P"\n')
        fh.write(f' zone t="{1:12d}"i={n1:12d}j={n2:12d}k={1:12d}\n')
        for j in range(n2):
            for i in range(n1):
                fh.write(_fortran_d(x1[i], 20, 10) + _fortran_d(x2[j], 20, 10) + _fortran_d(x3[k], 20, 10)
                         + _fortran_d(P[k, j, i], 30, 20) + "\n")
    return path


def rms_error(P: np.ndarray, exact: np.ndarray) -> float:
    """sqrt(sum over interior cells of (P - exact)^2 / (n1m n2m n3m)) (:79-117);
    `exact` ghosted like P or interior-shaped."""
    inner = P[1:-1, 1:-1, 1:-1]
    ex = exact[1:-1, 1:-1, 1:-1] if exact.shape == P.shape else exact
    return float(np.sqrt(((inner - ex) ** 2).sum() / inner.size))


def _fortran_e(v: float, w: int, d: int) -> str:
    """Fortran Ew.d: 0.ddddE+ee, right-justified in w columns."""
    return _fortran_d(v, w, d).replace("D", "E")


def read_restart_to_device(directory: str, P, n3m_global: int, pbc, z0: int = 0, stream=None):
    """Load this rank's block of the shared restart file `cont_P.bin` into the
    interior of the device field P (torch CUDA float64, ghosted shape
    (rows+2, n2m+2, n1m+2)) and fill the ghost cells as the driver's halo
    update does at one rank: periodic copies along the periodic axes (pbc),
    wall ghosts left as they were.  Returns P."""
    import torch
    from . import _check, _dptr, _stream_ptr, lib
    host = read_restart_shared(directory, tuple(P.shape), n3m_global, z0)
    rows, n2m, n1m = P.shape[0] - 2, P.shape[1] - 2, P.shape[2] - 2
    staged = torch.from_numpy(np.ascontiguousarray(host[1:-1, 1:-1, 1:-1])).pin_memory()
    P[1:-1, 1:-1, 1:-1].copy_(staged, non_blocking=True)
    _check("ppf_ghost_update", lib().ppf_ghost_update(_dptr(P, "P"), n1m, n2m, rows, int(bool(pbc[0])),
                                                      int(bool(pbc[1])), int(bool(pbc[2])), None, None, None, 0,
                                                      _stream_ptr(stream)))
    return P


def node_field(P, dx1, dx2, dx3, stream=None):
    """Node values (n3m, n2m, n1m) of the ghosted device field P for the 3-D
    instant field (ppf_cell_to_node); dx* device arrays of the cell widths."""
    import torch
    from . import _check, _dptr, _stream_ptr, lib
    n3m, n2m, n1m = P.shape[0] - 2, P.shape[1] - 2, P.shape[2] - 2
    G = torch.empty((n3m, n2m, n1m), dtype=torch.float64, device=P.device)
    _check("ppf_cell_to_node", lib().ppf_cell_to_node(_dptr(P, "P"), n1m, n2m, n3m, _dptr(dx1, "dx1", n1m + 2),
                                                      _dptr(dx2, "dx2", n2m + 2), _dptr(dx3, "dx3", n3m + 2),
                                                      _dptr(G, "G"), _stream_ptr(stream)))
    return G


def write_instant_field_3d(directory: str, P, x1, x2, x3, dx1, dx2, dx3, rank: int = 0) -> str:
    """Tecplot ASCII 3-D instant field of the device field P:
    `P_<rank:03d>.PLT` with the node values from the device (node_field) and
    the face coordinates x1(i), x2(j), x3(k), i, j, k = 1..n*m, in the
    reference's order and formats (cuda_post.f90:294-331)."""
    G = node_field(P, dx1, dx2, dx3).cpu().numpy()
    n3m, n2m, n1m = G.shape
    x1, x2, x3 = (np.asarray(a, dtype=np.float64) for a in (x1, x2, x3))
    path = os.path.join(directory, f"P_{rank:03d}.PLT")
    with open(path, "w") as fh:
        fh.write(' VARIABLES="X","Y","Z","P"\n')
        fh.write(f' zone t="{1:12d}"i={n1m:12d}j={n2m:12d}k={n3m:12d}\n')
        for k in range(1, n3m + 1):
            zs = _fortran_e(x3[k], 11, 4) + " "
            for j in range(1, n2m + 1):
                ys = _fortran_e(x2[j], 11, 4) + " "
                row = G[k - 1, j - 1]
                fh.write("".join(_fortran_e(x1[i], 11, 4) + " " + ys + zs + _fortran_e(row[i - 1], 11, 4) + " \n"
                                 for i in range(1, n1m + 1)))
    return path
