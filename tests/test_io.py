"""Field files of the reference's drivers (pascal_poisson_fft_b200.io)."""
import os

import numpy as np

from pascal_poisson_fft_b200 import io as FIO


def test_rank_tag_and_restart_name():
    assert FIO.rank_tag(1, 0, 3) == "01_00_03" + " " * 9
    assert os.path.basename(FIO.restart_path("/x", (0, 2, 11))) == "cont_P_00_02_11         .bin"


def test_restart_round_trip_is_fortran_layout(tmp_path):
    rng = np.random.default_rng(1)
    P = rng.standard_normal((6, 5, 7))          # P(0:6, 0:4, 0:5) in Fortran terms
    path = FIO.write_restart(str(tmp_path), P, (0, 0, 1))
    raw = np.fromfile(path, dtype=np.float64)
    assert raw.size == P.size
    # the first values run along x (Fortran column-major)
    assert np.array_equal(raw[:7], P[0, 0, :])
    assert np.array_equal(FIO.read_restart(str(tmp_path), P.shape, (0, 0, 1)), P)


def test_shared_restart_by_z_slabs(tmp_path):
    rng = np.random.default_rng(2)
    n1, n2, n3 = 6, 5, 9
    G = rng.standard_normal((n3 + 2, n2 + 2, n1 + 2))
    for z0, rows in ((0, 3), (3, 4), (7, 2)):
        slab = np.zeros((rows + 2, n2 + 2, n1 + 2))
        slab[1:-1] = G[1 + z0:1 + z0 + rows]
        FIO.write_restart_shared(str(tmp_path), slab, n3, z0)
    raw = np.fromfile(str(tmp_path / "cont_P.bin")).reshape(n3, n2, n1)
    assert np.array_equal(raw, G[1:-1, 1:-1, 1:-1])
    back = FIO.read_restart_shared(str(tmp_path), (4 + 2, n2 + 2, n1 + 2), n3, 3)
    assert np.array_equal(back[1:-1, 1:-1, 1:-1], G[4:8, 1:-1, 1:-1])


def test_instant_field_and_rms(tmp_path):
    P = np.arange(4 * 3 * 5, dtype=np.float64).reshape(4, 3, 5)
    x1, x2, x3 = np.linspace(0, 1, 5), np.linspace(0, 2, 3), np.linspace(0, 3, 4)
    path = FIO.write_instant_xy(str(tmp_path), P, x1, x2, x3)
    lines = open(path).read().splitlines()
    assert lines[0].strip() == 'VARIABLES="X","Y","Z","P"'
    assert len(lines) == 2 + 3 * 5
    vals = [float(t.replace("D", "E")) for t in lines[2 + 5 * 1 + 2].split()]
    assert vals == [x1[2], x2[1], x3[1], P[1, 1, 2]]
    assert FIO.rms_error(P, P + 2.0) == 2.0
