"""Field IO of the GPU example driver with the field in device memory: the
restart load into the device field with the one-rank halo update, the 3-D
instant field's cell-to-node interpolation and file, and the ghost update
outside a solve (01_Fortran/examples/cuda_post.f90:224-258, 294-353;
main.f90:136-139; cuda_subdomain.f90:199-220)."""
import numpy as np
import pytest

import pascal_poisson_fft_b200 as ppf
from pascal_poisson_fft_b200 import io
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _t(a):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def c2g_reference(P, dx1, dx2, dx3):
    """calc_C2g (cuda_post.f90:338-353) over every node i, j, k = 1..n*m, numpy."""
    n3, n2, n1 = P.shape[0] - 2, P.shape[1] - 2, P.shape[2] - 2
    i = np.arange(1, n1 + 1)[None, None, :]
    j = np.arange(1, n2 + 1)[None, :, None]
    k = np.arange(1, n3 + 1)[:, None, None]
    X = lambda a, b, c: P[c, b, a]
    wz = dx3[k] + dx3[k - 1]
    wx = dx1[i] + dx1[i - 1]
    X1 = (X(i - 1, j - 1, k) * dx3[k - 1] + X(i - 1, j - 1, k - 1) * dx3[k]) / wz
    X2 = (X(i, j - 1, k) * dx3[k - 1] + X(i, j - 1, k - 1) * dx3[k]) / wz
    Xy1 = (X2 * dx1[i - 1] + X1 * dx1[i]) / wx
    X1 = (X(i - 1, j, k) * dx3[k - 1] + X(i - 1, j, k - 1) * dx3[k]) / wz
    X2 = (X(i, j, k) * dx3[k - 1] + X(i, j, k - 1) * dx3[k]) / wz
    Xy2 = (X2 * dx1[i - 1] + X1 * dx1[i]) / wx
    return (Xy2 * dx2[j - 1] + Xy1 * dx2[j]) / (dx2[j] + dx2[j - 1])


def test_cell_to_node_matches_the_reference_formula():
    rng = np.random.default_rng(61)
    n1, n2, n3 = 12, 9, 7
    P = rng.standard_normal((n3 + 2, n2 + 2, n1 + 2))
    dx = [rng.uniform(0.5, 1.5, n + 2) for n in (n1, n2, n3)]
    dx[2][0] = 0.0   # a wall below the first cell, as the driver's metric has
    G = io.node_field(_t(P), *[_t(d) for d in dx]).cpu().numpy()
    # the same products, sums and quotients in the same order: bit-exact
    np.testing.assert_array_equal(G, c2g_reference(P, *dx))


def test_instant_field_3d_file(tmp_path):
    rng = np.random.default_rng(62)
    n1, n2, n3 = 4, 3, 2
    P = rng.standard_normal((n3 + 2, n2 + 2, n1 + 2))
    x = [np.cumsum(np.r_[0.0, rng.uniform(0.5, 1.0, n + 1)]) for n in (n1, n2, n3)]
    dx = [np.r_[np.diff(xx), 0.0] for xx in x]
    path = io.write_instant_field_3d(str(tmp_path), _t(P), *x, *[_t(d) for d in dx], rank=3)
    lines = open(path).read().splitlines()
    assert path.endswith("P_003.PLT")
    assert lines[0] == ' VARIABLES="X","Y","Z","P"'
    assert lines[1] == ' zone t="           1"i=           4j=           3k=           2'
    assert len(lines) == 2 + n1 * n2 * n3
    assert all(len(l) == 48 for l in lines[2:])
    G = c2g_reference(P, *dx)
    vals = np.array([[float(l[12 * c:12 * c + 11]) for c in range(4)] for l in lines[2:]])
    # k outer, then j, then i, with the face coordinates of the node
    kk, jj, ii = np.meshgrid(np.arange(1, n3 + 1), np.arange(1, n2 + 1), np.arange(1, n1 + 1), indexing="ij")
    np.testing.assert_allclose(vals[:, 0], x[0][ii.ravel()], rtol=1e-3, atol=0)
    np.testing.assert_allclose(vals[:, 2], x[2][kk.ravel()], rtol=1e-3, atol=0)
    np.testing.assert_allclose(vals[:, 3], G.ravel(), rtol=1e-3, atol=1e-12)


@pytest.mark.parametrize("pbc", [(1, 0, 1), (0, 1, 0), (1, 1, 1)])
def test_restart_load_into_device_field(tmp_path, pbc):
    import torch
    rng = np.random.default_rng(63)
    n1, n2, n3 = 10, 8, 6
    src = rng.standard_normal((n3 + 2, n2 + 2, n1 + 2))
    io.write_restart_shared(str(tmp_path), src, n3)
    P = torch.zeros((n3 + 2, n2 + 2, n1 + 2), dtype=torch.float64, device="cuda")
    io.read_restart_to_device(str(tmp_path), P, n3, pbc)
    got = P.cpu().numpy()
    # interior from the file; periodic ghosts as the one-rank halo update
    # copies them (x, then y, then z, each over the whole face); wall ghosts
    # untouched (zero)
    ref = np.zeros_like(src)
    ref[1:-1, 1:-1, 1:-1] = src[1:-1, 1:-1, 1:-1]
    if pbc[0]:
        ref[:, :, 0], ref[:, :, -1] = ref[:, :, -2].copy(), ref[:, :, 1].copy()
    if pbc[1]:
        ref[:, 0, :], ref[:, -1, :] = ref[:, -2, :].copy(), ref[:, 1, :].copy()
    if pbc[2]:
        ref[0], ref[-1] = ref[-2].copy(), ref[1].copy()
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("pbc", [(1, 1, 0), (0, 0, 0), (0, 1, 1)])
def test_ghost_update_matches_the_oracle(pbc):
    rng = np.random.default_rng(64)
    n1, n2, n3 = 16, 12, 10
    P = rng.standard_normal((n3 + 2, n2 + 2, n1 + 2))
    dmx = [rng.uniform(0.5, 1.5, n + 2) for n in (n1, n2, n3)]
    ref = P.copy()
    O.fill_ghosts(ref, pbc, *dmx)
    Pd = _t(P)
    dmx_d = [_t(d) for d in dmx]   # held: a freed block would be handed to the next array
    rc = ppf.lib().ppf_ghost_update(Pd.data_ptr(), n1, n2, n3, *pbc, *[d.data_ptr() for d in dmx_d], 1, None)
    assert rc == 0, ppf.lib().ppf_last_error()
    np.testing.assert_allclose(Pd.cpu().numpy(), ref, rtol=1e-14, atol=1e-15)
