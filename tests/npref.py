"""Independent numpy/scipy restatement of the solve (test infrastructure).

A second, separately written implementation of the same discrete method,
used only to pin the C oracle: transforms come from ``scipy.fft``
(pocketfft), the tridiagonal solves from a vectorised Thomas sweep, the
ghost cells from the reference's fill order.  Field arrays are shaped
(n3m, n2m, n1m) -- the reference's column-major f(1:n1m,1:n2m,1:n3m).

Reference formulas: modified wavenumbers 01_Fortran/src/fft_3d_poisson.f90:288-351;
z coefficients and pin :1121-1170, :1215-1254; mean removal :628-664;
ghost cells :798-852 and :666-796; mesh 01_Fortran/examples/mpi_subdomain.f90:397-472.
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft


def mesh(nm, L, uniform, gamma, pbc):
    idx = np.arange(0, nm + 2)
    if uniform:
        x = (idx - 1) * L / nm
    else:
        x = L * 0.5 * (1.0 + np.tanh(0.5 * gamma * (2.0 * (idx - 1) / nm - 1.0)) / np.tanh(gamma * 0.5))
    x = x.astype(np.float64)
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


def wavenumbers(n1m, n2m, L1, L2, pbc1, pbc2):
    h1, h2 = L1 / n1m, L2 / n2m

    def dct_wn(m, n, h):
        return 4.0 * np.sin(0.5 * m * np.pi / n) ** 2 / (h * h)

    def fft_wn(m, n, h):
        return 2.0 * (1.0 - np.cos(2.0 * m * np.pi / n)) / (h * h)

    i = np.arange(n1m)
    j = np.arange(n2m)
    kx = fft_wn(i, n1m, h1) if pbc1 else dct_wn(i, n1m, h1)
    if not pbc2:
        ky = dct_wn(j, n2m, h2)
    else:
        jm = j.copy()
        if pbc1:
            jm = np.where(j + 1 > n2m // 2 + 1, n2m - j, j)
        ky = fft_wn(jm, n2m, h2)
    return kx, ky


def z_coeffs(n3m, dx3, dmx3):
    k = np.arange(1, n3m + 1)
    am = 1.0 / dx3[k] / dmx3[k]
    ap = 1.0 / dx3[k] / dmx3[k + 1]
    am[0] = 0.0
    ap[-1] = 0.0
    return am, ap


def thomas(am, ap, lam, d, pin=None):
    """Vectorised Thomas along axis 0: (am_k, -am_k-ap_k-lam, ap_k) x = d.
    ``pin`` is a boolean mask over systems whose row 0 becomes the identity
    with zero right-hand side."""
    nz = d.shape[0]
    a = np.broadcast_to(am[:, None], (nz,) + lam.shape).copy()
    c = np.broadcast_to(ap[:, None], (nz,) + lam.shape).copy()
    b = (-am - ap)[:, None] - lam[None, :]
    d = d.copy()
    if pin is not None:
        a[0][pin] = 0.0
        b[0][pin] = 1.0
        c[0][pin] = 0.0
        d[0][pin] = 0.0
    cp = np.empty_like(c)
    dp = np.empty_like(d)
    cp[0] = c[0] / b[0]
    dp[0] = d[0] / b[0]
    for k in range(1, nz):
        r = 1.0 / (b[k] - a[k] * cp[k - 1])
        dp[k] = r * (d[k] - a[k] * dp[k - 1])
        cp[k] = r * c[k]
    x = np.empty_like(dp)
    x[-1] = dp[-1]
    for k in range(nz - 2, -1, -1):
        x[k] = dp[k] - cp[k] * x[k + 1]
    return x


def _dct(a, axis):
    if np.iscomplexobj(a):
        return sfft.dct(a.real, type=2, axis=axis) + 1j * sfft.dct(a.imag, type=2, axis=axis)
    return sfft.dct(a, type=2, axis=axis)


def _idct(a, axis):
    if np.iscomplexobj(a):
        return sfft.idct(a.real, type=2, axis=axis) + 1j * sfft.idct(a.imag, type=2, axis=axis)
    return sfft.idct(a, type=2, axis=axis)


def fill_ghosts(P, pbc, dmx1, dmx2, dmx3):
    """In-place ghost fill of P (shape (n3m+2, n2m+2, n1m+2))."""
    dmx = (dmx1, dmx2, dmx3)
    axes = (2, 1, 0)  # numpy axis of x, y, z
    for d in range(3):
        if pbc[d]:
            continue
        dm = dmx[d]
        ax = axes[d]
        na = P.shape[ax] - 1
        sl = dm[1] + dm[2]
        alo = sl * sl / (sl * sl - dm[1] * dm[1])
        blo = dm[1] * dm[1] / (sl * sl - dm[1] * dm[1])
        su = dm[na] + dm[na - 1]
        ahi = su * su / (su * su - dm[na] * dm[na])
        bhi = dm[na] * dm[na] / (su * su - dm[na] * dm[na])
        Pm = np.moveaxis(P, ax, 0)
        Pm[0] = alo * Pm[1] - blo * Pm[2]
        Pm[na] = ahi * Pm[na - 1] - bhi * Pm[na - 2]
    for d in range(3):
        if not pbc[d]:
            continue
        ax = axes[d]
        na = P.shape[ax] - 1
        Pm = np.moveaxis(P, ax, 0)
        s0 = Pm[1].copy()
        s1 = Pm[na - 1].copy()
        Pm[0] = s1
        Pm[na] = s0


def solve(f, L1, L2, pbc, dmx1, dmx2, dmx3, dx3):
    n3m, n2m, n1m = f.shape
    pbc1, pbc2, pbc3 = (bool(p) for p in pbc)
    kx, ky = wavenumbers(n1m, n2m, L1, L2, pbc1, pbc2)
    am, ap = z_coeffs(n3m, dx3, dmx3)
    F = sfft.rfft(f, axis=2) if pbc1 else _dct(f, 2)
    if pbc2:
        F = sfft.fft(F, axis=1) if np.iscomplexobj(F) else sfft.rfft(F, axis=1)
    else:
        F = _dct(F, 1)
    nky, nkx = F.shape[1], F.shape[2]
    lam = (kx[:nkx][None, :] + ky[:nky][:, None])
    pin = np.zeros(lam.shape, dtype=bool)
    pin[0, 0] = True
    U = thomas(am, ap, lam.reshape(-1), F.reshape(n3m, -1), pin.reshape(-1)).reshape(F.shape)
    if pbc2:
        U = sfft.ifft(U, axis=1) if pbc1 else sfft.irfft(U, n=n2m, axis=1)
    else:
        U = _idct(U, 1)
    u = sfft.irfft(U, n=n1m, axis=2) if pbc1 else _idct(U, 2)
    u = np.real(u)
    u = u - u.sum() / (n1m * n2m * n3m)
    P = np.zeros((n3m + 2, n2m + 2, n1m + 2))
    P[1:-1, 1:-1, 1:-1] = u
    fill_ghosts(P, (pbc1, pbc2, pbc3), dmx1, dmx2, dmx3)
    return P


def residual(f, u, L1, L2, pbc, dx3, dmx3):
    """r = f - L_h u on interior fields (n3m, n2m, n1m)."""
    n3m, n2m, n1m = f.shape
    hx, hy = L1 / n1m, L2 / n2m
    if pbc[0]:
        uxm, uxp = np.roll(u, 1, 2), np.roll(u, -1, 2)
    else:
        uxm = np.concatenate([u[:, :, :1], u[:, :, :-1]], 2)
        uxp = np.concatenate([u[:, :, 1:], u[:, :, -1:]], 2)
    if pbc[1]:
        uym, uyp = np.roll(u, 1, 1), np.roll(u, -1, 1)
    else:
        uym = np.concatenate([u[:, :1], u[:, :-1]], 1)
        uyp = np.concatenate([u[:, 1:], u[:, -1:]], 1)
    uzm = np.concatenate([u[:1], u[:-1]], 0)
    uzp = np.concatenate([u[1:], u[-1:]], 0)
    am, ap = z_coeffs(n3m, dx3, dmx3)
    lu = (uxm - 2 * u + uxp) / hx ** 2 + (uym - 2 * u + uyp) / hy ** 2 \
        + am[:, None, None] * (uzm - u) + ap[:, None, None] * (uzp - u)
    return f - lu
