"""Host check of the band-restricted Thomas solve used inside the IB Schur
operator (k_spectral_band): when the right-hand side of a tridiagonal system
vanishes outside rows [rlo, rhi] and only those rows of the solution are
wanted, the forward sweep may start at rlo from zero and the back
substitution at x(rhi+1) = S(rhi+1) y(rhi+1), y(rhi+1) = -MULT(rhi) y(rhi),
with S(j) = x(j)/y(j) of the homogeneous tail tabulated once:
S(Ny-1) = 1/D'(Ny-1), S(j) = (1 + DU(j) MULT(j) S(j+1)) / D'(j).

The systems are the wall-normal Poisson operators of a stretched channel
grid (src/poisson.f90:43-80): Dyy plus the modified wavenumbers kxx + kzz,
with the (0, 0) mode pinned as the reference pins it (D(1) scaled by 3/2).
"""
import numpy as np
import pytest

from oracle import channel_oracle as co


def thomas_factors(dl, d, du):
    """No-pivot factorisation of zgtsv (MULT = DL/D, D' -= MULT*DU)."""
    n = len(d)
    dp = d.astype(np.complex128).copy()
    for j in range(n - 1):
        mu = dl[j] / dp[j]
        dp[j + 1] = dp[j + 1] - mu * du[j]
    rdp = 1.0 / dp
    return rdp


def full_solve(dl, du, rdp, b):
    n = len(b)
    y = b.astype(np.complex128).copy()
    for j in range(1, n):
        y[j] = y[j] - dl[j - 1] * rdp[j - 1] * y[j - 1]
    x = np.zeros_like(y)
    x[n - 1] = y[n - 1] * rdp[n - 1]
    for j in range(n - 2, -1, -1):
        x[j] = (y[j] - du[j] * x[j + 1]) * rdp[j]
    return x


def tail_table(dl, du, rdp):
    n = len(rdp)
    s = np.zeros(n, dtype=np.complex128)
    s[n - 1] = rdp[n - 1]
    for j in range(n - 2, -1, -1):
        mu = dl[j] * rdp[j]
        s[j] = (1.0 + du[j] * mu * s[j + 1]) * rdp[j]
    return s


def band_solve(dl, du, rdp, tail, b, rlo, rhi):
    n = len(b)
    nr = rhi - rlo + 1
    y = np.zeros(nr, dtype=np.complex128)
    prev = 0.0
    for r in range(nr):
        j = rlo + r
        v = b[j]
        if r > 0:
            v = v - dl[j - 1] * rdp[j - 1] * prev
        y[r] = v
        prev = v
    xn = 0.0
    if rhi + 1 < n:
        xn = -dl[rhi] * rdp[rhi] * tail[rhi + 1] * prev
    x = np.zeros(nr, dtype=np.complex128)
    for r in range(nr - 1, -1, -1):
        j = rlo + r
        x[r] = (y[r] - du[j] * xn) * rdp[j]
        xn = x[r]
    return x


def channel_operators():
    """Dyy of the stretched 34x65x34 channel grid from the oracle (the
    reference's Dd, Dl, Du, src/initialization.f90) and its wavenumbers."""
    p = co.channel_params(34, 65, 34, 2.0, 1.0, 1e-3, alpha=2.0, grid_type=1, cfl=-1e-3)
    g = co.Grid(p)
    nyg = len(g.Dd) - 1
    dd = np.asarray(g.Dd[2:nyg], dtype=np.float64)
    dl = np.append(np.asarray(g.Dl[3:nyg], dtype=np.float64), 0.0)   # Dyy(j+1, j)
    du = np.append(np.asarray(g.Du[2:nyg - 1], dtype=np.float64), 0.0)  # Dyy(j, j+1)
    k2 = sorted({0.0, float(g.kxx[1] + g.kzz[0]), float(g.kxx[3] + g.kzz[5]),
                 float(g.kxx[16] + g.kzz[16])})
    return dl, dd, du, k2


@pytest.mark.parametrize("band", [(0, 5), (10, 19), (40, 63), (63, 63), (0, 63), (30, 30)])
def test_band_solve_matches_full_thomas(band):
    dl, d0, du, k2s = channel_operators()
    n = len(d0)
    rlo, rhi = band
    rhi = min(rhi, n - 1)
    rng = np.random.default_rng(rlo * 100 + rhi)
    for k2 in k2s:
        d = d0 + k2
        if k2 == 0.0:
            d = d.copy()
            d[0] *= 1.5                           # the pinned (0, 0) mode, src/poisson.f90:69
        rdp = thomas_factors(dl, d, du)
        tail = tail_table(dl, du, rdp)
        b = np.zeros(n, dtype=np.complex128)
        b[rlo:rhi + 1] = rng.standard_normal(rhi - rlo + 1) + 1j * rng.standard_normal(rhi - rlo + 1)
        xf = full_solve(dl, du, rdp, b)[rlo:rhi + 1]
        xb = band_solve(dl, du, rdp, tail, b, rlo, rhi)
        assert np.abs(xb - xf).max() <= 1e-12 * np.abs(xf).max(), (band, k2)
