"""The banded z-Fourier preconditioner of the Schur solve (C3D_PRECOND_BAND).

It has no counterpart in the reference (whose BiCGSTAB,
src/projection.f90:146-186, is unpreconditioned), so it is checked against
its own definition built here from the GPU's Schur operator: the columns of S
are read back one unit vector at a time, the library's probing (unit probes
of one colour class at z row 0: markers 8 lattice columns apart for the dudn
components, 32 for the pressure jump) is repeated on them, the band
B (lattice neighbours |d| <= 2 along the ring or row, every z distance,
repeated along z) is assembled densely, and ``precond_apply`` must return
B^-1 v: backward error below 1e-12 and within 1e-8 of a dense LU solve,
with the lattice's z transforms done by FFT and, for one lattice length, by
the direct DFT.
Then BiCGSTAB with it reaches the tolerance in fewer iterations than the
unpreconditioned solver.
"""
import math

import numpy as np
import pytest

from oracle import channel_oracle as co
from oracle import ib_oracle as ibo

pytestmark = pytest.mark.gpu

BAND_CASES = ["center_wall", "wall_standing_wave", "double_cylinders_z", "two_cylinders_z",
              "traveling_wave_x", "standing_wave"]
SPACING = (8, 8, 8, 32)


def segments(case, ib, p):
    nb = ib.body.nb
    lat = nb // p["nzb"]
    if case in ("center_wall", "wall_standing_wave"):
        return lat, [(0, lat)]
    if case == "double_cylinders_z":
        n1 = int(np.sum(np.asarray(ib.body.blocks[0]) < lat))
        return lat, [(0, n1), (n1, lat - n1)]
    return lat, [(0, lat // 2), (lat // 2, lat // 2)]


def colours(segs, P):
    col = []
    for _, n in segs:
        full = (n // P) * P
        col += [i % P if i < full else P + (i - full) for i in range(n)]
    return np.array(col)


def band_matrix(S, lat, nzl, segs):
    nb = lat * nzl
    n = 4 * nb
    nbr = np.zeros((lat, 5), dtype=np.int64)
    for st, ln in segs:
        for i in range(ln):
            for d in range(-2, 3):
                nbr[st + i, d + 2] = st + (i + d) % ln
    T = np.zeros((4, lat, 5, 4, nzl))          # [cp][i1][d][c][iz]
    for c in range(4):
        col = colours(segs, SPACING[c])
        for k in np.unique(col):
            sel = np.nonzero(col == k)[0]
            e = np.zeros(n)
            e[c * nb + sel] = 1.0
            R = (S @ e).reshape(4, nzl, lat)
            for i1 in sel:
                T[:, i1, :, c, :] = R[:, :, nbr[i1]].transpose(0, 2, 1)
    B = np.zeros((n, n))
    iz = np.arange(nzl)
    for i1 in range(lat):
        for d in range(5):
            j1 = nbr[i1, d]
            for c in range(4):
                for cp in range(4):
                    # B[(cp, j1, izp), (c, i1, iz)] = T[cp, i1, d, c, izp - iz]
                    rows = cp * nb + j1 + lat * iz[:, None]
                    cols = c * nb + i1 + lat * iz[None, :]
                    B[rows, cols] = T[cp, i1, d, c, (iz[:, None] - iz[None, :]) % nzl]
    return B


def dense_schur(ch, n):
    S = np.zeros((n, n))
    e = np.zeros(n)
    for i in range(n):
        e[:] = 0.0
        e[i] = 1.0
        S[:, i] = ch.schur(e)
    return S


# the lattice's z transforms run as FFTs when its length is 2^a 3^b (16,
# 12, 6 and 3 above) and as direct DFTs otherwise (10)
@pytest.mark.parametrize("case,extra", [(c, None) for c in BAND_CASES] + [("center_wall", {"nzb": 10})])
def test_band_preconditioner_is_the_probed_band_inverse(case, extra):
    import test_gpu_ib as tib
    from channel3d_parallel_b200 import lib as L
    p, g, st, ib, ch = tib.build(case, extra=extra)
    try:
        ch.set_mode(precond=L.PRECOND_BAND)
        nb = ib.body.nb
        lat, segs = segments(case, ib, p)
        S = dense_schur(ch, 4 * nb)
        B = band_matrix(S, lat, nb // lat, segs)
        rng = np.random.default_rng(11)
        v = rng.standard_normal(4 * nb)
        x = ch.precond_apply(v)
        bw = np.abs(B @ x - v).max() / (np.abs(B).sum(axis=1).max() * np.abs(x).max())
        assert bw < 1e-12, bw
        ref = np.linalg.solve(B, v)
        assert np.abs(x - ref).max() <= 1e-8 * np.abs(ref).max()
        s = ch.stats()
        assert s["precond_builds"] == 1
    finally:
        ch.close()


@pytest.mark.parametrize("case", ["wall_standing_wave", "two_cylinders_z", "traveling_wave_x"])
def test_band_bicgstab_converges_faster_than_unpreconditioned(case):
    import test_gpu_ib as tib
    from channel3d_parallel_b200 import lib as L
    iters = {}
    for mode in (L.PRECOND_NONE, L.PRECOND_BAND):
        p, g, st, ib, ch = tib.build(case, cg_tol=1e-13, cg_max_iter=400)
        try:
            ch.set_mode(precond=mode)
            ch.compute_time_step_RK3(2)
            s = ch.stats()
            assert s["last_residual"] < 1e-13
            iters[mode] = s["bicgstab_iters"] / s["bicgstab_solves"]
        finally:
            ch.close()
    assert iters[L.PRECOND_BAND] < iters[L.PRECOND_NONE], iters


def test_band_unsupported_for_plates():
    import test_gpu_ib as tib
    from channel3d_parallel_b200 import lib as L
    import channel3d_parallel_b200 as c3d
    p, g, st, ib, ch = tib.build("wall_plates", cg_max_iter=5)
    try:
        with pytest.raises(c3d.C3DError):
            ch.set_mode(precond=L.PRECOND_BAND)
    finally:
        ch.close()
