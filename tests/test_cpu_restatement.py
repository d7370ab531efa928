"""The C++/OpenMP restatement (timed CPU baseline) against the NumPy oracle.

Tolerances (max-norm error relative to the max-norm of the oracle field):
  U, V, W after 1 and 10 RK3 steps        1e-12
  P (stage-1 potential / dt)               1e-10
  dPdx                                     the GPU parity bound
  FFT vs numpy.fft                         1e-13 relative to max |X|
  zgtsv vs LAPACK (scipy), pivoting        1e-12 relative
"""
import math

import numpy as np
import pytest
from scipy.linalg import lapack

from oracle import channel_oracle as co
from oracle import cpu_rk3

CASES = {
    "cfg0_34x65x34": (34, 65, 34, math.pi, math.pi / 2, 1),
    "odd_ny_radix3": (50, 34, 26, 2.0, 1.0, 1),
    "uniform_small": (18, 17, 14, 1.0, 0.7, 0),
}


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module", autouse=True)
def built():
    cpu_rk3.build()


@pytest.mark.parametrize("case", list(CASES))
def test_rk3_steps_match_oracle(case):
    nx, ny, nz, lx, lz, gt = CASES[case]
    p = co.channel_params(nx, ny, nz, lx, lz, 1.0 / 5600.0, grid_type=gt)
    g = co.Grid(p)
    st = co.seeded_initial_state(g, p["dpdx"])
    cc = cpu_rk3.CpuChannel(g, nthreads=2)
    try:
        cc.set_state(st)
        done = 0
        for n in (1, 9):
            cc.steps(n)
            for _ in range(n):
                co.compute_time_step_RK3(g, st, 1e-3)
            done += n
            errs = {nm: rel(cc.get_field(nm), getattr(st, nm)) for nm in ("U", "V", "W")}
            assert max(errs.values()) < 1e-12, (done, errs)
            assert rel(cc.get_field("P"), st.P) < 1e-10
            assert abs(cc.dPdx - st.dPdx) <= 1e-9 * abs(st.dPdx) + 50 * 2.2e-16 * abs(st.Qflow_x_0) / 1e-3
    finally:
        cc.close()


@pytest.mark.parametrize("n", [27, 32, 40, 54, 128, 192, 256, 384])
def test_fft_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    X = cpu_rk3.fft(x, -1)
    ref = np.fft.fft(x)
    assert np.abs(X - ref).max() <= 1e-13 * np.abs(ref).max()
    xi = cpu_rk3.fft(ref, +1) / n
    assert np.abs(xi - x).max() <= 1e-13 * np.abs(x).max()


def test_fft_rejects_other_lengths():
    with pytest.raises(ValueError):
        cpu_rk3.fft(np.ones(14), -1)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_zgtsv_matches_lapack_with_pivoting(seed):
    rng = np.random.default_rng(seed)
    n = 40
    c = lambda m: rng.standard_normal(m) + 1j * rng.standard_normal(m)
    # off-diagonals larger than the diagonal: row interchanges are taken
    dl, d, du, b = 3.0 * c(n - 1), 0.2 * c(n), 3.0 * c(n - 1), c(n)
    x, info = cpu_rk3.zgtsv(dl, d, du, b)
    _, _, _, xr, info_r = lapack.zgtsv(dl, d, du, b.reshape(-1, 1))
    assert info == info_r == 0
    assert np.abs(x - xr[:, 0]).max() <= 1e-12 * np.abs(xr).max()
    A = np.diag(d) + np.diag(dl, -1) + np.diag(du, 1)
    assert np.abs(A @ x - b).max() <= 1e-11 * np.abs(b).max()


def test_zgtsv_reports_singular():
    x, info = cpu_rk3.zgtsv(np.zeros(2), np.array([0.0, 1.0, 1.0]), np.zeros(2), np.ones(3))
    assert info == 1
