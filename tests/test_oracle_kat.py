"""Known-answer tests that pin the CPU oracle (the reference ships no golden
data, so the oracle is checked against the mathematics of each operator)."""
import math

import numpy as np
import pytest
from scipy.linalg import lapack

from oracle import channel_oracle as co


@pytest.fixture(scope="module")
def small():
    p = co.channel_params(34, 33, 26, math.pi, math.pi / 2, 1.0 / 5600.0)
    return p, co.Grid(p)


def _Lh(g, phi):
    """Discrete operator div(G phi) with the reference's boundary conditions."""
    phi = phi.copy()
    phi[g.nxg - 1, :, :] = phi[2, :, :]
    phi[2:g.nxg, :, g.nzp + 2] = phi[2:g.nxg, :, 2]
    Gx, Gy, Gz = co.gradient(g, phi)
    co.apply_boundary_conditions(g, Gx, Gy, Gz)
    return co.divergence(g, Gx, Gy, Gz)


def _interior(g):
    return slice(2, g.nxp + 2), slice(2, g.nyg), slice(2, g.nzp + 2)


def test_grid_matches_reference_formulas(small):
    p, g = small
    # x faces: x(i) = Lxp*(i-1)/(nx-2)  (src/input_output.f90:146-149)
    assert np.allclose(g.x[1:], p["lxp"] * np.arange(g.nx) / (g.nx - 2), rtol=0, atol=1e-15)
    # tanh grid is symmetric and spans [0, Ly]
    y = g.y[1:]
    assert y[0] == 0.0 and abs(y[-1] - 2.0) < 1e-15
    assert np.allclose(y + y[::-1], 2.0, atol=1e-14)
    # ghost centres mirror the walls (src/initialization.f90:193-195)
    assert abs(g.yg[1] + g.yg[2]) < 1e-15


@pytest.mark.parametrize("mode", [(3, 0), (0, 2), (5, 4), (0, 0), (16, 12)])
def test_poisson_single_mode(small, mode):
    """A single Fourier mode times an arbitrary y profile is recovered."""
    p, g = small
    I, J, K = _interior(g)
    rng = np.random.default_rng(3)
    prof = rng.random(g.nyg - 2)
    xs, zs = np.arange(g.nxp), np.arange(g.nzp)
    phi = g.rhs_p_array()
    phi[I, J, K] = (np.cos(2 * np.pi * mode[0] * xs / g.nxp)[:, None, None]
                    * np.cos(2 * np.pi * mode[1] * zs / g.nzp)[None, None, :]
                    * prof[None, :, None])
    sol = co.solve_poisson_equation(g, _Lh(g, phi))
    d = sol[I, J, K] - phi[I, J, K]
    if mode == (0, 0):
        d = d - d.mean()          # pinned null space: a constant shift
    assert np.abs(d).max() < 1e-12


def test_poisson_random_field(small):
    p, g = small
    I, J, K = _interior(g)
    phi = g.rhs_p_array()
    phi[I, J, K] = np.random.default_rng(5).random((g.nxp, g.nyg - 2, g.nzp))
    sol = co.solve_poisson_equation(g, _Lh(g, phi))
    d = sol[I, J, K] - phi[I, J, K]
    assert (d.max() - d.min()) < 1e-12


def test_projection_divergence_free(small):
    p, g = small
    st = co.seeded_initial_state(g, p["dpdx"])
    d = co.divergence(g, st.U, st.V, st.W)
    assert np.abs(d[2:g.nxg - 1, 2:g.nyg, 2:g.nzg - 1]).max() < 1e-12
    co.compute_time_step_RK3(g, st, 1e-3)
    d = co.divergence(g, st.U, st.V, st.W)
    assert np.abs(d[2:g.nxg - 1, 2:g.nyg, 2:g.nzg - 1]).max() < 1e-12


def test_constant_mass_flow(small):
    p, g = small
    st = co.seeded_initial_state(g, p["dpdx"])
    q0 = st.Qflow_x_0
    for _ in range(2):
        co.compute_time_step_RK3(g, st, 1e-3)
    q, n = co.mean_mass_flow_u(g, st.U)
    assert abs(q / n - q0) < 1e-13


def test_poiseuille_balance_uniform_grid():
    """Exact parabola on a uniform y grid: convective terms vanish and
    nu*d2u/dy2 + dPdx = 0 away from the first cell (the odd ghost is not
    the parabola's mirror image)."""
    nu = 1.0 / 5600.0
    p = co.channel_params(18, 33, 14, 1.0, 0.5, nu, grid_type=0)
    g = co.Grid(p)
    st = co.State(g)
    ym = g.yg
    for j in range(1, g.nyg + 1):
        st.U[:, j, :] = 1.5 * ym[j] * (2.0 - ym[j])
    co.apply_boundary_conditions(g, st.U, st.V, st.W)
    r = co.compute_rhs_u(g, st.U, st.V, st.W, 3.0 * nu)
    assert np.abs(r[:, 1:-1, :]).max() < 1e-15 * 1e3


def test_rhs_linear_in_viscous_part(small):
    """With U,V,W scaled by s, the RHS is convective*s^2 + viscous*s + dPdx."""
    p, g = small
    st = co.seeded_initial_state(g, p["dpdx"])
    f = lambda s: co.compute_rhs_u(g, s * st.U, s * st.V, s * st.W, 0.0)
    r1, r2, r3 = f(1.0), f(2.0), f(3.0)
    # second difference in s is 2*convective; third-order combination vanishes
    assert np.abs(r3 - 3 * r2 + 3 * r1).max() < 1e-11 * max(1.0, np.abs(r1).max())


def test_thomas_matches_zgtsv_to_roundoff():
    """The unpivoted elimination used on the GPU versus LAPACK zgtsv (the
    reference's call, src/poisson.f90:72) on the stretched 129-face grid."""
    p = co.channel_params(194, 129, 194, 4 * math.pi, 4 * math.pi / 3, 1 / 5600)
    g = co.Grid(p)
    nyg = g.nyg
    dd, dl, du = g.Dd[2:nyg], g.Dl[3:nyg], g.Du[2:nyg - 1]
    rng = np.random.default_rng(0)
    for (i, k) in [(0, 0), (1, 0), (0, 1), (3, 7), (96, 96)]:
        D = (dd + g.kxx[i]) + g.kzz[k]
        if i == 0 and k == 0:
            D = D.copy(); D[0] *= 1.5
        b = rng.standard_normal(len(D)) + 1j * rng.standard_normal(len(D))
        x1 = lapack.zgtsv(dl.astype(complex), D.astype(complex), du.astype(complex), b[:, None])[3][:, 0]
        dm, bb = D.copy(), b.copy()
        for j in range(len(D) - 1):
            m = dl[j] / dm[j]
            dm[j + 1] -= m * du[j]
            bb[j + 1] -= m * bb[j]
        bb[-1] /= dm[-1]
        for j in range(len(D) - 2, -1, -1):
            bb[j] = (bb[j] - du[j] * bb[j + 1]) / dm[j]
        assert np.abs(bb - x1).max() / np.abs(x1).max() < 1e-11


def test_pressure_solves_the_inhomogeneous_neumann_problem():
    """compute_pressure (src/pressure.f90): the 3-point Laplacian of P, with the
    y ghosts P(1) = P(2) - dy*bc_1 and P(nyg) = P(nyg-1) + dy*bc_2, equals the
    divergence of the right-hand sides in every (x, z) Fourier mode except the
    pinned mean (whose row 2 carries the factor 3/2)."""
    import math
    p = co.channel_params(34, 33, 26, math.pi, 1.0, 1 / 5600)
    g = co.Grid(p)
    st = co.seeded_initial_state(g, p["dpdx"])
    co.compute_time_step_RK3(g, st, 1e-3)
    bc1, bc2 = co.compute_pressure_bc(g, st.V)
    rhs = co.compute_pressure_rhs(g, st, bc1, bc2)
    P = co.compute_pressure(g, st).copy()
    nxp, nzp, nyg = g.nxp, g.nzp, g.nyg
    Pi = P[2:nxp + 2, :, 2:nzp + 2]                  # periodic interior, all j
    lap_xz = ((np.roll(Pi, -1, 0) - 2 * Pi + np.roll(Pi, 1, 0)) / g.dx ** 2
              + (np.roll(Pi, -1, 2) - 2 * Pi + np.roll(Pi, 1, 2)) / g.dz ** 2)
    y, yg = g.y, g.yg
    res = np.zeros((nxp, nyg - 2, nzp))
    for j in range(2, nyg):
        a = 1.0 / (y[j] - y[j - 1]) / (yg[j + 1] - yg[j])
        c = 1.0 / (y[j] - y[j - 1]) / (yg[j] - yg[j - 1])
        lap_y = a * Pi[:, j + 1, :] - (a + c) * Pi[:, j, :] + c * Pi[:, j - 1, :]
        res[:, j - 2, :] = lap_xz[:, j, :] + lap_y - rhs[2:nxp + 2, j, 2:nzp + 2]
    scale = np.abs(rhs[2:nxp + 2, 2:nyg, 2:nzp + 2]).max()
    # every non-mean mode solves the discrete problem
    fluct = res - res.mean(axis=(0, 2), keepdims=True)
    assert np.abs(fluct).max() < 1e-9 * scale
    # the mean mode solves it on every row but the pinned one
    assert np.abs(res.mean(axis=(0, 2))[1:]).max() < 1e-9 * scale
    # the wall conditions are not trivial for this state
    assert np.abs(bc1[2:g.nxg, 2:g.nzg]).max() > 0
