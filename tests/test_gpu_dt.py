"""compute_dt with a positive CFL number (src/time_integration.f90:219-267)
on the GPU against the oracle.

The reference scans Max(dx/|U|) over the interior (so a zero velocity gives
an infinite convective bound, which drops out of the Minval), takes the
viscous bound CFL*d^2/nu per direction, the smaller of the two, and caps dt
at 0.1.  Every case below is compared exactly: the scan is a max of
quotients and the rest is scalar arithmetic in the reference's order.
"""
import math

import numpy as np
import pytest

from oracle import channel_oracle as co

pytestmark = pytest.mark.gpu

NU = 1.0 / 5600.0


def make(cfl, nu=NU, grid=(34, 65, 34, math.pi, math.pi / 2, 1)):
    import channel3d_parallel_b200 as c3d
    nx, ny, nz, lx, lz, gt = grid
    p = co.channel_params(nx, ny, nz, lx, lz, nu, grid_type=gt, cfl=cfl)
    g = co.Grid(p)
    st = co.seeded_initial_state(g, p["dpdx"])
    ch = c3d.Channel(nx_global=nx, ny_global=ny, nz_global=nz, Lxp=lx, Lzp=lz, nu=nu, CFL=cfl,
                     x_mass_cte=1, grid_type=gt, alpha_stretch=2.0, dPdx=p["dpdx"])
    ch.set_grid(g.x[1:], g.y[1:], g.z[1:])
    return p, g, st, ch


def upload(ch, st):
    for name, a in (("U", st.U), ("V", st.V), ("W", st.W)):
        ch.upload(name, a[1:, 1:, 1:])


@pytest.mark.parametrize("cfl", [0.05, 0.3])
def test_compute_dt_cfl_positive(cfl):
    p, g, st, ch = make(cfl)
    try:
        upload(ch, st)
        ref = co.compute_dt(g, st)
        assert 0.0 < ref <= 0.1
        assert ch.compute_dt() == ref
    finally:
        ch.close()


def test_compute_dt_zero_velocities_give_infinite_bounds():
    """U = 0 at interior points: dx/|U| is +Inf there, so the U bound is
    infinite and dt comes from V, W or the viscous bound; with V and W zero
    as well every convective bound is infinite and dt is the viscous one."""
    p, g, st, ch = make(0.5)
    try:
        st.U[5, 7, 9] = 0.0
        st.U[10:12, 20, 3:6] = 0.0
        upload(ch, st)
        ref = co.compute_dt(g, st)
        assert math.isfinite(ref)
        assert ch.compute_dt() == ref
        st.U[:] = 0.0
        st.V[:] = 0.0
        st.W[:] = 0.0
        upload(ch, st)
        ref = co.compute_dt(g, st)
        nu = p["nu"]
        vis = min(0.5 * g.dxmin ** 2 / nu, 0.5 * g.dymin ** 2 / nu, 0.5 * g.dzmin ** 2 / nu)
        assert ref == min(vis, 0.1)
        assert ch.compute_dt() == ref
    finally:
        ch.close()


def test_compute_dt_is_capped_at_one_tenth():
    """A large viscosity-free bound and a slow field: dt = min(dt, 0.1)."""
    p, g, st, ch = make(5.0, nu=1e-9)
    try:
        for a in (st.U, st.V, st.W):
            a *= 1e-3
        upload(ch, st)
        assert co.compute_dt(g, st) == 0.1
        assert ch.compute_dt() == 0.1
    finally:
        ch.close()


def test_compute_dt_negative_cfl_is_fixed_step():
    p, g, st, ch = make(-2.5e-3)
    try:
        upload(ch, st)
        assert ch.compute_dt() == 2.5e-3 == co.compute_dt(g, st)
    finally:
        ch.close()
