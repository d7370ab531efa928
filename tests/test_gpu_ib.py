"""GPU parity of the immersed-boundary path against the CPU oracle.

Tolerances (max-norm relative): E / E1n / R and Heaviside fields 1e-12 (the
delta weights come from the device's sqrt/asin); Schur operator 1e-11; IB
RK3 steps after 1 and 10 steps, U, V, W and the surface unknowns fb, 1e-10
with both Schur solves converged to 1e-14.  R is a fixed-order gather, so
the Schur operator and whole IB steps repeat bit for bit.
"""
import math

import numpy as np
import pytest

from oracle import channel_oracle as co
from oracle import ib_oracle as ibo

pytestmark = pytest.mark.gpu

NU = 3.076923076923077e-04

CASES = {
    # planar static wall at y = Ly/2 on a uniform grid (examples/input_parameters_ib_planar_wall)
    "center_wall": dict(nx_global=18, ny_global=33, nz_global=18, Lxp=1.718, Lzp=0.859,
                        grid_type=0, alpha_stretch=0.0, body_type="center_wall", nxb=16, nzb=16,
                        cfl=-0.01),
    # one plane at y = 0.2 with a standing wave inside the uniform wall buffer
    # of grid type 2 (uniform up to y = 0.42, every stencil row in it)
    "wall_standing_wave": dict(nx_global=34, ny_global=49, nz_global=14, Lxp=2.0, Lzp=0.6,
                               grid_type=2, alpha_stretch=2.0, min_buffer_width=0.45,
                               body_type="wall_standing_wave", nxb=32, nzb=12,
                               body_param_1=0.02, body_param_2=2 * math.pi / 5.0,
                               body_param_3=1.0, body_param_4=0.2, cfl=-1e-3),
    # two concentric z cylinders on a uniform grid (examples/input_parameters_ib_double_rotating_cylinders)
    "double_cylinders_z": dict(nx_global=34, ny_global=33, nz_global=14, Lxp=2.0, Lzp=1.0,
                               grid_type=0, alpha_stretch=0.0, body_type="double_cylinders_z",
                               nxb=0, nzb=6, body_param_1=0.15, body_param_2=0.3,
                               body_param_3=0.015, cfl=-0.01),
    # cfg3's body: two separate counter-rotating spanwise cylinders (extension)
    "two_cylinders_z": dict(nx_global=34, ny_global=33, nz_global=14, Lxp=4.5, Lzp=1.0,
                            grid_type=0, alpha_stretch=0.0, body_type="two_cylinders_z",
                            nxb=8, nzb=6, body_param_1=0.15, body_param_2=0.5,
                            body_param_3=1.5, body_param_4=0.3, cfl=-0.005),
    # cfg4's body: wall-mounted bending plates, 32 x 16 markers each (extension)
    "wall_plates": dict(nx_global=34, ny_global=65, nz_global=18, Lxp=2.0, Lzp=1.0,
                        grid_type=2, alpha_stretch=2.0, min_buffer_width=0.3,
                        body_type="wall_plates", nxb=2, nzb=2, body_param_1=0.2,
                        body_param_2=0.01, body_param_3=2 * math.pi, body_param_4=7,
                        cfl=-1e-3),
    # both walls with a wave travelling in x and a cosine ramp-up of its
    # amplitude over the first 10 steps (src/immersed_boundary_geometry.f90:271-390)
    "traveling_wave_x": dict(nx_global=34, ny_global=65, nz_global=10, Lxp=2.0, Lzp=0.5,
                             grid_type=2, alpha_stretch=2.0, min_buffer_width=0.1,
                             body_type="traveling_wave_x", nxb=16, nzb=3, body_param_1=0.05,
                             body_param_2=0.5, body_param_3=math.pi, body_ramp_up_time=0.05,
                             cfl=-0.005),
    # both walls with a standing wave (examples/input_parameters_ib_standing_wave)
    "standing_wave": dict(nx_global=34, ny_global=65, nz_global=10, Lxp=2.0, Lzp=0.5,
                          grid_type=2, alpha_stretch=2.0, min_buffer_width=0.1,
                          body_type="standing_wave", nxb=16, nzb=3, body_param_1=0.05,
                          body_param_2=0.5, body_param_3=1.0, cfl=-0.02),
}


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def build(case, cg_tol=1e-12, cg_max_iter=200, x_mass_cte=1, extra=None):
    import channel3d_parallel_b200 as c3d
    kw = dict(CASES[case])
    kw.update(extra or {})
    nx, ny, nz = kw.pop("nx_global"), kw.pop("ny_global"), kw.pop("nz_global")
    lx, lz = kw.pop("Lxp"), kw.pop("Lzp")
    gt, al = kw.pop("grid_type"), kw.pop("alpha_stretch")
    cfl = kw.pop("cfl")
    p = co.channel_params(nx, ny, nz, lx, lz, NU, alpha=al, grid_type=gt, cfl=cfl,
                          x_mass_cte=x_mass_cte, cg_tol=cg_tol, cg_max_iter=cg_max_iter,
                          **{k.lower(): v for k, v in kw.items()})
    g = co.Grid(p)
    st = co.seeded_initial_state(g, p["dpdx"], amplitude=0.05, dt=-cfl)
    ib = ibo.IBState(g, p, t=0.0)
    ibo.compute_heaviside(g, ib)
    q, n = co.mean_mass_flow_u(g, st.U, ib.Hu)
    st.Qflow_x_0 = q / n
    ch = c3d.Channel(nx_global=nx, ny_global=ny, nz_global=nz, Lxp=lx, Lzp=lz, nu=NU, CFL=cfl,
                     x_mass_cte=x_mass_cte, grid_type=gt, alpha_stretch=al, dPdx=p["dpdx"],
                     cg_tol=cg_tol, cg_max_iter=cg_max_iter, **kw)
    ch.set_grid(g.x[1:], g.y[1:], g.z[1:])
    for name, ref in (("U", st.U), ("V", st.V), ("W", st.W)):
        ch.upload(name, ref[1:, 1:, 1:])
    ch.compute_dt()
    ch.compute_heaviside()
    ch.set_scalars(dPdx=st.dPdx, t=0.0, Qflow_x_0=st.Qflow_x_0)
    return p, g, st, ib, ch


@pytest.fixture(params=list(CASES))
def setup(request):
    p, g, st, ib, ch = build(request.param)
    yield request.param, p, g, st, ib, ch
    ch.close()


def test_marker_geometry(setup):
    case, p, g, st, ib, ch = setup
    b = ib.body
    assert ch.dims["nb"] == b.nb
    for name, ref in (("XB", b.xb), ("YB", b.yb), ("ZB", b.zb), ("SB", b.sb),
                      ("NORMALS", b.normals), ("UB", b.ub)):
        got = ch.download(name)
        assert np.abs(got - ref).max() <= 1e-14 * max(1.0, np.abs(ref).max()), name


def test_interpolation_and_spreading(setup):
    case, p, g, st, ib, ch = setup
    rng = np.random.default_rng(7)
    U, V, W = (rng.standard_normal(a.shape) for a in (st.U, st.V, st.W))
    co.apply_boundary_conditions(g, U, V, W)
    for name, A in (("U", U), ("V", V), ("W", W)):
        ch.upload(name, A[1:, 1:, 1:])
    assert rel(ch.regT(), ib.ops.E(U, V, W)) < 1e-12
    assert rel(ch.regT_1n(), ib.ops.E1n(U, V, W)) < 1e-12
    Pr = g.rhs_p_array()
    Pr[2:, 2:, 2:] = rng.standard_normal(Pr[2:, 2:, 2:].shape)
    ch.upload("P_INTERIM", Pr[2:, 2:, 2:])
    assert rel(ch.regTc_1n("P_INTERIM"), ib.ops.E1n_c(Pr)) < 1e-12
    nb = ib.body.nb
    f = rng.standard_normal(nb)
    for comp, (fname, shape) in enumerate((("U_REG", st.U.shape), ("V_REG", st.V.shape),
                                           ("W_REG", st.W.shape))):
        ch.reg(comp + 1, f)
        ref = ib.ops.R(comp, f, shape)
        assert rel(ch.download(fname), ref[1:, 1:, 1:]) < 1e-12, fname


def test_heaviside(setup):
    case, p, g, st, ib, ch = setup
    for name, ref in (("HU_INTERIOR", ib.Hu), ("HV_INTERIOR", ib.Hv), ("HW_INTERIOR", ib.Hw)):
        assert np.abs(ch.download(name) - ref[1:, 1:, 1:]).max() < 1e-11, name
    assert np.abs(ch.download("HC_EXTERIOR") - ib.Hc_ext[2:, 2:, 2:]).max() < 1e-11
    assert rel(ch.download("E1NHC_EXT"), ib.E1nHc_ext) < 1e-10
    assert rel(ch.download("E1NH_EXT"), ib.E1nH_ext) < 1e-10


def test_spread_and_schur_are_bitwise_reproducible(setup):
    case, p, g, st, ib, ch = setup
    nb = ib.body.nb
    f = np.random.default_rng(5).standard_normal(4 * nb)
    assert np.array_equal(ch.schur(f), ch.schur(f))
    ch.reg(2, f[:nb])
    r1 = ch.download("V_REG")
    ch.reg(2, f[:nb])
    assert np.array_equal(r1, ch.download("V_REG"))


def test_schur_operator(setup):
    case, p, g, st, ib, ch = setup
    rng = np.random.default_rng(9)
    f = rng.standard_normal(4 * ib.body.nb)
    dt = -p["cfl"]
    assert rel(ch.schur(f), ibo.schur(g, ib, f, dt)) < 1e-11


STEP_TOL = 1e-14     # BiCGSTAB tolerance of the step parity runs (both sides converge)


@pytest.mark.parametrize("nsteps", [1, 10])
@pytest.mark.parametrize("mode", ["none", "band"])
@pytest.mark.parametrize("case", [c for c in CASES if c != "wall_plates"])
def test_ib_rk3_steps(case, mode, nsteps):
    """IB RK3 steps against the oracle (unpreconditioned BiCGSTAB, the
    reference's), both Schur solves converged to 1e-14: U, V, W and the
    surface unknowns fb within 1e-10 (max-norm relative) after 1 and 10 steps,
    with the reference's solver and with the banded preconditioner."""
    from channel3d_parallel_b200 import lib as L
    p, g, st, ib, ch = build(case, cg_tol=STEP_TOL, cg_max_iter=600)
    try:
        ch.set_mode(precond=L.PRECOND_BAND if mode == "band" else L.PRECOND_NONE)
        dt = -p["cfl"]
        ch.compute_time_step_RK3(nsteps)
        for _ in range(nsteps):
            ibo.compute_time_step_RK3_ib(g, st, ib, dt)
        errs = {name: rel(ch.download(name), ref[1:, 1:, 1:])
                for name, ref in (("U", st.U), ("V", st.V), ("W", st.W))}
        errs["FB"] = rel(ch.download("FB"), ib.fb)
        assert max(errs.values()) < 1e-10, errs
        s = ch.stats()
        assert s["bicgstab_solves"] == 3 * nsteps
        assert s["last_residual"] < STEP_TOL
        assert ib.last_err < STEP_TOL
    finally:
        ch.close()


@pytest.mark.parametrize("case", ["wall_standing_wave", "two_cylinders_z"])
def test_ib_steps_repeat_bitwise(case):
    """Two handles advanced from the same state give identical fields and
    surface unknowns (no order-dependent sums anywhere in the IB step)."""
    out = []
    for _ in range(2):
        p, g, st, ib, ch = build(case, cg_tol=1e-13, cg_max_iter=400)
        try:
            ch.compute_time_step_RK3(3)
            out.append([ch.download(n) for n in ("U", "V", "W", "FB")])
        finally:
            ch.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_wall_plates_steps():
    """The plates of the test grid are resolved more finely than the grid
    (2-4 markers per cell): the Schur system there is close to singular and
    stops at cg_max_iter, so two unconverged Krylov runs agree only to their
    amplified round-off.  What holds regardless: the step completes and the
    projected velocity is divergence-free."""
    p, g, st, ib, ch = build("wall_plates", cg_max_iter=50)
    try:
        ch.compute_time_step_RK3(2)
        assert ch.check_finite() == 0
        assert ch.check_divergence() < 1e-10
        assert ch.stats()["bicgstab_solves"] == 6
    finally:
        ch.close()


@pytest.mark.parametrize("cfg", ["cfg2", "cfg3"])
def test_full_size_schur_operator(cfg):
    """The Schur operator on the full-size IB configurations (192x129x192 with
    the standing-wave plane, 36,864 markers; 256x129x128 with two rotating
    cylinders, 51,200 markers) against the oracle at 1e-11: operator set-up,
    Heaviside fields, spreading, the banded Poisson solve with 255/127-row
    slabs and the gathers at the sizes the benchmark runs."""
    import os
    import sys
    import channel3d_parallel_b200 as c3d
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    c = dict(bench.IB_CONFIGS[cfg])
    nx, ny, nz = c.pop("grid")
    c.pop("desc")
    nu = c.pop("nu")
    lx, lz = c.pop("Lxp"), c.pop("Lzp")
    gt, al = c.pop("grid_type"), c.pop("alpha_stretch")
    p = co.channel_params(nx, ny, nz, lx, lz, nu, alpha=al, grid_type=gt, cfl=-1e-3, x_mass_cte=1,
                          **{k.lower(): v for k, v in c.items()})
    g = co.Grid(p)
    ib = ibo.IBState(g, p, t=0.0)
    ibo.compute_heaviside(g, ib)
    with c3d.Channel(nx_global=nx, ny_global=ny, nz_global=nz, Lxp=lx, Lzp=lz, nu=nu, CFL=-1e-3, x_mass_cte=1,
                     grid_type=gt, alpha_stretch=al, **c) as ch:
        ch.set_grid(g.x[1:], g.y[1:], g.z[1:])
        ch.compute_dt()
        ch.compute_heaviside()
        assert ch.dims["nb"] == ib.body.nb
        f = np.random.default_rng(3).standard_normal(4 * ib.body.nb)
        assert rel(ch.schur(f), ibo.schur(g, ib, f, 1e-3)) < 1e-11
