"""GPU parity of the FP64 path against the CPU oracle, through the C-ABI.

Tolerances (max-norm error relative to the max-norm of the oracle field):
  copies (boundary conditions)            bit-exact
  right-hand sides, divergence            1e-12
  Poisson solve, projection               1e-11  (Thomas vs LAPACK zgtsv, FFT rounding)
  RK3 steps (1 and 10)                    1e-10  (north-star bar)
"""
import math

import numpy as np
import pytest

from oracle import channel_oracle as co

pytestmark = pytest.mark.gpu

CASES = {
    # name: (nx_global, ny_global, nz_global, Lxp, Lzp, grid_type)
    "cfg0_34x65x34": (34, 65, 34, math.pi, math.pi / 2, 1),
    "odd_ny_radix3": (50, 34, 26, 2.0, 1.0, 1),
    "uniform_small": (18, 17, 14, 1.0, 0.7, 0),
    # 127 interior rows: a kx slab spans a 4-CTA cluster (FP64)
    "tall_ny_clusters": (18, 129, 18, 1.0, 0.5, 1),
    # Nz = 54 = 2 * 3^3: three radix-3 stages, 216-thread slab CTAs
    "nz54_radix3": (26, 20, 56, 1.7, 0.9, 1),
    # Nz = 256 > 192: the wide slab CTAs (256 threads, two per SM)
    "nz256_wide_slab": (18, 17, 258, 1.0, 2.0, 1),
}


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def make_pair(case, amplitude=0.1, seed=0):
    import channel3d_parallel_b200 as c3d
    nx, ny, nz, lx, lz, gt = CASES[case]
    nu = 1.0 / 5600.0
    p = co.channel_params(nx, ny, nz, lx, lz, nu, grid_type=gt)
    g = co.Grid(p)
    st = co.seeded_initial_state(g, p["dpdx"], amplitude=amplitude, seed=seed)
    ch = c3d.Channel(nx_global=nx, ny_global=ny, nz_global=nz, Lxp=lx, Lzp=lz, nu=nu,
                     CFL=-1e-3, x_mass_cte=1, grid_type=gt, alpha_stretch=2.0, dPdx=p["dpdx"])
    ch.set_grid(g.x[1:], g.y[1:], g.z[1:])
    ch.upload("U", st.U[1:, 1:, 1:])
    ch.upload("V", st.V[1:, 1:, 1:])
    ch.upload("W", st.W[1:, 1:, 1:])
    ch.set_scalars(dPdx=st.dPdx, t=0.0, Qflow_x_0=st.Qflow_x_0)
    ch.compute_dt()
    return p, g, st, ch


@pytest.fixture(params=list(CASES))
def pair(request):
    p, g, st, ch = make_pair(request.param)
    yield p, g, st, ch
    ch.close()


def test_library_grid_matches_oracle():
    import channel3d_parallel_b200 as c3d
    p = co.channel_params(34, 65, 34, math.pi, math.pi / 2, 1 / 5600)
    g = co.Grid(p)
    with c3d.Channel(nx_global=34, ny_global=65, nz_global=34, Lxp=math.pi, Lzp=math.pi / 2,
                     nu=1 / 5600, CFL=-1e-3, grid_type=1, alpha_stretch=2.0) as ch:
        gr = ch.grid()
    for k in ("x", "y", "z", "xg", "yg", "zg"):
        ref = getattr(g, k)[1:]
        assert np.abs(gr[k] - ref).max() <= 4e-16 * max(1.0, np.abs(ref).max()), k


def test_boundary_conditions_bit_exact(pair):
    p, g, st, ch = pair
    rng = np.random.default_rng(11)
    U, V, W = (rng.standard_normal(a.shape) for a in (st.U, st.V, st.W))
    ch.upload("U", U[1:, 1:, 1:]); ch.upload("V", V[1:, 1:, 1:]); ch.upload("W", W[1:, 1:, 1:])
    ch.apply_boundary_conditions("UVW")
    co.apply_boundary_conditions(g, U, V, W)
    assert np.array_equal(ch.download("U"), U[1:, 1:, 1:])
    assert np.array_equal(ch.download("V"), V[1:, 1:, 1:])
    assert np.array_equal(ch.download("W"), W[1:, 1:, 1:])


def test_rhs(pair):
    p, g, st, ch = pair
    ru = co.compute_rhs_u(g, st.U, st.V, st.W, st.dPdx)
    rv = co.compute_rhs_v(g, st.U, st.V, st.W, st.dPdy)
    rw = co.compute_rhs_w(g, st.U, st.V, st.W, st.dPdz)
    assert rel(ch.compute_rhs_u(), ru) < 1e-12
    assert rel(ch.compute_rhs_v(), rv) < 1e-12
    assert rel(ch.compute_rhs_w(), rw) < 1e-12


def test_divergence_and_poisson(pair):
    p, g, st, ch = pair
    # perturb so the field is not divergence-free
    rng = np.random.default_rng(2)
    U = st.U.copy(); U[2:g.nx, 2:g.nyg, 2:g.nzg] += 0.01 * rng.standard_normal(U[2:g.nx, 2:g.nyg, 2:g.nzg].shape)
    co.apply_boundary_conditions(g, U, st.V, st.W)
    ch.upload("U", U[1:, 1:, 1:])
    ch.divergence()
    d_ref = co.divergence(g, U, st.V, st.W)
    d_gpu = ch.download("RHS_P")
    assert rel(d_gpu, d_ref[2:, 2:, 2:]) < 1e-12
    ch.solve_poisson_equation(rk_step=1)
    s_ref = co.solve_poisson_equation(g, d_ref.copy(), st, rk_step=1, dt=1e-3)
    s_gpu = ch.download("RHS_P")
    assert rel(s_gpu, s_ref[2:, 2:, 2:]) < 1e-11
    assert rel(ch.download("P"), st.P[1:, 1:, 1:]) < 1e-11


def test_non_IB_projection(pair):
    p, g, st, ch = pair
    rng = np.random.default_rng(4)
    U = st.U.copy(); U[2:g.nx, 2:g.nyg, 2:g.nzg] += 0.01 * rng.standard_normal(U[2:g.nx, 2:g.nyg, 2:g.nzg].shape)
    co.apply_boundary_conditions(g, U, st.V, st.W)
    st.U = U
    ch.upload("U", U[1:, 1:, 1:])
    ch.compute_non_IB_projection(rk_step=0)
    co.compute_non_IB_projection(g, st, 1e-3)
    for name, ref in (("U", st.U), ("V", st.V), ("W", st.W)):
        assert rel(ch.download(name), ref[1:, 1:, 1:]) < 1e-11, name
    assert rel(ch.download("P_INTERIM"), st.P_interim[2:, 2:, 2:]) < 1e-11


@pytest.mark.parametrize("nsteps", [1, 10])
def test_rk3_steps(pair, nsteps):
    p, g, st, ch = pair
    ch.compute_time_step_RK3(nsteps)
    for _ in range(nsteps):
        co.compute_time_step_RK3(g, st, 1e-3)
    errs = {name: rel(ch.download(name), ref[1:, 1:, 1:])
            for name, ref in (("U", st.U), ("V", st.V), ("W", st.W), ("P", st.P))}
    assert max(errs.values()) < 1e-10, errs
    s = ch.stats()
    # dPdx = (dPdx_prev + shift/dt)/2 with shift = Q0 - Q(U), a difference of
    # nearly equal bulk fluxes: round-off of Q (a few eps*Q0) divided by dt
    dt = 1e-3
    assert abs(s["dPdx"] - st.dPdx) <= 1e-9 * abs(st.dPdx) + 50 * 2.2e-16 * abs(st.Qflow_x_0) / dt
    assert s["steps"] == nsteps
    # Nz > 192 only fits the wide slab CTAs; small grids run in one wave of
    # clusters either way and take the narrow shape
    assert s["slab_narrow"][0] == (0 if g.nz - 2 > 192 else 1)
    assert ch.check_divergence() < 1e-12
    assert ch.check_finite() == 0


def test_mass_flow_entries(pair):
    p, g, st, ch = pair
    q, n = co.mean_mass_flow_u(g, st.U)
    assert abs(ch.compute_mean_mass_flow_U() - q / n) < 1e-14
    assert abs(ch.compute_dPx_for_constant_mass_flow() - (st.Qflow_x_0 - q / n)) < 1e-14


def test_product_initial_state_matches_oracle():
    import channel3d_parallel_b200 as c3d
    nx, ny, nz, lx, lz, gt = CASES["cfg0_34x65x34"]
    p = co.channel_params(nx, ny, nz, lx, lz, 1 / 5600, grid_type=gt)
    g = co.Grid(p)
    st = co.seeded_initial_state(g, p["dpdx"])
    with c3d.Channel(nx_global=nx, ny_global=ny, nz_global=nz, Lxp=lx, Lzp=lz, nu=1 / 5600,
                     CFL=-1e-3, x_mass_cte=1, grid_type=gt, alpha_stretch=2.0) as ch:
        ch.set_grid(g.x[1:], g.y[1:], g.z[1:])
        q0 = c3d.seeded_initial_state(ch, p["dpdx"], 1 / 5600)
        assert abs(q0 - st.Qflow_x_0) < 1e-13
        for name, ref in (("U", st.U), ("V", st.V), ("W", st.W)):
            assert rel(ch.download(name), ref[1:, 1:, 1:]) < 1e-12


def test_nan_is_reported():
    """A non-finite value uploaded from the host comes back as C3D_ERR_NAN."""
    import channel3d_parallel_b200 as c3d
    p, g, st, ch = make_pair("uniform_small")
    try:
        U = st.U.copy()
        U[5, 5, 5] = np.nan
        ch.upload("U", U[1:, 1:, 1:])
        with pytest.raises(c3d.C3DError) as e:
            ch.check_finite()
        assert e.value.code == -3
    finally:
        ch.close()


def test_partial_box_transfer():
    p, g, st, ch = make_pair("uniform_small")
    try:
        full = ch.download("V")
        sub = ch.download("V", lb=(3, 2, 4), ub=(9, 7, 8))
        assert np.array_equal(sub, full[2:9, 1:7, 3:8])
        ch.upload("V", np.zeros((7, 6, 5)), lb=(3, 2, 4))
        full2 = ch.download("V")
        assert np.all(full2[2:9, 1:7, 3:8] == 0.0)
    finally:
        ch.close()


def test_full_size_one_step_parity():
    """192x129x192 (the throughput configuration): one RK3 step against the
    oracle, plus size-independent properties over further steps."""
    import channel3d_parallel_b200 as c3d
    nu = 1.0 / 5600.0
    p = co.channel_params(194, 129, 194, 4 * math.pi, 4 * math.pi / 3, nu)
    g = co.Grid(p)
    st = co.seeded_initial_state(g, p["dpdx"])
    with c3d.Channel(nx_global=194, ny_global=129, nz_global=194, Lxp=4 * math.pi,
                     Lzp=4 * math.pi / 3, nu=nu, CFL=-1e-3, x_mass_cte=1, grid_type=1,
                     alpha_stretch=2.0, dPdx=p["dpdx"]) as ch:
        ch.set_grid(g.x[1:], g.y[1:], g.z[1:])
        for name, ref in (("U", st.U), ("V", st.V), ("W", st.W)):
            ch.upload(name, ref[1:, 1:, 1:])
        ch.set_scalars(dPdx=st.dPdx, Qflow_x_0=st.Qflow_x_0)
        ch.compute_time_step_RK3(1)
        co.compute_time_step_RK3(g, st, 1e-3)
        for name, ref in (("U", st.U), ("V", st.V), ("W", st.W), ("P", st.P)):
            assert rel(ch.download(name), ref[1:, 1:, 1:]) < 1e-10, name
        ch.compute_time_step_RK3(4)
        # 97 slabs: 4-CTA wide clusters run in two waves, 8-CTA narrow ones
        # would take three
        assert ch.stats()["slab_cluster"][0] == 4 and ch.stats()["slab_narrow"][0] == 0
        assert ch.check_divergence() < 1e-12
        assert abs(ch.compute_mean_mass_flow_U() - st.Qflow_x_0) < 1e-13


def test_handles_of_different_sizes_coexist():
    """Kernel shared-memory limits are process-wide: a small handle created
    after a large one must not lower the large one's limits."""
    import channel3d_parallel_b200 as c3d
    nu = 1.0 / 5600.0
    p = co.channel_params(194, 129, 194, 4 * math.pi, 4 * math.pi / 3, nu)
    g = co.Grid(p)
    st = co.seeded_initial_state(g, p["dpdx"])
    with c3d.Channel(nx_global=194, ny_global=129, nz_global=194, Lxp=4 * math.pi,
                     Lzp=4 * math.pi / 3, nu=nu, CFL=-1e-3, x_mass_cte=1, grid_type=1,
                     alpha_stretch=2.0, dPdx=p["dpdx"]) as big:
        big.set_grid(g.x[1:], g.y[1:], g.z[1:])
        for name, ref in (("U", st.U), ("V", st.V), ("W", st.W)):
            big.upload(name, ref[1:, 1:, 1:])
        big.set_scalars(dPdx=st.dPdx, Qflow_x_0=st.Qflow_x_0)
        ps, gs, sts, small = make_pair("uniform_small")
        try:
            small.compute_time_step_RK3(2)
            big.compute_time_step_RK3(2)
            assert big.check_divergence() < 1e-12
            assert small.check_divergence() < 1e-12
        finally:
            small.close()


def make_flux_pair(case):
    """A pair with the y and z constant-flux corrections enabled."""
    import channel3d_parallel_b200 as c3d
    nx, ny, nz, lx, lz, gt = CASES[case]
    nu = 1.0 / 5600.0
    p = co.channel_params(nx, ny, nz, lx, lz, nu, grid_type=gt, y_mass_cte=1, z_mass_cte=1)
    g = co.Grid(p)
    st = co.seeded_initial_state(g, p["dpdx"])
    ch = c3d.Channel(nx_global=nx, ny_global=ny, nz_global=nz, Lxp=lx, Lzp=lz, nu=nu,
                     CFL=-1e-3, x_mass_cte=1, y_mass_cte=1, z_mass_cte=1, grid_type=gt,
                     alpha_stretch=2.0, dPdx=p["dpdx"])
    ch.set_grid(g.x[1:], g.y[1:], g.z[1:])
    for name in ("U", "V", "W"):
        ch.upload(name, getattr(st, name)[1:, 1:, 1:])
    ch.set_scalars(dPdx=st.dPdx, t=0.0, Qflow_x_0=st.Qflow_x_0)
    ch.set_flow_targets(st.Qflow_x_0, st.Qflow_y_0, st.Qflow_z_0)
    return g, st, ch


@pytest.mark.parametrize("case", ["cfg0_34x65x34", "odd_ny_radix3", "uniform_small"])
def test_flux_entries_y_z(case):
    """compute_mean_mass_flow_V/W and compute_dPy/dPz (the latter through the
    routine's declared W extents) against the oracle."""
    g, st, ch = make_flux_pair(case)
    try:
        q, n = co.mean_mass_flow_v(g, st.V)
        assert abs(ch.compute_mean_mass_flow_V() - q / n) < 1e-15
        q, n = co.mean_mass_flow_w(g, st.W)
        assert abs(ch.compute_mean_mass_flow_W() - q / n) < 1e-15
        assert abs(ch.compute_dPy_for_constant_mass_flow()
                   - co.compute_dPy_for_constant_mass_flow(g, st.V, st.Qflow_y_0)) < 1e-15
        assert abs(ch.compute_dPz_for_constant_mass_flow()
                   - co.compute_dPz_for_constant_mass_flow(g, st.W, st.Qflow_z_0)) < 1e-15
    finally:
        ch.close()


@pytest.mark.parametrize("case", ["cfg0_34x65x34", "uniform_small"])
@pytest.mark.parametrize("nsteps", [1, 10])
def test_rk3_steps_with_y_and_z_flux_corrections(case, nsteps):
    """x, y and z constant-flux corrections (src/time_integration.f90:187-211)."""
    g, st, ch = make_flux_pair(case)
    try:
        ch.compute_time_step_RK3(nsteps)
        for _ in range(nsteps):
            co.compute_time_step_RK3(g, st, 1e-3)
        errs = {name: rel(ch.download(name), ref[1:, 1:, 1:])
                for name, ref in (("U", st.U), ("V", st.V), ("W", st.W))}
        assert max(errs.values()) < 1e-10, errs
        s = ch.stats()
        tol = lambda ref, q: 1e-9 * abs(ref) + 50 * 2.2e-16 * max(abs(q), 1.0) / 1e-3
        assert abs(s["dPdx"] - st.dPdx) <= tol(st.dPdx, st.Qflow_x_0)
        assert abs(s["dPdy"] - st.dPdy) <= tol(st.dPdy, st.Qflow_y_0)
        assert abs(s["dPdz"] - st.dPdz) <= tol(st.dPdz, st.Qflow_z_0)
        assert abs(s["qflow_y_0"] - st.Qflow_y_0) == 0.0
    finally:
        ch.close()


@pytest.mark.parametrize("case", ["cfg0_34x65x34", "odd_ny_radix3", "uniform_small"])
@pytest.mark.parametrize("nsteps", [1, 10])
def test_euler_steps(case, nsteps):
    """compute_time_step_Euler (src/time_integration.f90:25-81)."""
    p, g, st, ch = make_pair(case)
    try:
        ch.compute_time_step_Euler(nsteps)
        for _ in range(nsteps):
            co.compute_time_step_Euler(g, st, 1e-3)
        errs = {name: rel(ch.download(name), ref[1:, 1:, 1:])
                for name, ref in (("U", st.U), ("V", st.V), ("W", st.W))}
        assert max(errs.values()) < 1e-10, errs
        s = ch.stats()
        assert abs(s["dPdx"] - st.dPdx) <= 1e-9 * abs(st.dPdx) + 50 * 2.2e-16 * abs(st.Qflow_x_0) / 1e-3
        assert abs(s["t"] - st.t) < 1e-15
        assert ch.check_divergence() < 1e-12
    finally:
        ch.close()


def test_euler_steps_with_y_flux_correction():
    g, st, ch = make_flux_pair("cfg0_34x65x34")
    try:
        ch.compute_time_step_Euler(3)
        for _ in range(3):
            co.compute_time_step_Euler(g, st, 1e-3)
        errs = {name: rel(ch.download(name), ref[1:, 1:, 1:])
                for name, ref in (("U", st.U), ("V", st.V), ("W", st.W))}
        assert max(errs.values()) < 1e-10, errs
        s = ch.stats()
        assert abs(s["dPdy"] - st.dPdy) <= 1e-9 * abs(st.dPdy) + 50 * 2.2e-16 / 1e-3
        # Euler has no z correction: dPdz stays at its initial value
        assert s["dPdz"] == st.dPdz
    finally:
        ch.close()


@pytest.mark.parametrize("case", ["cfg0_34x65x34", "odd_ny_radix3", "uniform_small", "nz256_wide_slab"])
def test_compute_pressure(case):
    """compute_pressure (src/pressure.f90:21-341) after two RK3 steps: the whole
    P array (solution, wall ghosts, periodic copies, untouched x/z ghost planes)."""
    p, g, st, ch = make_pair(case)
    try:
        ch.compute_time_step_RK3(2)
        for _ in range(2):
            co.compute_time_step_RK3(g, st, 1e-3)
        ch.compute_pressure()
        co.compute_pressure(g, st)
        assert rel(ch.download("P"), st.P[1:, 1:, 1:]) < 1e-10
    finally:
        ch.close()


FULL_CASES = {
    # the IB configurations' channels without the body: 256x129x128 (uniform
    # y, Lx = 4.5, Lz = 2) and the Re_tau = 550 channel 384x257x384 (Lx = 2 pi,
    # Lz = pi, nu = 1/20000, tanh y grid): Nx = 256 and 384 x transforms,
    # Nz = 128 and 384 slabs, and 255 and 127 wall-normal rows per kx slab
    "cfg3_256x129x128": (258, 129, 130, 4.5, 2.0, 0, 1.0 / 5600.0),
    "cfg4_384x257x384": (386, 257, 386, 2.0 * math.pi, math.pi, 1, 1.0 / 20000.0),
}


@pytest.mark.parametrize("case", list(FULL_CASES))
def test_full_size_ib_grids_one_step_parity(case):
    """One RK3 step on the grids of the IB configurations against the C++
    restatement of the oracle's step (oracle/cpu_rk3.cpp, checked against the
    NumPy oracle in tests/test_cpu_restatement.py): U, V, W, P within 1e-10,
    the mass-flow shift behind dPdx within 2e-15, and max|div u| < 1e-12."""
    import channel3d_parallel_b200 as c3d
    from oracle import cpu_rk3
    nx, ny, nz, lx, lz, gt, nu = FULL_CASES[case]
    p = co.channel_params(nx, ny, nz, lx, lz, nu, grid_type=gt, alpha=2.0 if gt else 0.0)
    g = co.Grid(p)
    st = co.seeded_initial_state(g, p["dpdx"])
    cpu_rk3.build()
    cc = cpu_rk3.CpuChannel(g)
    try:
        cc.set_state(st)
        cc.steps(1)
        with c3d.Channel(nx_global=nx, ny_global=ny, nz_global=nz, Lxp=lx, Lzp=lz, nu=nu, CFL=-1e-3,
                         x_mass_cte=1, grid_type=gt, alpha_stretch=2.0 if gt else 0.0,
                         dPdx=p["dpdx"]) as ch:
            ch.set_grid(g.x[1:], g.y[1:], g.z[1:])
            for name, ref in (("U", st.U), ("V", st.V), ("W", st.W)):
                ch.upload(name, ref[1:, 1:, 1:])
            ch.set_scalars(dPdx=st.dPdx, Qflow_x_0=st.Qflow_x_0)
            ch.compute_time_step_RK3(1)
            for name in ("U", "V", "W", "P"):
                ref = cc.get_field(name)
                assert rel(ch.download(name), ref[1:, 1:, 1:]) < 1e-10, name
            # dPdx = (dPdx_old + shift/dt)/2 with the shift Qflow_x_0 - Q a
            # difference of two unit bulk fluxes: it carries their round-off
            # divided by dt, so it is compared on the shift (2e-15)
            assert abs(ch.stats()["dPdx"] - cc.dPdx) <= 2e-15 / 1e-3
            assert ch.check_divergence() < 1e-12
    finally:
        cc.close()
