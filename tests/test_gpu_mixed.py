"""Mixed-precision Poisson (FP32 spectral solve, FP64 kx=kz=0 mode, FP64
residual and one refinement projection) against the FP64 oracle.

Bars (max-norm relative): before refinement 1e-6, after refinement 1e-10
for U, V, W over 1 and 10 RK3 steps; max|div u| < 1e-12 after refinement.
The pressure P after refinement within 3e-9: P is the stage-1 potential
itself (over dt), whose error after one FP32 refinement sweep is 1e-10 to
1e-9 of its size (7e-11 at 32x65x32, 1.1e-9 on the 129-row grid after 10
steps); the projected velocities see only its gradient.  Before refinement
within 1e-5.
"""
import math

import numpy as np
import pytest

from oracle import channel_oracle as co

pytestmark = pytest.mark.gpu

CASES = {
    "cfg0_34x65x34": (34, 65, 34, math.pi, math.pi / 2),
    "odd_ny_radix3": (50, 34, 26, 2.0, 1.0),
    "tall_ny_clusters": (18, 129, 18, 1.0, 0.5),
    # Nz = 54 = 2 * 3^3
    "nz54_radix3": (26, 20, 56, 1.7, 0.9),
    "nz256_wide_slab": (18, 17, 258, 1.0, 2.0),
}


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def make(case, mode):
    import channel3d_parallel_b200 as c3d
    nx, ny, nz, lx, lz = CASES[case]
    nu = 1.0 / 5600.0
    p = co.channel_params(nx, ny, nz, lx, lz, nu)
    g = co.Grid(p)
    st = co.seeded_initial_state(g, p["dpdx"])
    ch = c3d.Channel(nx_global=nx, ny_global=ny, nz_global=nz, Lxp=lx, Lzp=lz, nu=nu, CFL=-1e-3,
                     x_mass_cte=1, grid_type=1, alpha_stretch=2.0, dPdx=p["dpdx"])
    ch.set_grid(g.x[1:], g.y[1:], g.z[1:])
    for name, ref in (("U", st.U), ("V", st.V), ("W", st.W)):
        ch.upload(name, ref[1:, 1:, 1:])
    ch.set_scalars(dPdx=st.dPdx, Qflow_x_0=st.Qflow_x_0)
    ch.set_mode(poisson=mode)
    return g, st, ch


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("nsteps", [1, 10])
def test_mixed_refined_matches_fp64_oracle(case, nsteps):
    from channel3d_parallel_b200 import lib as L
    g, st, ch = make(case, L.POISSON_MIXED)
    try:
        ch.compute_time_step_RK3(nsteps)
        for _ in range(nsteps):
            co.compute_time_step_RK3(g, st, 1e-3)
        errs = {n: rel(ch.download(n), r[1:, 1:, 1:]) for n, r in (("U", st.U), ("V", st.V), ("W", st.W))}
        assert max(errs.values()) < 1e-10, errs
        assert rel(ch.download("P"), st.P[1:, 1:, 1:]) < 3e-9
        assert ch.check_divergence() < 1e-12
        s = ch.stats()
        assert s["refinement_sweeps"] == 1
        assert s["slab_narrow"][1] == (0 if g.nz - 2 > 192 else 1)
    finally:
        ch.close()


@pytest.mark.parametrize("case", list(CASES))
def test_mixed_unrefined_within_1e6(case):
    from channel3d_parallel_b200 import lib as L
    g, st, ch = make(case, L.POISSON_MIXED_UNREFINED)
    try:
        ch.compute_time_step_RK3(1)
        co.compute_time_step_RK3(g, st, 1e-3)
        errs = {n: rel(ch.download(n), r[1:, 1:, 1:]) for n, r in (("U", st.U), ("V", st.V), ("W", st.W))}
        assert max(errs.values()) < 1e-6, errs
        assert rel(ch.download("P"), st.P[1:, 1:, 1:]) < 1e-5
        # and it is genuinely a lower-precision solve
        assert max(errs.values()) > 1e-12, errs
    finally:
        ch.close()
