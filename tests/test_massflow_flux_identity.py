"""The identity behind the time step's fused constant-x-mass-flow correction.

The library takes the bulk flux of u for the correction of
src/time_integration.f90:187-193 from U* (in the divergence transform of the
last stage) instead of from the projected u: on the periodic, uniformly
spaced x grid the bulk flux of d(phi)/dx telescopes to zero, so the two are
equal up to rounding.  Checked here on the oracle (the reference's own
operators): a non-solenoidal U* with its boundary conditions, the flux
before and after compute_non_IB_projection.
"""
import math

import numpy as np

from oracle import channel_oracle as co


def _case(nxg, nyg, nzg, seed):
    nu = 1.0 / 5600.0
    p = co.channel_params(nxg, nyg, nzg, math.pi, math.pi / 2, nu)
    g = co.Grid(p)
    st = co.seeded_initial_state(g, p["dpdx"], amplitude=0.1, seed=seed, project=False)
    return g, st


def test_flux_of_u_unchanged_by_projection():
    for dims, seed in (((18, 17, 14), 0), ((34, 33, 30), 1), ((20, 25, 56), 2)):
        g, st = _case(*dims, seed)
        q_star, norm = co.mean_mass_flow_u(g, st.U)
        div0 = np.abs(co.divergence(g, st.U, st.V, st.W)).max()
        co.compute_non_IB_projection(g, st, 1e-3)
        co.apply_boundary_conditions(g, st.U, st.V, st.W)
        q_new, norm2 = co.mean_mass_flow_u(g, st.U)
        assert norm == norm2
        # a genuinely non-solenoidal U*: the projection changes u by O(div),
        # but not its bulk flux
        assert div0 > 1.0
        assert abs(q_new - q_star) <= 1e-13 * abs(q_star), (dims, q_star, q_new)
