"""The allocation-free bulk-flux entry point (c3d_mean_mass_flow_u_noalloc).

It serves callers that cannot call cudaMalloc (a driver checking the flux
inside its time loop, where an allocation would synchronise the device, or a
program whose device memory belongs to another runtime's pool).  Its scratch
is a static device array shared by all calls, so this file is collected last
and the test also runs alone in a fresh process.
"""
import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13   # absolute, on a flux of order one (same bar as the mass-flow parity test)


def test_noalloc_flux_matches_handle_entry_twice():
    import torch
    import channel3d_parallel_b200 as c3d
    from channel3d_parallel_b200 import lib as L

    nu = 1.0 / 5600.0
    with c3d.Channel(nx_global=34, ny_global=65, nz_global=34, Lxp=math.pi, Lzp=math.pi / 2,
                     nu=nu, CFL=-1e-3, x_mass_cte=1, grid_type=1, alpha_stretch=2.0) as ch:
        c3d.seeded_initial_state(ch, 3.0 * nu, nu)
        lib = L.load()
        d = ch.dims
        g = ch.grid()
        yg = torch.tensor(g["yg"], dtype=torch.float64, device="cuda")
        q = torch.zeros(1, dtype=torch.float64, device="cuda")
        for call in range(2):
            # perturb between calls so the second result differs from the first
            U = ch.download("U")
            if call == 1:
                U = U * 1.25
                ch.upload("U", U)
            Ud = torch.tensor(U.reshape(-1, order="F"), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            rc = lib.c3d_mean_mass_flow_u_noalloc(Ud.data_ptr(), d["nx"], d["nyg"], d["nzg"],
                                                  yg.data_ptr(), q.data_ptr(), None)
            assert rc == 0, lib.c3d_last_error(0)
            torch.cuda.synchronize()
            ref = ch.compute_mean_mass_flow_U()
            assert abs(float(q.item()) - ref) < TOL, (call, float(q.item()), ref)

        # sizes beyond the static scratch are rejected before any launch
        rc = lib.c3d_mean_mass_flow_u_noalloc(Ud.data_ptr(), d["nx"], d["nyg"], 5000,
                                              yg.data_ptr(), q.data_ptr(), None)
        assert rc == L.ERR_PARAM
        assert b"exceed the static scratch" in lib.c3d_last_error(0)
