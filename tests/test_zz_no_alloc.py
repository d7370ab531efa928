"""The allocation-free bulk-flux entry point (c3d_mean_mass_flow_u_noalloc).

It serves callers that cannot call cudaMalloc (a driver checking the flux
inside its time loop, where an allocation would synchronise the device, or a
program whose device memory belongs to another runtime's pool).  Its scratch
is a static device array shared by all calls, so this file is collected last;
``test_noalloc_in_fresh_process`` runs the comparison again alone in a new
Python process, where the entry's first call on the device is the one that
resolves the array's address.
"""
import ctypes as C
import math
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-13   # absolute, on a flux of order one (same bar as the mass-flow parity test)
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_CHILD = "C3D_NOALLOC_CHILD"


def _oracle_flux(p, U):
    """Bulk flux of the oracle (src/mass_flow.f90:24-53, Hu = 1) for a
    downloaded U(1:nx, 1:nyg, 1:nzg)."""
    from oracle import channel_oracle as co
    g = co.Grid(p)
    Uo = g.u_array()
    Uo[1:, 1:, 1:] = U
    q, norm = co.mean_mass_flow_u(g, Uo)
    return q / norm


def test_noalloc_flux_matches_oracle_and_handle_entry_twice():
    import torch
    import channel3d_parallel_b200 as c3d
    from channel3d_parallel_b200 import lib as L
    from oracle import channel_oracle as co

    nu = 1.0 / 5600.0
    p = co.channel_params(34, 65, 34, math.pi, math.pi / 2, nu)
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
            free_before = torch.cuda.mem_get_info()[0]
            rc = lib.c3d_mean_mass_flow_u_noalloc(Ud.data_ptr(), d["nx"], d["nyg"], d["nzg"],
                                                  yg.data_ptr(), q.data_ptr(), None)
            assert rc == 0, lib.c3d_last_error(0)
            torch.cuda.synchronize()
            if call == 1:
                # the first call may load the library's module (and with it
                # the static array); the second call must not take any memory
                assert torch.cuda.mem_get_info()[0] == free_before
            got = float(q.item())
            assert abs(got - _oracle_flux(p, U)) < TOL, (call, got)
            assert abs(got - ch.compute_mean_mass_flow_U()) < TOL, (call, got)

        # sizes beyond the static scratch are rejected before any launch
        rc = lib.c3d_mean_mass_flow_u_noalloc(Ud.data_ptr(), d["nx"], d["nyg"], 5000,
                                              yg.data_ptr(), q.data_ptr(), None)
        assert rc == L.ERR_PARAM
        assert b"exceed the static scratch" in lib.c3d_last_error(0)


@pytest.mark.skipif(os.environ.get(_CHILD) == "1", reason="already the fresh process")
def test_noalloc_in_fresh_process():
    env = dict(os.environ, **{_CHILD: "1"})
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-x", "-m", "gpu", "-p", "no:cacheprovider",
                        os.path.join(ROOT, "tests", "test_zz_no_alloc.py") +
                        "::test_noalloc_flux_matches_oracle_and_handle_entry_twice"],
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
