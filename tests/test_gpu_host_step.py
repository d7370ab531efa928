"""c3d_time_step_rk3_host: RK3 steps with u, v, w kept in the caller's arrays
(the reference's time loop, app/main.f90:101-117), every step uploading the
three arrays and writing the new fields back in place.

The fields it leaves in the host arrays must be bit-identical to the same
number of device-resident steps (c3d_time_step_rk3 between one upload and one
download: the round trips are exact copies), and both must match the oracle
at the RK3 bar (1e-10 relative max-norm)."""
import numpy as np
import pytest

from oracle import channel_oracle as co
from tests.test_gpu_parity import make_pair, rel

pytestmark = pytest.mark.gpu


def pinned_like(a):
    import torch
    t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
    v = t.numpy().reshape(a.shape, order="F")
    v[...] = a
    return t, v


@pytest.mark.parametrize("case,nsteps,pinned", [("cfg0_34x65x34", 3, True),
                                                ("odd_ny_radix3", 2, False),
                                                ("nz256_wide_slab", 4, True)])
def test_host_resident_steps_match_device_steps_and_oracle(case, nsteps, pinned):
    p, g, st, ch = make_pair(case)
    p2, g2, st2, ch2 = make_pair(case)
    try:
        host = {}
        keep = []
        for name in ("U", "V", "W"):
            a = ch.download(name)
            if pinned:
                t, v = pinned_like(a)
                keep.append(t)
                host[name] = v
            else:
                host[name] = np.asfortranarray(a.copy())
        ch.compute_time_step_RK3_host(host["U"], host["V"], host["W"], nsteps)
        ch2.compute_time_step_RK3(nsteps)
        for name in ("U", "V", "W"):
            assert np.array_equal(host[name], ch2.download(name)), name
            # the device copy holds the same state as the host arrays
            assert np.array_equal(host[name], ch.download(name)), name
        for _ in range(nsteps):
            co.compute_time_step_RK3(g, st, 1e-3)
        errs = {name: rel(host[name], ref[1:, 1:, 1:])
                for name, ref in (("U", st.U), ("V", st.V), ("W", st.W))}
        assert max(errs.values()) < 1e-10, errs
        assert ch.stats()["steps"] == nsteps
        assert abs(ch.stats()["dPdx"] - ch2.stats()["dPdx"]) == 0.0
    finally:
        ch.close()
        ch2.close()


def test_host_resident_steps_see_host_changes_between_calls():
    """A change the caller makes to its arrays between calls is what the next
    step advances (the upload reads the arrays every step): after one step
    the arrays are replaced by another state, and two more steps must equal
    two device-resident steps of that state under the same scalars."""
    p, g, st, ch = make_pair("cfg0_34x65x34")
    p2, g2, st2, ch2 = make_pair("cfg0_34x65x34", amplitude=0.05, seed=3)
    try:
        host = {n: np.asfortranarray(ch.download(n).copy()) for n in ("U", "V", "W")}
        ch.compute_time_step_RK3_host(host["U"], host["V"], host["W"], 1)
        for n in ("U", "V", "W"):
            host[n][...] = ch2.download(n)
        s = ch.stats()
        ch2.set_scalars(dPdx=s["dPdx"], t=s["t"], Qflow_x_0=st.Qflow_x_0)
        ch.compute_time_step_RK3_host(host["U"], host["V"], host["W"], 2)
        ch2.compute_time_step_RK3(2)
        for n in ("U", "V", "W"):
            assert np.array_equal(host[n], ch2.download(n)), n
    finally:
        ch.close()
        ch2.close()


def test_host_resident_step_rejects_bad_arrays():
    p, g, st, ch = make_pair("uniform_small")
    try:
        U = ch.download("U")
        V = ch.download("V")
        W = ch.download("W")
        with pytest.raises(ValueError):
            ch.compute_time_step_RK3_host(np.ascontiguousarray(U), V, W, 1)
        with pytest.raises(ValueError):
            ch.compute_time_step_RK3_host(U[:-1], V, W, 1)
        with pytest.raises(ValueError):
            ch.compute_time_step_RK3_host(U.astype(np.float32), V, W, 1)
        assert ch.stats()["steps"] == 0
    finally:
        ch.close()
