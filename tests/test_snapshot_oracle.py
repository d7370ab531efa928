"""The oracle's snapshot restatement (output_data / read_input_data layout)."""
import math

import numpy as np

from oracle import channel_oracle as co
from oracle import snapshot as sn


def test_snapshot_roundtrip_and_layout(tmp_path):
    p = co.channel_params(18, 17, 14, 1.0, 0.7, 1 / 5600, grid_type=0)
    g = co.Grid(p)
    st = co.seeded_initial_state(g, p["dpdx"])
    st.t = 0.25
    b = sn.snapshot_bytes(g, st, 1e-3)
    f = tmp_path / "snap.1"
    f.write_bytes(b)
    d = sn.read_snapshot(f)
    for k, ref in (("U", st.U), ("V", st.V), ("W", st.W), ("P", st.P)):
        assert np.array_equal(d[k], ref[1:, 1:, 1:]), k
    assert np.array_equal(d["x"], g.x[1:]) and np.array_equal(d["zm"], g.zm[1:g.nz])
    assert (d["t"], d["dt"], d["dpdx"], d["nu"]) == (0.25, 1e-3, st.dPdx, p["nu"])
    assert np.all(d["Hu_interior"] == 1.0) and d["fb"].size == 0
    # big-endian: the first record is the 4-byte count nx then x(1) = 0
    assert int.from_bytes(b[:4], "big") == g.nx
    assert np.frombuffer(b[4:12], dtype=">f8")[0] == g.x[1]
    # the original format is the prefix up to P
    o = sn.snapshot_bytes(g, st, 1e-3, original_format=True)
    assert b.startswith(o) and len(o) < len(b)


def test_statistics_profiles_of_a_laminar_profile():
    """Umean of U = U(y) is the interpolated profile; V, W moments vanish."""
    p = co.channel_params(18, 17, 14, 1.0, 0.7, 1 / 5600, grid_type=0)
    g = co.Grid(p)
    st = co.State(g)
    prof = 1.0 + 0.1 * np.arange(g.nyg + 1)
    st.U[:, :, :] = prof[None, :, None]
    s = sn.compute_statistics(g, st)
    assert np.allclose(s["Umean"], prof[1:], rtol=0, atol=1e-15)
    assert np.allclose(s["U2mean"], prof[1:] ** 2, rtol=1e-15)
    assert np.all(s["Vmean"] == 0) and np.all(s["W2mean"] == 0)
    m = sn.monitor_values(g, st)
    assert m["maxU"] == prof[2:g.nyg].max()
