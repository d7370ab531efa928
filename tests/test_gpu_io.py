"""Snapshots, statistics and monitor values through the C-ABI against the
oracle (oracle/snapshot.py).

Tolerances: snapshot bytes are compared exactly, given the library's own
field values; the statistics profiles and monitor means 1e-12 relative
(summation order), maxima exact.
"""
import math

import numpy as np
import pytest

from oracle import channel_oracle as co
from oracle import ib_oracle as ibo
from oracle import snapshot as sn

pytestmark = pytest.mark.gpu


def make(case=(34, 65, 34, math.pi, math.pi / 2, 1), steps=2):
    import channel3d_parallel_b200 as c3d
    nx, ny, nz, lx, lz, gt = case
    nu = 1.0 / 5600.0
    p = co.channel_params(nx, ny, nz, lx, lz, nu, grid_type=gt)
    g = co.Grid(p)
    st = co.seeded_initial_state(g, p["dpdx"])
    ch = c3d.Channel(nx_global=nx, ny_global=ny, nz_global=nz, Lxp=lx, Lzp=lz, nu=nu, CFL=-1e-3,
                     x_mass_cte=1, grid_type=gt, alpha_stretch=2.0, dPdx=p["dpdx"])
    ch.set_grid(g.x[1:], g.y[1:], g.z[1:])
    for name in ("U", "V", "W"):
        ch.upload(name, getattr(st, name)[1:, 1:, 1:])
    ch.set_scalars(dPdx=st.dPdx, t=0.0, Qflow_x_0=st.Qflow_x_0)
    ch.compute_time_step_RK3(steps)
    for _ in range(steps):
        co.compute_time_step_RK3(g, st, 1e-3)
    return p, g, st, ch


def library_state(g, ch):
    """An oracle State holding the library's current values."""
    s = co.State(g)
    for name in ("U", "V", "W", "P"):
        a = getattr(s, name)
        a[1:, 1:, 1:] = ch.download(name)
    st = ch.stats()
    s.t, s.dPdx = st["t"], st["dPdx"]
    return s, st["dt"]


@pytest.mark.parametrize("original", [False, True])
def test_write_snapshot_bytes(tmp_path, original):
    p, g, st, ch = make()
    try:
        f = tmp_path / "snap"
        ch.write_snapshot(f, original_format=original)
        s, dt = library_state(g, ch)
        assert f.read_bytes() == sn.snapshot_bytes(g, s, dt, original_format=original)
        # and the library's values are the oracle's (RK3 parity bar)
        d = sn.read_snapshot(f)
        for k, ref in (("U", st.U), ("V", st.V), ("W", st.W), ("P", st.P)):
            assert np.abs(d[k] - ref[1:, 1:, 1:]).max() <= 1e-10 * np.abs(ref).max(), k
    finally:
        ch.close()


def test_read_snapshot_roundtrip(tmp_path):
    import channel3d_parallel_b200 as c3d
    p, g, st, ch = make()
    try:
        f = tmp_path / "snap"
        ch.write_snapshot(f)
        # a handle with another grid: read_input_data replaces it
        with c3d.Channel(nx_global=34, ny_global=65, nz_global=34, Lxp=math.pi, Lzp=math.pi / 2,
                         nu=1 / 5600, CFL=-1e-3, x_mass_cte=1, grid_type=1, alpha_stretch=1.0) as other:
            other.read_snapshot(f)
            for name in ("U", "V", "W"):
                assert np.array_equal(other.download(name), ch.download(name)), name
            for k in ("x", "y", "z", "xg", "yg", "zg"):
                assert np.array_equal(other.grid()[k], ch.grid()[k]), k
            # the state read back advances exactly as the original
            other.set_scalars(dPdx=ch.stats()["dPdx"], t=ch.stats()["t"], Qflow_x_0=st.Qflow_x_0)
            ch.compute_time_step_RK3(1)
            other.compute_time_step_RK3(1)
            assert np.array_equal(other.download("U"), ch.download("U"))
    finally:
        ch.close()


def test_read_snapshot_errors(tmp_path):
    import channel3d_parallel_b200 as c3d
    p, g, st, ch = make()
    try:
        f = tmp_path / "snap"
        ch.write_snapshot(f)
        with c3d.Channel(nx_global=34, ny_global=33, nz_global=34, Lxp=math.pi, Lzp=math.pi / 2,
                         nu=1 / 5600, CFL=-1e-3) as other:
            with pytest.raises(c3d.C3DError) as e:
                other.read_snapshot(f)
            assert e.value.code == -1 and "ny_f/=ny" in str(e.value)
        with pytest.raises(c3d.C3DError) as e:
            ch.read_snapshot(tmp_path / "missing")
        assert e.value.code == -5
        trunc = tmp_path / "trunc"
        trunc.write_bytes(f.read_bytes()[:5000])
        with pytest.raises(c3d.C3DError) as e:
            ch.read_snapshot(trunc)
        assert e.value.code == -5
    finally:
        ch.close()


def test_statistics_and_monitor():
    p, g, st, ch = make(steps=3)
    try:
        got = ch.compute_statistics()
        ref = sn.compute_statistics(g, st)
        # scales: a mean against its rms (mean V is round-off of a zero-mean field)
        rms = {c: np.sqrt(np.abs(ref[c + "2mean"]).max()) for c in "UVW"}
        scale = {"Umean": rms["U"], "Vmean": rms["V"], "Wmean": rms["W"], "U2mean": rms["U"] ** 2,
                 "V2mean": rms["V"] ** 2, "W2mean": rms["W"] ** 2, "UVmean": rms["U"] * rms["V"]}
        for k in ch.STAT_NAMES:
            assert np.abs(got[k] - ref[k]).max() <= 1e-12 * scale[k], k
        for k in ("utau", "wtau", "Retau_u", "Retau_w", "Qflow_x", "Qflow_y", "Qflow_z"):
            assert abs(got[k] - ref[k]) <= 1e-9 * abs(ref[k]) + 1e-15, (k, got[k], ref[k])
        assert got["nonfinite"] is False
        m, r = ch.output_monitor(), sn.monitor_values(g, st)
        for k in ("meanU", "meanV", "meanW", "maxU", "maxV", "maxW"):
            assert abs(m[k] - r[k]) <= 1e-10 * abs(r[k]) + 1e-15, (k, m[k], r[k])
        assert m["max_divergence"] < 1e-12 and m["max_slip"] == 0.0
    finally:
        ch.close()


def test_write_statistics_text(tmp_path):
    p, g, st, ch = make(steps=1)
    try:
        f = tmp_path / "out.1.stats.txt"
        ch.write_statistics(f, 1)
        lines = f.read_text().splitlines()
        assert lines[0].startswith("%") and len(lines) == 1 + g.nyg
        head = lines[0][1:]
        vals = [float(head[15 * q:15 * q + 15]) for q in range(4)]
        ints = [int(head[60 + 12 * q:60 + 12 * q + 12]) for q in range(4)]
        s = ch.compute_statistics()
        assert vals[0] == pytest.approx(1e-3, abs=1e-8) and vals[3] == pytest.approx(1 / 5600, abs=1e-8)
        assert vals[1] == pytest.approx(s["Retau_u"], abs=1e-8)
        assert ints == [34, 65, 34, 1]
        row = [float(lines[1][15 * q:15 * q + 15]) for q in range(8)]
        assert row[0] == pytest.approx(g.yg[1], abs=1e-8)
        assert row[1] == pytest.approx(s["Umean"][0], abs=1e-8)
    finally:
        ch.close()


def test_snapshot_with_body(tmp_path):
    """Marker arrays, tangents and Heaviside fields of an IB snapshot."""
    from tests.test_gpu_ib import build
    p, g, st, ib, ch = build("wall_standing_wave")
    try:
        ch.compute_time_step_RK3(1)
        f = tmp_path / "snap"
        ch.write_snapshot(f)
        d = sn.read_snapshot(f)
        ib.refresh(ch.stats()["t"])          # geometry at the library's current time
        b = ib.body
        assert d["nxb"] == p["nxb"] and d["nzb"] == p["nzb"]
        for k, ref in (("xb", b.xb), ("yb", b.yb), ("zb", b.zb), ("sb", b.sb), ("normals", b.normals),
                       ("tangents_1", b.tangents_1), ("tangents_2", b.tangents_2), ("ub", b.ub)):
            assert d[k].shape == ref.shape and np.abs(d[k] - ref).max() <= 1e-14, k
        for k, name in (("Hu_interior", "HU_INTERIOR"), ("Hv_interior", "HV_INTERIOR"),
                        ("Hw_interior", "HW_INTERIOR")):
            assert np.array_equal(d[k], ch.download(name)), k
        assert np.array_equal(d["fb"], ch.download("FB"))
        m = ch.output_monitor()
        assert m["max_slip"] > 0.0
    finally:
        ch.close()
