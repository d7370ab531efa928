"""Snapshot format, statistics and monitor values -- TEST INFRASTRUCTURE ONLY.

Restates, for one domain:
  output_data       src/input_output.f90:498-728 (binary snapshot)
  read_input_data   src/input_output.f90:335-489 (mesh and U, V, W)
  compute_statistics src/statistics.f90:22-148
  output_monitor    src/monitor.f90:21-110 (the values it prints)
The snapshot is a big-endian stream without record markers (the layout that
tools/file_io.py reads and writes): 4-byte integer counts and extents,
8-byte reals, arrays in Fortran order.
"""
import numpy as np

from . import channel_oracle as co

_I4, _F8 = np.dtype(">i4"), np.dtype(">f8")


def _vec(a):
    a = np.asarray(a, dtype=np.float64)
    return np.array([a.size], dtype=_I4).tobytes() + a.astype(_F8).tobytes()


def _field(a):
    a = np.asarray(a, dtype=np.float64)
    return np.array(a.shape, dtype=_I4).tobytes() + np.asfortranarray(a).ravel(order="F").astype(_F8).tobytes()


def snapshot_bytes(g, st, dt, body=None, fb=None, H=None, original_format=False):
    """Bytes of output_data for the oracle state ``st`` (Fortran-indexed
    arrays).  ``body``: an ib_oracle.Body (None: no markers); ``fb`` the
    surface unknowns (4 nb); ``H``: (Hu, Hv, Hw) Fortran-indexed, default 1
    (app/main.f90:80-85)."""
    out = [_vec(g.x[1:]), _vec(g.y[1:]), _vec(g.z[1:]),
           _vec(g.xm[1:g.nx]), _vec(g.ym[1:g.ny]), _vec(g.zm[1:g.nz])]
    for a in (st.U, st.V, st.W, st.P):
        out.append(_field(a[1:, 1:, 1:]))
    if original_format:
        return b"".join(out)
    if H is None:
        H = (np.ones_like(st.U), np.ones_like(st.V), np.ones_like(st.W))
    for a in H:
        out.append(_field(a[1:, 1:, 1:]))
    out.append(np.array([st.t, dt, st.dPdx, g.p["nu"]], dtype=_F8).tobytes())
    if body is None:
        empty = np.zeros(0)
        xb = yb = zb = ub = sb = nrm = t1 = t2 = empty
        fb = empty
        nxb = g.p["nxb"]
    else:
        xb, yb, zb, ub, sb = body.xb, body.yb, body.zb, body.ub, body.sb
        nrm, t1, t2 = body.normals, body.tangents_1, body.tangents_2
        # double_cylinders_z recomputes nxb (src/immersed_boundary_geometry.f90:131)
        nxb = len(body.xb) // g.p["nzb"] if body.kind == "double_cylinders_z" else g.p["nxb"]
    out += [_vec(xb), _vec(yb), _vec(zb)]
    out.append(np.array([nxb, g.p["nzb"]], dtype=_I4).tobytes())
    out += [_vec(fb), _vec(ub), _vec(sb), _vec(nrm), _vec(t1), _vec(t2)]
    return b"".join(out)


def read_snapshot(path):
    """Every record of a snapshot (the layout of output_data), as a dict."""
    raw = open(path, "rb").read()
    pos = 0

    def take(dtype, n):
        nonlocal pos
        a = np.frombuffer(raw, dtype=dtype, count=n, offset=pos)
        pos += n * dtype.itemsize
        return a

    d = {}
    for k in ("x", "y", "z", "xm", "ym", "zm"):
        d[k] = take(_F8, int(take(_I4, 1)[0])).astype(np.float64)
    for k in ("U", "V", "W", "P", "Hu_interior", "Hv_interior", "Hw_interior"):
        if pos >= len(raw):
            return d
        n = take(_I4, 3)
        d[k] = take(_F8, int(np.prod(n))).astype(np.float64).reshape(tuple(int(v) for v in n), order="F")
    d["t"], d["dt"], d["dpdx"], d["nu"] = take(_F8, 4).astype(np.float64)
    for k in ("xb", "yb", "zb"):
        d[k] = take(_F8, int(take(_I4, 1)[0])).astype(np.float64)
    d["nxb"], d["nzb"] = (int(v) for v in take(_I4, 2))
    for k in ("fb", "ub", "sb", "normals", "tangents_1", "tangents_2"):
        d[k] = take(_F8, int(take(_I4, 1)[0])).astype(np.float64)
    assert pos == len(raw)
    return d


def compute_statistics(g, st, Hu=None, Hv=None):
    """src/statistics.f90:22-148 for one domain (the branch of the last
    rank): profiles at yg(1:nyg) and utau, wtau, Retau_u, Retau_w, Qflow_x,
    Qflow_y, Qflow_z (Qflow_z is compute_mean_mass_flow_V applied to W, :133,
    i.e. W read through V's declared extents)."""
    nx, ny, nxg, nyg, nzg, nz = g.nx, g.ny, g.nxg, g.nyg, g.nzg, g.nz
    U, V, W = st.U, st.V, st.W
    term1 = np.zeros((nxg + 1, nyg + 1, nzg + 1))
    term1[2:nxg, 1:nyg + 1, 1:nzg + 1] = 0.5 * (U[1:nx, 1:, 1:] + U[2:nx + 1, 1:, 1:])   # interpolate_x
    term2 = np.zeros((nxg + 1, nyg + 1, nzg + 1))
    term2[1:, 2:nyg, 1:] = 0.5 * (V[1:, 1:ny, 1:] + V[1:, 2:ny + 1, 1:])                 # interpolate_y
    term2[:, 1, :] = -term2[:, 2, :]
    term2[:, nyg, :] = -term2[:, nyg - 1, :]
    I, K, KW = slice(2, nxg - 1), slice(2, nzg - 1), slice(2, nz)
    t1, t2, w = term1[I, 1:nyg + 1, K], term2[I, 1:nyg + 1, K], W[I, 1:nyg + 1, KW]
    cnt, cntw = (nxg - 3) * (nzg - 3), (nxg - 3) * (nz - 2)
    prof = {
        "Umean": t1.sum(axis=(0, 2)) / cnt, "Vmean": t2.sum(axis=(0, 2)) / cnt,
        "Wmean": w.sum(axis=(0, 2)) / cntw,
        "U2mean": (t1 ** 2.0).sum(axis=(0, 2)) / cnt, "V2mean": (t2 ** 2.0).sum(axis=(0, 2)) / cnt,
        "W2mean": (w ** 2.0).sum(axis=(0, 2)) / cntw, "UVmean": (t1 * t2).sum(axis=(0, 2)) / cnt,
    }
    yg, y, nu, Ly = g.yg, g.y, g.p["nu"], g.Ly
    Um, Wm = prof["Umean"], prof["Wmean"]
    dUb = (Um[1] - Um[0]) / (yg[2] - yg[1])
    dUt = (Um[nyg - 1] - Um[nyg - 2]) / (yg[nyg] - yg[nyg - 1])
    dWb = (Wm[1] - Wm[0]) / (yg[2] - yg[1])
    dWt = (Wm[nyg - 1] - Wm[nyg - 2]) / (yg[nyg] - yg[nyg - 1])
    with np.errstate(invalid="ignore"):
        utau = ((0.0 - 0.0 - nu * dUt + nu * dUb) / Ly) ** 0.5
        wtau = ((0.0 - 0.0 - nu * dWt + nu * dWb) / Ly) ** 0.5
    prof["utau"], prof["wtau"] = float(np.real(utau)), float(np.real(wtau))
    prof["Retau_u"] = prof["utau"] * (y[ny] - y[1]) / 2.0 / nu
    prof["Retau_w"] = prof["wtau"] * (y[ny] - y[1]) / 2.0 / nu
    q, n = co.mean_mass_flow_u(g, U, Hu)
    prof["Qflow_x"] = q / n
    q, n = co.mean_mass_flow_v(g, V, Hv)
    prof["Qflow_y"] = q / n
    # W through compute_mean_mass_flow_V's dummy Dimension(nxg,ny,nzg)
    # (the loops stop at offset nxg*ny*nz - 2, inside W; the view's last
    # plane, beyond W when ny > nz, is never read and is filled with NaN)
    flat = np.asarray(W)[1:, 1:, 1:].ravel(order="F")
    full = np.full(nxg * ny * nzg, np.nan)
    m = min(full.size, flat.size)
    full[:m] = flat[:m]
    view = np.zeros((nxg + 1, ny + 1, nzg + 1))
    view[1:, 1:, 1:] = full.reshape((nxg, ny, nzg), order="F")
    q, n = co.mean_mass_flow_v(g, view, Hv)
    prof["Qflow_z"] = q / n
    prof["nonfinite"] = not (np.isfinite(U).all() and np.isfinite(V).all() and np.isfinite(W).all())
    return prof


def monitor_values(g, st):
    """The values output_monitor prints (src/monitor.f90:21-80, 210-221)."""
    nx, ny, nz, nxg, nyg, nzg = g.nx, g.ny, g.nz, g.nxg, g.nyg, g.nzg
    vol = float((nx - 1) * (ny - 1) * (nz - 1))
    u = st.U[2:nx, 2:nyg, 2:nzg]
    v = st.V[2:nxg, 2:ny, 2:nzg]
    w = st.W[2:nxg, 2:nyg, 2:nz]
    div = co.divergence(g, st.U, st.V, st.W)
    return {"meanU": u.sum() / vol, "meanV": v.sum() / vol, "meanW": w.sum() / vol,
            "maxU": u.max(), "maxV": v.max(), "maxW": w.max(),
            "max_divergence": float(np.abs(div).max())}
