"""FP64 CPU restatement of the immersed-boundary part of the hot path
(test infrastructure; parity unpinned -- see ``oracle/__init__.py``).

Follows src/immersed_boundary_geometry.f90, src/immersed_boundary_operators.f90,
src/heaviside.f90 and src/projection.f90:48-186 in the single-domain view:
a stencil point on the periodic duplicate centre plane nzg-1 is the plane 2
it duplicates -- reading it reads plane 2, and spreading into it adds to
plane 2 (what the reference's support-plane exchange does,
src/boundary_conditions.f90:737-906).

Arrays are Fortran-indexed as in ``channel_oracle``; marker vectors are plain
0-based NumPy vectors of length nb / 3nb / 4nb in the reference's block order.
"""
import math

import numpy as np

from . import channel_oracle as co

SUPP = 2
NW = (2 * SUPP + 1) ** 3
PI = co.PI


# ---------------------------------------------------------------------------
# geometry, src/immersed_boundary_geometry.f90
# ---------------------------------------------------------------------------
class Body:
    """Marker set of one configuration (module globals xb, yb, zb, ub,
    normals, sb, y_ref_index, nbodies and the per-body mean-removal blocks)."""

    def __init__(self, g, p, t=0.0, markers=None):
        self.g, self.p = g, p
        self.kind = p["body_type"]
        self.moving = self.kind in ("standing_wave", "traveling_wave_x", "wall_standing_wave",
                                    "wall_plates")
        self.markers = markers
        self.update(t)

    def update(self, t):
        """setup_IB_geometry at time t (src/immersed_boundary_geometry.f90:70-398)."""
        g, p, kind = self.g, self.p, self.kind
        nxb, nzb = p["nxb"], p["nzb"]
        Lxp, Lzp = g.Lxp, g.Lzp
        if kind == "center_wall":                                   # :80-115
            nb = nxb * nzb
            dxb, dzb = Lxp / nxb, Lzp / nzb
            i = np.tile(np.arange(1, nxb + 1), nzb)
            j = np.repeat(np.arange(1, nzb + 1), nxb)
            self.xb = (i - 0.5) * dxb
            self.yb = np.full(nb, 0.5 * p["ly_channel"])
            self.zb = (j - 0.5) * dzb
            self.ub = np.zeros(3 * nb)
            self.y_ref = np.full(nb, p["ny_global"] // 2)
            self.sb = np.full(nb, dxb * dzb)
            self.normals = np.zeros(3 * nb)
            self.normals[nb:2 * nb] = -1.0
            self.tangents_1 = np.zeros(3 * nb)                  # :111-115
            self.tangents_1[:nb] = 1.0
            self.tangents_2 = np.zeros(3 * nb)
            self.tangents_2[2 * nb:] = -1.0
            self.blocks = [np.arange(nb)]
        elif kind in ("standing_wave", "wall_standing_wave"):       # :176-269
            self._standing_wave(t, two_walls=(kind == "standing_wave"))
        elif kind == "traveling_wave_x":                            # :271-390
            self._traveling_wave(t)
        elif kind == "double_cylinders_z":                          # :117-174
            self._double_cylinders()
        elif kind == "two_cylinders_z":
            self._two_cylinders()
        elif kind == "wall_plates":
            self._wall_plates(t)
        elif kind == "markers":
            m = self.markers
            self.xb, self.yb, self.zb = m["xb"].copy(), m["yb"].copy(), m["zb"].copy()
            self.ub, self.normals, self.sb = m["ub"].copy(), m["normals"].copy(), m["sb"].copy()
            self.tangents_1 = np.asarray(m.get("tangents_1", np.zeros(3 * len(m["xb"])))).copy()
            self.tangents_2 = np.asarray(m.get("tangents_2", np.zeros(3 * len(m["xb"])))).copy()
            self.y_ref = m["y_ref"].copy()
            self.blocks = [np.asarray(b) for b in m["blocks"]]
        else:
            raise ValueError(f"body_type {kind!r}")
        self.nb = len(self.xb)

    def _standing_wave(self, t, two_walls):
        g, p = self.g, self.p
        nxb, nzb = p["nxb"], p["nzb"]
        Lxp, Lzp = g.Lxp, g.Lzp
        dxb, dzb = Lxp / nxb, Lzp / nzb
        A, om, b3 = p["body_param_1"], p["body_param_2"], p["body_param_3"]
        nw = 2 if two_walls else 1
        y0 = 0.0 if two_walls else p.get("body_param_4", 0.0)
        nb = nw * nxb * nzb
        xb, yb, zb = np.zeros(nb), np.zeros(nb), np.zeros(nb)
        ub, nrm, t1 = np.zeros(3 * nb), np.zeros(3 * nb), np.zeros(3 * nb)
        sb = np.zeros(nb)
        yref = np.zeros(nb, dtype=np.int64)
        bot, top = [], []
        for j in range(1, nzb + 1):
            for i in range(1, nxb + 1):
                k = i + nw * nxb * (j - 1) - 1        # 0-based marker index
                x = (i - 0.5) * dxb
                xb[k] = x
                yb[k] = y0 + A * math.sin(2.0 * PI * b3 * x / Lxp) * math.cos(om * t)
                zb[k] = (j - 0.5) * dzb
                yref[k] = 1
                bot.append(k)
                if two_walls:
                    xb[k + nxb] = x
                    yb[k + nxb] = p["ly_channel"] + A * math.sin(2.0 * PI * b3 * x / Lxp) * math.cos(om * t)
                    zb[k + nxb] = (j - 0.5) * dzb
                    yref[k + nxb] = p["ny_global"]
                    top.append(k + nxb)
        for j in range(1, nzb + 1):
            for i in range(1, nxb + 1):
                k = i + nw * nxb * (j - 1) - 1
                phase = 2.0 * PI * b3 * xb[k] / Lxp
                vy = -A * om * math.sin(phase) * math.sin(om * t)
                ub[nb + k] = vy
                slope = A * 2.0 * PI * b3 / Lxp * math.cos(phase) * math.cos(om * t)
                t1[k] = 1.0 / math.sqrt(1.0 + slope ** 2)
                t1[nb + k] = slope / math.sqrt(1.0 + slope ** 2)
                nrm[k] = t1[nb + k]
                nrm[nb + k] = -t1[k]
                if two_walls:
                    ub[nb + k + nxb] = vy
                    t1[k + nxb] = 1.0 / math.sqrt(1.0 + slope ** 2)
                    t1[nb + k + nxb] = slope / math.sqrt(1.0 + slope ** 2)
                    nrm[k + nxb] = -t1[nb + k + nxb]
                    nrm[nb + k + nxb] = t1[k + nxb]
        for j in range(1, nzb + 1):                                 # :253-269
            for i in range(1, nxb + 1):
                k = i + nw * nxb * (j - 1) - 1
                first = nw * nxb * (j - 1)
                last = nxb - 1 + nw * nxb * (j - 1)
                if i == 1:
                    a1 = math.sqrt((xb[k] - (xb[last] - Lxp)) ** 2 + (yb[k] - yb[last]) ** 2)
                    a2 = math.sqrt((xb[k] - xb[k + 1]) ** 2 + (yb[k] - yb[k + 1]) ** 2)
                elif i == nxb:
                    a1 = math.sqrt((xb[k] - xb[k - 1]) ** 2 + (yb[k] - yb[k - 1]) ** 2)
                    a2 = math.sqrt((xb[k] - (xb[first] + Lxp)) ** 2 + (yb[k] - yb[first]) ** 2)
                else:
                    a1 = math.sqrt((xb[k] - xb[k - 1]) ** 2 + (yb[k] - yb[k - 1]) ** 2)
                    a2 = math.sqrt((xb[k] - xb[k + 1]) ** 2 + (yb[k] - yb[k + 1]) ** 2)
                sb[k] = dzb * (0.5 * a1 + 0.5 * a2)
                if two_walls:
                    sb[k + nxb] = dzb * (0.5 * a1 + 0.5 * a2)
        self.xb, self.yb, self.zb, self.ub, self.normals, self.sb = xb, yb, zb, ub, nrm, sb
        self.tangents_1 = t1                                        # :236-244
        self.tangents_2 = np.zeros(3 * nb)
        self.tangents_2[2 * nb:] = 1.0
        self.y_ref = yref
        self.blocks = [np.array(bot)] + ([np.array(top)] if two_walls else [])

    def _traveling_wave(self, t):
        g, p = self.g, self.p
        nxb, nzb = p["nxb"], p["nzb"]
        Lxp, Lzp = g.Lxp, g.Lzp
        dxb, dzb = Lxp / nxb, Lzp / nzb
        b1, b2, b3, tr = p["body_param_1"], p["body_param_2"], p["body_param_3"], p["body_ramp_up_time"]
        if t < tr and tr > 0.0:
            tau = t / tr
            amp = b1 * 0.5 * (1.0 - math.cos(PI * tau))
            damp = b1 * 0.5 * (PI / tr) * math.sin(PI * tau)
        else:
            amp, damp = b1, 0.0
        phi = PI
        nb = 2 * nxb * nzb
        xb, yb, zb = np.zeros(nb), np.zeros(nb), np.zeros(nb)
        ub, nrm, t1, sb = np.zeros(3 * nb), np.zeros(3 * nb), np.zeros(3 * nb), np.zeros(nb)
        yref = np.zeros(nb, dtype=np.int64)
        bot, top = [], []
        for j in range(1, nzb + 1):
            for i in range(1, nxb + 1):
                k = i + 2 * nxb * (j - 1) - 1
                x = (i - 0.5) * dxb
                xb[k] = xb[k + nxb] = x
                ph = b3 * (x - b2 * t)
                yb[k] = amp / (b2 * b3) * math.sin(ph)
                yb[k + nxb] = p["ly_channel"] + amp / (b2 * b3) * math.sin(ph + phi)
                zb[k] = zb[k + nxb] = (j - 0.5) * dzb
                yref[k], yref[k + nxb] = 1, p["ny_global"]
                bot.append(k); top.append(k + nxb)
        for j in range(1, nzb + 1):
            for i in range(1, nxb + 1):
                k = i + 2 * nxb * (j - 1) - 1
                ph = b3 * (xb[k] - b2 * t)
                ub[nb + k] = -amp * math.cos(ph) + (damp / (b2 * b3)) * math.sin(ph)
                ub[nb + k + nxb] = -amp * math.cos(ph + phi) + (damp / (b2 * b3)) * math.sin(ph + phi)
                sbot = amp / b2 * math.cos(ph)
                stop = amp / b2 * math.cos(ph + phi)
                t1[k] = 1.0 / math.sqrt(1.0 + sbot ** 2)
                t1[k + nxb] = 1.0 / math.sqrt(1.0 + stop ** 2)
                t1[nb + k] = sbot / math.sqrt(1.0 + sbot ** 2)
                t1[nb + k + nxb] = stop / math.sqrt(1.0 + stop ** 2)
                nrm[k] = t1[nb + k]
                nrm[k + nxb] = -t1[nb + k + nxb]
                nrm[nb + k] = -t1[k]
                nrm[nb + k + nxb] = t1[k + nxb]
        for j in range(1, nzb + 1):
            for i in range(1, nxb + 1):
                for wall in (0, 1):
                    k = i + wall * nxb + 2 * nxb * (j - 1) - 1
                    first = wall * nxb + 2 * nxb * (j - 1)
                    last = nxb - 1 + wall * nxb + 2 * nxb * (j - 1)
                    if i == 1:
                        a1 = math.sqrt((xb[k] - (xb[last] - Lxp)) ** 2 + (yb[k] - yb[last]) ** 2)
                        a2 = math.sqrt((xb[k] - xb[k + 1]) ** 2 + (yb[k] - yb[k + 1]) ** 2)
                    elif i == nxb:
                        a1 = math.sqrt((xb[k] - xb[k - 1]) ** 2 + (yb[k] - yb[k - 1]) ** 2)
                        a2 = math.sqrt((xb[k] - (xb[first] + Lxp)) ** 2 + (yb[k] - yb[first]) ** 2)
                    else:
                        a1 = math.sqrt((xb[k] - xb[k - 1]) ** 2 + (yb[k] - yb[k - 1]) ** 2)
                        a2 = math.sqrt((xb[k] - xb[k + 1]) ** 2 + (yb[k] - yb[k + 1]) ** 2)
                    sb[k] = dzb * (0.5 * a1 + 0.5 * a2)
        self.xb, self.yb, self.zb, self.ub, self.normals, self.sb = xb, yb, zb, ub, nrm, sb
        self.tangents_1 = t1                                        # :344-352
        self.tangents_2 = np.zeros(3 * nb)
        self.tangents_2[2 * nb:] = 1.0
        self.y_ref = yref
        self.blocks = [np.array(bot), np.array(top)]

    def _double_cylinders(self):
        g, p = self.g, self.p
        nzb = p["nzb"]
        Lxp, Lzp = g.Lxp, g.Lzp
        r1, r2 = p["body_param_1"], p["body_param_2"]
        dzb = Lzp / nzb
        dxb = dzb * g.dx / g.dz                                      # compute_nb :35-36
        nxb1 = int(2 * 3.14159 * r1 / dxb)
        nxb2 = int(2 * 3.14159 * r2 / dxb)
        nxb = nxb1 + nxb2
        nb = nxb * nzb
        xc, yc = 0.5 * Lxp, 0.5 * p["ly_channel"]
        dsb1 = 2 * 3.14159 * r1 / nxb1
        dsb2 = 2 * 3.14159 * r2 / nxb2
        xb, yb, zb = np.zeros(nb), np.zeros(nb), np.zeros(nb)
        ub, nrm, sb = np.zeros(3 * nb), np.zeros(3 * nb), np.zeros(nb)
        t1 = np.zeros(3 * nb)
        inner, outer = [], []
        for j in range(1, nzb + 1):
            for i in range(1, nxb1 + 1):
                k = i + (j - 1) * nxb - 1
                th = float(i - 1) * dsb1 / r1
                xb[k] = r1 * math.cos(th) + xc
                yb[k] = r1 * math.sin(th) + yc
                zb[k] = (j - 0.5) * dzb
                ub[k] = -math.sin(th) * p["body_param_3"]
                ub[nb + k] = math.cos(th) * p["body_param_3"]
                sb[k] = dsb1 * dzb
                nrm[k] = -math.cos(th)
                nrm[nb + k] = -math.sin(th)
                t1[k] = math.sin(th)                                # :146-147
                t1[nb + k] = -math.cos(th)
                inner.append(k)
            for i in range(1, nxb2 + 1):
                k = i + (j - 1) * nxb + nxb1 - 1
                th = float(i - 1) * dsb2 / r2
                xb[k] = r2 * math.cos(th) + xc
                yb[k] = r2 * math.sin(th) + yc
                zb[k] = (j - 0.5) * dzb
                sb[k] = dsb2 * dzb
                nrm[k] = math.cos(th)
                nrm[nb + k] = math.sin(th)
                t1[k] = -math.sin(th)                               # :160-161
                t1[nb + k] = math.cos(th)
                outer.append(k)
        self.xb, self.yb, self.zb, self.ub, self.normals, self.sb = xb, yb, zb, ub, nrm, sb
        self.tangents_1 = t1
        self.tangents_2 = np.zeros(3 * nb)                          # :164-166
        self.tangents_2[2 * nb:] = 1.0
        self.y_ref = np.ones(nb, dtype=np.int64)
        self.blocks = [np.array(inner), np.array(outer)]

    def _two_cylinders(self):
        """Two separate spanwise cylinders (no reference analog; conventions
        of double_cylinders_z, src/immersed_boundary_geometry.f90:117-174):
        radius body_param_1, surface speeds +-body_param_2, centres
        (body_param_3, Ly/2) and (2 body_param_3, Ly/2 + body_param_4); normals
        into each cylinder; one body per cylinder."""
        g, p = self.g, self.p
        nxb, nzb = p["nxb"], p["nzb"]
        r, us = p["body_param_1"], p["body_param_2"]
        dzb = g.Lzp / nzb
        dsb = 2.0 * PI * r / nxb
        nb = 2 * nxb * nzb
        xc = (p["body_param_3"], 2.0 * p["body_param_3"])
        yc = (0.5 * p["ly_channel"], 0.5 * p["ly_channel"] + p["body_param_4"])
        sgn = (1.0, -1.0)
        xb, yb, zb = np.zeros(nb), np.zeros(nb), np.zeros(nb)
        ub, nrm, sb = np.zeros(3 * nb), np.zeros(3 * nb), np.zeros(nb)
        t1 = np.zeros(3 * nb)
        blocks = ([], [])
        for j in range(1, nzb + 1):
            for c in range(2):
                for i in range(1, nxb + 1):
                    k = i + c * nxb + 2 * nxb * (j - 1) - 1
                    th = (i - 1) * 2.0 * PI / nxb
                    xb[k] = xc[c] + r * math.cos(th)
                    yb[k] = yc[c] + r * math.sin(th)
                    zb[k] = (j - 0.5) * dzb
                    ub[k] = -sgn[c] * us * math.sin(th)
                    ub[nb + k] = sgn[c] * us * math.cos(th)
                    sb[k] = dsb * dzb
                    nrm[k] = -math.cos(th)
                    nrm[nb + k] = -math.sin(th)
                    t1[k] = math.sin(th)
                    t1[nb + k] = -math.cos(th)
                    blocks[c].append(k)
        self.xb, self.yb, self.zb, self.ub, self.normals, self.sb = xb, yb, zb, ub, nrm, sb
        self.tangents_1 = t1
        self.tangents_2 = np.zeros(3 * nb)
        self.tangents_2[2 * nb:] = 1.0
        self.y_ref = np.ones(nb, dtype=np.int64)
        self.blocks = [np.array(blocks[0]), np.array(blocks[1])]

    def _wall_plates(self, t):
        """Wall-mounted bending plates (no reference analog): nxb x nzb plates
        of height h = body_param_1 and width half the spanwise pitch, 32 x 16
        markers each, rows from 3 dymin above the wall to the tip;
        x = x_p + a (y/h)^2 sin(omega t + phi), a = body_param_2,
        omega = body_param_3, phi from splitmix64 seeded with body_param_4."""
        g, p = self.g, self.p
        nxb, nzb = p["nxb"], p["nzb"]
        my, mz = 32, 16
        hh, amp, om = p["body_param_1"], p["body_param_2"], p["body_param_3"]
        pitchx, pitchz = g.Lxp / nxb, g.Lzp / nzb
        wz = 0.5 * pitchz
        lat = nxb * my
        nb = nxb * nzb * my * mz
        phase = splitmix64_phases(int(round(p["body_param_4"])), nxb * nzb)
        xb, yb, zb = np.zeros(nb), np.zeros(nb), np.zeros(nb)
        ub, nrm, sb = np.zeros(3 * nb), np.zeros(3 * nb), np.zeros(nb)
        t1 = np.zeros(3 * nb)
        for pj in range(1, nzb + 1):
            for m in range(1, mz + 1):
                for pi_ in range(1, nxb + 1):
                    for kk in range(1, my + 1):
                        ix, iz = (pi_ - 1) * my + kk - 1, (pj - 1) * mz + m - 1
                        k = ix + lat * iz
                        ph = phase[(pi_ - 1) + nxb * (pj - 1)]
                        y0 = 3.0 * g.dymin
                        y = y0 + (kk - 1) * (hh - y0) / (my - 1)
                        eta = y / hh
                        sn, cs = math.sin(om * t + ph), math.cos(om * t + ph)
                        xb[k] = (pi_ - 0.5) * pitchx + amp * eta * eta * sn
                        yb[k] = y
                        zb[k] = (pj - 0.5) * pitchz + (m - 0.5 - 0.5 * mz) * (wz / mz)
                        ub[k] = amp * eta * eta * om * cs
                        slope = 2.0 * amp * y / (hh * hh) * sn
                        nn = math.sqrt(1.0 + slope * slope)
                        nrm[k] = 1.0 / nn
                        nrm[nb + k] = -slope / nn
                        t1[k] = slope / nn                          # along the plate, up
                        t1[nb + k] = 1.0 / nn
                        sb[k] = ((hh - 3.0 * g.dymin) / (my - 1)) * (wz / mz)
        self.xb, self.yb, self.zb, self.ub, self.normals, self.sb = xb, yb, zb, ub, nrm, sb
        self.tangents_1 = t1
        self.tangents_2 = np.zeros(3 * nb)
        self.tangents_2[2 * nb:] = 1.0
        self.y_ref = np.ones(nb, dtype=np.int64)
        self.blocks = [np.arange(nb)]


def splitmix64_phases(seed, n):
    """n phases 2 pi u, u in [0, 1) from the splitmix64 stream of ``seed``."""
    mask = (1 << 64) - 1
    st = seed & mask
    out = np.zeros(n)
    for q in range(n):
        st = (st + 0x9E3779B97F4A7C15) & mask
        z = st
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        z ^= z >> 31
        out[q] = 2.0 * PI * (z >> 11) * (1.0 / 9007199254740992.0)
    return out


def remove_mean_per_body(body, f):
    """src/immersed_boundary_geometry.f90:400-470 (in place on a length-nb vector)."""
    for b in body.blocks:
        f[b] = f[b] - np.sum(f[b]) / len(b)
    return f


# ---------------------------------------------------------------------------
# operators, src/immersed_boundary_operators.f90
# ---------------------------------------------------------------------------
_S3 = math.sqrt(3.0)


def deltafnc(x1, x2, dr):
    """Yang3 discrete delta / dr, :270-294 (vectorised)."""
    r = np.abs(x1 - x2)
    r1 = r / dr
    r2 = r1 * r1
    with np.errstate(invalid="ignore"):
        a = (17.0 / 48.0 + _S3 * PI / 108.0 + r1 / 4.0 - r2 / 4.0
             + (1.0 - 2.0 * r1) / 16.0 * np.sqrt(-12.0 * r2 + 12.0 * r1 + 1.0)
             - _S3 / 12.0 * np.arcsin(_S3 / 2.0 * (2.0 * r1 - 1.0)))
        b = (55.0 / 48.0 - _S3 * PI / 108 - 13.0 * r1 / 12.0 + r2 / 4.0
             + (2.0 * r1 - 3.0) / 48.0 * np.sqrt(-12.0 * r2 + 36.0 * r1 - 23.0)
             + _S3 / 36.0 * np.arcsin(_S3 / 2.0 * (2.0 * r1 - 3.0)))
    out = np.where(r1 <= 1.0, a, np.where(r1 <= 2.0, b, 0.0))
    return out / dr


class Operators:
    """setup_IB_operators (:19-256): for each of the u, v, w and centre
    locations, per marker and per stencil point (k, j, i order, i fastest),
    the weight, the normal offset dxn and the folded field index."""

    def __init__(self, g, body):
        self.g, self.body = g, body
        self.build()

    def build(self):
        g, b = self.g, self.body
        nxg_, nzg_ = g.nx, g.nz           # nx_global, nz_global
        nxm_, nzm_ = g.nxm, g.nzm         # nxm_global, nzm_global
        dx, dz, dymin = g.dx, g.dz, g.dymin
        xb, yb, zb = b.xb, b.yb, b.zb
        nb = b.nb
        nrm = b.normals
        yref = b.y_ref
        x_piv = np.floor(xb / dx).astype(np.int64) + 1                      # :29-41
        xm_piv = np.floor((xb + 0.5 * dx) / dx).astype(np.int64)
        yr = g.y[yref]
        y_piv = np.floor((yb - yr) / dymin).astype(np.int64) + yref
        ym_piv = np.floor((yb - (yr + 0.5 * dymin)) / dymin).astype(np.int64) + yref
        z_piv = np.floor(zb / dz).astype(np.int64) + 1
        zm_piv = np.floor((zb + 0.5 * dz) / dz).astype(np.int64) + 1
        ks, js, is_ = np.meshgrid(np.arange(-SUPP, SUPP + 1), np.arange(-SUPP, SUPP + 1),
                                  np.arange(-SUPP, SUPP + 1), indexing="ij")
        ks, js, is_ = ks.ravel(), js.ravel(), is_.ravel()     # count order: k, j, i (i fastest)
        self.ops = {}
        scale = dx * dymin * dz

        def zfold_centre(kkp):
            # kk_periodic == nzg_global-1 is the duplicate of plane 2
            return np.where(kkp == g.nzg - 1, 2, kkp)

        def finish(name, ii_p, xs, x_grid, jj_idx, y_grid, kk_idx, z_grid, iy):
            w = scale * deltafnc(x_grid, xb[:, None], dx) * deltafnc(y_grid, yb[:, None], dymin) \
                * deltafnc(z_grid, zb[:, None], dz)
            dxn = (nrm[:nb, None] * (x_grid - xb[:, None]) + nrm[nb:2 * nb, None] * (y_grid - yb[:, None])
                   + nrm[2 * nb:, None] * (z_grid - zb[:, None]))
            self.ops[name] = dict(ix=xs, iy=iy, iz=kk_idx, w=w, dxn=dxn)

        # u: faces in x, centres in y and z (:44-90)
        ii = x_piv[:, None] + is_[None, :]
        jj = ym_piv[:, None] + js[None, :]
        kk = zm_piv[:, None] + ks[None, :]
        xsh = np.floor((ii - 1).astype(np.float64) / (nxg_ - 2)).astype(np.int64)
        iip = ii - xsh * (nxg_ - 2)
        zsh = np.floor((kk - 2).astype(np.float64) / nzm_).astype(np.int64)
        kkp = kk - zsh * (nzm_ - 1)
        ux = np.where(iip == 1, nxg_ - 1, iip)
        finish("u", iip, ux, g.x[iip] + xsh * g.Lxp, None, g.ym[jj], zfold_centre(kkp),
               g.zm[kkp - 1] + zsh * g.Lzp, jj + 1)
        # v: centres in x and z, faces in y (:93-138)
        ii = xm_piv[:, None] + is_[None, :]
        jj = y_piv[:, None] + js[None, :]
        kk = zm_piv[:, None] + ks[None, :]
        xsh = np.floor((ii - 1).astype(np.float64) / (nxm_ - 1)).astype(np.int64)
        iip = ii - xsh * (nxm_ - 1)
        zsh = np.floor((kk - 2).astype(np.float64) / nzm_).astype(np.int64)
        kkp = kk - zsh * (nzm_ - 1)
        finish("v", iip, iip + 1, g.xm[iip] + xsh * g.Lxp, None, g.y[jj], zfold_centre(kkp),
               g.zm[kkp - 1] + zsh * g.Lzp, jj)
        # w: centres in x and y, faces in z (:141-184); x window starts one cell lower
        ii = xm_piv[:, None] + is_[None, :] - 1
        jj = ym_piv[:, None] + js[None, :]
        kk = z_piv[:, None] + ks[None, :]
        xsh = np.floor((ii - 1).astype(np.float64) / (nxm_ - 1)).astype(np.int64)
        iip = ii - xsh * (nxm_ - 1)
        zsh = np.floor((kk - 2).astype(np.float64) / (nzg_ - 2)).astype(np.int64)
        kkp = kk - zsh * (nzg_ - 2)
        finish("w", iip, iip + 1, g.xm[iip] + xsh * g.Lxp, None, g.ym[jj], kkp,
               g.z[kkp] + zsh * g.Lzp, jj + 1)
        # c: centres (:187-234)
        ii = xm_piv[:, None] + is_[None, :]
        jj = ym_piv[:, None] + js[None, :]
        kk = zm_piv[:, None] + ks[None, :]
        xsh = np.floor((ii - 1).astype(np.float64) / (nxm_ - 1)).astype(np.int64)
        iip = ii - xsh * (nxm_ - 1)
        zsh = np.floor((kk - 2).astype(np.float64) / nzm_).astype(np.int64)
        kkp = kk - zsh * (nzm_ - 1)
        finish("c", iip, iip + 1, g.xm[iip] + xsh * g.Lxp, None, g.ym[jj], zfold_centre(kkp),
               g.zm[kkp - 1] + zsh * g.Lzp, jj + 1)

    # E: interpolation, local_regT (:409-454)
    def E(self, U, V, W):
        out = []
        for name, F in (("u", U), ("v", V), ("w", W)):
            o = self.ops[name]
            out.append(np.sum(o["w"] * F[o["ix"], o["iy"], o["iz"]], axis=1))
        return np.concatenate(out)

    # E1n for velocities, local_regT_1n (:456-501)
    def E1n(self, U, V, W):
        out = []
        for name, F in (("u", U), ("v", V), ("w", W)):
            o = self.ops[name]
            out.append(np.sum(o["w"] * F[o["ix"], o["iy"], o["iz"]] * o["dxn"], axis=1))
        return np.concatenate(out)

    # E1n for a centre field stored with rhs_p extents, local_regTc_1n (:503-526)
    def E1n_c(self, Pr):
        o = self.ops["c"]
        return np.sum(o["w"] * Pr[o["ix"], o["iy"], o["iz"]] * o["dxn"], axis=1)

    # R: spreading, local_reg (:544-603) into a zeroed field
    def R(self, comp, f, shape):
        g, b = self.g, self.body
        F = np.zeros(shape)
        o = self.ops["uvw"[comp]]
        factor = 1.0 / (g.dx * g.dymin * g.dz)
        vals = o["w"] * factor * b.sb[:, None] * f[:, None]
        np.add.at(F, (o["ix"].ravel(), o["iy"].ravel(), o["iz"].ravel()), vals.ravel())
        return F


# ---------------------------------------------------------------------------
# IB state, Heaviside, Schur complement, BiCGSTAB, projection
# ---------------------------------------------------------------------------
class IBState:
    def __init__(self, g, p, t=0.0, markers=None):
        self.g, self.p = g, p
        self.body = Body(g, p, t, markers)
        self.ops = Operators(g, self.body)
        nb = self.body.nb
        self.fb = np.zeros(4 * nb)
        self.Hu = g.u_array() + 1.0
        self.Hv = g.v_array() + 1.0
        self.Hw = g.w_array() + 1.0
        self.E1nHc_ext = np.zeros(nb)
        self.E1nH_ext = np.zeros(3 * nb)
        self.cg_accum_iter = 0
        self.last_iters = 0
        self.last_err = 0.0

    def refresh(self, t):
        self.body.update(t)
        self.ops = Operators(self.g, self.body)


def compute_heaviside(g, ib, st=None, rk_step=0, dt=None):
    """src/heaviside.f90:20-54."""
    b, ops = ib.body, ib.ops
    nb = b.nb
    Ur = ops.R(0, b.normals[:nb], g.u_array().shape)
    Vr = ops.R(1, b.normals[nb:2 * nb], g.v_array().shape)
    Wr = ops.R(2, b.normals[2 * nb:], g.w_array().shape)
    co.apply_boundary_conditions(g, Ur, Vr, Wr)
    Hc = co.divergence(g, Ur, Vr, Wr)
    Hc = -Hc
    co.solve_poisson_equation(g, Hc, st, rk_step, dt)
    Hce = 1.0 - Hc
    Hce[:2, :, :] = 0.0; Hce[:, :2, :] = 0.0; Hce[:, :, :2] = 0.0   # padding outside rhs_p bounds
    nx, ny, nz, nxg, nyg, nzg = g.nx, g.ny, g.nz, g.nxg, g.nyg, g.nzg
    Hu, Hv, Hw = g.u_array(), g.v_array(), g.w_array()
    # interpolate_x(Hc_ext, Hu_ext(2:nx-1, 2:nyg-1, 2:nzg)) etc. (src/interpolation.f90)
    Hu[2:nx, 2:nyg, 2:nzg + 1] = 0.5 * (Hce[2:nx, 2:nyg, 2:nzg + 1] + Hce[3:nx + 1, 2:nyg, 2:nzg + 1])
    Hv[2:nxg, 2:ny, 2:nzg + 1] = 0.5 * (Hce[2:nxg, 2:ny, 2:nzg + 1] + Hce[2:nxg, 3:ny + 1, 2:nzg + 1])
    Hw[2:nxg, 2:nyg, 2:nz + 1] = 0.5 * (Hce[2:nxg, 2:nyg, 2:nz + 1] + Hce[2:nxg, 2:nyg, 3:nz + 2])
    co.apply_boundary_conditions(g, Hu, Hv, Hw)
    Hui, Hvi, Hwi = 1.0 - Hu, 1.0 - Hv, 1.0 - Hw
    for A in (Hui, Hvi, Hwi):
        A[0, :, :] = 0.0; A[:, 0, :] = 0.0; A[:, :, 0] = 0.0
    co.apply_boundary_conditions(g, Hui, Hvi, Hwi)
    ib.Hu, ib.Hv, ib.Hw = Hui, Hvi, Hwi
    ib.Hc_ext = Hce
    ib.E1nHc_ext = ops.E1n_c(Hce)
    ib.E1nH_ext = ops.E1n(Hu, Hv, Hw)


def schur(g, ib, f, dt, st=None, rk_step=0):
    """src/projection.f90:98-144."""
    b, ops = ib.body, ib.ops
    nb, nu = b.nb, g.p["nu"]
    Sf = np.zeros(4 * nb)
    dudn, pj = f[:3 * nb], f[3 * nb:]
    aux = [dt * nu * dudn[c * nb:(c + 1) * nb] - dt * pj * b.normals[c * nb:(c + 1) * nb] for c in range(3)]
    Ur = ops.R(0, aux[0], g.u_array().shape)
    Vr = ops.R(1, aux[1], g.v_array().shape)
    Wr = ops.R(2, aux[2], g.w_array().shape)
    co.apply_boundary_conditions(g, Ur, Vr, Wr)
    rhs = co.divergence(g, Ur, Vr, Wr)
    co.solve_poisson_equation(g, rhs, st, rk_step, dt)
    rhs = rhs / dt
    E1np = ops.E1n_c(rhs)
    Sf[3 * nb:] = -E1np
    remove_mean_per_body(b, Sf[3 * nb:])
    Sf[3 * nb:] = Sf[3 * nb:] - ib.E1nHc_ext * pj
    rhs = dt * rhs
    Gx, Gy, Gz = co.gradient(g, rhs)
    co.apply_boundary_conditions(g, Gx, Gy, Gz)
    Gx, Gy, Gz = Gx - Ur, Gy - Vr, Gz - Wr
    Eu = ops.E(Gx, Gy, Gz)
    Sf[:3 * nb] = Eu - ib.E1nH_ext * dudn
    return Sf


def bicgstab(g, ib, x, bvec, dt, st=None, rk_step=0, Minv=None, tol=None, max_iter=None):
    """src/projection.f90:146-186 (unpreconditioned when Minv is None); with a
    diagonal Minv, the right-preconditioned form S M^-1 y = b, x = M^-1 y."""
    p = g.p
    tol = p["cg_tol"] if tol is None else tol
    max_iter = p["cg_max_iter"] if max_iter is None else max_iter
    A = lambda v: schur(g, ib, v, dt, st, rk_step)
    M = (lambda v: v) if Minv is None else (lambda v: Minv * v)
    eps = tol * tol
    it = 0
    r = bvec - A(x)
    rhat = r.copy()
    rho_o = alpha = om = 1.0
    nu_ = np.zeros_like(x)
    pv = np.zeros_like(x)
    err = 1.0
    while it < max_iter and err >= eps:
        rho_n = float(np.dot(rhat, r))
        bta = (rho_n / rho_o) * (alpha / om)
        rho_o = rho_n
        pv = r + bta * (pv - om * nu_)
        ph = M(pv)
        nu_ = A(ph)
        alpha = rho_n / float(np.dot(rhat, nu_))
        h = x + alpha * ph
        sv = r - alpha * nu_
        sh = M(sv)
        tv = A(sh)
        om = float(np.dot(tv, sv)) / float(np.dot(tv, tv))
        x = h + om * sh
        r = sv - om * tv
        err = float(np.dot(r, r))
        it += 1
    ib.cg_accum_iter += it
    ib.last_iters = it
    ib.last_err = math.sqrt(err)
    return x


def compute_IB_projection(g, st, ib, dt, rk_step=0):
    """src/projection.f90:48-96; st.U/V/W hold the non-IB-projected field and
    st.U_interim/.. the field before that projection."""
    b, ops = ib.body, ib.ops
    nb, nu = b.nb, g.p["nu"]
    Eu = ops.E(st.U, st.V, st.W)
    rhs = np.zeros(4 * nb)
    rhs[:3 * nb] = -Eu + b.ub
    E1np = ops.E1n_c(st.P_interim)
    rhs[3 * nb:] = -E1np
    remove_mean_per_body(b, rhs[3 * nb:])
    ib.fb = bicgstab(g, ib, ib.fb, rhs, dt, st, rk_step)
    dudn, pj = ib.fb[:3 * nb], ib.fb[3 * nb:]
    aux = [dt * nu * dudn[c * nb:(c + 1) * nb] - dt * pj * b.normals[c * nb:(c + 1) * nb] for c in range(3)]
    Ur = ops.R(0, aux[0], g.u_array().shape)
    Vr = ops.R(1, aux[1], g.v_array().shape)
    Wr = ops.R(2, aux[2], g.w_array().shape)
    co.apply_boundary_conditions(g, Ur, Vr, Wr)
    rhs_p = co.divergence(g, Ur, Vr, Wr)
    co.solve_poisson_equation(g, rhs_p, st, rk_step, dt)
    rhs_p = rhs_p / dt
    rhs_p = st.P_interim - rhs_p
    rhs_p = dt * rhs_p
    Gx, Gy, Gz = co.gradient(g, rhs_p)
    st.U = st.U_interim - Ur - Gx
    st.V = st.V_interim - Vr - Gy
    st.W = st.W_interim - Wr - Gz
    co.apply_boundary_conditions(g, st.U, st.V, st.W)
    ib.rhs_last = rhs


def compute_time_step_RK3_ib(g, st, ib, dt):
    """src/time_integration.f90:86-213 with an immersed body."""
    p = g.p
    nx, ny, nz, nxg, nyg, nzg = g.nx, g.ny, g.nz, g.nxg, g.nyg, g.nzg
    to = st.t
    Uo, Vo, Wo = st.U.copy(), st.V.copy(), st.W.copy()
    Iu, Ju, Ku = slice(2, nx), slice(2, nyg), slice(2, nzg)
    Iv, Jv, Kv = slice(2, nxg), slice(2, ny), slice(2, nzg)
    Iw, Jw, Kw = slice(2, nxg), slice(2, nyg), slice(2, nz)
    epg = p["exterior_pressure_gradient"]
    F = []
    for s in range(3):
        F.append((co.compute_rhs_u(g, st.U, st.V, st.W, st.dPdx, ib.Hu, epg),
                  co.compute_rhs_v(g, st.U, st.V, st.W, st.dPdy, ib.Hv, epg),
                  co.compute_rhs_w(g, st.U, st.V, st.W, st.dPdz, ib.Hw, epg)))
        c = co.RK_COEF[s]
        for comp, (A, Ao, sl) in enumerate(((st.U, Uo, (Iu, Ju, Ku)), (st.V, Vo, (Iv, Jv, Kv)),
                                            (st.W, Wo, (Iw, Jw, Kw)))):
            if s == 0:
                A[sl] = Ao[sl] + dt * c[0] * F[0][comp]
            elif s == 1:
                A[sl] = Ao[sl] + dt * (c[0] * F[0][comp] + c[1] * F[1][comp])
            else:
                A[sl] = Ao[sl] + dt * (c[0] * F[0][comp] + c[1] * F[1][comp] + c[2] * F[2][comp])
        st.t = to + co.RK_T[s] * dt
        if ib.body.moving:
            ib.refresh(st.t)
            compute_heaviside(g, ib, st, s + 1, dt)
        co.apply_boundary_conditions(g, st.U, st.V, st.W)
        st.U_interim, st.V_interim, st.W_interim = st.U.copy(), st.V.copy(), st.W.copy()
        co.compute_non_IB_projection(g, st, dt, rk_step=s + 1)
        co.apply_boundary_conditions(g, st.U, st.V, st.W)
        compute_IB_projection(g, st, ib, dt, rk_step=s + 1)
        co.apply_boundary_conditions(g, st.U, st.V, st.W)
    if p["x_mass_cte"] == 1:
        dPdx_prev = st.dPdx
        shift = co.compute_dPx_for_constant_mass_flow(g, st.U, st.Qflow_x_0, ib.Hu)
        st.U[Iu, Ju, Ku] = st.U[Iu, Ju, Ku] + shift
        st.dPdx = 0.5 * (dPdx_prev + shift / dt)
        co.apply_boundary_conditions(g, st.U, st.V, st.W)
    return st
