"""Host-side mirror of the reference's module interfaces over the C-ABI.

``Channel`` owns one libc3d handle: one z slab of the reference's global
arrays resident in GPU memory.  Its methods carry the names of the Fortran
module procedures they replace (``compute_time_step_RK3``,
``solve_poisson_equation``, ``compute_non_IB_projection``, ``regT``, ...)
and the same argument meaning; errors come back as ``C3DError`` instead of
``Stop``.  Arrays cross the boundary in Fortran order with the reference's
index bounds (see ``bounds``).
"""
import ctypes as C
import math
import os

import numpy as np

from . import lib as L

PI = 4.0 * math.atan(1.0)

_NAMELIST_ORDER = [
    "Lxp", "Lzp", "Ly_channel", "alpha_stretch", "nx_global", "ny_global", "nz_global",
    "nxb", "nzb", "CFL", "nu", "dPdx", "dPdz", "Qflow_x_0", "Qflow_z_0", "x_mass_cte",
    "y_mass_cte", "z_mass_cte", "nsteps", "nsave", "nstats", "nmonitor", "filein", "fileout",
    "nstep_init", "t_init", "init_type", "grid_type", "body_type",
    "exterior_pressure_gradient", "body_param_3", "body_param_1", "body_param_2",
    "body_ramp_up_time", "min_buffer_width", "cg_tol", "cg_max_iter", "perturb_scale",
    "body_param_4"]


def namelist_text(**params):
    """A ``&params`` namelist (src/input_output.f90:27-40) from keyword values."""
    canon = {k.lower(): k for k in _NAMELIST_ORDER}
    lines = ["&params"]
    for key, val in params.items():
        name = canon.get(key.lower())
        if name is None:
            raise KeyError(f"unknown namelist variable {key!r}")
        if isinstance(val, bool):
            s = ".true." if val else ".false."
        elif isinstance(val, str):
            s = "'" + val + "'"
        elif isinstance(val, int):
            s = str(val)
        else:
            s = repr(float(val)).replace("e", "d")
            if "d" not in s and "." not in s:
                s += "d0"
        lines.append(f"  {name} = {s}")
    lines.append("/")
    return "\n".join(lines) + "\n"


class Channel:
    """One solver handle (one GPU-resident domain)."""

    def __init__(self, namelist_path=None, text=None, **params):
        self._lib = L.load()
        h = C.c_int(0)
        if namelist_path is not None:
            rc = self._lib.c3d_create(str(namelist_path).encode(), C.byref(h))
        else:
            if text is None:
                text = namelist_text(**params)
            rc = self._lib.c3d_create_from_text(text.encode(), C.byref(h))
        L.check(rc, 0)
        self.handle = h.value
        d = L.Dims()
        self._check(self._lib.c3d_get_dims(self.handle, C.byref(d)))
        self.dims = {n: getattr(d, n) for n, _ in L.Dims._fields_}

    # ------------------------------------------------------------------ infra
    def _check(self, rc):
        return L.check(rc, self.handle)

    def close(self):
        if getattr(self, "handle", 0):
            self._lib.c3d_destroy(self.handle)
            self.handle = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def bounds(self, name):
        """(lb, ub) Fortran index bounds of a field or marker array."""
        d = self.dims
        nx, ny, nz, nxg, nyg, nzg, nb = (d["nx"], d["ny"], d["nz"], d["nxg"], d["nyg"],
                                         d["nzg"], d["nb"])
        u = (nx, nyg, nzg)
        v = (nxg, ny, nzg)
        w = (nxg, nyg, nz)
        r = (nxg - 1, nyg - 1, nzg)
        tab = {
            "U": ((1, 1, 1), u), "V": ((1, 1, 1), v), "W": ((1, 1, 1), w),
            "P": ((1, 1, 1), (nxg, nyg, nzg)),
            "RHS_P": ((2, 2, 2), r), "P_INTERIM": ((2, 2, 2), r), "HC_EXTERIOR": ((2, 2, 2), r),
            "RHS_U": ((2, 2, 2), (nx - 1, nyg - 1, nzg - 1)),
            "RHS_V": ((2, 2, 2), (nxg - 1, ny - 1, nzg - 1)),
            "RHS_W": ((2, 2, 2), (nxg - 1, nyg - 1, nz - 1)),
            "U_WORK": ((1, 1, 1), u), "V_WORK": ((1, 1, 1), v), "W_WORK": ((1, 1, 1), w),
            "U_REG": ((1, 1, 1), u), "V_REG": ((1, 1, 1), v), "W_REG": ((1, 1, 1), w),
            "HU_INTERIOR": ((1, 1, 1), u), "HV_INTERIOR": ((1, 1, 1), v),
            "HW_INTERIOR": ((1, 1, 1), w),
            "FB": ((1, 1, 1), (4 * nb, 1, 1)), "UB": ((1, 1, 1), (3 * nb, 1, 1)),
            "XB": ((1, 1, 1), (nb, 1, 1)), "YB": ((1, 1, 1), (nb, 1, 1)),
            "ZB": ((1, 1, 1), (nb, 1, 1)), "NORMALS": ((1, 1, 1), (3 * nb, 1, 1)),
            "SB": ((1, 1, 1), (nb, 1, 1)), "E1NH_EXT": ((1, 1, 1), (3 * nb, 1, 1)),
            "E1NHC_EXT": ((1, 1, 1), (nb, 1, 1)),
        }
        return tab[name.upper()]

    def _id(self, name):
        n = name.upper()
        return L.FIELD[n] if n in L.FIELD else L.MARKER[n]

    def upload(self, name, arr, lb=None, ub=None):
        """Copy a host array (Fortran order) into a device field or sub-box."""
        flb, fub = self.bounds(name)
        lb = tuple(lb) if lb is not None else flb
        a = np.asfortranarray(arr, dtype=np.float64)
        if a.ndim == 1:
            a = a.reshape((-1, 1, 1), order="F")
        if ub is None:
            ub = tuple(lb[i] + a.shape[i] - 1 for i in range(3))
        cl, cu = L.box(lb, ub)
        self._check(self._lib.c3d_upload(self.handle, self._id(name), L.dptr(a), cl, cu))

    def download(self, name, lb=None, ub=None):
        """Return a device field (or sub-box) as a Fortran-ordered array."""
        flb, fub = self.bounds(name)
        lb = tuple(lb) if lb is not None else flb
        ub = tuple(ub) if ub is not None else fub
        shape = tuple(ub[i] - lb[i] + 1 for i in range(3))
        a = np.zeros(shape, dtype=np.float64, order="F")
        cl, cu = L.box(lb, ub)
        self._check(self._lib.c3d_download(self.handle, self._id(name), L.dptr(a), cl, cu))
        if name.upper() in L.MARKER:
            return a.reshape(-1, order="F")
        return a

    def set_grid(self, x, y, z):
        x, y, z = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z))
        self._check(self._lib.c3d_set_grid(self.handle, L.dptr(x), L.dptr(y), L.dptr(z)))

    def grid(self):
        d = self.dims
        out = {k: np.zeros(d[n]) for k, n in (("x", "nx"), ("y", "ny"), ("z", "nz"),
                                               ("xg", "nxg"), ("yg", "nyg"), ("zg", "nzg"))}
        self._check(self._lib.c3d_get_grid(self.handle, *(L.dptr(out[k]) for k in
                                                          ("x", "y", "z", "xg", "yg", "zg"))))
        return out

    def set_scalars(self, dPdx=0.0, dPdy=0.0, dPdz=0.0, t=0.0, Qflow_x_0=0.0):
        self._check(self._lib.c3d_set_scalars(self.handle, dPdx, dPdy, dPdz, t, Qflow_x_0))

    def synchronize(self):
        self._check(self._lib.c3d_synchronize(self.handle))

    # ------------------------------------------------- time_integration.f90
    def compute_time_step_RK3(self, nsteps=1):
        """compute_dt + compute_time_step_RK3 (src/time_integration.f90:86-267)."""
        return self._check(self._lib.c3d_time_step_rk3(self.handle, int(nsteps)))

    def compute_time_step_RK3_host(self, U, V, W, nsteps=1):
        """compute_time_step_RK3 with u, v, w kept in the caller's arrays
        (app/main.f90:101-117): each step uploads U, V, W, advances one step
        and writes them back in place.  The arrays must be float64,
        Fortran-contiguous and of the full field extents; page-locked memory
        (e.g. numpy views of pinned torch tensors) lets the copies overlap."""
        for name, a in (("U", U), ("V", V), ("W", W)):
            shape = self.bounds(name)[1]
            if (not isinstance(a, np.ndarray) or a.dtype != np.float64 or a.shape != tuple(shape)
                    or not a.flags.f_contiguous or not a.flags.writeable):
                raise ValueError(f"{name} must be a writeable Fortran-ordered float64 array of shape {shape}")
        return self._check(self._lib.c3d_time_step_rk3_host(self.handle, L.dptr(U), L.dptr(V), L.dptr(W),
                                                            int(nsteps)))

    def compute_time_step_Euler(self, nsteps=1):
        """compute_dt + compute_time_step_Euler (src/time_integration.f90:25-81)."""
        return self._check(self._lib.c3d_time_step_euler(self.handle, int(nsteps)))

    def compute_dt(self):
        dt = C.c_double(0.0)
        self._check(self._lib.c3d_compute_dt(self.handle, C.byref(dt)))
        return dt.value

    # ------------------------------------------------------ equations.f90
    def compute_rhs_u(self):
        self._check(self._lib.c3d_compute_rhs_u(self.handle))
        return self.download("RHS_U")

    def compute_rhs_v(self):
        self._check(self._lib.c3d_compute_rhs_v(self.handle))
        return self.download("RHS_V")

    def compute_rhs_w(self):
        self._check(self._lib.c3d_compute_rhs_w(self.handle))
        return self.download("RHS_W")

    # -------------------------------------- poisson.f90 / projection.f90
    def divergence(self):
        self._check(self._lib.c3d_divergence(self.handle))

    def solve_poisson_equation(self, rk_step=0):
        self._check(self._lib.c3d_solve_poisson_equation(self.handle, int(rk_step)))

    def compute_non_IB_projection(self, rk_step=0):
        self._check(self._lib.c3d_compute_non_IB_projection(self.handle, int(rk_step)))

    def compute_IB_projection(self):
        return self._check(self._lib.c3d_compute_IB_projection(self.handle))

    def schur(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64)
        out = np.zeros_like(f)
        self._check(self._lib.c3d_schur(self.handle, L.dptr(f), L.dptr(out)))
        return out

    def precond_apply(self, v):
        """M v for the preconditioner selected by set_mode (built if needed)."""
        v = np.ascontiguousarray(v, dtype=np.float64)
        out = np.zeros_like(v)
        self._check(self._lib.c3d_precond_apply(self.handle, L.dptr(v), L.dptr(out)))
        return out

    def bicgstab(self, rhs):
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        return self._check(self._lib.c3d_bicgstab(self.handle, L.dptr(rhs)))

    # ------------------------------------------ boundary_conditions.f90
    def apply_boundary_conditions(self, which="UVW"):
        code = {"UVW": 0, "REG": 1, "WORK": 2}[which.upper()]
        self._check(self._lib.c3d_apply_boundary_conditions(self.handle, code))

    # ----------------------------------------------------- mass_flow.f90
    def compute_dPx_for_constant_mass_flow(self):
        v = C.c_double(0.0)
        self._check(self._lib.c3d_compute_dPx_for_constant_mass_flow(self.handle, C.byref(v)))
        return v.value

    def compute_dPy_for_constant_mass_flow(self):
        """src/mass_flow.f90:190-221: Qflow_y_0 - Int_V/norm."""
        v = C.c_double(0.0)
        self._check(self._lib.c3d_compute_dPy_for_constant_mass_flow(self.handle, C.byref(v)))
        return v.value

    def compute_dPz_for_constant_mass_flow(self):
        """src/mass_flow.f90:236-267: Qflow_z_0 - Int_W/norm (W read through
        the routine's declared extents, as the reference does)."""
        v = C.c_double(0.0)
        self._check(self._lib.c3d_compute_dPz_for_constant_mass_flow(self.handle, C.byref(v)))
        return v.value

    def compute_mean_mass_flow_U(self):
        v = C.c_double(0.0)
        self._check(self._lib.c3d_compute_mean_mass_flow_u(self.handle, C.byref(v)))
        return v.value

    def compute_mean_mass_flow_V(self):
        v = C.c_double(0.0)
        self._check(self._lib.c3d_compute_mean_mass_flow_v(self.handle, C.byref(v)))
        return v.value

    def compute_mean_mass_flow_W(self):
        v = C.c_double(0.0)
        self._check(self._lib.c3d_compute_mean_mass_flow_w(self.handle, C.byref(v)))
        return v.value

    def set_flow_targets(self, Qflow_x_0, Qflow_y_0=0.0, Qflow_z_0=0.0):
        """Qflow_x_0, Qflow_y_0, Qflow_z_0 (src/global.f90:180)."""
        self._check(self._lib.c3d_set_flow_targets(self.handle, Qflow_x_0, Qflow_y_0, Qflow_z_0))

    # ------------------------------------- input_output, statistics, monitor
    def write_snapshot(self, path, original_format=False):
        """output_data (src/input_output.f90:498-728) to ``path``."""
        self._check(self._lib.c3d_write_snapshot(self.handle, os.fsencode(path), int(bool(original_format))))

    def read_snapshot(self, path):
        """read_input_data (src/input_output.f90:335-489): mesh and U, V, W."""
        self._check(self._lib.c3d_read_snapshot(self.handle, os.fsencode(path)))

    STAT_NAMES = ("Umean", "Vmean", "Wmean", "U2mean", "V2mean", "W2mean", "UVmean")

    def compute_statistics(self):
        """compute_statistics (src/statistics.f90:22-148): the seven y
        profiles at yg(1:nyg) and utau, wtau, Retau_u, Retau_w, Qflow_x/y/z."""
        nyg = self.dims["nyg"]
        prof = np.zeros(7 * nyg)
        sc = np.zeros(8)
        self._check(self._lib.c3d_compute_statistics(self.handle, prof.ctypes.data_as(L._D),
                                                      sc.ctypes.data_as(L._D)))
        out = {n: prof[q * nyg:(q + 1) * nyg].copy() for q, n in enumerate(self.STAT_NAMES)}
        out.update(dict(zip(("utau", "wtau", "Retau_u", "Retau_w", "Qflow_x", "Qflow_y", "Qflow_z"),
                            map(float, sc[:7]))))
        out["nonfinite"] = bool(sc[7])
        return out

    def write_statistics(self, path, istep):
        """output_statistics (src/input_output.f90:733-754) to ``path``."""
        self._check(self._lib.c3d_write_statistics(self.handle, os.fsencode(path), int(istep)))

    def output_monitor(self):
        """The values output_monitor prints (src/monitor.f90:21-110)."""
        out = np.zeros(8)
        self._check(self._lib.c3d_monitor(self.handle, out.ctypes.data_as(L._D)))
        return dict(zip(("meanU", "meanV", "meanW", "maxU", "maxV", "maxW", "max_divergence", "max_slip"),
                        map(float, out)))

    def compute_pressure(self):
        self._check(self._lib.c3d_compute_pressure(self.handle))

    # ------------------------------------- immersed_boundary_*.f90, heaviside.f90
    def setup_IB_geometry(self):
        self._check(self._lib.c3d_setup_IB_geometry(self.handle))

    def setup_IB_operators(self):
        self._check(self._lib.c3d_setup_IB_operators(self.handle))

    def compute_heaviside(self):
        self._check(self._lib.c3d_compute_heaviside(self.handle))

    def regT(self):
        out = np.zeros(3 * self.dims["nb"])
        self._check(self._lib.c3d_regT(self.handle, L.dptr(out)))
        return out

    def regT_1n(self):
        out = np.zeros(3 * self.dims["nb"])
        self._check(self._lib.c3d_regT_1n(self.handle, L.dptr(out)))
        return out

    def regTc_1n(self, field="P_INTERIM"):
        out = np.zeros(self.dims["nb"])
        self._check(self._lib.c3d_regTc_1n(self.handle, self._id(field), L.dptr(out)))
        return out

    def reg(self, component, f):
        f = np.ascontiguousarray(f, dtype=np.float64)
        self._check(self._lib.c3d_reg(self.handle, int(component), L.dptr(f)))

    # ------------------------------------------------ options / telemetry
    def set_mode(self, poisson=L.POISSON_FP64, precond=L.PRECOND_NONE):
        self._check(self._lib.c3d_set_mode(self.handle, poisson, precond))

    def stats(self):
        s = L.Stats()
        self._check(self._lib.c3d_get_stats(self.handle, C.byref(s)))
        out = {}
        for n, _ in L.Stats._fields_:
            v = getattr(s, n)
            out[n] = list(v) if isinstance(v, C.Array) else v
        return out

    def check_divergence(self):
        v = C.c_double(0.0)
        self._check(self._lib.c3d_check_divergence(self.handle, C.byref(v)))
        return v.value

    def check_finite(self):
        return self._check(self._lib.c3d_check_finite(self.handle))

    def last_step_time_ms(self):
        v = C.c_double(0.0)
        self._check(self._lib.c3d_last_step_time_ms(self.handle, C.byref(v)))
        return v.value

    def profile_kernels(self, nrep=10):
        """Average device ms of each kernel class (lib.KERNEL_CLASSES order)."""
        out = np.zeros(len(L.KERNEL_CLASSES))
        self._check(self._lib.c3d_profile_kernels(self.handle, int(nrep), L.dptr(out), len(out)))
        return dict(zip(L.KERNEL_CLASSES, out.tolist()))

    def kernel_launches(self):
        v = C.c_int64(0)
        self._check(self._lib.c3d_kernel_launches(self.handle, C.byref(v)))
        return v.value

    # ---- learned preconditioner of the Schur solve ----
    def precond_collect(self, enable=True, max_store=48, max_sets=16):
        """While enabled, every band the solver probes (PRECOND_BAND solves)
        is kept as a training set of the learned preconditioner (at most
        ``max_sets``; ``max_store`` is unused)."""
        self._check(self._lib.c3d_precond_collect(self.handle, int(bool(enable)), int(max_store),
                                                  int(max_sets)))

    def precond_probe(self):
        """Probe the band of the Schur operator at the current geometry (unit
        corrections and their Schur responses) and keep it as a training set."""
        self._check(self._lib.c3d_precond_probe(self.handle))

    def precond_train(self, epochs=400, lr=2e-3):
        """Train the network on the collected sets; returns the relative loss."""
        v = C.c_double(0.0)
        self._check(self._lib.c3d_precond_train(self.handle, int(epochs), float(lr), C.byref(v)))
        return v.value

    def precond_info(self):
        pairs, sets, epochs, loss = C.c_int64(0), C.c_int(0), C.c_int(0), C.c_double(0)
        self._check(self._lib.c3d_precond_info(self.handle, C.byref(pairs), C.byref(sets),
                                               C.byref(epochs), C.byref(loss)))
        return {"pairs": pairs.value, "sets": sets.value, "epochs": epochs.value,
                "loss": loss.value}

    def precond_params(self):
        """(parameters[PRECOND_NPARAM], sig[8]) as float32 arrays."""
        buf = np.zeros(L.PRECOND_NPARAM + 8, dtype=np.float32)
        self._check(self._lib.c3d_precond_get_params(self.handle, L.fptr(buf), len(buf)))
        return buf[:L.PRECOND_NPARAM].copy(), buf[L.PRECOND_NPARAM:].copy()

    def precond_set_params(self, params, sig=None):
        p = np.ascontiguousarray(params, dtype=np.float32)
        sg = None if sig is None else np.ascontiguousarray(sig, dtype=np.float32)
        self._check(self._lib.c3d_precond_set_params(self.handle, L.fptr(p), len(p),
                                                     L.fptr(sg) if sg is not None else None))

    def precond_eval(self, feats, moments, sig):
        """Network output, loss and parameter gradient on caller data."""
        f = np.ascontiguousarray(feats, dtype=np.float32)
        mo = np.ascontiguousarray(moments, dtype=np.float32)
        sg = np.ascontiguousarray(sig, dtype=np.float32)
        m = f.shape[0]
        out = np.zeros((m, 16), dtype=np.float32)
        grad = np.zeros(L.PRECOND_NPARAM, dtype=np.float32)
        loss = C.c_double(0.0)
        self._check(self._lib.c3d_precond_eval(self.handle, L.fptr(f), L.fptr(mo), m, L.fptr(sg),
                                               L.fptr(out), L.fptr(grad), C.byref(loss)))
        return out, grad, loss.value


def laminar_perturbed_fields(grid, dims, dPdx, nu, Ly=2.0, amplitude=0.1, seed=0):
    """Host fields of the seeded initial state: laminar profile
    dPdx/(Ly*nu)*y*(Ly-y) (src/input_output.f90:275-280) plus uniform
    perturbations of peak ``amplitude`` from NumPy PCG64(seed), drawn in
    Fortran order for U, then V, then W, with the wall values of
    src/input_output.f90:288-313.  Returns Fortran-ordered U, V, W."""
    nx, ny, nz, nxg, nyg, nzg = (dims[k] for k in ("nx", "ny", "nz", "nxg", "nyg", "nzg"))
    y = grid["y"]
    rng = np.random.Generator(np.random.PCG64(seed))
    ps = 2.0 * amplitude
    U = np.zeros((nx, nyg, nzg), order="F")
    for jj in range(1, ny):           # Fortran jj = 1..ny-1
        ymv = 0.5 * (y[jj - 1] + y[jj])
        if 0.0 < ymv < Ly:
            U[:, jj, :] = dPdx / (Ly * nu) * ymv * (Ly - ymv)

    def draw(shape):
        return ps * (rng.random(shape[::-1]).T - 0.5)

    U += draw(U.shape)
    U[:, 0, :] = -U[:, 1, :]
    U[:, ny, :] = -U[:, ny - 1, :]
    V = np.zeros((nxg, ny, nzg), order="F") + draw((nxg, ny, nzg))
    V[:, 0, :] = 0.0
    V[:, ny - 1, :] = 0.0
    W = np.zeros((nxg, nyg, nz), order="F") + draw((nxg, nyg, nz))
    W[:, 0, :] = -W[:, 1, :]
    W[:, ny, :] = -W[:, ny - 1, :]
    return np.asfortranarray(U), np.asfortranarray(V), np.asfortranarray(W)


def seeded_initial_state(ch, dPdx, nu, amplitude=0.1, seed=0, dt=1e-3):
    """Set the seeded initial state on the device: host fields of
    ``laminar_perturbed_fields``, boundary conditions, one projection (dt
    cancels), boundary conditions, and Qflow_x_0 and Qflow_z_0 from the
    result (app/main.f90:90-92); Qflow_y_0 and dPdy are zero (:93-94).
    Returns Qflow_x_0."""
    g = ch.grid()
    U, V, W = laminar_perturbed_fields(g, ch.dims, dPdx, nu, amplitude=amplitude, seed=seed)
    ch.upload("U", U)
    ch.upload("V", V)
    ch.upload("W", W)
    ch.apply_boundary_conditions("UVW")
    ch.set_scalars(dPdx=dPdx, t=0.0, Qflow_x_0=0.0)
    if ch.compute_dt() <= 0:
        raise ValueError("dt must be positive for the initial projection")
    ch.compute_non_IB_projection(rk_step=0)
    ch.apply_boundary_conditions("UVW")
    q = ch.compute_mean_mass_flow_U()
    ch.set_scalars(dPdx=dPdx, t=0.0, Qflow_x_0=q)
    ch.set_flow_targets(q, 0.0, ch.compute_mean_mass_flow_W())
    return q
