"""Benchmark: RK3 steps/s of the channel at 192x129x192 (FP64) on B200.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                [--poisson fp64|mixed] [--no-cpu-baseline]

A step is one compute_time_step_RK3 of the 192x129x192 Re_tau=180 channel
(nx_global=194, ny_global=129, nz_global=194; Lx=4pi, Lz=4pi/3, tanh y grid
with stretching 2.0, nu=1/5600, dt=1e-3, constant mass flow) from the seeded
laminar+perturbation state.  The working set (~0.5 GB of FP64 fields) is
larger than L2, so no flush is needed between steps.

value : steps/s from CUDA events on the library's stream around K steps
        (fields resident in HBM), max over ranks, summed over ranks (replicas).
e2e   : the same metric through the C-ABI with the fields in pinned host
        arrays (c3d_time_step_rk3_host): every step uploads U, V, W, advances
        one step and downloads U, V, W into the same arrays; the download of
        one step and the upload of the next overlap slab by slab.
        e2e.blocking_calls_value: the same round trip as blocking
        upload / step / download calls.
--impl reference: the C++/OpenMP restatement of the reference's FP64 step
        (oracle/cpu_rk3.cpp; the Fortran/MPI/FFTW reference cannot be built
        on this host) with all host threads, one full RK3 step of the same
        workload per timed step.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX, NY, NZ = 194, 129, 194
LX, LZ = 4.0 * math.pi, 4.0 * math.pi / 3.0
NU = 1.0 / 5600.0
DT = 1e-3
WORKLOAD = "channel Re_tau=180 192x129x192 (nx_global=194, ny_global=129, nz_global=194), RK3, dt=1e-3"


def max_over_ranks(x, pg=None, device="cuda"):
    """The largest of a per-rank time over the process group (x itself
    without one): a whole-job rate is the ranks' work over the slowest
    rank's time."""
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], device=device, dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        return d["hbm_gbs"], "measured"
    except Exception:
        return 6650.0, "fallback"


def make_channel(poisson):
    import channel3d_parallel_b200 as c3d
    ch = c3d.Channel(nx_global=NX, ny_global=NY, nz_global=NZ, Lxp=LX, Lzp=LZ, nu=NU,
                     CFL=-DT, x_mass_cte=1, grid_type=1, alpha_stretch=2.0, dPdx=3.0 * NU)
    if poisson == "mixed":
        ch.set_mode(poisson=c3d.lib.POISSON_MIXED)
    c3d.seeded_initial_state(ch, 3.0 * NU, NU)
    return ch


def cpu_restatement(nthreads=0):
    """The C++/OpenMP restatement of the FP64 RK3 step on the workload's
    seeded initial state (the Fortran/MPI/FFTW reference cannot be built on
    this host), with all host threads by default."""
    from oracle import channel_oracle as co
    from oracle import cpu_rk3
    cpu_rk3.build()
    p = co.channel_params(NX, NY, NZ, LX, LZ, NU)
    g = co.Grid(p)
    st = co.seeded_initial_state(g, p["dpdx"])
    cc = cpu_rk3.CpuChannel(g, nthreads=nthreads)
    cc.set_state(st)
    return cc


def cpu_baseline_sample(min_seconds=10.0, max_steps=50):
    """Seconds per RK3 step of the C++/OpenMP restatement on the host: one
    untimed step, then whole steps until min_seconds have passed."""
    cc = cpu_restatement()
    cc.steps(1)
    n, t0 = 0, time.perf_counter()
    while n < 3 or (time.perf_counter() - t0 < min_seconds and n < max_steps):
        cc.steps(1)
        n += 1
    sec = (time.perf_counter() - t0) / n
    threads = cc.threads
    cc.close()
    return sec, n, threads


def measure_mixed(steps=10):
    """Mixed-precision Poisson against the FP64 path: steps/s of each and the
    max-norm relative difference of u, v, w after ``steps`` steps from the same
    seeded state."""
    import numpy as np
    out = {}
    fields = {}
    for mode in ("fp64", "mixed"):
        ch = make_channel(mode)
        ch.compute_time_step_RK3(steps)
        fields[mode] = {n: ch.download(n) for n in ("U", "V", "W")}
        ch.compute_time_step_RK3(50)
        out[mode] = {"steps_per_s": 1e3 / ch.last_step_time_ms(), "max_div": ch.check_divergence()}
        if mode == "mixed":
            out[mode]["refinement_sweeps"] = ch.stats()["refinement_sweeps"]
        ch.close()
    out["max_rel_diff_after_%d_steps" % steps] = {
        n: float(np.abs(fields["mixed"][n] - fields["fp64"][n]).max() / np.abs(fields["fp64"][n]).max())
        for n in ("U", "V", "W")}
    return out


def measure_accuracy():
    """Accuracy beside the timings: max-norm relative error of u, v, w, p
    (and the IB surface unknowns fb) against the FP64 CPU restatement of the
    reference's step, with max|div u|, for the FP64 and the mixed-precision
    Poisson paths: one step at 192x129x192, ten steps at 32x65x32, and ten IB
    steps of a planar standing-wave wall (34x49x14, band preconditioner)
    against the NumPy oracle."""
    import numpy as np
    import channel3d_parallel_b200 as c3d
    from oracle import channel_oracle as co
    from oracle import cpu_rk3
    cpu_rk3.build()

    def rel(a, b):
        return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))

    out = {}
    cases = {"192x129x192_1step": (194, 129, 194, LX, LZ, 1), "32x65x32_10steps": (34, 65, 34, math.pi,
                                                                                math.pi / 2, 10)}
    for name, (nx, ny, nz, lx, lz, nsteps) in cases.items():
        p = co.channel_params(nx, ny, nz, lx, lz, NU)
        g = co.Grid(p)
        st = co.seeded_initial_state(g, p["dpdx"])
        cc = cpu_rk3.CpuChannel(g)
        cc.set_state(st)
        cc.steps(nsteps)
        ref = {k: cc.get_field(k)[1:, 1:, 1:] for k in ("U", "V", "W", "P")}
        cc.close()
        res = {}
        for mode, pm in (("fp64", c3d.lib.POISSON_FP64), ("mixed", c3d.lib.POISSON_MIXED),
                         ("mixed_unrefined", c3d.lib.POISSON_MIXED_UNREFINED)):
            with c3d.Channel(nx_global=nx, ny_global=ny, nz_global=nz, Lxp=lx, Lzp=lz, nu=NU, CFL=-DT,
                             x_mass_cte=1, grid_type=1, alpha_stretch=2.0, dPdx=p["dpdx"]) as ch:
                ch.set_mode(poisson=pm)
                ch.set_grid(g.x[1:], g.y[1:], g.z[1:])
                for k in ("U", "V", "W"):
                    ch.upload(k, getattr(st, k)[1:, 1:, 1:])
                ch.set_scalars(dPdx=st.dPdx, Qflow_x_0=st.Qflow_x_0)
                ch.compute_time_step_RK3(nsteps)
                res[mode] = {k: rel(ch.download(k), ref[k]) for k in ("U", "V", "W", "P")}
                res[mode]["max_div"] = ch.check_divergence()
        out[name] = res
    # IB: ten steps of the planar standing wave against the NumPy oracle
    from oracle import ib_oracle as ibo
    kw = dict(nx_global=34, ny_global=49, nz_global=14, Lxp=2.0, Lzp=0.6, grid_type=2, alpha_stretch=2.0,
              min_buffer_width=0.45, body_type="wall_standing_wave", nxb=32, nzb=12, body_param_1=0.02,
              body_param_2=2 * math.pi / 5.0, body_param_3=1.0, body_param_4=0.2)
    nu = 3.076923076923077e-04
    p = co.channel_params(34, 49, 14, 2.0, 0.6, nu, alpha=2.0, grid_type=2, cfl=-1e-3, x_mass_cte=1,
                          cg_tol=1e-14, cg_max_iter=600, min_buffer_width=0.45, body_type="wall_standing_wave",
                          nxb=32, nzb=12, body_param_1=0.02, body_param_2=2 * math.pi / 5.0, body_param_3=1.0,
                          body_param_4=0.2)
    g = co.Grid(p)
    st = co.seeded_initial_state(g, p["dpdx"], amplitude=0.05, dt=1e-3)
    ib = ibo.IBState(g, p, t=0.0)
    ibo.compute_heaviside(g, ib)
    q, n = co.mean_mass_flow_u(g, st.U, ib.Hu)
    st.Qflow_x_0 = q / n
    for k in ("nx_global", "ny_global", "nz_global", "Lxp", "Lzp", "grid_type", "alpha_stretch"):
        kw.pop(k)
    with c3d.Channel(nx_global=34, ny_global=49, nz_global=14, Lxp=2.0, Lzp=0.6, nu=nu, CFL=-1e-3, x_mass_cte=1,
                     grid_type=2, alpha_stretch=2.0, dPdx=p["dpdx"], cg_tol=1e-14, cg_max_iter=600, **kw) as ch:
        ch.set_grid(g.x[1:], g.y[1:], g.z[1:])
        for k in ("U", "V", "W"):
            ch.upload(k, getattr(st, k)[1:, 1:, 1:])
        ch.compute_dt()
        ch.compute_heaviside()
        ch.set_scalars(dPdx=st.dPdx, t=0.0, Qflow_x_0=st.Qflow_x_0)
        ch.set_mode(precond=c3d.lib.PRECOND_BAND)
        ch.compute_time_step_RK3(10)
        for _ in range(10):
            ibo.compute_time_step_RK3_ib(g, st, ib, 1e-3)
        res = {k: rel(ch.download(k), getattr(st, k)[1:, 1:, 1:]) for k in ("U", "V", "W")}
        res["fb"] = rel(ch.download("FB"), ib.fb)
        res["max_div"] = ch.check_divergence()
        out["ib_wall_standing_wave_34x49x14_10steps"] = res
    return out


IB_CONFIGS = {
    # cfg2: the 192x129x192 channel with an immersed plane at y = 0.2 above the
    # lower wall (y = -0.8 in wall-centred coordinates), 192x192 markers,
    # standing wave 0.02 sin(2 pi x/Lx) cos(2 pi t/5).  The IB operators take
    # the y pivot and delta width from dymin (src/immersed_boundary_operators.f90:
    # 35-37, 86-89), so every stencil must lie in uniform y cells: grid_type 2
    # with min_buffer_width 0.45 makes the wall buffer uniform up to y = 0.26,
    # above the plane's highest stencil row (0.22 + 2.5 dymin = 0.245).  With a
    # 0.3 buffer (uniform only up to 0.18) the plane sits in stretched cells,
    # the operators are inconsistent there and the Schur system is indefinite
    "cfg2": dict(grid=(194, 129, 194), Lxp=4.0 * math.pi, Lzp=4.0 * math.pi / 3.0, nu=1.0 / 5600.0,
                 grid_type=2, alpha_stretch=2.0, min_buffer_width=0.45, body_type="wall_standing_wave",
                 nxb=192, nzb=192, body_param_1=0.02, body_param_2=2 * math.pi / 5, body_param_3=1.0,
                 body_param_4=0.2,
                 desc="plane y=0.2, 192x192 markers, standing wave A=0.02 omega=2pi/5"),
    # cfg3: 256x129x128 on a uniform grid (the cylinders' stencils need uniform
    # cells); Lx = 4.5 holds the cylinders at x = 1.5 and 3.0, Lz = 2 gives
    # nearly square x-z cells; 200 x 128 markers per cylinder of radius 0.15,
    # surface speeds +-0.5
    "cfg3": dict(grid=(258, 129, 130), Lxp=4.5, Lzp=2.0, nu=1.0 / 5600.0, grid_type=0, alpha_stretch=0.0,
                 body_type="two_cylinders_z", nxb=200, nzb=128, body_param_1=0.15, body_param_2=0.5,
                 body_param_3=1.5, body_param_4=0.3,
                 desc="two counter-rotating z cylinders r=0.15 at (1.5,0), (3.0,0.3), 2x200x128 markers"),
    # cfg4: Re_tau=550 channel 384x257x384 (Lx=2pi, Lz=pi, nu=1/20000), 16x8
    # wall-mounted plates of height 0.1, 32x16 markers each, tip amplitude 0.01,
    # seeded phases; the wall buffer (min_buffer_width 0.25) is uniform up to
    # y = 0.139, above the plates' highest stencil row (0.1 + 2.5 dymin)
    "cfg4": dict(grid=(386, 257, 386), Lxp=2.0 * math.pi, Lzp=math.pi, nu=1.0 / 20000.0, grid_type=2,
                 alpha_stretch=2.0, min_buffer_width=0.25, body_type="wall_plates", nxb=16, nzb=8,
                 body_param_1=0.1, body_param_2=0.01, body_param_3=2 * math.pi, body_param_4=7,
                 desc="16x8 wall plates h=0.1, 32x16 markers each, tip amplitude 0.01"),
}


def make_ib_channel(maxit, cfg="cfg2", tol=1e-10):
    import channel3d_parallel_b200 as c3d
    c = dict(IB_CONFIGS[cfg])
    nx, ny, nz = c.pop("grid")
    c.pop("desc")
    nu = c.pop("nu")
    ch = c3d.Channel(nx_global=nx, ny_global=ny, nz_global=nz, CFL=-DT, x_mass_cte=1, nu=nu,
                     dPdx=3.0 * nu, cg_tol=tol, cg_max_iter=maxit, **c)
    ch.compute_heaviside()
    c3d.seeded_initial_state(ch, 3.0 * nu, nu)
    return ch


def measure_ib(maxit=300, steps=2, modes=("none", "jacobi", "band", "learned"), cfgs=("cfg2",),
               band_maxit=600):
    """Schur BiCGSTAB of the IB projection at the 1e-10 tolerance for each
    preconditioner, after one untimed warm-up step (graph capture, first
    preconditioner build): iterations and device ms per solve (3 solves per step),
    ms per iteration (two Schur applications), the residual reached, and for
    the band preconditioner its builds (probes of the Schur operator and the
    banded factorisations) in device ms."""
    import channel3d_parallel_b200 as c3d
    L = c3d.lib
    mode_id = {"none": L.PRECOND_NONE, "jacobi": L.PRECOND_JACOBI, "band": L.PRECOND_BAND,
               "learned": L.PRECOND_LEARNED, "spai": L.PRECOND_SPAI}

    def run(ch, n):
        s0 = ch.stats()
        ch.compute_time_step_RK3(n)
        step_ms = ch.last_step_time_ms()     # whole IB RK3 step, device timeline
        s1 = ch.stats()
        ns = s1["bicgstab_solves"] - s0["bicgstab_solves"]
        it = s1["bicgstab_iters"] - s0["bicgstab_iters"]
        ms = s1["bicgstab_ms"] - s0["bicgstab_ms"]
        bms = s1["precond_build_ms"] - s0["precond_build_ms"]
        return {"iters_per_solve": it / ns, "ms_per_solve": ms / ns, "ms_per_iter": ms / max(it, 1),
                "build_ms_per_solve": bms / ns, "builds": s1["precond_builds"] - s0["precond_builds"],
                "total_ms_per_solve": (ms + bms) / ns, "iters_per_step": it / n,
                "last_residual": s1["last_residual"], "converged": s1["last_residual"] < 1e-10,
                "fallbacks": s1["precond_fallbacks"] - s0["precond_fallbacks"],
                "max_div": ch.check_divergence(), "ib_rows": list(s1["ib_rows"]),
                "ms_per_step": step_ms}

    out = {}
    for cfg in cfgs:
        c = IB_CONFIGS[cfg]
        res = {"config": c["desc"], "grid": list(c["grid"]), "cg_tol": 1e-10, "modes": {}}
        for name in modes:
            cap = band_maxit if name in ("band", "learned") else maxit
            ch = make_ib_channel(cap, cfg)
            res["markers"] = ch.dims["nb"]
            try:
                if name == "learned":
                    res["modes"][name] = learned_run(ch, run, steps)
                else:
                    ch.set_mode(precond=mode_id[name])
                    ch.compute_time_step_RK3(1)      # warm-up: graph capture, first builds
                    res["modes"][name] = run(ch, steps)
                    res["modes"][name]["cg_max_iter"] = cap
            except c3d.C3DError as e:
                res["modes"][name] = {"unavailable": str(e)}
            finally:
                ch.close()
        # Bytes of one Schur application on the band of y rows it touches
        # (the stencil rows and one row either side; Nb = Nx * rows * Nz):
        # spread writes 3 fields (24 Nb), divergence reads them (24) and
        # writes the x spectrum (8.08 = 16 B x 97/192 per cell at 192), the
        # band y-z solve reads and writes it (16.17), the inverse x transform
        # reads it and writes phi (8.08 + 8), the gathers read phi and the
        # three fields (32): 120.3 B per band cell.
        rows = next((m.get("ib_rows") for m in res["modes"].values() if m.get("ib_rows")), None)
        if rows and rows[1] >= rows[0]:
            nx, nz = c["grid"][0] - 2, c["grid"][2] - 2
            spec = 16.0 * (nx // 2 + 1) / nx
            nb_cells = nx * (rows[1] - rows[0] + 3) * nz
            per_cell = 24 + 24 + spec + 2 * spec + spec + 8 + 32
            byt = per_cell * nb_cells
            res["schur_bytes"] = {"band_rows": rows, "band_cells": nb_cells, "bytes_per_cell": per_cell,
                                  "bytes_per_application": byt,
                                  "hbm_ms_per_application": byt / (measured_peaks()[0] * 1e9) * 1e3}
            for m in res["modes"].values():
                if "ms_per_iter" in m:
                    m["iter_frac_of_hbm_bound"] = 2 * res["schur_bytes"]["hbm_ms_per_application"] / m["ms_per_iter"]
        out[cfg] = res
    return out


def profile_schur(cfg, apps):
    """N applications of the Schur operator S (src/projection.f90:98-144)
    and of the probed band preconditioner, as plain stream launches (no time
    step, no BiCGSTAB): the kernels of one BiCGSTAB iteration's operators in
    isolation, for launch lists and captures.  Host vectors in and out."""
    import numpy as np
    import channel3d_parallel_b200 as c3d
    ch = make_ib_channel(600, cfg)
    try:
        ch.setup_IB_operators()
        ch.set_mode(precond=c3d.lib.PRECOND_BAND)
        ch.precond_probe()
        f = np.random.default_rng(0).standard_normal(4 * ch.dims["nb"])
        ch.schur(f)
        t0 = time.perf_counter()
        for _ in range(apps):
            ch.schur(f)
            ch.precond_apply(f)
        wall = (time.perf_counter() - t0) / apps * 1e3
        return {"cfg": cfg, "schur_apps": apps, "wall_ms_per_schur_and_band_apply": wall,
                "ib_rows": list(ch.stats()["ib_rows"])}
    finally:
        ch.close()


def learned_run(ch, run, steps):
    """Learned preconditioner: trained on probe pairs at three geometries
    (RK stages of band-preconditioned steps), then used."""
    import channel3d_parallel_b200 as c3d
    L = c3d.lib
    ch.set_mode(precond=L.PRECOND_BAND)
    t0 = time.perf_counter()
    for _ in range(3):
        ch.precond_probe()
        ch.compute_time_step_RK3(1)
    t_probe = time.perf_counter() - t0
    t0 = time.perf_counter()
    loss = ch.precond_train(epochs=400, lr=2e-3)
    t_train = time.perf_counter() - t0
    ch.set_mode(precond=L.PRECOND_LEARNED)
    ch.compute_time_step_RK3(1)                  # warm-up: graph capture, buffers
    r = run(ch, steps)
    r.update({"train_loss": loss, "train_s": t_train, "probe_and_step_s": t_probe,
              "pairs": ch.precond_info()["pairs"]})
    return r


def run_reference(args):
    """Reference arm: the reference's algorithm on the host cores.  The
    Fortran/MPI/FFTW reference cannot be built here, so this times its
    C++/OpenMP restatement (oracle/cpu_rk3.cpp) with all host threads: W
    untimed steps, then K timed steps (fewer if K steps would take more than
    about two minutes; the line says how many were timed)."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    cc = cpu_restatement()
    cc.steps(max(1, args.warmup))
    t0 = time.perf_counter()
    cc.steps(1)
    first = time.perf_counter() - t0
    budget = max(1, min(args.steps, int(120.0 / max(first, 1e-6))))
    n = 1
    if budget > 1:
        cc.steps(budget - 1)
        n = budget
    sec = (time.perf_counter() - t0) / n
    threads = cc.threads
    cc.close()
    val = 1.0 / sec
    line = {
        "impl": "reference", "metric": "RK3 steps/s at 192x129x192 (FP64)", "value": val,
        "unit": "steps/s", "n_gpus": args.gpus, "steps": n, "warmup": args.warmup,
        "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "grid": [NX, NY, NZ], "cells": (NX - 2) * (NY - 1) * (NZ - 2),
                   "poisson": "fp64", "parallelism": f"replicas x{args.gpus}",
                   "l2": "working set > L2 (no flush)"},
        "cpu_baseline": {"value": val, "unit": "steps/s", "cores": threads, "kind": "port",
                         "sample": f"{n} full RK3 steps of the workload ({args.steps} requested) on the "
                                   "C++/OpenMP restatement of the reference's step, "
                                   f"{threads} OpenMP threads"},
        "e2e": {"value": val, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import numpy as np
    import torch
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    ch = make_channel(args.poisson)
    dims = ch.dims
    # warm-up (also captures the step graph)
    ch.compute_time_step_RK3(args.warmup)
    ch.synchronize()
    l0 = ch.kernel_launches()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    time.sleep(0.3)
    ch.compute_time_step_RK3(args.steps)     # CUDA events inside the library
    ms_step = ch.last_step_time_ms()
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = ch.kernel_launches() - l0
    ms_step = max_over_ranks(ms_step, pg)
    if pg:
        pg.barrier()
    value = ws / (ms_step * 1e-3)
    div = ch.check_divergence()
    if args.device_only:
        ch.close()
        if pg:
            pg.destroy_process_group()
        if rank == 0:
            print(json.dumps({"metric": "RK3 steps/s at 192x129x192", "value": value,
                              "unit": "steps/s", "ms_per_step": ms_step,
                              "gpu_launches": launches, "max_div": div}), flush=True)
        return

    # ---- per-kernel device times (roofline of the dominant kernel)
    prof = ch.profile_kernels(nrep=10)
    N = (NX - 2) * (NY - 1) * (NZ - 2)
    # algorithmic bytes per cell: each FP64 value read or written once
    # (spectrum: 97 complex per 192 real = 8.08 B per cell)
    sp = 16.0 * (NX - 2 + 2) / 2 / (NX - 2)
    bytes_per_cell = {"rhs_stage": 72.0, "grad_sub": 8.0 * 7, "div_xfft": 8.0 * 3 + sp,
                      "xfft_inv": sp + 8.0, "spectral_yz": 2 * sp}
    dom = max(("rhs_stage", "grad_sub", "div_xfft", "xfft_inv", "spectral_yz"),
              key=lambda k: prof[k])
    alg = bytes_per_cell[dom] * N
    peak, peak_kind = measured_peaks()
    achieved = alg / (prof[dom] * 1e-3) / 1e9
    # the whole step against the same peak: three stages of RHS, divergence +
    # x FFT, slab, inverse x FFT and projection update (72 FP64 field passes)
    step_bytes = 3 * sum(bytes_per_cell.values()) * N
    step_roofline = {"bytes_per_step": step_bytes, "achieved": step_bytes / (ms_step * 1e-3) / 1e9,
                     "peak": peak, "unit": "GB/s", "frac": step_bytes / (ms_step * 1e-3) / 1e9 / peak}
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile):
        try:
            traffic = json.load(open(tfile)).get(dom)
        except Exception:
            traffic = None

    # ---- end to end through the C-ABI with pinned host buffers: the fields
    # live in the caller's arrays and every step uploads U, V, W, advances one
    # step and downloads them into the same arrays (c3d_time_step_rk3_host,
    # whose slabbed copies let step n's download overlap step n+1's upload)
    pin = {}
    for name in ("U", "V", "W"):
        a = ch.download(name)
        t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
        t.numpy()[:] = a.reshape(-1, order="F")
        pin[name] = (t, t.numpy().reshape(a.shape, order="F"))
    nbytes = sum(v[1].nbytes for v in pin.values())
    e2e_steps = max(3, min(args.steps, 20))
    hU, hV, hW = (pin[n][1] for n in ("U", "V", "W"))
    ch.compute_time_step_RK3_host(hU, hV, hW, 2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ch.compute_time_step_RK3_host(hU, hV, hW, e2e_steps)
    e2e_sec = (time.perf_counter() - t0) / e2e_steps
    e2e_sec = max_over_ranks(e2e_sec, pg)
    e2e_val = ws / e2e_sec
    # the same round trip as one blocking call per copy and per step
    # (upload U, V, W; one step; download U, V, W), without the overlap
    from channel3d_parallel_b200 import lib as L
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        for name in ("U", "V", "W"):
            ch.upload(name, pin[name][1])
        ch.compute_time_step_RK3(1)
        for name in ("U", "V", "W"):
            cl, cu = L.box(*ch.bounds(name))
            L.check(ch._lib.c3d_download(ch.handle, L.FIELD[name], L.dptr(pin[name][1]), cl, cu), ch.handle)
    e2e_sync_sec = max_over_ranks((time.perf_counter() - t0) / e2e_steps, pg)

    extras = {}
    if ws == 1 and not args.no_extras:
        extras["mixed_vs_fp64"] = measure_mixed()
        extras["accuracy"] = measure_accuracy()
        extras["ib_schur"] = measure_ib(maxit=args.ib_maxit, cfgs=tuple(args.ib_cfgs.split(",")))
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        sec, nst, threads = cpu_baseline_sample()
        cpu = {"value": 1.0 / sec, "unit": "steps/s", "cores": threads, "kind": "port",
               "sample": f"{nst} full RK3 steps of the workload on the C++/OpenMP restatement "
                         "of the reference's step (FP64)"}
    ch.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": "RK3 steps/s at 192x129x192 (FP64)" if args.poisson == "fp64"
        else "RK3 steps/s at 192x129x192 (mixed-precision Poisson)",
        "value": value, "unit": "steps/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.poisson == "fp64" else "f64+f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "grid": [NX, NY, NZ], "cells": N, "poisson": args.poisson,
                   "parallelism": f"replicas x{ws}", "l2": "working set > L2 (no flush)"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "alg_bytes_per_launch": alg,
                     "kernel_ms": prof[dom]},
        "step_roofline": step_roofline,
        "kernel_ms": prof,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_val, "unit": "steps/s", "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": nbytes, "entry": "c3d_time_step_rk3_host",
                "blocking_calls_value": ws / e2e_sync_sec},
        "gpu_launches": launches,
        "clocks": clk,
        "max_div": div,
    }
    line.update(extras)
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--poisson", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the mixed-precision and IB Schur-solve measurements")
    ap.add_argument("--ib-maxit", type=int, default=300,
                    help="BiCGSTAB iteration cap of the IB measurement without the band preconditioner")
    ap.add_argument("--ib-cfgs", default="cfg2,cfg3,cfg4",
                    help="IB configurations to measure (cfg2, cfg3, cfg4)")
    ap.add_argument("--only-ib", action="store_true",
                    help="only the IB Schur-solve measurement (--steps steps per preconditioner)")
    ap.add_argument("--ib-modes", default="none,jacobi,band,learned")
    ap.add_argument("--device-only", action="store_true",
                    help="only the device-timed step loop (used for profiler captures)")
    ap.add_argument("--schur-apps", type=int, default=0,
                    help="only N Schur-operator and band-preconditioner applications at the first of "
                         "--ib-cfgs, outside any time step (a profiler target)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.schur_apps > 0:
        print(json.dumps(profile_schur(args.ib_cfgs.split(",")[0], args.schur_apps)), flush=True)
        return
    if args.only_ib:
        print(json.dumps(measure_ib(maxit=args.ib_maxit, steps=args.steps,
                                    modes=tuple(args.ib_modes.split(",")),
                                    cfgs=tuple(args.ib_cfgs.split(",")))), flush=True)
        return
    if args.impl == "reference":
        if args.steps > 20:
            args.steps = 10     # each CPU step is a full RK3 step (seconds)
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
