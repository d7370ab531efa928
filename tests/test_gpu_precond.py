"""GPU tests of the learned Schur preconditioner.

Network: forward output and parameter gradient of the tcgen05 kernels
against the CPU oracle with the same BF16 rounding points (tolerance 2e-2
relative: FP32 accumulation in a different order can move values across a
BF16 rounding boundary).

Solver: the network predicts the band of the Schur operator that the banded
z-Fourier preconditioner otherwise measures by probing.  Trained on probe
sets the solver generates, it must reach the same 1e-14 tolerance, match the
FP64 oracle (1e-10, as the other IB step tests), and need at most half the
iterations of the Jacobi-preconditioned solve; a network forced to break
down (non-finite parameters) hands over to the probed band and still
converges.
"""
import numpy as np
import pytest

from oracle import channel_oracle as co
from oracle import ib_oracle as ibo
from oracle import mlp_oracle as mo

from test_gpu_ib import build, rel

pytestmark = pytest.mark.gpu


def small_channel():
    import channel3d_parallel_b200 as c3d
    return c3d.Channel(nx_global=18, ny_global=17, nz_global=14, Lxp=1.0, Lzp=0.7, nu=1e-3,
                       CFL=-1e-3, grid_type=0, alpha_stretch=0.0)


@pytest.mark.parametrize("m", [128, 300, 16384])
def test_network_forward_and_gradient_match_oracle(m):
    p, X, mom, sig = mo.random_case(m, seed=m)
    with small_channel() as ch:
        ch.precond_set_params(p, sig)
        out, grad, loss = ch.precond_eval(X, mom, sig)
    L, _, out_ref, g_ref = mo.loss_and_grad(p.astype(np.float64), X, mom, sig, bf=True)
    assert np.abs(out - out_ref).max() <= 2e-2 * np.abs(out_ref).max()
    assert abs(loss - L) <= 2e-2 * abs(L)
    for name, a, b in (("W1", mo.OFF_W1, mo.OFF_B1), ("b1", mo.OFF_B1, mo.OFF_W2),
                       ("W2", mo.OFF_W2, mo.OFF_B2), ("b2", mo.OFF_B2, mo.OFF_W3),
                       ("W3", mo.OFF_W3, mo.OFF_B3), ("b3", mo.OFF_B3, mo.NPARAM)):
        err = np.linalg.norm(grad[a:b] - g_ref[a:b]) / np.linalg.norm(g_ref[a:b])
        assert err < 2e-2, (name, err)


def iters_per_solve(s0, s1):
    return (s1["bicgstab_iters"] - s0["bicgstab_iters"]) / max(1, s1["bicgstab_solves"] - s0["bicgstab_solves"])


TOL = 1e-14     # both sides converge far enough for the 1e-10 step parity


def count_iters(case, mode, nsteps, warm=0):
    import channel3d_parallel_b200 as c3d
    p, g, st, ib, ch = build(case, cg_tol=TOL, cg_max_iter=600)
    try:
        if warm:
            ch.compute_time_step_RK3(warm)
        ch.set_mode(precond=mode)
        s0 = ch.stats()
        ch.compute_time_step_RK3(nsteps)
        return iters_per_solve(s0, ch.stats())
    finally:
        ch.close()


@pytest.mark.parametrize("case,ratio,warm", [("wall_standing_wave", 0.5, 0), ("traveling_wave_x", None, 0)])
def test_learned_band_trains_and_beats_jacobi(case, ratio, warm):
    """Training sets: the band probed at five geometries 2 steps apart (the
    solver's unit corrections and their Schur responses); then three steps
    with the network's band and the learned warm start, which must converge
    to 1e-14 and match the oracle; for the standing wave with no hand-over
    to the probed band and at most half the Jacobi iterations.  The
    travelling wave is trained during its 10-step amplitude ramp and run
    after it (outside the training geometries; its test flow diverges after
    about 13 steps in every preconditioner mode alike, so the run cannot
    train after the ramp): reported, not asserted."""
    import channel3d_parallel_b200 as c3d
    L = c3d.lib
    p, g, st, ib, ch = build(case, cg_tol=TOL, cg_max_iter=600)
    dt = -p["cfl"]
    try:
        ch.set_mode(precond=L.PRECOND_BAND)
        if warm:
            ch.compute_time_step_RK3(warm)
        ch.precond_collect(True, max_sets=8)
        for _ in range(5):
            ch.precond_probe()
            ch.compute_time_step_RK3(2)
        ch.precond_collect(False)
        info = ch.precond_info()
        assert info["sets"] >= 5 and info["pairs"] > 0
        loss = ch.precond_train(epochs=1500, lr=2e-3)
        assert 0.0 <= loss < 0.05, loss
        ch.set_mode(precond=L.PRECOND_LEARNED)
        s0 = ch.stats()
        ch.compute_time_step_RK3(3)
        s1 = ch.stats()
        it_lrn = iters_per_solve(s0, s1)
        assert s1["last_residual"] < TOL
        for _ in range(warm + 13):
            ibo.compute_time_step_RK3_ib(g, st, ib, dt)
        errs = {name: rel(ch.download(name), ref[1:, 1:, 1:])
                for name, ref in (("U", st.U), ("V", st.V), ("W", st.W))}
        assert max(errs.values()) < 1e-10, errs
    finally:
        ch.close()
    it_jac = count_iters(case, L.PRECOND_JACOBI, 3, warm=warm + 10)
    it_band = count_iters(case, L.PRECOND_BAND, 3, warm=warm + 10)
    print(f"{case}: iterations per solve jacobi {it_jac:.1f}, probed band {it_band:.1f}, "
          f"learned {it_lrn:.1f}, loss {loss:.4f}, hand-overs {s1['precond_fallbacks'] - s0['precond_fallbacks']}")
    if ratio is not None:
        assert s1["precond_fallbacks"] == s0["precond_fallbacks"]
        assert it_lrn <= ratio * it_jac, (it_lrn, it_jac)


def test_broken_network_hands_over_to_the_probed_band():
    import channel3d_parallel_b200 as c3d
    L = c3d.lib
    p, g, st, ib, ch = build("wall_standing_wave", cg_tol=TOL, cg_max_iter=600)
    dt = -p["cfl"]
    try:
        ch.set_mode(precond=L.PRECOND_BAND)
        ch.precond_probe()                       # fixes the target scales
        # a diverged training run: non-finite parameters, so the predicted
        # band cannot be factored
        ch.precond_set_params(np.full(L.PRECOND_NPARAM, np.nan, np.float32), np.ones(8, np.float32))
        ch.set_mode(precond=L.PRECOND_LEARNED)
        ch.compute_time_step_RK3(1)
        s = ch.stats()
        assert s["precond_fallbacks"] >= 1
        assert s["last_residual"] < TOL
        ibo.compute_time_step_RK3_ib(g, st, ib, dt)
        for name, ref in (("U", st.U), ("V", st.V), ("W", st.W)):
            assert rel(ch.download(name), ref[1:, 1:, 1:]) < 1e-10, name
    finally:
        ch.close()


def test_badly_fitting_network_hands_over_to_the_probed_band():
    """An untrained network (random weights of unit scale) predicts a band
    unlike S's: the solve stalls or is slow against the probed band's recent
    solves (or the predicted band is singular), the probed band takes over,
    and the steps still converge to the tolerance and match the oracle."""
    import channel3d_parallel_b200 as c3d
    L = c3d.lib
    p, g, st, ib, ch = build("wall_standing_wave", cg_tol=TOL, cg_max_iter=600)
    dt = -p["cfl"]
    try:
        ch.set_mode(precond=L.PRECOND_BAND)
        ch.precond_probe()
        ch.compute_time_step_RK3(1)              # the probed band's iteration count
        rng = np.random.default_rng(5)
        ch.precond_set_params(rng.standard_normal(L.PRECOND_NPARAM).astype(np.float32),
                              np.ones(8, np.float32))
        ch.set_mode(precond=L.PRECOND_LEARNED)
        s0 = ch.stats()
        ch.compute_time_step_RK3(2)
        s1 = ch.stats()
        assert s1["precond_fallbacks"] > s0["precond_fallbacks"]
        assert s1["last_residual"] < TOL
        for _ in range(3):
            ibo.compute_time_step_RK3_ib(g, st, ib, dt)
        for name, ref in (("U", st.U), ("V", st.V), ("W", st.W)):
            assert rel(ch.download(name), ref[1:, 1:, 1:]) < 1e-10, name
    finally:
        ch.close()


def test_learned_unsupported_for_plates():
    import channel3d_parallel_b200 as c3d
    p, g, st, ib, ch = build("wall_plates", cg_max_iter=5)
    try:
        with pytest.raises(c3d.C3DError):
            ch.set_mode(precond=c3d.lib.PRECOND_LEARNED)
        with pytest.raises(c3d.C3DError):
            ch.precond_probe()
    finally:
        ch.close()
