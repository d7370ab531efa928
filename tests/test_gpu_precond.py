"""GPU tests of the learned Schur preconditioner.

Network: forward output and parameter gradient of the tcgen05 kernels
against the CPU oracle with the same BF16 rounding points (tolerance 2e-2
relative: FP32 accumulation in a different order can move values across a
BF16 rounding boundary).  Solver: with the learned preconditioner the IB
steps converge to the same tolerance and match the FP64 oracle (1e-9, as
the other IB step tests); a network forced to break down (all-zero
output) falls back to Jacobi and still converges."""
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


def run_oracle(g, st, ib, dt, n):
    for _ in range(n):
        ibo.compute_time_step_RK3_ib(g, st, ib, dt)


def test_learned_preconditioner_matches_oracle_and_trains():
    import channel3d_parallel_b200 as c3d
    p, g, st, ib, ch = build("wall_standing_wave", cg_tol=1e-12, cg_max_iter=400)
    dt = -p["cfl"]
    try:
        # collect from Jacobi-preconditioned solves, then train
        ch.set_mode(precond=c3d.lib.PRECOND_JACOBI)
        ch.precond_collect(True, max_store=64, max_sets=8)
        ch.compute_time_step_RK3(2)
        info = ch.precond_info()
        assert info["sets"] >= 1 and info["pairs"] > 0
        s0 = ch.stats()
        it_jac = s0["bicgstab_iters"] / s0["bicgstab_solves"]
        ch.precond_collect(False)
        loss = ch.precond_train(epochs=300, lr=2e-3)
        assert 0.0 <= loss < 1.0
        ch.set_mode(precond=c3d.lib.PRECOND_LEARNED)
        ch.compute_time_step_RK3(2)
        s1 = ch.stats()
        run_oracle(g, st, ib, dt, 4)
        for name, ref in (("U", st.U), ("V", st.V), ("W", st.W)):
            assert rel(ch.download(name), ref[1:, 1:, 1:]) < 1e-9, name
        assert s1["last_residual"] < p["cg_tol"]
        assert s1["precond_mode"] in (c3d.lib.PRECOND_LEARNED, c3d.lib.PRECOND_JACOBI)
        it_lrn = (s1["bicgstab_iters"] - s0["bicgstab_iters"]) / (s1["bicgstab_solves"] - s0["bicgstab_solves"])
        print(f"iterations per solve: jacobi {it_jac:.1f}, learned {it_lrn:.1f}, loss {loss:.3f}")
    finally:
        ch.close()


def test_broken_network_falls_back_to_jacobi():
    import channel3d_parallel_b200 as c3d
    p, g, st, ib, ch = build("wall_standing_wave", cg_tol=1e-12, cg_max_iter=400)
    dt = -p["cfl"]
    try:
        ch.precond_set_params(np.zeros(c3d.lib.PRECOND_NPARAM, np.float32), np.ones(8, np.float32))
        ch.set_mode(precond=c3d.lib.PRECOND_LEARNED)
        ch.compute_time_step_RK3(1)
        s = ch.stats()
        assert s["precond_fallbacks"] >= 1
        assert s["last_residual"] < p["cg_tol"]
        run_oracle(g, st, ib, dt, 1)
        for name, ref in (("U", st.U), ("V", st.V), ("W", st.W)):
            assert rel(ch.download(name), ref[1:, 1:, 1:]) < 1e-9, name
    finally:
        ch.close()


def iters_per_solve(s0, s1):
    return (s1["bicgstab_iters"] - s0["bicgstab_iters"]) / max(1, s1["bicgstab_solves"] - s0["bicgstab_solves"])


def test_spai_and_probe_trained_network_match_oracle():
    import channel3d_parallel_b200 as c3d
    p, g, st, ib, ch = build("wall_standing_wave", cg_tol=1e-12, cg_max_iter=400)
    dt = -p["cfl"]
    try:
        res = {}
        for name, mode in (("jacobi", c3d.lib.PRECOND_JACOBI), ("spai", c3d.lib.PRECOND_SPAI)):
            ch.set_mode(precond=mode)
            s0 = ch.stats()
            ch.compute_time_step_RK3(1)
            res[name] = iters_per_solve(s0, ch.stats())
            ch.precond_probe()                     # one training set per geometry
        loss = ch.precond_train(epochs=400, lr=2e-3)
        assert 0.0 <= loss < 1.0
        ch.set_mode(precond=c3d.lib.PRECOND_LEARNED)
        s0 = ch.stats()
        ch.compute_time_step_RK3(2)
        s1 = ch.stats()
        res["learned"] = iters_per_solve(s0, s1)
        run_oracle(g, st, ib, dt, 4)
        for name, ref in (("U", st.U), ("V", st.V), ("W", st.W)):
            assert rel(ch.download(name), ref[1:, 1:, 1:]) < 1e-9, name
        assert s1["last_residual"] < p["cg_tol"]
        print("iterations per solve:", {k: round(v, 1) for k, v in res.items()}, "loss", round(loss, 3),
              "fallbacks", s1["precond_fallbacks"])
    finally:
        ch.close()
