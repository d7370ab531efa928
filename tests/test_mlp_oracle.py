"""CPU checks of the preconditioner-network oracle: the analytic gradient
against central finite differences (float64, no BF16 rounding), and the
BF16 rounding helper against known values."""
import numpy as np

from oracle import mlp_oracle as mo


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159265, 65504.0, 1e-3], np.float32)
    got = mo.bf16(x)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: rounds to even (1.0)
    assert got[0] == 1.0 and got[1] == 1.0
    assert got[2] == 1.0078125
    assert abs(got[3] + 3.140625) < 1e-12
    assert np.all(np.abs(got - x) <= np.abs(x) * 2.0 ** -8)


def test_gradient_matches_finite_differences():
    p, X, mom, sig = mo.random_case(40, seed=3)
    p = p.astype(np.float64)
    L, _, _, g = mo.loss_and_grad(p, X, mom, sig, bf=False)
    rng = np.random.default_rng(0)
    idx = np.concatenate([rng.choice(np.arange(mo.OFF_W1, mo.OFF_B1), 6),
                          rng.choice(np.arange(mo.OFF_B1, mo.OFF_W2), 3),
                          rng.choice(np.arange(mo.OFF_W2, mo.OFF_B2), 6),
                          rng.choice(np.arange(mo.OFF_B2, mo.OFF_W3), 3),
                          rng.choice(np.arange(mo.OFF_W3, mo.OFF_B3), 6),
                          np.arange(mo.OFF_B3, mo.NPARAM)])
    for i in idx:
        h = 1e-6 * max(1.0, abs(p[i]))
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (mo.loss(pp, X, mom, sig, bf=False)[0] - mo.loss(pm, X, mom, sig, bf=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])


def test_loss_is_zero_at_least_squares_optimum():
    # with Ahat = Cer Crr^-1 for every row and Cee = diag(Cer Crr^-1 Cer^T), L = 0
    p, X, mom, sig = mo.random_case(5, seed=1)
    Crr, Cer, _ = mo.normalised(mom.astype(np.float64), sig)
    A = Cer @ np.linalg.inv(Crr)
    L = np.einsum("bij,bjk,bik->b", A, Crr, A) - 2 * np.einsum("bij,bij->b", A, Cer)
    Cee_opt = -L
    assert np.all(Cee_opt >= -1e-9)
