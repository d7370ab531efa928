"""CPU restatement of the learned Schur preconditioner network (test
infrastructure only: the GPU path never calls it).

The reference has no learned part (its bicgstab, src/projection.f90:146-186,
is unpreconditioned); this oracle states the model and loss that the CUDA
kernels implement so that their forward pass and gradients can be checked:

    out = W3 relu(W2 relu(W1 x + b1) + b2) + b3        (32 -> 128 -> 128 -> 16)
    Ahat = out reshaped 4x4 (row-major)
    L_b = tr(Ahat Crr Ahat^T) - 2 tr(Ahat Cer^T) + tr(Cee)

with the moments normalised by sig = (sig_r[4], sig_e[4]):
Crr_ij / (sig_r_i sig_r_j), Cer_ij / (sig_e_i sig_r_j), Cee_i / sig_e_i^2.

With ``bf16=True`` the values the GPU keeps in BF16 are rounded the same way
(round to nearest even): inputs, weights, hidden activations, dO, dZ2, dZ1.
Products accumulate in float64 here (FP32 on the GPU).
"""
import numpy as np

F, H, O = 32, 128, 16
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * F
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + O * H
NPARAM = OFF_B3 + O


def bf16(a):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    x = np.ascontiguousarray(a, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return rounded.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(H, F), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H),
            p[OFF_B2:OFF_W3], p[OFF_W3:OFF_B3].reshape(O, H), p[OFF_B3:NPARAM])


def _r(a, on):
    return bf16(a) if on else np.asarray(a, dtype=np.float64)


def forward(p, X, bf=True):
    W1, b1, W2, b2, W3, b3 = unpack(p)
    Xb = _r(X, bf)
    H1 = _r(np.maximum(Xb @ _r(W1, bf).T + b1, 0.0), bf)
    H2 = _r(np.maximum(H1 @ _r(W2, bf).T + b2, 0.0), bf)
    out = H2 @ _r(W3, bf).T + b3
    return out, (Xb, H1, H2)


def normalised(mom, sig):
    sr, se = np.asarray(sig[:4], np.float64), np.asarray(sig[4:], np.float64)
    Crr = mom[:, :16].reshape(-1, 4, 4) / np.outer(sr, sr)
    Cer = mom[:, 16:32].reshape(-1, 4, 4) / np.outer(se, sr)
    Cee = (mom[:, 32:36] / se ** 2).sum(axis=1)
    return Crr, Cer, Cee


def loss(p, X, mom, sig, bf=True):
    out, _ = forward(p, X, bf)
    A = out.reshape(-1, 4, 4)
    Crr, Cer, Cee = normalised(np.asarray(mom, np.float64), sig)
    AC = A @ Crr
    L = np.einsum("bij,bij->b", AC, A) - 2 * np.einsum("bij,bij->b", A, Cer) + Cee
    return L.sum(), Cee.sum()


def loss_and_grad(p, X, mom, sig, bf=True):
    """Unnormalised loss, its normaliser sum tr(Cee), output and gradient."""
    W1, b1, W2, b2, W3, b3 = unpack(p)
    out, (Xb, H1, H2) = forward(p, X, bf)
    A = out.reshape(-1, 4, 4)
    Crr, Cer, Cee = normalised(np.asarray(mom, np.float64), sig)
    AC = A @ Crr
    L = np.einsum("bij,bij->b", AC, A) - 2 * np.einsum("bij,bij->b", A, Cer) + Cee
    G = (2.0 * (AC - Cer)).reshape(-1, O)
    dO = _r(G, bf)
    dH2 = dO @ _r(W3, bf)
    g2 = dH2 * (H2 > 0)
    dZ2 = _r(g2, bf)
    dH1 = dZ2 @ _r(W2, bf)
    g1 = dH1 * (H1 > 0)
    dZ1 = _r(g1, bf)
    grad = np.zeros(NPARAM)
    grad[OFF_W3:OFF_B3] = (dO.T @ H2).ravel()
    grad[OFF_B3:NPARAM] = dO.sum(axis=0)
    grad[OFF_W2:OFF_B2] = (dZ2.T @ H1).ravel()
    grad[OFF_B2:OFF_W3] = g2.sum(axis=0)
    grad[OFF_W1:OFF_B1] = (dZ1.T @ Xb).ravel()
    grad[OFF_B1:OFF_W2] = g1.sum(axis=0)
    return L.sum(), Cee.sum(), out, grad


def random_case(m, seed=0):
    """Parameters, features, moments and sig of a reproducible test case."""
    rng = np.random.default_rng(seed)
    p = np.zeros(NPARAM)
    p[OFF_W1:OFF_B1] = rng.standard_normal(H * F) * np.sqrt(2.0 / F)
    p[OFF_B1:OFF_W2] = rng.standard_normal(H) * 0.1
    p[OFF_W2:OFF_B2] = rng.standard_normal(H * H) * np.sqrt(2.0 / H)
    p[OFF_B2:OFF_W3] = rng.standard_normal(H) * 0.1
    p[OFF_W3:OFF_B3] = rng.standard_normal(O * H) * 0.05
    p[OFF_B3:NPARAM] = np.eye(4).ravel() + rng.standard_normal(O) * 0.1
    X = rng.uniform(-1.0, 1.0, (m, F))
    R = rng.standard_normal((m, 4, 6))
    Crr = R @ R.transpose(0, 2, 1) / 6
    Cer = rng.standard_normal((m, 4, 4)) * 0.5 + np.eye(4)
    Cee = rng.uniform(0.5, 2.0, (m, 4))
    mom = np.concatenate([Crr.reshape(m, 16), Cer.reshape(m, 16), Cee], axis=1)
    sig = np.concatenate([rng.uniform(0.5, 2.0, 4), rng.uniform(0.5, 2.0, 4)])
    return (p.astype(np.float32), X.astype(np.float32), mom.astype(np.float32),
            sig.astype(np.float32))
