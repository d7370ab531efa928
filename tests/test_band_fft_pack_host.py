"""Host check of the packing the band preconditioner's lattice FFTs use
(k_band_fwd_fft / k_band_inv_fft against the direct DFTs k_band_fwd /
k_band_inv of the same file).

Forward: two real marker columns a, b share one complex row z = a + i b;
from Z = FFT(z) the half spectra are A[q] = (Z[q] + conj Z[N-q]) / 2 and
B[q] = (Z[q] - conj Z[N-q]) / 2i, q = 0 .. N/2, which must equal the direct
DFTs sum_iz a[iz] exp(-2 pi i q iz / N).

Inverse: the direct kernel forms v[iz] = (1/N) sum_q w_q Re(X[q] exp(+2 pi i
q iz / N)), w_q = 2 except q = 0 and q = N/2.  The packed form drops the
imaginary parts of X[0] and X[N/2], extends A and B to the whole circle as
Hermitian spectra, inverts Z = A + i B once and takes a = Re z / N,
b = Im z / N.  Half spectra with non-zero imaginary parts at q = 0 and N/2
(the band solve's output need not be exactly Hermitian there) must give the
same values.
"""
import numpy as np
import pytest

LENGTHS = [3, 6, 10, 12, 16, 128, 192]


def direct_forward(x):
    n = len(x)
    nq = n // 2 + 1
    iz = np.arange(n)
    return np.array([np.sum(x * np.exp(-2j * np.pi * q * iz / n)) for q in range(nq)])


def direct_inverse(X, n):
    iz = np.arange(n)
    v = np.zeros(n)
    for q, xq in enumerate(X):
        w = 1.0 if (q == 0 or 2 * q == n) else 2.0
        v += w * np.real(xq * np.exp(2j * np.pi * q * iz / n))
    return v / n


def packed_forward(a, b):
    n = len(a)
    Z = np.fft.fft(a + 1j * b)
    q = np.arange(n // 2 + 1)
    zn = np.conj(Z[(n - q) % n])
    return (Z[q] + zn) / 2.0, (Z[q] - zn) / 2j


def packed_inverse(A, B, n):
    A = A.copy()
    B = B.copy()
    Z = np.zeros(n, dtype=np.complex128)
    for q in range(len(A)):
        edge = q == 0 or 2 * q == n
        if edge:
            A[q] = A[q].real
            B[q] = B[q].real
        Z[q] = A[q] + 1j * B[q]
        if not edge:
            Z[n - q] = np.conj(A[q]) + 1j * np.conj(B[q])
    z = np.fft.ifft(Z) * n          # unnormalised inverse, as the engine's
    return z.real / n, z.imag / n


@pytest.mark.parametrize("n", LENGTHS)
def test_packed_forward_matches_direct_dft(n):
    rng = np.random.default_rng(n)
    a, b = rng.standard_normal(n), rng.standard_normal(n)
    A, B = packed_forward(a, b)
    for got, x in ((A, a), (B, b)):
        ref = direct_forward(x)
        assert np.abs(got - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("n", LENGTHS)
def test_packed_inverse_matches_direct_real_inverse(n):
    rng = np.random.default_rng(100 + n)
    nq = n // 2 + 1
    A = rng.standard_normal(nq) + 1j * rng.standard_normal(nq)
    B = rng.standard_normal(nq) + 1j * rng.standard_normal(nq)
    a, b = packed_inverse(A, B, n)
    for got, X in ((a, A), (b, B)):
        ref = direct_inverse(X, n)
        assert np.abs(got - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())
