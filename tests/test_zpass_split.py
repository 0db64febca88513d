"""CPU restatement of the two-thread z-line transform of the register z pass
(csrc/mv_zpass.cuh; complex64 at Lz = 64, complex128 at Lz = 32): each thread b of a line
computes the outputs X[2m + b] as one Lz/2-point FFT of the twiddled input x[n] W^{nb} (the
line holds data only at n < N_z <= Lz/2), and the inverse keeps the layers 2n + b from one
Lz/2-point inverse FFT of W^{-bk} (X[k] + (-1)^b X[k + Lz/2]). Checked against the full
zero-padded transforms with numpy, with the kernel's own index arithmetic."""

import numpy as np
import pytest


def split_forward(x, L):
    """X (length L) of x zero-padded to L, computed as the two half-length transforms."""
    H = L // 2
    n = np.arange(H)
    xp = np.zeros(H, complex)
    xp[: x.size] = x
    X = np.empty(L, complex)
    for b in (0, 1):
        y = xp * np.exp(-2j * np.pi * n * b / L)
        X[b::2] = np.fft.fft(y)  # rows kz = 2 m + b of the tile
    return X


def split_inverse(X, L, nz):
    """The layers n < nz of the unnormalised inverse transform of X, computed as the two
    half-length inverse transforms (outputs 2 m + b)."""
    H = L // 2
    k = np.arange(H)
    out = np.empty(L, complex)
    for b in (0, 1):
        z = np.exp(2j * np.pi * b * k / L) * (X[:H] + (-1) ** b * X[H:])
        out[b::2] = np.fft.ifft(z) * H  # unnormalised: sum_k z[k] exp(+2 pi i m k / H)
    return out[:nz]


@pytest.mark.parametrize("L,nz", [(64, 32), (64, 17), (64, 1), (32, 16), (16, 5)])
def test_split_forward_equals_padded_fft(L, nz):
    rng = np.random.default_rng(L + nz)
    x = rng.standard_normal(nz) + 1j * rng.standard_normal(nz)
    xp = np.zeros(L, complex)
    xp[:nz] = x
    np.testing.assert_allclose(split_forward(x, L), np.fft.fft(xp), rtol=0, atol=1e-12 * np.abs(x).sum())


@pytest.mark.parametrize("L,nz", [(64, 32), (64, 20), (32, 16), (16, 8)])
def test_split_inverse_equals_padded_ifft(L, nz):
    rng = np.random.default_rng(7 * L + nz)
    X = rng.standard_normal(L) + 1j * rng.standard_normal(L)
    want = (np.fft.ifft(X) * L)[:nz]
    np.testing.assert_allclose(split_inverse(X, L, nz), want, rtol=0, atol=1e-12 * np.abs(X).sum())


def test_split_round_trip_is_the_circular_convolution():
    """forward, a pointwise product, inverse: the linear convolution of the z layers with
    a kernel placed circularly, as the matvec's z pass computes it per wavevector."""
    L, nz = 64, 32
    rng = np.random.default_rng(3)
    x = rng.standard_normal(nz) + 1j * rng.standard_normal(nz)
    kz = rng.standard_normal(2 * nz - 1) + 1j * rng.standard_normal(2 * nz - 1)  # offsets -(nz-1)..nz-1
    kc = np.zeros(L, complex)
    for d in range(-(nz - 1), nz):
        kc[d % L] = kz[d + nz - 1]
    got = split_inverse(split_forward(x, L) * np.fft.fft(kc), L, nz) / L
    want = np.array([sum(kz[(m - n) + nz - 1] * x[n] for n in range(nz)) for m in range(nz)])
    np.testing.assert_allclose(got, want, rtol=0, atol=1e-11 * np.abs(want).max())
