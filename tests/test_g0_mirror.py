"""CPU checks of the mirror symmetry the octant G0 build relies on (csrc/setup.cu k_g0_x,
k_g0_spatial_oct and the parity-mirrored strided passes, launch_fft_strided with an odd-entry
mask): reflecting the axes in f (bit 0 x, bit 1 y, bit 2 z) maps the spatial kernel at offset
r to S_f K(r) S_f at the reflected offset, with S_f = diag((-1)^popc(par_c & f)) and par_c the
DOF parities of csrc/mv_common.cuh (dof_parity). Checked on the oracle's spatial kernel
(slab_kernel_spatial, which follows the reference's D4h-orbit construction) for the point and
the volume-averaged propagators, and on the half-line mirror reconstruction the strided passes
use: a line stored for idx <= L/2 and read as s x[L - idx] beyond gives the full transform."""

import numpy as np
import pytest

from oracle import slab_oracle as O

# [u_z, u_x, u_y, e_zz, e_xx, e_yy, 2e_xy, 2e_zy, 2e_zx]: bit 0 odd under x -> -x, bit 1 under
# y -> -y, bit 2 under z -> -z
DOF_PARITY = np.array([4, 1, 2, 0, 0, 0, 3, 6, 5])


def _sign(f):
    return np.array([-1.0 if bin(int(p) & f).count("1") % 2 else 1.0 for p in DOF_PARITY])


@pytest.mark.parametrize("va", [False, True])
def test_spatial_kernel_mirror_parity(va):
    M, Nz = 5, 3
    ref_alpha, ref_beta, ref_rho = 3000.0, 1732.0, 2500.0
    omega = 0.4 * ref_beta / 1.0
    ker = O.slab_kernel_spatial(M, Nz, 1.0, omega, ref_alpha, ref_beta, ref_rho, volume_averaged=va)
    # index [k, ix, iy] holds offset (k - (Nz - 1), ix - (M - 1), iy - (M - 1))
    scale = np.abs(ker).max()
    for f in range(1, 8):
        s = _sign(f)
        refl = ker
        if f & 1:
            refl = refl[:, ::-1, :]
        if f & 2:
            refl = refl[:, :, ::-1]
        if f & 4:
            refl = refl[::-1, :, :]
        want = s[:, None] * ker * s[None, :]
        assert np.abs(refl - want).max() <= 1e-12 * scale, f


@pytest.mark.parametrize("L,odd", [(128, False), (128, True), (80, True), (15, False), (33, True)])
def test_half_line_mirror_reconstruction(L, odd):
    """A mirror-symmetric line x[L - n] = s x[n] stored for n <= L/2 only, the rest read
    through the sign (the strided pass's MIRROR load): the same transform as the full line."""
    rng = np.random.default_rng(L + odd)
    s = -1.0 if odd else 1.0
    h = L // 2 + 1
    half = rng.standard_normal(h) + 1j * rng.standard_normal(h)
    full = np.zeros(L, complex)
    full[:h] = half
    for n in range(h, L):
        full[n] = s * full[L - n]
    # the symmetric line itself: x[L - n] = s x[n] for 0 < n < L (the self-mirror points of an
    # odd line set to satisfy it)
    if L % 2 == 0 and odd:
        full[L // 2] = 0.0
    if odd:
        full[0] = 0.0
    rec = np.zeros(L, complex)
    rec[:h] = full[:h]
    for q in range(h, L):
        rec[q] = s * rec[L - q]
    assert np.allclose(np.fft.fft(rec), np.fft.fft(full), rtol=0, atol=1e-12 * np.abs(full).sum())
    # the transform keeps the parity, so the next pass may mirror its output the same way
    X = np.fft.fft(full)
    assert np.allclose(X[1:][::-1], s * X[1:], atol=1e-10 * np.abs(X).max())
