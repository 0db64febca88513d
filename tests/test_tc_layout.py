"""CPU restatement of the operand layout of the tensor-core near-field stencil
(multiplescatteringcalculations_b200/csrc/pc_tc.cu), checked against the oracle stencil.

The kernel never materialises the per-offset operands: it stages each halo plane of a
16 x 8 tile (18 x 10 voxels) as BF16 rows of 4 K chunks in the K-major no-swizzle layout
(row r at 16 r bytes, chunk c at c * 2880 bytes, 160 bytes between 8-row groups) and starts
one MMA descriptor per offset at a shifted row; DOF 8 of the y- and x-neighbour rows sits in
chunks 2-3 so that 6 MMAs cover its 27 taps. This test rebuilds the ring of planes, the
packed weight tiles and every MMA's operand gather exactly as the kernel addresses them (in
FP64, with unstaged bytes NaN), runs the layer-chunked schedule of the kernel (planes staged
into slot (p + 1) & 3, layer j reading planes j - 1 .. j + 1), and compares with the oracle.
It pins the index arithmetic; the GPU tests pin the kernel itself.
"""

import numpy as np
import pytest

from oracle import slab_oracle as O

TX, TY, HX, HY = 16, 8, 18, 10
PROWS = HX * HY
LBO_A, SBO_A = PROWS * 16, HY * 16
PLANE = 4 * LBO_A
BTILE, LBO_B = 1024, 512
PARITY = [4, 1, 2, 0, 0, 0, 3, 6, 5]


def _allowed(o, a, b):
    dz, dx, dy = o // 9 - 1, (o // 3) % 3 - 1, o % 3 - 1
    zm = int(dx == 0) | (int(dy == 0) << 1) | (int(dz == 0) << 2)
    return not ((PARITY[a] ^ PARITY[b]) & zm)


def _put(mem, t, n, kl, v):
    mem[(t * BTILE + ((kl // 8) * 4 + n // 8) * 128 + (n % 8) * 16 + (kl % 8) * 2) // 2] = v


def _put_block(mem, t, blocks, o, a, b, kre):
    if not _allowed(o, a, b):
        return
    g = blocks[o, a, b]
    _put(mem, t, 2 * a, kre, g.real)
    _put(mem, t, 2 * a, kre + 1, -g.imag)
    _put(mem, t, 2 * a + 1, kre, g.imag)
    _put(mem, t, 2 * a + 1, kre + 1, g.real)


def pack_layer(blocks):
    """The 33 weight tiles of a layer (the kernel's nf_tc_pack_layer), values in FP64."""
    mem = np.zeros(33 * BTILE // 2)
    for o in range(27):
        for a in range(9):
            for b in range(8):
                _put_block(mem, o, blocks, o, a, b, 2 * b)
    for dz in (-1, 0, 1):
        for part in range(2):
            for c in range(2 - part):
                dx = (1 if c == 0 else 0) if part == 0 else -1
                for e in range(3):
                    o = ((dz + 1) * 3 + dx + 1) * 3 + (1 - e) + 1
                    for a in range(9):
                        _put_block(mem, 27 + 2 * (dz + 1) + part, blocks, o, a, 8, 8 * c + 2 * e)
    return mem


def _gather(mem, start, rows, lbo, sbo):
    """Operand (rows x 16) read through a K-major no-swizzle descriptor."""
    m = np.arange(rows)[:, None]
    k = np.arange(16)[None, :]
    return mem[(start + (k // 8) * lbo + (m // 8) * sbo + (m % 8) * 16 + (k % 8) * 2) // 2]


def tc_layer(tau, blocks, M, Nz, sms=148):
    """One stencil layer y = sum_o G_o tau(. - o) through the kernel's layout and schedule."""
    B = pack_layer(blocks)
    nty, ntx = -(-M // TY), -(-M // TX)
    ncol = nty * ntx
    nzc = min(Nz, max(1, (2 * sms) // ncol))
    zc = -(-Nz // nzc)
    out = np.full((Nz, M, M, 9), np.nan, dtype=complex)
    hy, hx = np.arange(PROWS) % HY, np.arange(PROWS) // HY
    for bid in range(ncol * (-(-Nz // zc))):
        col, chunk = bid % ncol, bid // ncol
        y0, x0, z0 = (col % nty) * TY, (col // nty) * TX, chunk * zc
        czc = min(zc, Nz - z0)
        ring = np.full(4 * PLANE // 2, np.nan)

        def stage(slot, z):
            xx, yy = x0 + hx - 1, y0 + hy - 1
            ok = (0 <= z < Nz) & (xx >= 0) & (xx < M) & (yy >= 0) & (yy < M)
            v = np.zeros((PROWS, 9), dtype=complex)
            v[ok] = tau[z, xx[ok], yy[ok]] if 0 <= z < Nz else 0
            base = (slot * PLANE + np.arange(PROWS) * 16) // 2
            for b in range(8):
                c, e = b // 4, b % 4
                ring[base + c * LBO_A // 2 + 2 * e] = v[:, b].real
                ring[base + c * LBO_A // 2 + 2 * e + 1] = v[:, b].imag
            t8 = np.concatenate([v[:, 8], np.zeros(HY + 3, dtype=complex)])
            for c, off in ((2, 0), (3, HY)):
                for e in range(4):
                    val = t8[np.arange(PROWS) + off + e] if e < 3 else np.zeros(PROWS)
                    ring[base + c * LBO_A // 2 + 2 * e] = np.real(val)
                    ring[base + c * LBO_A // 2 + 2 * e + 1] = np.imag(val)

        for p in (-1, 0, 1):
            stage((p + 1) & 3, z0 + p)
        for j in range(czc):
            D = np.zeros((128, 32))
            for o in range(27):
                dz, dx, dy = o // 9 - 1, (o // 3) % 3 - 1, o % 3 - 1
                a0 = ((j - dz + 1) & 3) * PLANE + ((1 - dx) * HY + (1 - dy)) * 16
                D += _gather(ring, a0, 128, LBO_A, SBO_A) @ _gather(B, o * BTILE, 32, LBO_B, 128).T
            for dz in (-1, 0, 1):
                for part in range(2):
                    a0 = ((j - dz + 1) & 3) * PLANE + (2 * HY * 16 if part else 0) + 2 * LBO_A
                    t = 27 + 2 * (dz + 1) + part
                    D += _gather(ring, a0, 128, LBO_A, SBO_A) @ _gather(B, t * BTILE, 32, LBO_B, 128).T
            m = np.arange(128)
            xx, yy = x0 + (m >> 3), y0 + (m & 7)
            keep = (xx < M) & (yy < M)
            out[z0 + j, xx[keep], yy[keep]] = D[keep, 0:18:2] + 1j * D[keep, 1:18:2]
            if j + 2 <= czc:  # plane j + 2 into the slot the layer j - 1 released
                stage((j + 3) & 3, z0 + j + 2)
    return out


def _case(M, Nz, seed):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((Nz, M, M, 9)) + 1j * rng.standard_normal((Nz, M, M, 9))
    t4 = rng.standard_normal((4, Nz, M, M)) + 1j * rng.standard_normal((4, Nz, M, M))
    blocks = (rng.standard_normal((27, 9, 9)) + 1j * rng.standard_normal((27, 9, 9))) * O.nearfield_symmetry_mask()
    want = O.nearfield_stencil(x.ravel(), t4, blocks, M, Nz).reshape(Nz, M, M, 9)
    tau = O.apply_t0(t4, x).reshape(Nz, M, M, 9)
    return tau, blocks, want


def test_tc_layout_one_layer_per_block_ragged():
    M, Nz = 12, 5  # ragged against the 16 x 8 tile; 148 SMs give one layer per block
    tau, blocks, want = _case(M, Nz, 0)
    got = tc_layer(tau, blocks, M, Nz)
    assert not np.isnan(got).any()
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.parametrize("sms", [12, 1])
def test_tc_layout_several_layers_per_block(sms):
    """20 x 20 x 7: 6 tile columns; 12 SMs give chunks of 2, 2, 2, 1 layers per block, 1 SM
    one chunk of 7 layers (the 4-slot ring of planes wraps around)."""
    M, Nz = 20, 7
    tau, blocks, want = _case(M, Nz, 1)
    got = tc_layer(tau, blocks, M, Nz, sms=sms)
    assert not np.isnan(got).any()
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
