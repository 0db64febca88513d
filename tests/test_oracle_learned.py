"""The oracle's restatement of the learned near-field preconditioner's objective
and gradients (oracle/slab_oracle.py, section 9), pinned by finite differences and
by the adjoint identities it relies on. CPU only."""

import numpy as np

from oracle import slab_oracle as O

ALPHA, BETA, RHO = 3000.0, 1732.0, 2500.0


def _case(M=4, Nz=3, seed=0):
    om = 0.7 * BETA
    rng = np.random.default_rng(seed)
    dl, dm, dr = (rng.uniform(-0.2, 0.2, (Nz, M, M)) * s for s in (7.5e9, 7.5e9, 2500.0))
    t4 = O.t0_scalars(om, 1.0, ALPHA, BETA, RHO, dl, dm, dr)
    kh = O.build_slab_kernels(M, Nz, 1.0, om, ALPHA, BETA, RHO)
    blocks = O.nearfield_blocks(M, Nz, 1.0, om, ALPHA, BETA, RHO)
    return rng, t4, kh, blocks


def test_adjoints():
    M, Nz = 4, 3
    rng, t4, kh, blocks = _case(M, Nz)
    n = Nz * M * M * 9
    x, y = (rng.standard_normal(n) + 1j * rng.standard_normal(n) for _ in range(2))
    a = np.vdot(y, O.nearfield_stencil(x, t4, blocks, M, Nz))
    b = np.vdot(O.nearfield_stencil_adjoint(y, t4, blocks, M, Nz), x)
    assert abs(a - b) < 1e-12 * abs(a)
    # the slab operator's adjoint from the kernel's symmetries (reciprocity, mirror)
    a = np.vdot(y, O.slab_matvec(x, t4, kh, M, Nz))
    b = np.vdot(O.slab_operator_adjoint(y, t4, kh, M, Nz), x)
    assert abs(a - b) < 1e-5 * abs(a)


def test_residual_objective_gradients_by_finite_differences():
    M, Nz = 4, 3
    rng, t4, kh, blocks = _case(M, Nz, seed=1)
    n = Nz * M * M * 9
    coef = np.array([1.0, 0.9 + 0.1j, 0.7 - 0.2j])
    w = 0.05 * (rng.standard_normal((2, 27, 9, 9)) + 1j * rng.standard_normal((2, 27, 9, 9)))
    r = rng.standard_normal(n) + 1j * rng.standard_normal(n)

    def f(c, ww):
        return O.nearfield_residual_loss_grad(r, t4, kh, blocks, M, Nz, c, ww)

    L0, gc, gw = f(coef, w)
    h = 1e-6
    # dL/dconj(theta) = (dL/dRe + i dL/dIm) / 2
    for k in range(3):
        e = np.zeros(3, complex)
        e[k] = h
        fd = ((f(coef + e, w)[0] - f(coef - e, w)[0]) + 1j * (f(coef + 1j * e, w)[0] - f(coef - 1j * e, w)[0])) / (4 * h)
        assert abs(fd - gc[k]) < 1e-3 * abs(gc).max()
    mask = O.nearfield_symmetry_mask()
    for (l, o, a, b) in [(0, 4, 0, 0), (1, 13, 3, 4), (0, 22, 6, 6), (1, 0, 1, 7)]:
        assert mask[o, a, b]
        e = np.zeros_like(w)
        e[l, o, a, b] = h
        fd = ((f(coef, w + e)[0] - f(coef, w - e)[0]) + 1j * (f(coef, w + 1j * e)[0] - f(coef, w - 1j * e)[0])) / (4 * h)
        assert abs(fd - gw[l, o, a, b]) < 1e-3 * abs(gw).max()
    assert np.all(gw[:, ~mask] == 0)
