"""CPU oracle for the slab Foldy-Lax solve ``(I - G0 T0) psi = psi0``.

TEST INFRASTRUCTURE ONLY. This module is the checker, never the product: only
``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import it. The shipped package never imports, links or executes
anything under ``oracle/``.

It restates, in vectorised numpy/scipy FP64, the reference's CPU path
(tmnestor/MultipleScatteringCalculations, ``cubic_scattering/``). Each function
cites the reference file:line it follows. Conventions are the reference's:
axis order (z, x, y) with z down, 9 DOF per voxel
[u_z, u_x, u_y, e_zz, e_xx, e_yy, 2e_xy, 2e_zy, 2e_zx], field layout
``psi[N_z, M, M, 9]``, ``a`` is the cube half-width (d = 2a).

Parity of this restatement with the reference itself is pinned by the golden
fixtures in ``tests/golden/`` (generated by ``tests/golden/make_golden.py``,
which imports the reference where it is available) and checked by
``tests/test_oracle_golden.py``.

Additions that the reference does not have (clearly marked): a Bloch-phased
periodic fold (the reference folds without phase, ``slab_scattering.py:337-346``)
and the matching demodulated R_PP.
"""

from __future__ import annotations

from math import factorial

import numpy as np
from scipy.sparse.linalg import LinearOperator, gmres

from . import va_tables as _va

N_TAYLOR = 8
# g0 = int_{[-1,1]^3} 1/|x| d^3x, written with the Pell identity as the
# reference does (effective_contrasts.py:104-105).
G0_CUBE = (4.0 / 3.0) * np.log(70226 + 40545 * np.sqrt(3.0)) - 2.0 * np.pi

# Voigt index -> Cartesian pair, (z=0, x=1, y=2) (resonance_tmatrix.py:141-148)
VOIGT_PAIRS = [(0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1)]


# ---------------------------------------------------------------------------
# 1. Per-voxel T0 (effective_contrasts.py:112-532, resonance_tmatrix.py:461-487)
# ---------------------------------------------------------------------------


def _taylor_coefficients(omega, alpha, beta, rho, n_taylor=N_TAYLOR):
    """phi_n, psi_n of the smooth Green's tensor (effective_contrasts.py:153-191)."""
    ikb = 1j * omega / beta
    ika = 1j * omega / alpha
    cf = 1.0 / (4.0 * np.pi * rho * beta**2)
    cg = 1.0 / (4.0 * np.pi * rho)
    n = np.arange(n_taylor)
    phi = np.array([ikb ** (2 * k + 1) / factorial(2 * k + 1) * cf for k in n])
    psi = np.array(
        [cg * (ika ** (2 * k + 3) / alpha**2 - ikb ** (2 * k + 3) / beta**2) / factorial(2 * k + 3) for k in n]
    )
    return phi, psi


def _cube_moments(a, n_max):
    """Monomial moments S0, S1, S2, S11 of [-a,a]^3 (effective_contrasts.py:194-234)."""
    mu = np.array([2.0 * a ** (2 * k + 1) / (2 * k + 1) for k in range(n_max + 3)])
    S0 = np.zeros(n_max + 1)
    S1 = np.zeros(n_max + 1)
    S2 = np.zeros(n_max + 1)
    S11 = np.zeros(n_max + 1)
    for m in range(n_max + 1):
        for p in range(m + 1):
            for q in range(m - p + 1):
                r = m - p - q
                c = factorial(m) / (factorial(p) * factorial(q) * factorial(r))
                S0[m] += c * mu[p] * mu[q] * mu[r]
                S1[m] += c * mu[p + 1] * mu[q] * mu[r]
                S2[m] += c * mu[p + 2] * mu[q] * mu[r]
                S11[m] += c * mu[p + 1] * mu[q + 1] * mu[r]
    return S0, S1, S2, S11


def cube_frequency_constants(omega, a, alpha, beta, rho, n_taylor=N_TAYLOR):
    """Gamma0, A^c, B^c, C^c of the cube (contrast independent).

    Gamma0: effective_contrasts.py:112-145; static Eshelby :237-275;
    smooth A/B/C :278-330.
    """
    a0 = (alpha**2 + beta**2) / (8.0 * np.pi * rho * alpha**2 * beta**2)
    b0 = (alpha**2 - beta**2) / (8.0 * np.pi * rho * alpha**2 * beta**2)
    phi, psi = _taylor_coefficients(omega, alpha, beta, rho, n_taylor)
    S0, S1, S2, S11 = _cube_moments(a, n_taylor - 1)
    N = n_taylor
    gamma0 = a**2 * (a0 + b0 / 3.0) * G0_CUBE + complex(np.sum(phi * S0[:N]) + np.sum(psi * S1[:N]))

    s3 = np.sqrt(3.0)
    j1 = 2.0 * np.pi / 3.0
    j2 = -2.0 * (s3 - np.pi) / 9.0
    k1 = 2.0 * (2.0 * s3 + np.pi) / 9.0
    A_stat = 2.0 * (-a0 * j1 - 3.0 * b0 * j2)
    B_stat = 2.0 * b0 * (j1 - 3.0 * j2)
    C_stat = 6.0 * b0 * (3.0 * j2 - k1)

    n = np.arange(N)
    n2 = n[2:]
    n1 = n[1:]
    A_s = (
        np.sum(4 * n2 * (n2 - 1) * phi[2:] * S1[: N - 2])
        + np.sum(4 * n2 * (n2 - 1) * psi[2:] * S11[: N - 2])
        + np.sum(2 * n1 * phi[1:] * S0[: N - 1])
        + np.sum(2 * n1 * psi[1:] * S1[: N - 1])
    )
    B_s = (
        np.sum(psi * S0[:N])
        + np.sum(4 * n1 * psi[1:] * S1[: N - 1])
        + np.sum(4 * n2 * (n2 - 1) * psi[2:] * S11[: N - 2])
    )
    C_s = np.sum(4 * n2 * (n2 - 1) * psi[2:] * (S2[: N - 2] - 3 * S11[: N - 2]))
    return complex(gamma0), complex(A_stat + A_s), complex(B_stat + B_s), complex(C_stat + C_s)


def t0_scalars(omega, a, alpha, beta, rho, dlam, dmu, drho):
    """The 4 complex scalars of T0 per voxel: (t_u, t_l, t_d, t_s).

    T0 = diag(t_u I3, [[t_l + t_d on the diagonal, t_l off it] for the normal
    strains], t_s I3 for the engineering shears), which is
    ``_sub_cell_tmatrix_9x9`` (resonance_tmatrix.py:461-487) of
    ``compute_cube_tmatrix`` (effective_contrasts.py:454-532) with the Voigt
    stiffness of voigt_tmatrix.py:131-169. T1/T2/T3 are the closed form of
    ``_compute_T123`` (effective_contrasts.py:338-378):
    T1 = dlam(A+4B+C) + 2B dmu, T2 = dmu(A+B), T3 = 2C dmu.
    """
    g0, A, B, C = cube_frequency_constants(omega, a, alpha, beta, rho)
    dlam = np.asarray(dlam, dtype=float)
    dmu = np.asarray(dmu, dtype=float)
    drho = np.asarray(drho, dtype=float)
    T1 = dlam * (A + 4.0 * B + C) + 2.0 * B * dmu
    T2 = dmu * (A + B)
    T3 = 2.0 * C * dmu
    amp_u = 1.0 / (1.0 - omega**2 * drho * g0)
    amp_th = 1.0 / (1.0 - 3.0 * T1 - 2.0 * T2 - T3)
    amp_off = 1.0 / (1.0 - 2.0 * T2)
    amp_diag = 1.0 / (1.0 - 2.0 * T2 - T3)
    drho_s = drho * amp_u
    dmu_off = dmu * amp_off
    dmu_diag = dmu * amp_diag
    dlam_s = (dlam + 2.0 / 3.0 * dmu) * amp_th - 2.0 / 3.0 * dmu * amp_diag
    V = (2.0 * a) ** 3
    return np.stack([omega**2 * drho_s * V, V * dlam_s, V * 2.0 * dmu_diag, V * 2.0 * dmu_off])


def t0_full(t4):
    """Expand (4, ...) scalars to the reference's (..., 9, 9) T-matrices
    (compute_slab_tmatrices, slab_scattering.py:169-205)."""
    t_u, t_l, t_d, t_s = t4
    shp = t_u.shape
    T = np.zeros(shp + (9, 9), dtype=complex)
    for i in range(3):
        T[..., i, i] = t_u
        T[..., 6 + i, 6 + i] = t_s
        for j in range(3):
            T[..., 3 + i, 3 + j] = t_l + (t_d if i == j else 0.0)
    return T


def apply_t0(t4, psi):
    """tau = T0 psi for psi (..., 9) using the 4-scalar form."""
    t_u, t_l, t_d, t_s = t4
    tau = np.empty_like(psi)
    tau[..., 0:3] = t_u[..., None] * psi[..., 0:3]
    tr = psi[..., 3] + psi[..., 4] + psi[..., 5]
    tau[..., 3:6] = t_l[..., None] * tr[..., None] + t_d[..., None] * psi[..., 3:6]
    tau[..., 6:9] = t_s[..., None] * psi[..., 6:9]
    return tau


# ---------------------------------------------------------------------------
# 2. Point 9x9 propagator (resonance_tmatrix.py:214-428), vectorised over r
# ---------------------------------------------------------------------------

_PHI_TERMS = ((2, "S", -1), (1, "S", -2), (0, "S", -3), (1, "P", -2), (0, "P", -3))
_PSI_TERMS = ((2, "S", -1), (1, "S", -2), (0, "S", -3), (2, "P", -1), (1, "P", -2), (0, "P", -3))


def _radial_functions(r, kP, kS):
    """phi, psi and their first two radial derivatives (resonance_tmatrix.py:214-271)."""
    coef_phi = [kS**2, 1j * kS, -1.0, -1j * kP, 1.0]
    coef_psi = [-(kS**2), -3j * kS, 3.0, kP**2, 3j * kP, -3.0]
    waves = {"S": (kS, np.exp(1j * kS * r)), "P": (kP, np.exp(1j * kP * r))}
    out = []
    for coefs, terms in ((coef_phi, _PHI_TERMS), (coef_psi, _PSI_TERMS)):
        f = np.zeros_like(r, dtype=complex)
        fp = np.zeros_like(f)
        fpp = np.zeros_like(f)
        for c, (_, w, p) in zip(coefs, terms):
            k, e = waves[w]
            ikr = 1j * k * r
            f += c * e * r**p
            fp += c * e * r ** (p - 1) * (ikr + p)
            fpp += c * e * r ** (p - 2) * (ikr**2 + 2 * p * ikr + p * (p - 1))
        out.append((f, fp, fpp))
    (phi, phi_p, phi_pp), (psi, psi_p, psi_pp) = out
    return phi, psi, phi_p, psi_p, phi_pp, psi_pp


def point_propagator(rvec, omega, alpha, beta, rho):
    """9x9 [[G, C], [H, S]] at separation(s) ``rvec`` (..., 3); zero at r = 0.

    G, dG, ddG: resonance_tmatrix.py:274-350; Voigt contraction with the
    engineering-shear column halving: :353-409; block: :412-428.
    """
    rvec = np.asarray(rvec, dtype=float)
    shp = rvec.shape[:-1]
    rv = rvec.reshape(-1, 3)
    r = np.linalg.norm(rv, axis=1)
    out = np.zeros((rv.shape[0], 9, 9), dtype=complex)
    ok = r >= 1.0e-14
    if not np.any(ok):
        return out.reshape(shp + (9, 9))
    rr = r[ok]
    g = rv[ok] / rr[:, None]
    kP = omega / alpha
    kS = omega / beta
    P = 1.0 / (4.0 * np.pi * rho * omega**2)
    phi, psi, phi_p, psi_p, phi_pp, psi_pp = _radial_functions(rr, kP, kS)
    d = np.eye(3)
    G = P * (phi[:, None, None] * d + psi[:, None, None] * np.einsum("ni,nj->nij", g, g))
    c1 = phi_p
    c2 = psi_p - 2.0 * psi / rr
    c3 = psi / rr
    Gd = P * (
        c1[:, None, None, None] * np.einsum("nk,ij->nijk", g, d)
        + c2[:, None, None, None] * np.einsum("ni,nj,nk->nijk", g, g, g)
        + c3[:, None, None, None] * (np.einsum("ik,nj->nijk", d, g) + np.einsum("jk,ni->nijk", d, g))
    )
    t1 = phi_p / rr
    t2 = phi_pp - phi_p / rr
    t3 = psi_p / rr - 2.0 * psi / rr**2
    t4 = psi / rr**2
    t7 = psi_pp - 5.0 * psi_p / rr + 8.0 * psi / rr**2
    e = lambda x: x[:, None, None, None, None]  # noqa: E731
    dd = np.einsum("ij,kl->ijkl", d, d)
    Gdd = P * (
        e(t1) * dd
        + e(t2) * np.einsum("ij,nk,nl->nijkl", d, g, g)
        + e(t3) * np.einsum("ni,nj,kl->nijkl", g, g, d)
        + e(t4) * (np.einsum("ik,jl->ijkl", d, d) + np.einsum("jk,il->ijkl", d, d))
        + e(t3) * (np.einsum("il,nj,nk->nijkl", d, g, g) + np.einsum("jl,ni,nk->nijkl", d, g, g))
        + e(t3) * (np.einsum("ik,nj,nl->nijkl", d, g, g) + np.einsum("jk,ni,nl->nijkl", d, g, g))
        + e(t7) * np.einsum("ni,nj,nk,nl->nijkl", g, g, g, g)
    )
    blk = np.zeros((rr.shape[0], 9, 9), dtype=complex)
    blk[:, :3, :3] = G
    for al, (p, q) in enumerate(VOIGT_PAIRS):
        if p == q:
            blk[:, :3, 3 + al] = Gd[:, :, p, p]
            blk[:, 3 + al, :3] = Gd[:, p, :, p]
        else:
            blk[:, :3, 3 + al] = Gd[:, :, p, q] + Gd[:, :, q, p]
            blk[:, 3 + al, :3] = Gd[:, p, :, q] + Gd[:, q, :, p]
        for be, (m, n) in enumerate(VOIGT_PAIRS):
            if p == q and m == n:
                v = Gdd[:, p, m, m, p]
            elif p == q:
                v = Gdd[:, p, m, n, p] + Gdd[:, p, n, m, p]
            elif m == n:
                v = Gdd[:, p, m, m, q] + Gdd[:, q, m, m, p]
            else:
                v = Gdd[:, p, m, n, q] + Gdd[:, p, n, m, q] + Gdd[:, q, m, n, p] + Gdd[:, q, n, m, p]
            blk[:, 3 + al, 3 + be] = v
    blk[:, :, 6:9] *= 0.5  # halve the shear columns of C and S (:404-407)
    out[ok] = blk
    return out.reshape(shp + (9, 9))


# ---------------------------------------------------------------------------
# 3. Volume-averaged nearest-neighbour 9x9 (inter_voxel_propagator.py)
# ---------------------------------------------------------------------------


def _sym_from_counts(vals, combos, rank):
    """Fully symmetric tensor from values indexed by index-count multisets."""
    import itertools

    T = np.zeros((3,) * rank)
    for v, c in zip(vals, combos):
        base = (0,) * c[0] + (1,) * c[1] + (2,) * c[2]
        for perm in set(itertools.permutations(base)):
            T[perm] = v
    return T


def _A_matrix(v6):
    A = np.diag(v6[:3]).astype(float)
    A[0, 1] = A[1, 0] = v6[3]
    A[0, 2] = A[2, 0] = v6[4]
    A[1, 2] = A[2, 1] = v6[5]
    return A


def _assemble_P(A, B, mu, eta):
    """P_ijkl = -1/(2 mu) [d_ik A_jl + d_jk A_il - 2 eta B_ijkl] (inter_voxel_propagator.py:392-413)."""
    d = np.eye(3)
    return -1.0 / (2.0 * mu) * (np.einsum("ik,jl->ijkl", d, A) + np.einsum("jk,il->ijkl", d, A) - 2.0 * eta * B)


def _oh_permutation(source, target):
    """Signed permutation P with P @ source = target, greedy matching as in
    inter_voxel_propagator.py:734-760 (so the chosen representative agrees)."""
    P = np.zeros((3, 3))
    used = [False, False, False]
    for i in range(3):
        for j in range(3):
            if not used[j] and abs(abs(target[i]) - abs(source[j])) < 1e-10 and abs(source[j]) > 1e-10:
                P[i, j] = np.sign(target[i]) * np.sign(source[j])
                used[j] = True
                break
            if not used[j] and abs(source[j]) < 1e-10 and abs(target[i]) < 1e-10:
                P[i, j] = 1.0
                used[j] = True
                break
    return P


def _p_to_voigt_s(P):
    """(3,3,3,3) -> (6,6) Voigt S with shear-column halving (inter_voxel_propagator.py:834-856)."""
    S = np.zeros((6, 6), dtype=P.dtype)
    for al, (p, q) in enumerate(VOIGT_PAIRS):
        mult = 2 if p != q else 1
        for be, (m, n) in enumerate(VOIGT_PAIRS):
            v = mult * P[p, q, m, n]
            if m != n:
                v += mult * P[p, q, n, m]
            S[al, be] = v
    S[:, 3:] *= 0.5
    return S


_VA_TYPES = {
    "face": (np.array([1.0, 0, 0]), "FACE"),
    "edge": (np.array([1.0, 1.0, 0]), "EDGE"),
    "corner": (np.array([1.0, 1.0, 1.0]), "CORNER"),
}


def va_propagator(R, alpha, beta, rho, omega, n_orders=2):
    """Volume-averaged NN 9x9 at integer lattice offset R = (dz, dx, dy).

    inter_voxel_propagator_9x9 (inter_voxel_propagator.py:1295-1355): S block
    from the dynamic strain propagator (:791-823, orders <= 3), G block from
    ``_build_G_block_canonical`` (:985-1057), C from ``_build_dG_rank3_canonical``
    (:1192-1269) and H = C^T. Real valued; the constants assume the unit cube.
    """
    n_abs = sorted(abs(int(x)) for x in R)[::-1]
    kind = {(1, 0, 0): "face", (1, 1, 0): "edge", (1, 1, 1): "corner"}[tuple(n_abs)]
    canon, tag = _VA_TYPES[kind]
    perm = _oh_permutation(canon, np.array(R, dtype=float))
    tA = getattr(_va, tag + "_A")
    tB = getattr(_va, tag + "_B")
    tD2 = getattr(_va, tag + "_D2W")
    tD3 = getattr(_va, tag + "_D3")
    tDW = getattr(_va, tag + "_DW")
    cs, cp = beta, alpha
    mu = rho * beta**2
    nu = (alpha**2 - 2.0 * beta**2) / (2.0 * (alpha**2 - beta**2))
    no = min(n_orders, 3)
    # S block: static + sum_n omega^(2n) P^(n), each rotated (:611-643, :791-823)
    Pc = _assemble_P(_A_matrix(tA[0]), _sym_from_counts(tB[0], _va.COMBOS4, 4), mu, 1.0 / (2.0 * (1.0 - nu)))
    Pt = np.einsum("ia,jb,kc,ld,abcd->ijkl", perm, perm, perm, perm, Pc)
    for n in range(1, no + 1):
        mu_n = rho * cs ** (2 * n + 2)
        eta_n = 1.0 - (cs / cp) ** (2 * n + 2)
        Pn = _assemble_P(_A_matrix(tA[n]), _sym_from_counts(tB[n], _va.COMBOS4, 4), mu_n, eta_n)
        Pt = Pt + omega ** (2 * n) * np.einsum("ia,jb,kc,ld,abcd->ijkl", perm, perm, perm, perm, Pn)
    S = _p_to_voigt_s(Pt)
    # G block (:985-1057)
    d = np.eye(3)
    D2 = _A_matrix(tD2[0])
    G = (1.0 / (4.0 * np.pi * mu)) * (d * 0.5 * np.trace(D2) - D2 / (4.0 * (1.0 - nu)))
    g_coef = [None, -(omega**2) / (8.0 * np.pi * rho * cs**4), omega**4 / (96.0 * np.pi * rho * cs**6),
              -(omega**6) / (2880.0 * np.pi * rho * cs**8)]
    lap = [None, 12.0, 30.0, 56.0]
    for n in range(1, no + 1):
        D2 = _A_matrix(tD2[n])
        eta_n = 1.0 - (cs / cp) ** (2 * n + 2)
        G = G + g_coef[n] * (d * np.trace(D2) / lap[n] - (eta_n / lap[n]) * D2)
    G = perm @ G @ perm.T
    # dG rank-3 (:1192-1269); the omega terms are skipped when omega == 0
    D3 = _sym_from_counts(tD3[0], _va.COMBOS3, 3)
    dG = (1.0 / (4.0 * np.pi * mu)) * (np.einsum("ij,k->ijk", d, np.array(tDW[0])) - D3 / (4.0 * (1.0 - nu)))
    if omega != 0.0:
        for n in range(1, no + 1):
            D3 = _sym_from_counts(tD3[n], _va.COMBOS3, 3)
            eta_n = 1.0 - (cs / cp) ** (2 * n + 2)
            dG = dG + g_coef[n] * (np.einsum("ij,k->ijk", d, np.array(tDW[n])) - (eta_n / lap[n]) * D3)
    dG = np.einsum("ia,jb,kc,abc->ijk", perm, perm, perm, dG)
    C = np.zeros((3, 6))
    for al, (m, n) in enumerate(VOIGT_PAIRS):
        C[:, al] = dG[:, m, m] if m == n else 0.5 * (dG[:, m, n] + dG[:, n, m])
    P9 = np.zeros((9, 9), dtype=complex)
    P9[:3, :3] = G
    P9[:3, 3:] = C
    P9[3:, :3] = C.T
    P9[3:, 3:] = S
    return P9


# ---------------------------------------------------------------------------
# 4. D4h orbit and the slab kernel (slab_scattering.py:211-351, lattice_greens.py:521-566)
# ---------------------------------------------------------------------------


def _d4h_matrices():
    rx = np.diag([1.0, -1, 1, 1, 1, 1, -1, 1, -1])
    ry = np.diag([1.0, 1, -1, 1, 1, 1, -1, -1, 1])
    p = np.zeros((9, 9))
    p[0, 0] = p[1, 2] = p[2, 1] = 1.0
    p[3, 3] = p[4, 5] = p[5, 4] = p[6, 6] = p[7, 8] = p[8, 7] = 1.0
    return rx, ry, p


_RX, _RY, _P90 = _d4h_matrices()


def _orbit(dx, dy):
    """D4h images (sdx, sdy, R9) of the fundamental offset (slab_scattering.py:233-259)."""
    I = np.eye(9)
    if dx == 0 and dy == 0:
        return [(0, 0, I)]
    base = [(dx, dy, I), (-dx, dy, _RX), (dx, -dy, _RY), (-dx, -dy, _RX @ _RY)]
    if dx == dy:
        return base
    return base + [(dy, dx, _P90), (-dy, dx, _RX @ _P90), (dy, -dx, _RY @ _P90), (-dy, -dx, _RX @ _RY @ _P90)]


def slab_kernel_spatial(M, N_z, a, omega, alpha, beta, rho, *, volume_averaged=False, n_orders=2):
    """Spatial kernel on the (2N_z-1, 2M-1, 2M-1) offset window, self term zero.

    Follows ``_build_slab_kernels`` (slab_scattering.py:303-335): the point
    propagator is evaluated on the fundamental domain 0 <= dy <= dx < M and
    expanded by the D4h orbit R P R^T; nearest neighbours (max |offset| <= 1)
    use the volume-averaged propagator at each signed offset when enabled.
    Index [k, ix, iy] holds offset (k-(N_z-1), ix-(M-1), iy-(M-1)). The orbit
    operations are applied in the reference's order (slab_scattering.py:241-259),
    vectorised over the fundamental points, so where two images of one point
    coincide the later operation wins, as in the reference loop.
    """
    d = 2.0 * a
    S = 2 * M - 1
    n_dz = 2 * N_z - 1
    ker = np.zeros((n_dz, S, S, 9, 9), dtype=complex)
    fd = np.array([(dx, dy) for dx in range(M) for dy in range(dx + 1)], dtype=int)
    I9 = np.eye(9)
    # (target offset as a function of (dx, dy), 9x9 transform, which points take part)
    ops = [
        (lambda x, y: (x, y), I9, "all"),
        (lambda x, y: (-x, y), _RX, "nz"),
        (lambda x, y: (x, -y), _RY, "nz"),
        (lambda x, y: (-x, -y), _RX @ _RY, "nz"),
        (lambda x, y: (y, x), _P90, "off"),
        (lambda x, y: (-y, x), _RX @ _P90, "off"),
        (lambda x, y: (y, -x), _RY @ _P90, "off"),
        (lambda x, y: (-y, -x), _RX @ _RY @ _P90, "off"),
    ]
    for k in range(n_dz):
        dz = k - (N_z - 1)
        keep = ~((fd[:, 0] == 0) & (fd[:, 1] == 0) & (dz == 0))
        pts = fd[keep]
        if pts.size == 0:
            continue
        r = np.stack([np.full(len(pts), dz * d), pts[:, 0] * d, pts[:, 1] * d], axis=1)
        blocks = point_propagator(r, omega, alpha, beta, rho)
        nn = np.maximum(abs(dz), np.maximum(pts[:, 0], pts[:, 1])) <= 1
        zero = (pts[:, 0] == 0) & (pts[:, 1] == 0)
        diag = pts[:, 0] == pts[:, 1]
        for tgt, R9, which in ops:
            sel = np.ones(len(pts), bool) if which == "all" else (~zero if which == "nz" else ~diag)
            if volume_averaged:
                sel = sel & ~nn
            if not np.any(sel):
                continue
            tx, ty = tgt(pts[sel, 0], pts[sel, 1])
            ker[k, tx + M - 1, ty + M - 1] = np.einsum("ab,nbc,dc->nad", R9, blocks[sel], R9)
        if volume_averaged:
            for dx, dy in pts[nn]:
                for sdx, sdy, _ in _orbit(int(dx), int(dy)):
                    ker[k, sdx + M - 1, sdy + M - 1] = va_propagator((dz, sdx, sdy), alpha, beta, rho, omega,
                                                                     n_orders)
    return ker


def fold_periodic(ker, M, phase_xy=None):
    """Fold the (.., 2M-1, 2M-1, ..) window onto M x M (slab_scattering.py:337-346).

    ``phase_xy`` is an addition of this build (the Bloch-phased fold): when
    given as (kx d, ky d) the offset (dx, dy) is weighted by
    exp(-i (kx dx + ky dy) d) before folding, which is the circulant kernel of
    the demodulated field psi e^{-i k_par . x}. ``None`` is the reference fold.
    """
    S = 2 * M - 1
    out = np.zeros(ker.shape[:1] + (M, M) + ker.shape[3:], dtype=complex)
    for ix in range(S):
        for iy in range(S):
            dx, dy = ix - (M - 1), iy - (M - 1)
            w = 1.0 if phase_xy is None else np.exp(-1j * (phase_xy[0] * dx + phase_xy[1] * dy))
            out[:, dx % M, dy % M] += w * ker[:, ix, iy]
    return out


def build_slab_kernels(M, N_z, a, omega, alpha, beta, rho, *, volume_averaged=False, n_orders=2, periodic=False,
                       phase_xy=None):
    """xy-FFT'd kernels (2N_z-1, H, H, 9, 9), H = M if periodic else 2M-1
    (``_build_slab_kernels``, slab_scattering.py:267-351)."""
    ker = slab_kernel_spatial(M, N_z, a, omega, alpha, beta, rho, volume_averaged=volume_averaged, n_orders=n_orders)
    if periodic:
        ker = fold_periodic(ker, M, phase_xy)
    return np.fft.fft2(ker, axes=(1, 2))


# ---------------------------------------------------------------------------
# 5. Matvec (slab_scattering.py:359-418) and the dense direct operator
# ---------------------------------------------------------------------------


def slab_matvec(psi_flat, T_local, kernel_hat, M, N_z, *, periodic=False, threads=1):
    """(I - G T) psi by 2D FFT per layer and the O(N_z^2) layer-pair sum.

    ``T_local`` is either the (N_z,M,M,9,9) matrices or the (4,N_z,M,M) scalars.
    ``threads`` > 1 runs the FFTs with scipy.fft workers and the output layers of
    the layer-pair sum in a thread pool (the same arithmetic, for CPU timing).
    """
    psi = psi_flat.reshape(N_z, M, M, 9)
    if T_local.ndim == 4 and T_local.shape[0] == 4:
        tau = apply_t0(T_local, psi)
    else:
        tau = np.einsum("lmnab,lmnb->lmna", T_local, psi)
    fft2, ifft2 = np.fft.fft2, np.fft.ifft2
    if threads > 1:
        import scipy.fft as sfft

        fft2 = lambda x, axes: sfft.fft2(x, axes=axes, workers=threads)  # noqa: E731
        ifft2 = lambda x, axes: sfft.ifft2(x, axes=axes, workers=threads)  # noqa: E731
    if periodic:
        H = M
        tau_hat = fft2(tau, axes=(1, 2))
    else:
        H = 2 * M - 1
        pad = np.zeros((N_z, H, H, 9), dtype=complex)
        pad[:, :M, :M] = tau
        tau_hat = fft2(pad, axes=(1, 2))
    acc = np.zeros((N_z, H, H, 9), dtype=complex)

    def layer(m):
        for n in range(N_z):
            acc[m] += np.einsum("xyij,xyj->xyi", kernel_hat[m - n + N_z - 1], tau_hat[n])

    if threads > 1:
        from concurrent.futures import ThreadPoolExecutor

        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(layer, range(N_z)))
    else:
        for m in range(N_z):
            layer(m)
    acc = ifft2(acc, axes=(1, 2))
    if not periodic:
        acc = acc[:, M - 1 :, M - 1 :]
    return (psi - acc).ravel()


def all_centres(M, N_z, a):
    """Cube centres (N_z, M, M, 3) in (z, x, y) (slab_scattering.py:90-99)."""
    d = 2.0 * a
    z = (np.arange(N_z) + 0.5) * d
    x = (np.arange(M) - (M - 1) / 2.0) * d
    zz, xx, yy = np.meshgrid(z, x, x, indexing="ij")
    return np.stack([zz, xx, yy], axis=-1)


def dense_operator(M, N_z, a, omega, alpha, beta, rho, T_local):
    """Assembled (I - P T) for small lattices (tests/test_slab_scattering.py:223-244)."""
    c = all_centres(M, N_z, a).reshape(-1, 3)
    n = c.shape[0]
    rv = c[:, None, :] - c[None, :, :]
    P = point_propagator(rv, omega, alpha, beta, rho)  # zero on the diagonal
    if T_local.ndim == 4 and T_local.shape[0] == 4:
        T = t0_full(T_local).reshape(n, 9, 9)
    else:
        T = T_local.reshape(n, 9, 9)
    PT = np.einsum("ijab,jbc->iajc", P, T).reshape(9 * n, 9 * n)
    return np.eye(9 * n) - PT


# ---------------------------------------------------------------------------
# 6. Incident plane wave (slab_scattering.py:426-478, sphere_scattering.py:1256-1287)
# ---------------------------------------------------------------------------


def polarisation(k_hat, wave_type):
    """Unit propagation, polarisation and which speed (slab_scattering.py:446-464)."""
    k_hat = np.asarray(k_hat, dtype=float)
    k_hat = k_hat / np.linalg.norm(k_hat)
    if wave_type == "P":
        return k_hat, k_hat.copy(), "P"
    if wave_type == "S":
        cross = np.cross(k_hat, np.array([1.0, 0.0, 0.0]))
        if np.linalg.norm(cross) < 1e-10:
            pol = np.array([0.0, 1.0, 0.0])
        else:
            pol = np.cross(cross, k_hat)
            pol = pol / np.linalg.norm(pol)
        return k_hat, pol, "S"
    raise ValueError(f"wave_type must be 'P' or 'S', got '{wave_type}'")


def incident_vector(k_hat, pol, k):
    """[pol, Voigt strain of the plane wave] (sphere_scattering.py:1256-1287)."""
    eps = 0.5j * k * (np.outer(k_hat, pol) + np.outer(pol, k_hat))
    v = np.zeros(9, dtype=complex)
    v[:3] = pol
    for i, (p, q) in enumerate(VOIGT_PAIRS):
        v[3 + i] = eps[p, q] if p == q else 2.0 * eps[p, q]
    return v


def incident_field(M, N_z, a, omega, alpha, beta, k_hat, wave_type):
    """psi0 (N_z, M, M, 9) (``_build_slab_incident_field``, slab_scattering.py:426-478)."""
    kh, pol, w = polarisation(k_hat, wave_type)
    k = omega / (alpha if w == "P" else beta)
    v = incident_vector(kh, pol, k)
    ph = np.exp(1j * k * np.einsum("k,lmnk->lmn", kh, all_centres(M, N_z, a)))
    return v[None, None, None, :] * ph[..., None]


# ---------------------------------------------------------------------------
# 7. Solve (slab_scattering.py:486-565)
# ---------------------------------------------------------------------------


def solve(M, N_z, a, alpha, beta, rho, dlam, dmu, drho, omega, k_hat, wave_type="P", gmres_tol=1e-6, max_iter=500,
          *, volume_averaged=False, n_orders=2, periodic=False, restart=20, phase_xy=None, threads=1, timings=None):
    """scipy GMRES on the FFT operator with x0 = psi0, as ``compute_slab_scattering``.

    ``restart=20`` is scipy's default that the reference call uses
    (slab_scattering.py:542). Returns a dict with psi, psi0, t4, n_matvec
    (including the final residual matvec, as the reference counts it) and the
    true relative residual.
    """
    import time

    t_0 = time.perf_counter()
    t4 = t0_scalars(omega, a, alpha, beta, rho, dlam, dmu, drho)
    t_1 = time.perf_counter()
    kh = build_slab_kernels(M, N_z, a, omega, alpha, beta, rho, volume_averaged=volume_averaged, n_orders=n_orders,
                            periodic=periodic, phase_xy=phase_xy)
    t_2 = time.perf_counter()
    psi0 = incident_field(M, N_z, a, omega, alpha, beta, k_hat, wave_type)
    b = psi0.ravel()
    if phase_xy is not None:
        b = (psi0 * bloch_demodulation(M, N_z, a, phase_xy)[..., None]).ravel()
    n = b.size
    cnt = [0]

    def mv(x):
        cnt[0] += 1
        return slab_matvec(x, t4, kh, M, N_z, periodic=periodic, threads=threads)

    A = LinearOperator((n, n), matvec=mv, dtype=complex)
    t_3 = time.perf_counter()
    x, info = gmres(A, b, x0=b.copy(), rtol=gmres_tol, maxiter=max_iter, restart=restart)
    res = np.linalg.norm(mv(x) - b) / np.linalg.norm(b)
    if timings is not None:
        timings.update(t0=t_1 - t_0, kernel=t_2 - t_1, solve=time.perf_counter() - t_3)
    psi = x.reshape(N_z, M, M, 9)
    if phase_xy is not None:
        psi = psi / bloch_demodulation(M, N_z, a, phase_xy)[..., None]
    return {"psi": psi, "psi0": psi0, "t4": t4, "n_matvec": cnt[0], "residual": float(res), "info": info}


def bloch_demodulation(M, N_z, a, phase_xy):
    """exp(-i (kx x + ky y)) at the cube centres (addition of this build)."""
    c = all_centres(M, N_z, a)
    d = 2.0 * a
    return np.exp(-1j * (phase_xy[0] * c[..., 1] + phase_xy[1] * c[..., 2]) / d)


# ---------------------------------------------------------------------------
# 8. Observables (slab_scattering.py:589-735)
# ---------------------------------------------------------------------------


def _voigt_to_tensor(v6):
    T = np.zeros(v6.shape[:-1] + (3, 3), dtype=complex)
    T[..., 0, 0], T[..., 1, 1], T[..., 2, 2] = v6[..., 0], v6[..., 1], v6[..., 2]
    T[..., 1, 2] = T[..., 2, 1] = v6[..., 3] / 2.0
    T[..., 0, 2] = T[..., 2, 0] = v6[..., 4] / 2.0
    T[..., 0, 1] = T[..., 1, 0] = v6[..., 5] / 2.0
    return T


def vertical_slowness(s, p):
    """sqrt(s^2 - p^2) on the Im >= 0 branch (kennett_layers.py:273-284)."""
    eta = np.sqrt(complex((s + p) * (s - p)))
    if eta.imag < 0.0 or (eta.imag == 0.0 and eta.real < 0.0):
        eta = -eta
    return eta


def rpp_periodic(psi, T_local, M, N_z, a, omega, alpha, rho, p=0.0, demod=None, moment="reference"):
    """Weyl-sum specular R_PP of a periodic slab (``slab_rpp_periodic``,
    slab_scattering.py:672-735). ``demod`` (addition of this build) multiplies
    the sources by the Bloch demodulation before the lateral mean.
    ``moment="plane_wave"`` (addition of this build) puts omega/alpha instead of
    the reference's kz in the strain-moment term; the two agree at p = 0."""
    if T_local.ndim == 4 and T_local.shape[0] == 4:
        src = apply_t0(T_local, psi)
    else:
        src = np.einsum("lmnab,lmnb->lmna", T_local, psi)
    if demod is not None:
        src = src * demod[..., None]
    d = 2.0 * a
    eta = vertical_slowness(complex(1.0 / alpha), p)
    kz = omega * eta
    rh = np.array([-eta * alpha, p * alpha, 0.0])
    z = (np.arange(N_z) + 0.5) * d
    tot = 0.0 + 0j
    for l in range(N_z):
        f = np.mean(src[l, :, :, :3], axis=(0, 1))
        sig = _voigt_to_tensor(np.mean(src[l, :, :, 3:], axis=(0, 1)))
        km = omega / alpha if moment == "plane_wave" else kz
        q = -np.dot(rh, f) - 1j * km * np.dot(rh, sig @ rh)
        tot += q * np.exp(1j * kz * z[l])
    return complex(-1j / (2.0 * kz * d**2 * rho * alpha**2) * tot)


def reflected_field(psi, T_local, M, N_z, a, omega, alpha, beta, rho, k_hat):
    """(R_PP, R_PS, R_SP) far-field sums per unit area (``slab_reflected_field``,
    slab_scattering.py:589-669)."""
    k_hat = np.asarray(k_hat, dtype=float)
    k_hat = k_hat / np.linalg.norm(k_hat)
    kP, kS = omega / alpha, omega / beta
    rh = -k_hat
    gP = 1.0 / (4.0 * np.pi * rho * alpha**2)
    gS = 1.0 / (4.0 * np.pi * rho * beta**2)
    if T_local.ndim == 4 and T_local.shape[0] == 4:
        src = apply_t0(T_local, psi)
    else:
        src = np.einsum("lmnab,lmnb->lmna", T_local, psi)
    c = all_centres(M, N_z, a)
    f = src[..., :3]
    sig = _voigt_to_tensor(src[..., 3:])
    phP = np.exp(-1j * kP * (c @ rh))
    phS = np.exp(-1j * kS * (c @ rh))
    sr = sig @ rh
    srr = sr @ rh
    QP = f @ rh - 1j * kP * srr
    uP = -gP * np.sum(phP * QP) * rh
    QS = f - 1j * kS * sr
    QSp = QS - (QS @ rh)[..., None] * rh
    uS = -gS * np.sum(phS[..., None] * QSp, axis=(0, 1, 2))
    area = (M * 2.0 * a) ** 2
    uP = uP / area
    uS = uS / area
    R_PP = complex(np.dot(rh, uP))
    cross = np.cross(rh, np.array([1.0, 0.0, 0.0]))
    if np.linalg.norm(cross) < 1e-10:
        sv = np.array([0.0, 1.0, 0.0])
    else:
        sv = np.cross(cross, rh)
        sv = sv / np.linalg.norm(sv)
    return R_PP, complex(np.dot(sv, uS)), R_PP


# ---------------------------------------------------------------------------
# 9. Near-field polynomial preconditioner (an addition of this build; the
#    reference solves without a preconditioner)
# ---------------------------------------------------------------------------


def nearfield_blocks(M, N_z, a, omega, alpha, beta, rho, *, volume_averaged=False, n_orders=2):
    """The 27 nearest-neighbour 9x9 blocks of the slab kernel, index
    o = ((dz+1)*3 + dx+1)*3 + dy+1, zero at the self term and for offsets the
    lattice does not have (N_z = 1 or M = 1)."""
    ker = slab_kernel_spatial(M, N_z, a, omega, alpha, beta, rho, volume_averaged=volume_averaged,
                              n_orders=n_orders)
    out = np.zeros((27, 9, 9), dtype=complex)
    for o in range(27):
        dz, dx, dy = o // 9 - 1, (o // 3) % 3 - 1, o % 3 - 1
        if abs(dz) < N_z and abs(dx) < M and abs(dy) < M:
            out[o] = ker[dz + N_z - 1, dx + M - 1, dy + M - 1]
    return out


_DOF_PARITY = np.array([4, 1, 2, 0, 0, 0, 3, 6, 5])  # bits: odd under x, y, z reflection


def nearfield_symmetry_mask():
    """(27, 9, 9) mask of the block entries the mirror symmetry allows: entry (a, b) of an
    offset with a zero component along an axis vanishes when the DOF pair is odd under
    that axis' reflection."""
    mask = np.ones((27, 9, 9), dtype=bool)
    odd = _DOF_PARITY[:, None] ^ _DOF_PARITY[None, :]
    for o in range(27):
        dz, dx, dy = o // 9 - 1, (o // 3) % 3 - 1, o % 3 - 1
        zm = (1 if dx == 0 else 0) | (2 if dy == 0 else 0) | (4 if dz == 0 else 0)
        mask[o] = (odd & zm) == 0
    return mask


def nearfield_stencil(x, t4, blocks, M, N_z):
    """y(v) = sum_o G_o (T0 x)(v - o) over the 27 offsets (the self block included:
    zero for the kernel, a pointwise block for a corrected layer), with the entries
    outside the mirror-symmetry pattern dropped, zero outside the slab; x flat
    (N_z, M, M, 9)."""
    blocks = blocks * nearfield_symmetry_mask()
    tau = apply_t0(t4, x.reshape(N_z, M, M, 9))
    tp = np.zeros((N_z + 2, M + 2, M + 2, 9), dtype=complex)
    tp[1:-1, 1:-1, 1:-1] = tau
    y = np.zeros((N_z, M, M, 9), dtype=complex)
    for o in range(27):
        dz, dx, dy = o // 9 - 1, (o // 3) % 3 - 1, o % 3 - 1
        y += tp[1 - dz:1 - dz + N_z, 1 - dx:1 - dx + M, 1 - dy:1 - dy + M] @ blocks[o].T
    return y.ravel()


def nearfield_precondition(x, t4, blocks, M, N_z, coef=(1, 1, 1), dblocks=None):
    """P x = sum_l c_l h_l, h_0 = x, h_l = (G_nn + dG_l) T0 h_{l-1}."""
    h = np.asarray(x, dtype=complex).ravel()
    out = coef[0] * h
    for l in range(1, len(coef)):
        b = blocks if dblocks is None else blocks + dblocks[l - 1]
        h = nearfield_stencil(h, t4, b, M, N_z)
        out = out + coef[l] * h
    return out


def round_bf16(x):
    """Round real values to bfloat16 as the device does (to float32 first, then to
    nearest even on the upper 16 bits); returned as float64."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32).astype(np.uint64)
    r = ((f + 0x7FFF + ((f >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def _cbf16(z):
    z = np.asarray(z)
    return round_bf16(z.real) + 1j * round_bf16(z.imag)


def nearfield_precondition_rounded(x, t4, blocks, M, N_z, coef=(1, 1, 1), dblocks=None, activations="bf16"):
    """The complex64 preconditioner with the device's roundings restated (an addition
    of this build): layer blocks G_nn + dG_l rounded to float32 and then to BF16; the
    stencil input tau = T0 h formed in float32 and, with activations="bf16" (the
    tensor-core form), rounded to BF16, kept in float32 with activations="fp32" (the
    CUDA-core BF16-weight form); the products summed in FP64 (the device sums in FP32);
    each layer output h_l stored in float32. What remains between this and the device is
    the FP32 summation order, so a wrong tap or operand shows up far above it."""
    if activations not in ("bf16", "fp32"):
        raise ValueError(activations)
    mask = nearfield_symmetry_mask()
    t4c = np.asarray(t4).reshape(4, N_z, M, M).astype(np.complex64)
    h = np.asarray(x).reshape(N_z, M, M, 9).astype(np.complex64)
    out = coef[0] * h.astype(complex)
    for l in range(1, len(coef)):
        b = blocks if dblocks is None else blocks + dblocks[l - 1]
        b = _cbf16(b.astype(np.complex64)) * mask
        tr = h[..., 3] + h[..., 4] + h[..., 5]
        tau = np.empty_like(h)
        for c in range(3):
            tau[..., c] = t4c[0] * h[..., c]
        for c in range(3, 6):
            tau[..., c] = t4c[1] * tr + t4c[2] * h[..., c]
        for c in range(6, 9):
            tau[..., c] = t4c[3] * h[..., c]
        tau = _cbf16(tau) if activations == "bf16" else tau.astype(complex)
        tp = np.zeros((N_z + 2, M + 2, M + 2, 9), dtype=complex)
        tp[1:-1, 1:-1, 1:-1] = tau
        y = np.zeros((N_z, M, M, 9), dtype=complex)
        for o in range(27):
            dz, dx, dy = o // 9 - 1, (o // 3) % 3 - 1, o % 3 - 1
            y += tp[1 - dz:1 - dz + N_z, 1 - dx:1 - dx + M, 1 - dy:1 - dy + M] @ b[o].T
        h = y.astype(np.complex64)
        out = out + coef[l] * h.astype(complex)
    return out.ravel()


def nearfield_stencil_adjoint(y, t4, blocks, M, N_z):
    """S^H y = T0^H (sum_o G_o^H y(. + o)): the adjoint of nearfield_stencil in the
    Euclidean inner product (T0 is complex symmetric, so T0^H = conj(T0))."""
    blocks = blocks * nearfield_symmetry_mask()
    yp = np.zeros((N_z + 2, M + 2, M + 2, 9), dtype=complex)
    yp[1:-1, 1:-1, 1:-1] = np.asarray(y).reshape(N_z, M, M, 9)
    z = np.zeros((N_z, M, M, 9), dtype=complex)
    for o in range(27):
        dz, dx, dy = o // 9 - 1, (o // 3) % 3 - 1, o % 3 - 1
        z += yp[1 + dz:1 + dz + N_z, 1 + dx:1 + dx + M, 1 + dy:1 + dy + M] @ blocks[o].conj()
    return apply_t0(np.conj(t4), z).ravel()


_ADJ_P = np.array([-1.0, -1.0, -1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0])  # displacements odd, strains even
_ADJ_D = np.array([1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 2.0, 2.0, 2.0])    # Voigt factors of the shear strains


def slab_operator_adjoint(y, t4, kernel_hat, M, N_z, *, periodic=False):
    """A^H y for A = I - G0 T0 (an addition of this build). Reciprocity makes K D
    symmetric and the mirror symmetry gives K(-r) = P K(r) P, so G0^T = P D^-1 G0 D P and
    A^H y = y - conj(T0) P D^-1 conj(G0 (D P conj(y))), G0 u = (u - A_tau u) / tau with
    A_tau the operator at T0 = tau I, tau = 1 / max|K| (so G0 tau u does not cancel)."""
    tau = 1.0 / np.abs(kernel_hat).max() * kernel_hat.shape[1] * kernel_hat.shape[2]
    ident = np.zeros_like(t4)
    ident[0] = ident[2] = ident[3] = tau
    y = np.asarray(y, dtype=complex).reshape(-1, 9)
    u = (_ADJ_D * _ADJ_P * np.conj(y)).ravel()
    g0u = (u - slab_matvec(u, ident, kernel_hat, M, N_z, periodic=periodic)) / tau
    w = (_ADJ_P / _ADJ_D * np.conj(g0u.reshape(-1, 9))).reshape(N_z, M, M, 9)
    return y.ravel() - apply_t0(np.conj(t4), w).ravel()


def nearfield_residual_loss_grad(r, t4, kernel_hat, blocks, M, N_z, coef, w=None, *, periodic=False):
    """Training objective of the learned near-field preconditioner and its gradients
    (an addition of this build). With P r = sum_l c_l h_l, h_0 = r, h_l = S_l h_{l-1},
    S_l = (G_nn + s w_l) T0, s = max |G_nn|, the residual of one GMRES step:
        loss = min_alpha || alpha A P r^ - r^ ||^2 = 1 - |<y, r^>|^2 / <y, y>,
        y = A P r^,  r^ = r / ||r||.
    Returns (loss, dL/dconj(c) (L+1,), dL/dconj(w) (L, 27, 9, 9)); the weight gradient
    is zero outside the mirror-symmetry pattern."""
    coef = np.asarray(coef, dtype=complex)
    L = len(coef) - 1
    s = np.abs(blocks).max()
    w = np.zeros((L, 27, 9, 9), dtype=complex) if w is None else np.asarray(w, dtype=complex)
    r = np.asarray(r, dtype=complex).ravel()
    r = r / np.linalg.norm(r)
    mask = nearfield_symmetry_mask()
    lay = [blocks + s * w[l] for l in range(L)]
    hs, taus = [r], []
    for l in range(L):
        taus.append(apply_t0(t4, hs[-1].reshape(N_z, M, M, 9)))
        hs.append(nearfield_stencil(hs[-1], t4, lay[l], M, N_z))
    z = sum(c * h for c, h in zip(coef, hs))
    y = slab_matvec(z, t4, kernel_hat, M, N_z, periodic=periodic)
    alpha = np.vdot(y, r) / np.vdot(y, y).real
    q = alpha * y - r
    loss = np.vdot(q, q).real
    d = slab_operator_adjoint(np.conj(alpha) * q, t4, kernel_hat, M, N_z, periodic=periodic)
    gc = np.array([np.vdot(h, d) for h in hs])
    gw = np.zeros((L, 27, 9, 9), dtype=complex)
    delta = np.conj(coef[L]) * d
    for l in range(L, 0, -1):
        tp = np.zeros((N_z + 2, M + 2, M + 2, 9), dtype=complex)
        tp[1:-1, 1:-1, 1:-1] = taus[l - 1]
        dv = delta.reshape(N_z, M, M, 9)
        for o in range(27):
            dz, dx, dy = o // 9 - 1, (o // 3) % 3 - 1, o % 3 - 1
            src = tp[1 - dz:1 - dz + N_z, 1 - dx:1 - dx + M, 1 - dy:1 - dy + M]
            gw[l - 1, o] = s * np.einsum("zxya,zxyb->ab", dv, np.conj(src)) * mask[o]
        if l > 1:
            delta = np.conj(coef[l - 1]) * d + nearfield_stencil_adjoint(delta, t4, lay[l - 1], M, N_z)
    return loss, gc, gw


# ---------------------------------------------------------------------------
# 10. Sphere FFT Foldy-Lax (sphere_scattering_fft.py:42-330) on the slab operator
# ---------------------------------------------------------------------------


def sphere_grid(radius, n_sub):
    """Cells of the n_sub^3 cube grid inside the sphere (sphere_scattering_fft.py:42-80):
    centre coordinates (-n/2 + 1/2 + i) d per axis, d = 2 a_sub, a_sub = radius / n_sub,
    kept when |centre| < radius. Returns (grid_idx (N, 3), centres (N, 3), a_sub)."""
    a_sub = radius / n_sub
    d = 2.0 * a_sub
    c1 = (-n_sub / 2.0 + 0.5 + np.arange(n_sub)) * d
    g = np.stack(np.meshgrid(c1, c1, c1, indexing="ij"), -1).reshape(-1, 3)
    idx = np.stack(np.meshgrid(*(np.arange(n_sub),) * 3, indexing="ij"), -1).reshape(-1, 3)
    keep = np.linalg.norm(g, axis=1) < radius
    return idx[keep], g[keep], a_sub


_VOIGT_PAIRS = ((0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1))


def sphere_incident(centres, omega, alpha, beta, k_hat=None, wave_type="S"):
    """The 9 incident patterns (9N, 9) of the coupled system
    (resonance_tmatrix.py:526-586): columns 0-2 a uniform displacement e_p, columns 3-8
    the displacement eps(e_alpha) (x - x_mean) with the Voigt strain e_alpha (engineering
    shear: off-diagonal tensor entries 1/2), all times exp(i k k_hat . x)."""
    k_hat = np.array([0.0, 0.0, 1.0]) if k_hat is None else np.asarray(k_hat, dtype=float)
    k_hat = k_hat / np.linalg.norm(k_hat)
    k = omega / (beta if wave_type == "S" else alpha)
    ph = np.exp(1j * k * (centres @ k_hat))
    dx = centres - centres.mean(axis=0)
    N = len(centres)
    U = np.zeros((N, 9, 9), dtype=complex)
    for p in range(3):
        U[:, p, p] = ph
    for al, (p, q) in enumerate(_VOIGT_PAIRS):
        e = np.zeros((3, 3))
        if p == q:
            e[p, p] = 1.0
        else:
            e[p, q] = e[q, p] = 0.5
        U[:, :3, 3 + al] = (dx @ e.T) * ph[:, None]
        U[:, 3 + al, 3 + al] = ph
    return U.reshape(9 * N, 9)


def sphere_foldy_lax_column(omega, radius, alpha, beta, rho, dlam, dmu, drho, n_sub, k_hat, wave_type, col,
                            gmres_tol=1e-12):
    """Column ``col`` of the sphere system alone (the unit of the CPU baseline):
    returns the exciting field on the inside cells (N, 9)."""
    grid_idx, centres, a_sub = sphere_grid(radius, n_sub)
    n = n_sub
    mask = np.zeros((n, n, n), dtype=bool)
    mask[tuple(grid_idx.T)] = True
    t4 = t0_scalars(omega, a_sub, alpha, beta, rho, dlam * mask, dmu * mask, drho * mask)
    kh = build_slab_kernels(n, n, a_sub, omega, alpha, beta, rho)
    U = sphere_incident(centres, omega, alpha, beta, k_hat, wave_type)
    A = LinearOperator((9 * n ** 3,) * 2, matvec=lambda v: slab_matvec(v, t4, kh, n, n), dtype=complex)
    b = np.zeros((n, n, n, 9), dtype=complex)
    b[tuple(grid_idx.T)] = U[:, col].reshape(len(centres), 9)
    x, _ = gmres(A, b.ravel(), x0=b.ravel().copy(), rtol=gmres_tol, maxiter=500, restart=30)
    return x.reshape(n, n, n, 9)[tuple(grid_idx.T)]


def sphere_foldy_lax(omega, radius, alpha, beta, rho, dlam, dmu, drho, n_sub, k_hat=None, wave_type="S",
                     gmres_tol=1e-12):
    """T_comp (9, 9) and psi_exc (9N, 9) of the sphere: the slab operator on the
    n_sub^3 lattice (cube half-width a_sub, aperiodic) with the contrast inside the
    sphere and none outside, so the outside cells carry no source and the inside block
    is the reference's (I - P T) (sphere_scattering_fft.py:83-125, 184-225); scipy GMRES
    per column from the Born guess; T_comp = sum over cells of T x."""
    grid_idx, centres, a_sub = sphere_grid(radius, n_sub)
    n = n_sub
    mask = np.zeros((n, n, n), dtype=bool)
    mask[tuple(grid_idx.T)] = True
    t4 = t0_scalars(omega, a_sub, alpha, beta, rho, dlam * mask, dmu * mask, drho * mask)
    kh = build_slab_kernels(n, n, a_sub, omega, alpha, beta, rho)
    U = sphere_incident(centres, omega, alpha, beta, k_hat, wave_type)
    N = len(centres)
    A = LinearOperator((9 * n ** 3,) * 2, matvec=lambda v: slab_matvec(v, t4, kh, n, n), dtype=complex)
    psi = np.zeros((9 * N, 9), dtype=complex)
    Tc = np.zeros((9, 9), dtype=complex)
    for col in range(9):
        b = np.zeros((n, n, n, 9), dtype=complex)
        b[tuple(grid_idx.T)] = U[:, col].reshape(N, 9)
        x, _ = gmres(A, b.ravel(), x0=b.ravel().copy(), rtol=gmres_tol, maxiter=500, restart=30)
        xf = x.reshape(n, n, n, 9)
        psi[:, col] = xf[tuple(grid_idx.T)].ravel()
        Tc[:, col] = apply_t0(t4, xf).reshape(-1, 9).sum(axis=0)
    return Tc, psi, centres, a_sub
