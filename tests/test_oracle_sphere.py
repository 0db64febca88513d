"""The oracle's restatement of the sphere FFT Foldy-Lax solver (oracle/slab_oracle.py,
section 10: the slab operator on the n_sub^3 lattice with the contrast inside the sphere
only) against fixtures of the reference's own CPU solver
(tests/golden/make_sphere_golden.py). CPU only."""

from pathlib import Path

import numpy as np
import pytest

from oracle import slab_oracle as O

GOLD = np.load(Path(__file__).parent / "golden" / "sphere.npz")


def _case(k):
    kh = GOLD[f"c{k}_k_hat"]
    return dict(omega=float(GOLD[f"c{k}_omega"]), radius=float(GOLD[f"c{k}_radius"]),
                n_sub=int(GOLD[f"c{k}_n_sub"]), k_hat=None if kh.size == 0 else kh, wave=str(GOLD[f"c{k}_wave"]))


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("k", range(int(GOLD["n_cases"])))
def test_sphere_oracle_matches_reference(k):
    c = _case(k)
    idx, cen, a_sub = O.sphere_grid(c["radius"], c["n_sub"])
    assert np.array_equal(cen, GOLD[f"c{k}_centres"]) and a_sub == GOLD[f"c{k}_a_sub"]
    Tc, psi, _, _ = O.sphere_foldy_lax(c["omega"], c["radius"], float(GOLD["alpha"]), float(GOLD["beta"]),
                                       float(GOLD["rho"]), float(GOLD["Dlambda"]), float(GOLD["Dmu"]),
                                       float(GOLD["Drho"]), c["n_sub"], c["k_hat"], c["wave"])
    assert _rel(Tc, GOLD[f"c{k}_T_comp"]) < 1e-10
    assert _rel(psi, GOLD[f"c{k}_psi_exc"]) < 1e-10
    # the per-cell T of the lattice's T0 build is the reference's sub-cell T-matrix
    t4 = O.t0_scalars(c["omega"], a_sub, float(GOLD["alpha"]), float(GOLD["beta"]), float(GOLD["rho"]),
                      np.full((1, 1, 1), float(GOLD["Dlambda"])), np.full((1, 1, 1), float(GOLD["Dmu"])),
                      np.full((1, 1, 1), float(GOLD["Drho"])))
    assert _rel(O.t0_full(t4)[0, 0, 0], GOLD[f"c{k}_T_loc"]) < 1e-12


def test_sphere_incident_patterns():
    _, cen, _ = O.sphere_grid(0.5, 4)
    U = O.sphere_incident(cen, 300.0, 5000.0, 3000.0, None, "S").reshape(len(cen), 9, 9)
    ph = np.exp(1j * 300.0 / 3000.0 * cen[:, 2])
    assert np.allclose(U[:, 0, 0], ph) and np.allclose(U[:, 3 + 3, 3 + 3], ph)
    # column of 2 e_xy: u = eps . dx with eps_xy = eps_yx = 1/2
    dx = cen - cen.mean(0)
    assert np.allclose(U[:, 1, 6], 0.5 * dx[:, 2] * ph) and np.allclose(U[:, 2, 6], 0.5 * dx[:, 1] * ph)
