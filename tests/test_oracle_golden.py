"""The oracle (CPU restatement) against the reference's own outputs.

The fixtures in tests/golden were produced by tests/golden/make_golden.py from
the reference package; these tests pin the oracle before anything is compared
with it.
"""

import numpy as np
import pytest
from numpy.testing import assert_allclose

from oracle import slab_oracle as O


def _medium(z):
    return tuple(float(v) for v in z["medium"])


def test_va_nn_blocks(golden):
    z = golden("va_nn.npz")
    al, be, rho = _medium(z)
    for no in range(4):
        for io, om in enumerate(z["omegas"]):
            for ir, R in enumerate(z["offsets"]):
                got = O.va_propagator(tuple(int(v) for v in R), al, be, rho, float(om), no)
                ref = z["blocks"][no, io, ir]
                assert_allclose(got, ref, rtol=0, atol=1e-15 * np.abs(ref).max())


def test_point_propagator(golden):
    z = golden("point_propagator.npz")
    al, be, rho = _medium(z)
    for io, om in enumerate(z["omegas"]):
        got = O.point_propagator(z["r"], float(om), al, be, rho)
        ref = z["blocks"][io]
        for g, r, x in zip(got, ref, z["r"]):
            # The P and S 1/r^3 terms cancel as k r -> 0, so rounding differences
            # between two FP64 evaluation orders grow like (k_S r)^-2.
            ksr = float(om) / be * np.linalg.norm(x)
            tol = 1e-13 * max(1.0, ksr**-2)
            assert_allclose(g, r, rtol=0, atol=tol * np.abs(r).max())


def test_t0(golden):
    z = golden("t0.npz")
    al, be, rho = _medium(z)
    for (om, a, dl, dm, dr), T in zip(z["cases"], z["T"]):
        t4 = O.t0_scalars(om, a, al, be, rho, np.array(dl), np.array(dm), np.array(dr))
        assert_allclose(O.t0_full(t4), T, rtol=1e-13, atol=1e-30)


@pytest.mark.parametrize("per", [0, 1])
@pytest.mark.parametrize("va", [0, 1])
def test_kernels(golden, per, va):
    z = golden("kernels_m3_nz2.npz")
    al, be, rho = _medium(z)
    got = O.build_slab_kernels(3, 2, float(z["a"]), float(z["omega"]), al, be, rho, volume_averaged=bool(va),
                               periodic=bool(per))
    ref = z[f"k_p{per}_va{va}"]
    assert got.shape == ref.shape
    assert_allclose(got, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("M,Nz", [(3, 2), (2, 3)])
@pytest.mark.parametrize("per", [0, 1])
def test_matvec(golden, M, Nz, per):
    z = golden("matvec_small.npz")
    al, be, rho = _medium(z)
    om, a = float(z["omega"]), float(z["a"])
    t4 = O.t0_scalars(om, a, al, be, rho, z[f"dlam_M{M}_Nz{Nz}"], z[f"dmu_M{M}_Nz{Nz}"], z[f"drho_M{M}_Nz{Nz}"])
    kh = O.build_slab_kernels(M, Nz, a, om, al, be, rho, periodic=bool(per))
    got = O.slab_matvec(z[f"x_M{M}_Nz{Nz}"], t4, kh, M, Nz, periodic=bool(per))
    assert_allclose(got, z[f"y_M{M}_Nz{Nz}_p{per}"], rtol=1e-11)


def test_incident(golden):
    z = golden("incident.npz")
    al, be, rho = _medium(z)
    for i, kh in enumerate(z["dirs"]):
        for w in ("P", "S"):
            got = O.incident_field(3, 2, float(z["a"]), float(z["omega"]), al, be, kh, w)
            assert_allclose(got, z[f"psi0_{i}_{w}"], rtol=1e-14, atol=1e-14)
    with pytest.raises(ValueError, match="wave_type"):
        O.polarisation(np.array([1.0, 0, 0]), "X")


@pytest.mark.parametrize("name,M,Nz,opt", [
    ("ap_P", 4, 2, {}), ("per_P", 4, 2, {"periodic": True}), ("va_P", 3, 2, {"volume_averaged": True}),
    ("ap_S", 3, 3, {}),
])
def test_small_solves(golden, name, M, Nz, opt):
    z = golden("solve_small.npz")
    al, be, rho = _medium(z)
    om, a = float(z["omega"]), float(z["a"])
    wt = "S" if name.endswith("S") else "P"
    r = O.solve(M, Nz, a, al, be, rho, z[f"{name}_dlam"], z[f"{name}_dmu"], z[f"{name}_drho"], om, z[f"{name}_khat"],
                wt, 1e-12, **opt)
    ref = z[f"{name}_psi"]
    assert np.linalg.norm(r["psi"] - ref) / np.linalg.norm(ref) < 1e-10
    rpp = O.rpp_periodic(r["psi"], r["t4"], M, Nz, a, om, al, rho)
    assert abs(rpp - z[f"{name}_rpp"]) <= 1e-9 * abs(z[f"{name}_rpp"])
    refl = O.reflected_field(r["psi"], r["t4"], M, Nz, a, om, al, be, rho, z[f"{name}_khat"])
    assert_allclose(np.array(refl), z[f"{name}_refl"], rtol=1e-9)


def test_headline_cpu_case(golden):
    """16x16x4, ka 0.2, i.i.d. +-10 %, periodic, normal P: psi and R_PP vs the reference."""
    z = golden("slab_16x16x4.npz")
    al, be, rho = _medium(z)
    r = O.solve(16, 4, float(z["a"]), al, be, rho, z["dlam"], z["dmu"], z["drho"], float(z["omega"]),
                np.array([1.0, 0, 0]), "P", 1e-12, periodic=True)
    assert np.linalg.norm(r["psi"] - z["psi"]) / np.linalg.norm(z["psi"]) < 1e-10
    rpp = O.rpp_periodic(r["psi"], r["t4"], 16, 4, float(z["a"]), float(z["omega"]), al, rho)
    assert abs(rpp - complex(z["rpp"])) <= 1e-9 * abs(complex(z["rpp"]))


def test_dense_direct(golden):
    """The FFT operator solved by GMRES equals the dense pairwise operator solved by LU."""
    z = golden("dense_m3_nz2.npz")
    al, be, rho = _medium(z)
    om, a = float(z["omega"]), float(z["a"])
    t4 = O.t0_scalars(om, a, al, be, rho, z["dlam"], z["dmu"], z["drho"])
    A = O.dense_operator(3, 2, a, om, al, be, rho, t4)
    b = O.incident_field(3, 2, a, om, al, be, np.array([1.0, 0, 0]), "P").ravel()
    x = np.linalg.solve(A, b)
    assert np.linalg.norm(x - z["psi"].ravel()) / np.linalg.norm(z["psi"]) < 1e-11
    r = O.solve(3, 2, a, al, be, rho, z["dlam"], z["dmu"], z["drho"], om, np.array([1.0, 0, 0]), "P", 1e-13)
    assert np.linalg.norm(r["psi"].ravel() - z["psi"].ravel()) / np.linalg.norm(z["psi"]) < 1e-10


def test_zero_contrast_identity():
    """Zero contrast: psi = psi0 and R_PP = 0 (tests/test_slab_scattering.py:328-346)."""
    z = np.zeros((2, 3, 3))
    r = O.solve(3, 2, 1.0, 5000.0, 3000.0, 2500.0, z, z, z, 150.0, np.array([1.0, 0, 0]), "P", 1e-10)
    assert_allclose(r["psi"], r["psi0"], atol=1e-12)
    assert abs(O.rpp_periodic(r["psi"], r["t4"], 3, 2, 1.0, 150.0, 5000.0, 2500.0)) < 1e-20


def test_bloch_fold_reduces_to_reference_at_normal_incidence():
    kh0 = O.build_slab_kernels(3, 2, 1.0, 150.0, 5000.0, 3000.0, 2500.0, periodic=True)
    kh1 = O.build_slab_kernels(3, 2, 1.0, 150.0, 5000.0, 3000.0, 2500.0, periodic=True, phase_xy=(0.0, 0.0))
    assert_allclose(kh1, kh0, rtol=1e-15, atol=0)


def _bloch_uniform_rpp(z, ic, p, M=4, moment="reference"):
    """Bloch-phased periodic solve of a uniform one-layer slab (H = 2, a = 1) at
    horizontal slowness p, P incidence, and its specular R_PP."""
    al, be, rho = z["medium"]
    om, a = float(z["omega"]), 1.0
    dl, dm, dr = (np.full((1, M, M), v) for v in z["contrasts"][ic])
    s = p * al
    kh = np.array([np.sqrt(1.0 - s * s), s, 0.0])
    phase = (om * p * 2.0 * a, 0.0)
    r = O.solve(M, 1, a, al, be, rho, dl, dm, dr, om, kh, "P", gmres_tol=1e-11, periodic=True, phase_xy=phase)
    return O.rpp_periodic(r["psi"], r["t4"], M, 1, a, om, al, rho, p=p,
                          demod=O.bloch_demodulation(M, 1, a, phase), moment=moment)


@pytest.mark.parametrize("ic", [0, 1])
def test_bloch_oblique_rpp_vs_kennett(golden, ic):
    """Oblique P incidence on a uniform layer through the Bloch-phased fold: with the
    plane-wave moment term the Weyl-sum R_PP matches the Kennett layer reflectivity
    within 1% at every slowness (weak and strong contrast); the reference's formula
    (kz in the moment term) agrees at p = 0 and falls below it as p grows."""
    z = golden("kennett.npz")
    K = z[f"rpp_p_c{ic}_H2"]
    for ip, p in enumerate(z["ps"]):
        R = _bloch_uniform_rpp(z, ic, float(p), moment="plane_wave")
        assert abs(R - K[ip]) < 0.01 * abs(K[ip])
    r0 = _bloch_uniform_rpp(z, ic, 0.0)
    assert abs(r0 - K[0]) < 0.01 * abs(K[0])
    r_ref = _bloch_uniform_rpp(z, ic, float(z["ps"][-1]))
    assert abs(r_ref) < 0.95 * abs(K[-1])
