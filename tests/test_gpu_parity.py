"""GPU parity of the CUDA path (through the C-ABI) with the oracle and the
reference's golden fixtures. Tolerances follow the reference tests
(tests/test_slab_scattering.py:259-273, 663-718; test_slab_scattering_gpu.py:45-141):
complex128 operator rtol 1e-10; complex64 operator rtol 2e-5 (FP32 FFT/accumulate);
solves judged by the FP64 true residual and the relative error of psi and R_PP.
"""

import numpy as np
import pytest
import torch
from numpy.testing import assert_allclose

from oracle import slab_oracle as O

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from multiplescatteringcalculations_b200 import (  # noqa: E402
    MaterialContrast,
    ReferenceMedium,
    SlabGeometry,
    SlabMaterial,
    SlabPlan,
    compute_slab_scattering_gpu,
    compute_slab_tmatrices,
    random_slab_material,
    slab_reflected_field,
    slab_rpp_periodic,
    t0_expand,
    uniform_random_material,
    uniform_slab_material,
)

REF = ReferenceMedium(5000.0, 3000.0, 2500.0)
CONTRAST = MaterialContrast(2e9, 1e9, 100.0)
OMEGA = 0.05 * REF.beta / 1.0
KZ = np.array([1.0, 0.0, 0.0])


def _medium(z):
    return ReferenceMedium(*[float(v) for v in z["medium"]])


def _rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300)


# ---- building blocks ----------------------------------------------------------------


def test_t0_matches_reference(golden):
    z = golden("t0.npz")
    ref = _medium(z)
    for (om, a, dl, dm, dr), T in zip(z["cases"], z["T"]):
        g = SlabGeometry(1, 1, float(a))
        mat = SlabMaterial(np.full((1, 1, 1), dl), np.full((1, 1, 1), dm), np.full((1, 1, 1), dr), ref)
        got = compute_slab_tmatrices(g, mat, float(om))[0, 0, 0]
        assert_allclose(got, T, rtol=1e-13, atol=1e-300 + 1e-15 * np.abs(T).max())


def test_incident_matches_reference(golden):
    z = golden("incident.npz")
    ref = _medium(z)
    plan = SlabPlan(SlabGeometry(3, 2, float(z["a"])), ref)
    for i, kh in enumerate(z["dirs"]):
        for w in ("P", "S"):
            got = plan.incident(float(z["omega"]), kh, w).cpu().numpy()
            assert_allclose(got, z[f"psi0_{i}_{w}"], rtol=1e-13, atol=1e-15)
    with pytest.raises(ValueError, match="wave_type"):
        plan.incident(float(z["omega"]), KZ, "X")


@pytest.mark.parametrize("M,Nz", [(3, 2), (2, 3)])
@pytest.mark.parametrize("per", [0, 1])
def test_matvec_matches_reference(golden, M, Nz, per):
    z = golden("matvec_small.npz")
    ref = _medium(z)
    g = SlabGeometry(M, Nz, float(z["a"]))
    mat = SlabMaterial(z[f"dlam_M{M}_Nz{Nz}"], z[f"dmu_M{M}_Nz{Nz}"], z[f"drho_M{M}_Nz{Nz}"], ref)
    plan = SlabPlan(g, ref, periodic=bool(per))
    plan.build_t0(mat, float(z["omega"]))
    plan.build_g0(float(z["omega"]))
    x = torch.from_numpy(z[f"x_M{M}_Nz{Nz}"].reshape(Nz, M, M, 9))
    y = plan.matvec(x, "complex128").cpu().numpy().ravel()
    assert_allclose(y, z[f"y_M{M}_Nz{Nz}_p{per}"], rtol=1e-10)
    y32 = plan.matvec(x, "complex64").cpu().numpy().ravel()
    assert _rel(y32, z[f"y_M{M}_Nz{Nz}_p{per}"]) < 2e-6


@pytest.mark.parametrize("M,Nz,per,va", [
    (8, 4, 0, 0), (8, 4, 1, 0), (5, 3, 1, 0), (7, 2, 1, 0), (11, 2, 1, 0), (6, 5, 0, 0), (4, 3, 0, 1), (4, 3, 1, 1),
    (12, 1, 0, 0), (1, 3, 0, 0), (3, 1, 1, 1),
])
def test_matvec_random_sizes_vs_oracle(M, Nz, per, va):
    """Odd/mixed-radix FFT lengths, one layer, one column, VA kernels."""
    rng = np.random.default_rng(M * 100 + Nz)
    g = SlabGeometry(M, Nz, 1.0)
    mat = random_slab_material(g, REF, CONTRAST, 0.5, seed=M + Nz)
    t4 = O.t0_scalars(OMEGA, 1.0, REF.alpha, REF.beta, REF.rho, mat.Dlambda, mat.Dmu, mat.Drho)
    kh = O.build_slab_kernels(M, Nz, 1.0, OMEGA, REF.alpha, REF.beta, REF.rho, periodic=bool(per),
                              volume_averaged=bool(va))
    x = rng.standard_normal(Nz * M * M * 9) + 1j * rng.standard_normal(Nz * M * M * 9)
    want = O.slab_matvec(x, t4, kh, M, Nz, periodic=bool(per))
    plan = SlabPlan(g, REF, periodic=bool(per))
    plan.build_t0(mat, OMEGA)
    plan.build_g0(OMEGA, volume_averaged=bool(va))
    got = plan.matvec(torch.from_numpy(x.reshape(Nz, M, M, 9))).cpu().numpy().ravel()
    assert _rel(got, want) < 1e-12
    assert_allclose(got, want, rtol=1e-10, atol=1e-12 * np.abs(want).max())


@pytest.mark.parametrize("M,Nz,per,va", [
    (8, 4, 0, 0),     # Lz 8 (one pruned radix-8 stage), Lxy 15
    (16, 8, 0, 0),    # Lz 16, Lxy 32 pruned
    (16, 16, 1, 1),   # Lz 32 volume averaged, Lxy 16 periodic (unpruned)
    (32, 5, 0, 1),    # Lz 16 volume averaged, Lxy 63 (radices 7, 3, 3)
    (64, 2, 1, 0),    # Lxy 64 periodic, Lz 4
    (20, 33, 0, 0),   # Lz 128 (one block per column set), Lxy 40
    (24, 12, 0, 0),   # Lz 32, Lxy 48
    (28, 6, 0, 0),    # Lz 16, Lxy 56
])
def test_matvec_compiled_lengths_vs_oracle(M, Nz, per, va):
    """The compile-time FFT kernels (power-of-two lengths, pruned first and last
    stages when the data fill at most half the padded line) in both precisions."""
    rng = np.random.default_rng(M * 1000 + Nz)
    g = SlabGeometry(M, Nz, 1.0)
    mat = random_slab_material(g, REF, CONTRAST, 0.5, seed=M * 7 + Nz)
    t4 = O.t0_scalars(OMEGA, 1.0, REF.alpha, REF.beta, REF.rho, mat.Dlambda, mat.Dmu, mat.Drho)
    kh = O.build_slab_kernels(M, Nz, 1.0, OMEGA, REF.alpha, REF.beta, REF.rho, periodic=bool(per),
                              volume_averaged=bool(va))
    x = rng.standard_normal(Nz * M * M * 9) + 1j * rng.standard_normal(Nz * M * M * 9)
    want = O.slab_matvec(x, t4, kh, M, Nz, periodic=bool(per))
    plan = SlabPlan(g, REF, periodic=bool(per))
    plan.build_t0(mat, OMEGA)
    plan.build_g0(OMEGA, volume_averaged=bool(va))
    xt = torch.from_numpy(x.reshape(Nz, M, M, 9))
    got = plan.matvec(xt, "complex128").cpu().numpy().ravel()
    assert _rel(got, want) < 1e-12
    got32 = plan.matvec(xt, "complex64").cpu().numpy().ravel()
    assert _rel(got32, want) < 1e-5


@pytest.mark.parametrize("M,Nz,per,va", [
    (8, 20, 1, 0),     # Lz 64 periodic, two threads per z line
    (6, 17, 0, 1),     # Lz 64 volume averaged (one octant kx per block)
    (10, 32, 0, 0),    # Lz 64, N_z = Lz/2
    (9, 9, 1, 1),      # Lz 32 volume averaged, Lxy 9 (octant kx chunks ragged)
    (13, 16, 0, 0),    # Lz 32, N_z = Lz/2, Lxy 25
    (7, 5, 1, 0),      # Lz 16
    (5, 3, 0, 1),      # Lz 8 volume averaged
])
def test_matvec_register_z_pass_vs_oracle(M, Nz, per, va):
    """The register form of the complex64 z pass (every power-of-two Lz up to 64,
    point and volume-averaged kernels, ragged kx chunks) against the oracle, and one
    and three right-hand sides against each other."""
    rng = np.random.default_rng(M * 10 + Nz)
    g = SlabGeometry(M, Nz, 1.0)
    mat = random_slab_material(g, REF, CONTRAST, 0.5, seed=M * 3 + Nz)
    t4 = O.t0_scalars(OMEGA, 1.0, REF.alpha, REF.beta, REF.rho, mat.Dlambda, mat.Dmu, mat.Drho)
    kh = O.build_slab_kernels(M, Nz, 1.0, OMEGA, REF.alpha, REF.beta, REF.rho, periodic=bool(per),
                              volume_averaged=bool(va))
    x = rng.standard_normal(Nz * M * M * 9) + 1j * rng.standard_normal(Nz * M * M * 9)
    want = O.slab_matvec(x, t4, kh, M, Nz, periodic=bool(per))
    plan = SlabPlan(g, REF, periodic=bool(per))
    plan.build_t0(mat, OMEGA)
    plan.build_g0(OMEGA, volume_averaged=bool(va))
    xt = torch.from_numpy(x.reshape(Nz, M, M, 9))
    got32 = plan.matvec(xt, "complex64").cpu().numpy().ravel()
    assert _rel(got32, want) < 5e-6
    x3 = torch.stack([xt, 2j * xt, xt.conj()]).to(torch.complex64)
    y3 = plan.matvec_multi(x3.permute(0, 4, 1, 2, 3).contiguous().to(plan.device), "complex64")
    for r in range(3):
        want_r = O.slab_matvec(x3[r].numpy().astype(np.complex128).ravel(), t4, kh, M, Nz, periodic=bool(per))
        assert _rel(y3[r].permute(1, 2, 3, 0).cpu().numpy().ravel(), want_r) < 5e-6
    plan.close()


@pytest.mark.parametrize("M,Nz,Lxy,va", [
    (32, 5, 64, 0),    # M = L/2
    (30, 4, 64, 0),    # M < L/2, not a multiple of 4 (warps holding rows inside and outside the lattice)
    (64, 3, 128, 0),   # the cfg2 shape
    (45, 6, 128, 1),   # odd M, volume averaged
])
def test_matvec_fused_plane_passes_vs_oracle(M, Nz, Lxy, va):
    """The complex64 matvec's fused plane kernels (aperiodic, Lx = Ly in {64, 128}):
    T0 + y + x per plane and x' + y' + output per plane."""
    rng = np.random.default_rng(M * 100 + Nz)
    g = SlabGeometry(M, Nz, 1.0)
    mat = random_slab_material(g, REF, CONTRAST, 0.5, seed=M + 3 * Nz)
    t4 = O.t0_scalars(OMEGA, 1.0, REF.alpha, REF.beta, REF.rho, mat.Dlambda, mat.Dmu, mat.Drho)
    kh = O.build_slab_kernels(M, Nz, 1.0, OMEGA, REF.alpha, REF.beta, REF.rho, volume_averaged=bool(va))
    x = rng.standard_normal(Nz * M * M * 9) + 1j * rng.standard_normal(Nz * M * M * 9)
    want = O.slab_matvec(x, t4, kh, M, Nz)
    plan = SlabPlan(g, REF, Lxy=Lxy)
    assert plan.fft_sizes()[1:] == (Lxy, Lxy)
    plan.build_t0(mat, OMEGA)
    plan.build_g0(OMEGA, volume_averaged=bool(va))
    xt = torch.from_numpy(x.reshape(Nz, M, M, 9))
    assert _rel(plan.matvec(xt, "complex64").cpu().numpy().ravel(), want) < 1e-5
    assert _rel(plan.matvec(xt, "complex128").cpu().numpy().ravel(), want) < 1e-12


@pytest.mark.parametrize("M,Nz,va", [(64, 3, 0), (40, 7, 1), (9, 4, 0), (33, 1, 0), (2, 2, 1)])
def test_fused_g0_build_equals_unfused(monkeypatch, M, Nz, va):
    """The aperiodic G0 build with the spatial evaluation fused into the x transform
    (mirror images by parity sign) against the unfused passes (MSC_G0_FUSED=0): the same
    operator to rounding and the same near-field blocks (power-of-two and mixed-radix lateral
    lengths, one layer, volume averaged; 2 x 2 lies below the fused kernel's minimum length)."""
    g = SlabGeometry(M, Nz, 1.0)
    mat = random_slab_material(g, REF, CONTRAST, 0.5, seed=M + 3 * Nz)
    rng = np.random.default_rng(M + Nz)
    x = rng.standard_normal(Nz * M * M * 9) + 1j * rng.standard_normal(Nz * M * M * 9)
    xt = torch.from_numpy(x.reshape(Nz, M, M, 9))
    out = []
    for flag in ("1", "0"):
        monkeypatch.setenv("MSC_G0_FUSED", flag)
        plan = SlabPlan(g, REF)
        plan.build_t0(mat, OMEGA)
        plan.build_g0(OMEGA, volume_averaged=bool(va))
        out.append((plan.matvec(xt, "complex128").cpu().numpy(), plan.nearfield_blocks()))
    assert _rel(out[0][0], out[1][0]) < 1e-13
    assert _rel(out[0][1], out[1][1]) < 1e-14


def test_bloch_matvec_compiled_lengths_vs_oracle():
    """Full (non-octant) spectrum with Lxy 16 periodic and Lz 16."""
    M, Nz = 16, 8
    g = SlabGeometry(M, Nz, 1.0)
    mat = random_slab_material(g, REF, CONTRAST, 0.5, seed=11)
    kpar = (0.011, 0.004)
    t4 = O.t0_scalars(OMEGA, 1.0, REF.alpha, REF.beta, REF.rho, mat.Dlambda, mat.Dmu, mat.Drho)
    kh = O.build_slab_kernels(M, Nz, 1.0, OMEGA, REF.alpha, REF.beta, REF.rho, periodic=True,
                              phase_xy=(kpar[0] * 2.0, kpar[1] * 2.0))
    rng = np.random.default_rng(3)
    x = rng.standard_normal(Nz * M * M * 9) + 1j * rng.standard_normal(Nz * M * M * 9)
    want = O.slab_matvec(x, t4, kh, M, Nz, periodic=True)
    plan = SlabPlan(g, REF, periodic=True)
    plan.build_t0(mat, OMEGA)
    plan.build_g0(OMEGA, kpar=kpar)
    xt = torch.from_numpy(x.reshape(Nz, M, M, 9))
    assert _rel(plan.matvec(xt, "complex128").cpu().numpy().ravel(), want) < 1e-12
    assert _rel(plan.matvec(xt, "complex64").cpu().numpy().ravel(), want) < 1e-5


def test_matvec_identity_when_T_zero():
    g = SlabGeometry(5, 3, 1.0)
    zero = MaterialContrast(0.0, 0.0, 0.0)
    plan = SlabPlan(g, REF)
    plan.build_t0(uniform_slab_material(g, REF, zero), OMEGA)
    plan.build_g0(OMEGA)
    x = torch.randn(3, 5, 5, 9, dtype=torch.complex128)
    assert_allclose(plan.matvec(x).cpu().numpy(), x.numpy(), atol=1e-14)


def test_bloch_fold_is_reference_fold_at_normal_incidence():
    g = SlabGeometry(6, 2, 1.0)
    mat = random_slab_material(g, REF, CONTRAST, 0.5, seed=2)
    x = torch.randn(2, 6, 6, 9, dtype=torch.complex128)
    ys = []
    for kp in (None, (0.0, 0.0)):
        plan = SlabPlan(g, REF, periodic=True)
        plan.build_t0(mat, OMEGA)
        plan.build_g0(OMEGA, kpar=kp)
        ys.append(plan.matvec(x).cpu().numpy())
    assert_allclose(ys[1], ys[0], rtol=1e-13, atol=1e-16)


def test_bloch_matvec_vs_oracle():
    M, Nz = 6, 2
    g = SlabGeometry(M, Nz, 1.0)
    mat = random_slab_material(g, REF, CONTRAST, 0.5, seed=4)
    kpar = (0.013, -0.007)
    t4 = O.t0_scalars(OMEGA, 1.0, REF.alpha, REF.beta, REF.rho, mat.Dlambda, mat.Dmu, mat.Drho)
    kh = O.build_slab_kernels(M, Nz, 1.0, OMEGA, REF.alpha, REF.beta, REF.rho, periodic=True,
                              phase_xy=(kpar[0] * 2.0, kpar[1] * 2.0))
    rng = np.random.default_rng(0)
    x = rng.standard_normal(Nz * M * M * 9) + 1j * rng.standard_normal(Nz * M * M * 9)
    want = O.slab_matvec(x, t4, kh, M, Nz, periodic=True)
    plan = SlabPlan(g, REF, periodic=True)
    plan.build_t0(mat, OMEGA)
    plan.build_g0(OMEGA, kpar=kpar)
    got = plan.matvec(torch.from_numpy(x.reshape(Nz, M, M, 9))).cpu().numpy().ravel()
    assert _rel(got, want) < 1e-12


# ---- solves ---------------------------------------------------------------------------


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("name,M,Nz,opt", [
    ("ap_P", 4, 2, {}), ("per_P", 4, 2, {"periodic": True}), ("va_P", 3, 2, {"volume_averaged": True}),
    ("ap_S", 3, 3, {}),
])
def test_small_solves_match_reference(golden, precision, name, M, Nz, opt):
    z = golden("solve_small.npz")
    ref = _medium(z)
    g = SlabGeometry(M, Nz, float(z["a"]))
    mat = SlabMaterial(z[f"{name}_dlam"], z[f"{name}_dmu"], z[f"{name}_drho"], ref)
    wt = "S" if name.endswith("S") else "P"
    res = compute_slab_scattering_gpu(g, mat, float(z["omega"]), z[f"{name}_khat"], wt, gmres_tol=1e-12,
                                      precision=precision, **opt)
    assert res.gmres_residual < 1e-12
    assert _rel(res.psi, z[f"{name}_psi"]) < 1e-10
    T = compute_slab_tmatrices(g, mat, float(z["omega"]))
    rpp = slab_rpp_periodic(res, T)
    assert abs(rpp - complex(z[f"{name}_rpp"])) <= 1e-9 * abs(complex(z[f"{name}_rpp"]))
    refl = np.array(slab_reflected_field(res, T))
    # R_PS can be orders below R_PP; its error is bounded relative to the largest amplitude
    want = z[f"{name}_refl"]
    assert_allclose(refl, want, rtol=1e-9, atol=1e-9 * np.abs(want).max())


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_headline_16x16x4_matches_reference(golden, precision):
    """16x16x4, ka 0.2, i.i.d. +-10 %, periodic, normal P, GMRES(30) to 1e-10:
    R_PP within 1e-7 of the reference's FP64 solve."""
    z = golden("slab_16x16x4.npz")
    ref = _medium(z)
    g = SlabGeometry(16, 4, float(z["a"]))
    mat = SlabMaterial(z["dlam"], z["dmu"], z["drho"], ref)
    res = compute_slab_scattering_gpu(g, mat, float(z["omega"]), KZ, "P", gmres_tol=1e-10, periodic=True,
                                      precision=precision, restart=30)
    assert res.gmres_residual < 1e-10
    assert _rel(res.psi0, z["psi0"]) < 1e-14
    assert _rel(res.psi, z["psi"]) < 1e-9
    rpp = slab_rpp_periodic(res, res.t0)
    assert abs(rpp - complex(z["rpp"])) <= 1e-7 * abs(complex(z["rpp"]))


def test_dense_direct_solution(golden):
    """GMRES on the FFT operator equals LU on the dense pairwise operator."""
    z = golden("dense_m3_nz2.npz")
    ref = _medium(z)
    g = SlabGeometry(3, 2, float(z["a"]))
    mat = SlabMaterial(z["dlam"], z["dmu"], z["drho"], ref)
    res = compute_slab_scattering_gpu(g, mat, float(z["omega"]), KZ, "P", gmres_tol=1e-13)
    assert _rel(res.psi, z["psi"]) < 1e-11


def test_zero_contrast_gives_incident_field():
    g = SlabGeometry(4, 2, 1.0)
    mat = uniform_slab_material(g, REF, MaterialContrast(0.0, 0.0, 0.0))
    for per in (False, True):
        res = compute_slab_scattering_gpu(g, mat, OMEGA, KZ, periodic=per)
        assert_allclose(res.psi, res.psi0, atol=1e-12)
        assert abs(slab_rpp_periodic(res, res.t0)) < 1e-20


def test_single_scatterer_centre_unchanged():
    g = SlabGeometry(3, 1, 1.0)
    z = np.zeros((1, 3, 3))
    dl, dm, dr = z.copy(), z.copy(), z.copy()
    dl[0, 1, 1], dm[0, 1, 1], dr[0, 1, 1] = CONTRAST.Dlambda, CONTRAST.Dmu, CONTRAST.Drho
    res = compute_slab_scattering_gpu(g, SlabMaterial(dl, dm, dr, REF), OMEGA, KZ, gmres_tol=1e-10)
    assert_allclose(res.psi[0, 1, 1], res.psi0[0, 1, 1], atol=1e-10)
    assert np.any(np.abs(res.psi[0, 0, 0] - res.psi0[0, 0, 0]) > 1e-15)


def test_born_scaling():
    g = SlabGeometry(4, 2, 1.0)
    w = MaterialContrast(2e5, 1e5, 0.01)
    w2 = MaterialContrast(4e5, 2e5, 0.02)
    r1 = compute_slab_scattering_gpu(g, uniform_slab_material(g, REF, w), OMEGA, KZ, gmres_tol=1e-12)
    r2 = compute_slab_scattering_gpu(g, uniform_slab_material(g, REF, w2), OMEGA, KZ, gmres_tol=1e-12)
    s1, s2 = r1.psi - r1.psi0, r2.psi - r2.psi0
    m = np.abs(s1) > 1e-15
    assert_allclose(np.abs(s2[m] / s1[m]), 2.0, rtol=0.02)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_bloch_oblique_rpp_vs_kennett_and_oracle(golden, precision):
    """Oblique P incidence (p = 1e-4 s/m, 30 degrees) on a uniform layer through the
    Bloch-phased periodic solve: R_PP in both moment forms equals the oracle's, and
    the plane-wave form is within 1% of the Kennett layer reflectivity."""
    z = golden("kennett.npz")
    ref = _medium(z)
    om, a, M = float(z["omega"]), 1.0, 4
    p = float(z["ps"][-1])
    g = SlabGeometry(M, 1, a)
    for ic in (0, 1):
        dl, dm, dr = (np.full((1, M, M), v) for v in z["contrasts"][ic])
        mat = SlabMaterial(dl, dm, dr, ref)
        s = p * ref.alpha
        kh = np.array([np.sqrt(1.0 - s * s), s, 0.0])
        res = compute_slab_scattering_gpu(g, mat, om, kh, "P", gmres_tol=1e-11, periodic=True, bloch=True,
                                          precision=precision)
        phase = (om * p * 2.0 * a, 0.0)
        ora = O.solve(M, 1, a, ref.alpha, ref.beta, ref.rho, dl, dm, dr, om, kh, "P", gmres_tol=1e-12,
                      periodic=True, phase_xy=phase)
        demod = O.bloch_demodulation(M, 1, a, phase)
        for moment in ("reference", "plane_wave"):
            got = slab_rpp_periodic(res, res.t0, p=p, moment=moment)
            want = O.rpp_periodic(ora["psi"], ora["t4"], M, 1, a, om, ref.alpha, ref.rho, p=p, demod=demod,
                                  moment=moment)
            assert abs(got - want) <= 1e-7 * abs(want)
        K = z[f"rpp_p_c{ic}_H2"][-1]
        assert abs(slab_rpp_periodic(res, res.t0, p=p, moment="plane_wave") - K) < 0.01 * abs(K)
    with pytest.raises(ValueError, match="moment"):
        slab_rpp_periodic(res, res.t0, p=p, moment="bogus")


def test_oblique_random_solve_vs_oracle():
    """Aperiodic oblique SV at ka 0.5 with +-20 % i.i.d. contrast: both precisions."""
    ref = ReferenceMedium(3000.0, 1732.0, 2500.0)
    g = SlabGeometry(10, 3, 1.0)
    om = 0.5 * ref.beta
    mat = uniform_random_material(g, ref, 0.2, seed=3)
    kh = np.array([np.cos(0.4), np.sin(0.4), 0.0])
    ora = O.solve(10, 3, 1.0, ref.alpha, ref.beta, ref.rho, mat.Dlambda, mat.Dmu, mat.Drho, om, kh, "S", 1e-13,
                  restart=30)
    for prec in ("mixed", "fp64"):
        for ortho in ("auto", "cgs1", "cgs2"):
            res = compute_slab_scattering_gpu(g, mat, om, kh, "S", gmres_tol=1e-11, precision=prec, restart=30,
                                              ortho=ortho)
            assert res.gmres_residual < 1e-11, (prec, ortho)
            assert _rel(res.psi, ora["psi"]) < 1e-9, (prec, ortho)


def test_nonconvergence_warns_and_reports():
    g = SlabGeometry(6, 3, 1.0)
    mat = random_slab_material(g, REF, CONTRAST, 0.5, seed=1)
    with pytest.warns(UserWarning, match="did not converge"):
        res = compute_slab_scattering_gpu(g, mat, OMEGA, KZ, gmres_tol=1e-14, max_iter=3)
    assert res.stats["n_matvec"] - res.stats["n_matvec64"] <= 3
    assert res.gmres_residual > 1e-14


def test_input_validation():
    g = SlabGeometry(2, 1, 1.0)
    mat = uniform_slab_material(g, REF, CONTRAST)
    with pytest.raises(ValueError, match="wave_type"):
        compute_slab_scattering_gpu(g, mat, OMEGA, KZ, "X")
    with pytest.raises(ValueError, match="bloch"):
        compute_slab_scattering_gpu(g, mat, OMEGA, KZ, bloch=True)
    with pytest.raises(ValueError, match="omega"):
        compute_slab_scattering_gpu(g, mat, -1.0, KZ)
    with pytest.raises(ValueError):
        compute_slab_scattering_gpu(g, mat, OMEGA, KZ, device="cpu")


def test_run_from_config_matches_oracle():
    """The YAML entry (reference schema) solves the same slab as the oracle."""
    from pathlib import Path

    from multiplescatteringcalculations_b200.solver_config import build_material, load_config, run_from_config

    cfg = load_config(Path(__file__).resolve().parent / "configs" / "slab_small.yml")
    res = run_from_config(cfg)
    mat = build_material(cfg)
    ora = O.solve(6, 3, 1.0, 5000.0, 3000.0, 2500.0, mat.Dlambda, mat.Dmu, mat.Drho, 150.0, KZ, "P", 1e-13)
    assert res.gmres_residual < 1e-10
    assert _rel(res.psi, ora["psi"]) < 1e-9


@pytest.mark.parametrize("M,Nz,periodic", [(12, 3, False), (64, 16, False), (16, 5, True)])
def test_matvec_soa_equals_matvec(M, Nz, periodic):
    """msc_matvec_soa applies the same operator on the component-major layout
    (9, N_z, M, M) that GMRES keeps its vectors in."""
    import ctypes as C

    from multiplescatteringcalculations_b200 import SlabPlan, _native, random_slab_material

    lib = _native.load()
    g = SlabGeometry(M, Nz, 1.0)
    mat = random_slab_material(g, REF, CONTRAST, 0.5, seed=M + Nz)
    plan = SlabPlan(g, REF, periodic=periodic)
    plan.build_t0(mat, OMEGA)
    plan.build_g0(OMEGA)
    for prec, dt, tol in ((_native.MSC_COMPLEX64, torch.complex64, 1e-6), (_native.MSC_COMPLEX128, torch.complex128,
                                                                            1e-13)):
        x = torch.randn(Nz, M, M, 9, dtype=dt, device=plan.device)
        y_ref = plan.matvec(x, "complex64" if prec == _native.MSC_COMPLEX64 else "complex128")
        xs = x.permute(3, 0, 1, 2).contiguous()
        ys = torch.empty_like(xs)
        assert lib.msc_matvec_soa(plan.handle, C.c_void_p(xs.data_ptr()), C.c_void_p(ys.data_ptr()), prec) == 0
        got = ys.permute(1, 2, 3, 0).cpu().numpy()
        assert _rel(got, y_ref.cpu().numpy()) < tol
    plan.close()


@pytest.mark.parametrize("M,Nz,periodic", [(64, 3, True), (128, 2, True), (256, 2, True), (100, 2, False)])
def test_complex64_matvec_large_planes(M, Nz, periodic):
    """Planes the fused plane kernels do not hold: the inverse y pass on the register
    four-step engine (Ly = 64, 128, 256; 100 x 100 aperiodic pads to 200, the shared-
    memory tiles) against the complex128 path, and at M = 64 against the oracle."""
    from multiplescatteringcalculations_b200 import SlabPlan, random_slab_material

    g = SlabGeometry(M, Nz, 1.0)
    mat = random_slab_material(g, REF, CONTRAST, 0.5, seed=M)
    plan = SlabPlan(g, REF, periodic=periodic)
    plan.build_t0(mat, OMEGA)
    plan.build_g0(OMEGA)
    torch.manual_seed(M)
    x = torch.randn(Nz, M, M, 9, dtype=torch.complex128, device=plan.device)
    y64 = plan.matvec(x, "complex128").cpu().numpy()
    y32 = plan.matvec(x, "complex64").cpu().numpy()
    assert _rel(y32, y64) < 5e-6
    if M == 64:
        t4 = O.t0_scalars(OMEGA, 1.0, REF.alpha, REF.beta, REF.rho, mat.Dlambda, mat.Dmu, mat.Drho)
        kh = O.build_slab_kernels(M, Nz, 1.0, OMEGA, REF.alpha, REF.beta, REF.rho, periodic=periodic)
        want = O.slab_matvec(x.cpu().numpy().ravel(), t4, kh, M, Nz, periodic=periodic).reshape(y64.shape)
        assert _rel(y64, want) < 1e-10
        assert _rel(y32, want) < 5e-6
    plan.close()


def test_autotuned_lateral_length():
    """Lxy="auto" (-1 in the C descriptor): the plan takes the smallest 2,3,5,7-smooth
    length >= 2M - 1 or the next power of two, whichever runs the complex64 operator
    faster; the choice is remembered for the shape, and the operator matches the oracle
    either way. Values below -1 are refused; periodic plans keep Lxy = M."""
    M, Nz = 24, 6
    g = SlabGeometry(M, Nz, 1.0)
    mat = random_slab_material(g, REF, CONTRAST, 0.5, seed=11)
    plan = SlabPlan(g, REF, Lxy="auto")
    L = plan.fft_sizes()[1]
    assert L in (48, 64)
    again = SlabPlan(g, REF, Lxy="auto")
    assert again.fft_sizes()[1] == L
    again.close()
    plan.build_t0(mat, OMEGA)
    plan.build_g0(OMEGA)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(Nz * M * M * 9) + 1j * rng.standard_normal(Nz * M * M * 9)
    t4 = O.t0_scalars(OMEGA, 1.0, REF.alpha, REF.beta, REF.rho, mat.Dlambda, mat.Dmu, mat.Drho)
    kh = O.build_slab_kernels(M, Nz, 1.0, OMEGA, REF.alpha, REF.beta, REF.rho)
    want = O.slab_matvec(x, t4, kh, M, Nz)
    xt = torch.from_numpy(x.reshape(Nz, M, M, 9))
    assert _rel(plan.matvec(xt, "complex128").cpu().numpy().ravel(), want) < 1e-12
    assert _rel(plan.matvec(xt, "complex64").cpu().numpy().ravel(), want) < 5e-6
    plan.close()
    with pytest.raises(ValueError):
        SlabPlan(g, REF, Lxy=-2)
    assert SlabPlan(SlabGeometry(8, 2, 1.0), REF, periodic=True, Lxy="auto").fft_sizes()[1] == 8
