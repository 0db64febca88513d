"""Generate the golden fixtures of the slab path from the reference itself.

Run from the repository root where the reference checkout is available:

    python tests/golden/make_golden.py [path-to-reference-checkout]

The path of the reference checkout comes from the argument or, without one, from
the environment variable ``MSC_REFERENCE_ROOT``. The script imports the reference package
``cubic_scattering`` read-only and writes small ``.npz`` files next to this
script. Those files pin the oracle (``oracle/slab_oracle.py``) and, through it,
the CUDA path. Nothing at test time reads the reference checkout; only these
committed fixtures travel.

Inputs are seeded (``numpy.random.default_rng``), so re-running the script
reproduces the files bit for bit on the same numpy/scipy versions.
"""

from __future__ import annotations

import itertools
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def main(ref_root: str | None = None) -> None:
    import os

    ref_root = ref_root or os.environ.get("MSC_REFERENCE_ROOT")
    if not ref_root:
        raise SystemExit("give the reference checkout's path as the argument or in MSC_REFERENCE_ROOT")
    sys.path.insert(0, ref_root)
    from cubic_scattering import slab_scattering as ss
    from cubic_scattering.effective_contrasts import MaterialContrast, ReferenceMedium, compute_cube_tmatrix
    from cubic_scattering.inter_voxel_propagator import inter_voxel_propagator_9x9
    from cubic_scattering.kennett_layers import IsotropicLayer, LayerStack, kennett_layers
    from cubic_scattering.resonance_tmatrix import _propagator_block_9x9, _sub_cell_tmatrix_9x9

    # Reference test fixture medium (tests/test_slab_scattering.py:31-43)
    ref = ReferenceMedium(alpha=5000.0, beta=3000.0, rho=2500.0)
    contrast = MaterialContrast(Dlambda=2e9, Dmu=1e9, Drho=100.0)
    a = 1.0
    omega = 0.05 * ref.beta / a

    # 1. VA nearest-neighbour blocks: all 26 offsets, orders 0..3, three frequencies
    offs = [R for R in itertools.product([-1, 0, 1], repeat=3) if R != (0, 0, 0)]
    va = np.zeros((4, 3, 26, 9, 9), dtype=complex)
    oms = np.array([0.0, 150.0, 900.0])
    for no in range(4):
        for io, om in enumerate(oms):
            for ir, R in enumerate(offs):
                va[no, io, ir] = inter_voxel_propagator_9x9(R, ref.alpha, ref.beta, ref.rho, om, no)
    np.savez_compressed(HERE / "va_nn.npz", offsets=np.array(offs), omegas=oms, blocks=va,
                        medium=np.array([ref.alpha, ref.beta, ref.rho]))

    # 2. Point propagator at seeded separations, incl. near field
    rng = np.random.default_rng(7)
    r = np.concatenate([rng.standard_normal((24, 3)) * 3.0, rng.standard_normal((8, 3)) * 0.05])
    pb = np.array([_propagator_block_9x9(x, omega, ref) for x in r])
    pb2 = np.array([_propagator_block_9x9(x, 900.0, ref) for x in r])
    np.savez_compressed(HERE / "point_propagator.npz", r=r, omegas=np.array([omega, 900.0]),
                        blocks=np.stack([pb, pb2]), medium=np.array([ref.alpha, ref.beta, ref.rho]))

    # 3. T0 9x9 for several (omega, a, contrast)
    cases = [(omega, 1.0, 2e9, 1e9, 100.0), (3000.0, 0.5, -1e9, 5e8, -200.0), (866.0, 2.0, 7.5e8, -7.5e8, 250.0),
             (346.4, 1.0, 0.0, 0.0, 0.0)]
    t0 = np.array([
        _sub_cell_tmatrix_9x9(compute_cube_tmatrix(om, aa, ref, MaterialContrast(dl, dm, dr)), om, aa)
        for om, aa, dl, dm, dr in cases
    ])
    np.savez_compressed(HERE / "t0.npz", cases=np.array(cases), T=t0, medium=np.array([ref.alpha, ref.beta, ref.rho]))

    # 4. Slab kernels (xy-FFT'd) M=3, N_z=2 for periodic x va
    kd = {}
    for per in (False, True):
        for vav in (False, True):
            g = ss.SlabGeometry(M=3, N_z=2, a=a)
            kd[f"k_p{int(per)}_va{int(vav)}"] = ss._build_slab_kernels(g, omega, ref, volume_averaged=vav, periodic=per)
    np.savez_compressed(HERE / "kernels_m3_nz2.npz", omega=omega, a=a, medium=np.array([ref.alpha, ref.beta, ref.rho]),
                        **kd)

    # 5. Matvec: random psi on a random binary medium, M=3, N_z=2 (and M=2,N_z=3)
    md = {}
    for M, Nz in ((3, 2), (2, 3)):
        g = ss.SlabGeometry(M=M, N_z=Nz, a=a)
        mat = ss.random_slab_material(g, ref, contrast, 0.5, seed=11)
        T = ss.compute_slab_tmatrices(g, mat, omega)
        rng = np.random.default_rng(123)
        x = rng.standard_normal(g.n_cubes * 9) + 1j * rng.standard_normal(g.n_cubes * 9)
        for per in (False, True):
            kh = ss._build_slab_kernels(g, omega, ref, periodic=per)
            md[f"y_M{M}_Nz{Nz}_p{int(per)}"] = ss._slab_matvec(x, T, kh, g, periodic=per)
        md[f"x_M{M}_Nz{Nz}"] = x
        md[f"dlam_M{M}_Nz{Nz}"] = mat.Dlambda
        md[f"dmu_M{M}_Nz{Nz}"] = mat.Dmu
        md[f"drho_M{M}_Nz{Nz}"] = mat.Drho
    np.savez_compressed(HERE / "matvec_small.npz", omega=omega, a=a, medium=np.array([ref.alpha, ref.beta, ref.rho]),
                        **md)

    # 6. Incident fields
    g = ss.SlabGeometry(M=3, N_z=2, a=a)
    inc = {}
    dirs = [(1.0, 0.0, 0.0), (np.cos(0.35), np.sin(0.35), 0.0), (np.cos(0.5), 0.2, np.sin(0.4))]
    for i, kh in enumerate(dirs):
        for w in ("P", "S"):
            inc[f"psi0_{i}_{w}"] = ss._build_slab_incident_field(g, omega, ref, np.array(kh), w)
    np.savez_compressed(HERE / "incident.npz", dirs=np.array(dirs), omega=omega, a=a,
                        medium=np.array([ref.alpha, ref.beta, ref.rho]), **inc)

    # 7. Small full solves through the reference API at tol 1e-12
    sol = {}
    small = [
        ("ap_P", dict(M=4, N_z=2), dict(k_hat=(1.0, 0.0, 0.0), wave_type="P"), dict()),
        ("per_P", dict(M=4, N_z=2), dict(k_hat=(1.0, 0.0, 0.0), wave_type="P"), dict(periodic=True)),
        ("va_P", dict(M=3, N_z=2), dict(k_hat=(1.0, 0.0, 0.0), wave_type="P"), dict(volume_averaged=True)),
        ("ap_S", dict(M=3, N_z=3), dict(k_hat=(np.cos(0.5), np.sin(0.5), 0.0), wave_type="S"), dict()),
    ]
    for name, gk, ik, opt in small:
        g = ss.SlabGeometry(a=a, **gk)
        mat = ss.random_slab_material(g, ref, contrast, 0.5, seed=5)
        res = ss.compute_slab_scattering(g, mat, omega, np.array(ik["k_hat"]), ik["wave_type"], gmres_tol=1e-12, **opt)
        T = ss.compute_slab_tmatrices(g, mat, omega)
        sol[f"{name}_psi"] = res.psi
        sol[f"{name}_dlam"] = mat.Dlambda
        sol[f"{name}_dmu"] = mat.Dmu
        sol[f"{name}_drho"] = mat.Drho
        sol[f"{name}_rpp"] = ss.slab_rpp_periodic(res, T)
        sol[f"{name}_refl"] = np.array(ss.slab_reflected_field(res, T))
        sol[f"{name}_khat"] = np.array(ik["k_hat"])
    np.savez_compressed(HERE / "solve_small.npz", omega=omega, a=a, medium=np.array([ref.alpha, ref.beta, ref.rho]),
                        **sol)

    # 8. The CPU-runnable headline case: 16x16x4, ka = 0.2 (a = half-width), i.i.d. U(+-10%) of
    #    (lambda0, mu0, rho0) drawn in that order from default_rng(0), periodic, normal P.
    ref1 = ReferenceMedium(alpha=3000.0, beta=1732.0, rho=2500.0)
    M, Nz = 16, 4
    om1 = 0.2 * ref1.beta / a
    rng = np.random.default_rng(0)
    shp = (Nz, M, M)
    dl = rng.uniform(-0.10, 0.10, shp) * ref1.lam
    dm = rng.uniform(-0.10, 0.10, shp) * ref1.mu
    dr = rng.uniform(-0.10, 0.10, shp) * ref1.rho
    g = ss.SlabGeometry(M=M, N_z=Nz, a=a)
    mat = ss.SlabMaterial(Dlambda=dl, Dmu=dm, Drho=dr, ref=ref1)
    res = ss.compute_slab_scattering(g, mat, om1, np.array([1.0, 0.0, 0.0]), "P", gmres_tol=1e-12, periodic=True)
    T = ss.compute_slab_tmatrices(g, mat, om1)
    np.savez_compressed(HERE / "slab_16x16x4.npz", psi=res.psi, psi0=res.psi0, dlam=dl, dmu=dm, drho=dr,
                        omega=om1, a=a, medium=np.array([ref1.alpha, ref1.beta, ref1.rho]),
                        rpp=ss.slab_rpp_periodic(res, T), n_matvec=res.n_gmres_iter, residual=res.gmres_residual)

    # 9. Kennett reflectivity of a uniform layer (normal and oblique p) for physics checks
    kn = {}
    cts = [MaterialContrast(2e9 * 1e-4, 1e9 * 1e-4, 100.0 * 1e-4), contrast]
    for ic, ct in enumerate(cts):
        for H in (2.0, 4.0):
            kn[f"rpp0_c{ic}_H{int(H)}"] = ss.kennett_reference_rpp(ref, ct, H, omega)
    lam_bg = ref.rho * (ref.alpha**2 - 2.0 * ref.beta**2)
    mu_bg = ref.rho * ref.beta**2
    ps = np.array([0.0, 0.5e-4, 1.0e-4])
    for ic, ct in enumerate(cts):
        lp, mp, rp = lam_bg + ct.Dlambda, mu_bg + ct.Dmu, ref.rho + ct.Drho
        stack = LayerStack(layers=[
            IsotropicLayer(alpha=ref.alpha, beta=ref.beta, rho=ref.rho, thickness=100.0),
            IsotropicLayer(alpha=float(np.sqrt((lp + 2 * mp) / rp)), beta=float(np.sqrt(mp / rp)), rho=rp,
                           thickness=2.0),
            IsotropicLayer(alpha=ref.alpha, beta=ref.beta, rho=ref.rho, thickness=np.inf),
        ])
        kn[f"rpp_p_c{ic}_H2"] = np.array([complex(kennett_layers(stack, p=float(p), omega=np.array([omega])).RPP[0])
                                          for p in ps])
    np.savez_compressed(HERE / "kennett.npz", omega=omega, ps=ps, medium=np.array([ref.alpha, ref.beta, ref.rho]),
                        contrasts=np.array([[c.Dlambda, c.Dmu, c.Drho] for c in cts]), **kn)

    # 10. Dense direct solve (the reference test's _direct_matvec operator) at M=3, N_z=2
    g = ss.SlabGeometry(M=3, N_z=2, a=a)
    mat = ss.random_slab_material(g, ref, contrast, 0.5, seed=9)
    T = ss.compute_slab_tmatrices(g, mat, omega)
    n = g.n_cubes * 9
    cen = g.all_centres().reshape(-1, 3)
    Tn = T.reshape(-1, 9, 9)
    A = np.eye(n, dtype=complex)
    for i in range(g.n_cubes):
        for j in range(g.n_cubes):
            if i != j:
                A[9 * i:9 * i + 9, 9 * j:9 * j + 9] -= _propagator_block_9x9(cen[i] - cen[j], omega, ref) @ Tn[j]
    b = ss._build_slab_incident_field(g, omega, ref, np.array([1.0, 0.0, 0.0]), "P").ravel()
    np.savez_compressed(HERE / "dense_m3_nz2.npz", psi=np.linalg.solve(A, b).reshape(2, 3, 3, 9), dlam=mat.Dlambda,
                        dmu=mat.Dmu, drho=mat.Drho, omega=omega, a=a, medium=np.array([ref.alpha, ref.beta, ref.rho]))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main(*sys.argv[1:])
