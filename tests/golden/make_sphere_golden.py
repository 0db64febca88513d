"""Generate the golden fixtures of the sphere FFT Foldy-Lax path from the reference.

Run from the repository root where the reference checkout is available:

    python tests/golden/make_sphere_golden.py [path-to-reference-checkout]

The path of the reference checkout comes from the argument or, without one, from
the environment variable ``MSC_REFERENCE_ROOT``. The script imports the reference package
``cubic_scattering`` read-only, runs its CPU solver ``compute_sphere_foldy_lax_fft``
(sphere_scattering_fft.py:228-330, scipy GMRES at rtol 1e-12) on small spheres and
writes ``sphere.npz`` next to this script. Nothing at test time reads the reference
checkout.
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

# (n_sub, radius, omega / (alpha or beta) * radius, wave, k_hat)
CASES = [
    (3, 0.5, ("beta", 0.05 * 0.5), "P", None),
    (5, 0.5, ("alpha", 0.1), "S", None),
    (6, 0.5, ("alpha", 0.3), "P", (0.6, 0.8, 0.0)),
]


def main(ref_root: str | None = None) -> None:
    import os

    ref_root = ref_root or os.environ.get("MSC_REFERENCE_ROOT")
    if not ref_root:
        raise SystemExit("give the reference checkout's path as the argument or in MSC_REFERENCE_ROOT")
    sys.path.insert(0, ref_root)
    from cubic_scattering.effective_contrasts import MaterialContrast, ReferenceMedium, compute_cube_tmatrix
    from cubic_scattering.resonance_tmatrix import _sub_cell_tmatrix_9x9
    from cubic_scattering.sphere_scattering_fft import compute_sphere_foldy_lax_fft

    # the reference tests' medium and contrast (tests/test_sphere_scattering_fft.py:37-38)
    ref = ReferenceMedium(alpha=5000.0, beta=3000.0, rho=2500.0)
    contrast = MaterialContrast(Dlambda=2.0e9, Dmu=1.0e9, Drho=100.0)
    out = {}
    for k, (n_sub, radius, (speed, kr), wave, k_hat) in enumerate(CASES):
        omega = kr * (ref.alpha if speed == "alpha" else ref.beta) / radius
        kh = None if k_hat is None else np.asarray(k_hat, dtype=float)
        r = compute_sphere_foldy_lax_fft(omega, radius, ref, contrast, n_sub, k_hat=kh, wave_type=wave,
                                         gmres_tol=1e-12, gmres_maxiter=500)
        T_loc = _sub_cell_tmatrix_9x9(compute_cube_tmatrix(omega, r.a_sub, ref, contrast), omega, r.a_sub)
        out[f"c{k}_n_sub"] = n_sub
        out[f"c{k}_radius"] = radius
        out[f"c{k}_omega"] = omega
        out[f"c{k}_wave"] = wave
        out[f"c{k}_k_hat"] = np.zeros(0) if kh is None else kh
        out[f"c{k}_T_comp"] = r.T_comp_9x9
        out[f"c{k}_psi_exc"] = r.psi_exc
        out[f"c{k}_centres"] = r.centres
        out[f"c{k}_a_sub"] = r.a_sub
        out[f"c{k}_T_loc"] = T_loc
    out["alpha"], out["beta"], out["rho"] = ref.alpha, ref.beta, ref.rho
    out["Dlambda"], out["Dmu"], out["Drho"] = contrast.Dlambda, contrast.Dmu, contrast.Drho
    out["n_cases"] = len(CASES)
    np.savez_compressed(HERE / "sphere.npz", **out)


if __name__ == "__main__":
    main(*sys.argv[1:])
