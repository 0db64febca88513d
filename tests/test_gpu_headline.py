"""The benchmark's headline slab against the oracle's FP64 CPU solve.

The slab is exactly the one the default benchmark times: 64 x 64 x 16 cubes (589,824
unknowns), a = 1 m half-width, ka = 0.5 (omega = 0.5 beta / a), P plane wave at 20
degrees in the x-z plane, contrasts from a Gaussian random field (correlation length 3
cells, std 15 %, seed 1000), aperiodic. The GPU solves to an FP64 true relative
residual of 1e-10 in mixed precision (complex64 GMRES(30) inside FP64 refinement) and
in plain FP64; the oracle (the reference's numpy/scipy algorithm, scipy GMRES(30))
solves to 1e-12. Both GPU fields must lie within 1e-8 of the oracle's and R_PP (the
reference's Weyl-sum formula) within 1e-7, the bounds the headline is stated with.
The oracle takes about 20-40 s on the host's cores.
"""

import os

import numpy as np
import pytest
import torch

from oracle import slab_oracle as O

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from multiplescatteringcalculations_b200 import (  # noqa: E402
    ReferenceMedium,
    SlabGeometry,
    compute_slab_scattering_gpu,
    gaussian_random_field_material,
    slab_rpp_periodic,
)

REF = ReferenceMedium(3000.0, 1732.0, 2500.0)


def _rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


@pytest.fixture(scope="module")
def headline():
    geom = SlabGeometry(64, 16, 1.0)
    mat = gaussian_random_field_material(geom, REF, correlation_length=3.0, std=0.15, seed=1000)
    th = np.deg2rad(20.0)
    kh = np.array([np.cos(th), np.sin(th), 0.0])
    omega = 0.5 * REF.beta / geom.a
    ora = O.solve(64, 16, 1.0, REF.alpha, REF.beta, REF.rho, mat.Dlambda, mat.Dmu, mat.Drho, omega, kh, "P", 1e-12,
                  2000, periodic=False, restart=30, threads=os.cpu_count() or 1)
    assert ora["residual"] < 1e-11
    rpp = O.rpp_periodic(ora["psi"], ora["t4"], 64, 16, 1.0, omega, REF.alpha, REF.rho)
    return geom, mat, kh, omega, ora, rpp


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_headline_slab_matches_oracle(headline, precision):
    geom, mat, kh, omega, ora, rpp_o = headline
    res = compute_slab_scattering_gpu(geom, mat, omega, kh, "P", gmres_tol=1e-10, max_iter=1000, precision=precision)
    assert res.gmres_residual <= 1e-10
    assert _rel(res.psi0, ora["psi0"]) < 1e-13
    assert _rel(res.psi, ora["psi"]) < 1e-8
    rpp = slab_rpp_periodic(res, res.t0)
    assert abs(rpp - rpp_o) <= 1e-7 * abs(rpp_o)
