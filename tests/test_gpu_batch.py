"""Batched solves (msc_batch_solve) on the GPU: every item of a batch of uneven
slabs equals its own single solve, with any number of workers, and a failing item
leaves the others intact."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from multiplescatteringcalculations_b200 import (  # noqa: E402
    BatchProblem,
    ReferenceMedium,
    SlabGeometry,
    compute_slab_scattering_batch,
    compute_slab_scattering_gpu,
    slab_rpp_periodic,
    uniform_random_material,
)

REF = ReferenceMedium(3000.0, 1732.0, 2500.0)


def _problems(n, seed=0):
    """Uneven slabs: M, N_z, ka, angle, wave, periodicity and Bloch phase drawn per item."""
    r = np.random.default_rng(seed)
    out = []
    for i in range(n):
        M = int(r.choice([4, 6, 8, 12, 16]))
        Nz = int(r.integers(1, 6))
        g = SlabGeometry(M, Nz, 1.0)
        mat = uniform_random_material(g, REF, 0.2, seed=100 + i)
        th = r.uniform(0, np.deg2rad(40))
        per = bool(r.random() < 0.5)
        out.append(BatchProblem(g, mat, r.uniform(0.1, 1.0) * REF.beta, np.array([np.cos(th), np.sin(th), 0.0]),
                                "P" if r.random() < 0.5 else "S", periodic=per, bloch=per and bool(r.random() < 0.5)))
    return out


@pytest.mark.parametrize("workers", [0, 1, 3])
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_items_equal_single_solves(workers, precision):
    probs = _problems(10, seed=workers)
    sols, info = compute_slab_scattering_batch(probs, gmres_tol=1e-11, max_iter=2000, precision=precision,
                                               workers=workers)
    assert info["workers"] >= 1
    for pr, s in zip(probs, sols):
        assert s.status == 0 and s.gmres_residual < 1e-11
        one = compute_slab_scattering_gpu(pr.geometry, pr.material, pr.omega, pr.k_hat, pr.wave_type,
                                          gmres_tol=1e-11, max_iter=2000, periodic=pr.periodic, bloch=pr.bloch,
                                          precision=precision)
        assert np.linalg.norm(s.psi - one.psi) <= 1e-9 * np.linalg.norm(one.psi)
        p = 0.0
        if pr.bloch:
            kh = pr.k_hat / np.linalg.norm(pr.k_hat)
            p = np.hypot(kh[1], kh[2]) / (REF.alpha if pr.wave_type == "P" else REF.beta)
        want = slab_rpp_periodic(one, one.t0, p=p)
        assert abs(s.rpp - want) <= 1e-8 * max(abs(want), 1e-30)


def test_batch_failing_item_is_isolated():
    probs = _problems(5, seed=7)
    probs[2] = BatchProblem(SlabGeometry(4, 2, 1.0), _problems(1, seed=9)[0].material, 500.0, np.array([1.0, 0, 0]))
    if probs[2].material.Dlambda.shape != (2, 4, 4):
        with pytest.raises(ValueError):
            compute_slab_scattering_batch(probs)
    probs = _problems(5, seed=7)
    probs[1].material.ref = ReferenceMedium(1000.0, 2000.0, 2500.0)  # alpha < beta: the plan is refused
    with pytest.warns(UserWarning, match="did not converge or failed"):
        sols, _ = compute_slab_scattering_batch(probs, gmres_tol=1e-10, workers=2)
    assert sols[1].status < 0
    for i in (0, 2, 3, 4):
        assert sols[i].status == 0 and sols[i].gmres_residual < 1e-10


def test_batch_without_fields_and_with_the_nearfield_preconditioner():
    probs = _problems(6, seed=3)
    sols, _ = compute_slab_scattering_batch(probs, gmres_tol=1e-10, return_fields=False, preconditioner="nearfield")
    for s in sols:
        assert s.psi is None and s.status == 0 and s.gmres_residual < 1e-10


@pytest.mark.parametrize("volume_averaged", [False, True])
def test_frequency_sweep_matches_oracle_per_frequency(volume_averaged):
    """compute_slab_rpp_sweep serves the frequency loop of the reference's ocean-bottom
    model (ocean_bottom.py:290-307): one periodic oblique slab per frequency, R_PP at the
    incidence slowness p by the reference's Weyl sum; each frequency against the
    oracle's FP64 solve and R_PP."""
    from multiplescatteringcalculations_b200 import compute_slab_rpp_sweep

    from oracle import slab_oracle as O

    ref = ReferenceMedium(3000.0, 1732.0, 2500.0)
    g = SlabGeometry(8, 3, 1.0)
    mat = uniform_random_material(g, ref, 0.15, seed=11)
    th = np.deg2rad(25.0)
    k_hat = np.array([np.cos(th), np.sin(th), 0.0])
    p = np.sin(th) / ref.alpha
    omegas = np.array([0.1, 0.25, 0.4, 0.6]) * ref.beta
    sw = compute_slab_rpp_sweep(g, mat, omegas, k_hat, p, gmres_tol=1e-11, max_iter=2000,
                                volume_averaged=volume_averaged, return_fields=True)
    assert list(sw.status) == [0] * len(omegas)
    for i, w in enumerate(omegas):
        ora = O.solve(8, 3, 1.0, ref.alpha, ref.beta, ref.rho, mat.Dlambda, mat.Dmu, mat.Drho, w, k_hat, "P",
                      1e-13, 2000, periodic=True, restart=30, volume_averaged=volume_averaged)
        rpp_o = O.rpp_periodic(ora["psi"], ora["t4"], 8, 3, 1.0, w, ref.alpha, ref.rho, p=p)
        assert np.linalg.norm(sw.psi[i] - ora["psi"]) <= 1e-9 * np.linalg.norm(ora["psi"])
        assert abs(sw.rpp[i] - rpp_o) <= 1e-8 * abs(rpp_o)
    with pytest.raises(ValueError):
        compute_slab_rpp_sweep(g, mat, [], k_hat, p)
    with pytest.raises(ValueError):
        compute_slab_rpp_sweep(g, mat, omegas, k_hat, -1.0)
