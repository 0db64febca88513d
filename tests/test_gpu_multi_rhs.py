"""Several right-hand sides at once (msc_matvec_multi, msc_solve_multi) against the
single-field operator and solver, which the oracle pins (tests/test_gpu_parity.py).

The multi-RHS matvec stages each block's slice of the G0 spectrum once and applies it to
the same columns of every field; it must equal the single-field application field by
field, for the fused plane passes (aperiodic 64 x 64 planes), the generic passes
(periodic, odd radices) and both precisions. The stacked solve must bound every right-
hand side's FP64 relative residual by tol and give each field to that accuracy.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from oracle import slab_oracle as O

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from multiplescatteringcalculations_b200 import (  # noqa: E402
    MaterialContrast,
    ReferenceMedium,
    SlabGeometry,
    SlabPlan,
    _native,
    random_slab_material,
)

REF = ReferenceMedium(5000.0, 3000.0, 2500.0)
CON = MaterialContrast(2e9, 1e9, 100.0)


def _rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


def _plan(M, Nz, periodic, om, seed=1):
    g = SlabGeometry(M, Nz, 1.0)
    mat = random_slab_material(g, REF, CON, 0.5, seed=seed)
    plan = SlabPlan(g, REF, periodic=periodic)
    plan.build_t0(mat, om)
    plan.build_g0(om)
    return g, mat, plan


@pytest.mark.parametrize("M,Nz,periodic,R", [(32, 16, False, 3), (12, 3, False, 9), (15, 5, True, 2), (8, 4, True, 1)])
def test_matvec_multi_equals_single(M, Nz, periodic, R):
    lib = _native.load()
    g, _, plan = _plan(M, Nz, periodic, 300.0)
    for prec, dt, tol in ((_native.MSC_COMPLEX64, torch.complex64, 1e-6),
                          (_native.MSC_COMPLEX128, torch.complex128, 1e-13)):
        x = torch.randn(R, 9, Nz, M, M, dtype=dt, device=plan.device)
        y = plan.matvec_multi(x, "complex64" if prec == _native.MSC_COMPLEX64 else "complex128")
        for r in range(R):
            xr = x[r].contiguous()
            yr = torch.empty_like(xr)
            assert lib.msc_matvec_soa(plan.handle, C.c_void_p(xr.data_ptr()), C.c_void_p(yr.data_ptr()), prec) == 0
            assert _rel(y[r].cpu().numpy(), yr.cpu().numpy()) < tol
        # twice in a row: nothing carried between calls
        assert torch.equal(plan.matvec_multi(x, "complex64" if prec == 0 else "complex128"), y)
    with pytest.raises(ValueError):
        _native.check(lib.msc_matvec_multi(plan.handle, 0, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), 1),
                      "msc_matvec_multi")
    plan.close()


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("periodic", [False, True])
def test_solve_multi_matches_single_solves(precision, periodic):
    M, Nz, om = 12, 4, 900.0
    g, mat, plan = _plan(M, Nz, periodic, om, seed=7)
    dirs = [np.array([1.0, 0.0, 0.0]), np.array([np.cos(0.4), np.sin(0.4), 0.0]),
            np.array([np.cos(0.7), 0.0, np.sin(0.7)])]
    B = torch.stack([plan.incident(om, d, w) for d in dirs for w in ("P", "S")])
    B[3] *= 1e-3  # uneven norms: each right-hand side is held to tol on its own
    tol = 1e-10
    X, stats = plan.solve_multi(B, tol=tol, max_iter=2000, precision=precision)
    assert len(stats) == B.shape[0]
    t4 = O.t0_scalars(om, 1.0, REF.alpha, REF.beta, REF.rho, mat.Dlambda, mat.Dmu, mat.Drho)
    kh = O.build_slab_kernels(M, Nz, 1.0, om, REF.alpha, REF.beta, REF.rho, periodic=periodic)
    for r in range(B.shape[0]):
        assert stats[r]["status"] == 0 and stats[r]["residual"] <= tol
        x1, st1 = plan.solve(B[r], tol=1e-12, max_iter=2000, precision="fp64")
        assert _rel(X[r].cpu().numpy(), x1.cpu().numpy()) < 1e-8
        # the FP64 residual reported equals the oracle operator's on the returned field
        b = B[r].cpu().numpy().ravel()
        res = np.linalg.norm(O.slab_matvec(X[r].cpu().numpy().ravel(), t4, kh, M, Nz, periodic=periodic) - b)
        assert res / np.linalg.norm(b) <= 2 * tol
    plan.close()


def test_solve_multi_with_the_nearfield_preconditioner():
    """Flexible GMRES on the stacked system: the preconditioner applies to each field."""
    M, Nz, om = 16, 6, 0.7 * 3000.0
    g, mat, plan = _plan(M, Nz, False, om, seed=9)
    B = torch.stack([plan.incident(om, np.array([1.0, 0.0, 0.0]), w) for w in ("P", "S")])
    plan.set_nearfield(2)
    X, stats = plan.solve_multi(B, tol=1e-9, max_iter=2000, precision="mixed", preconditioner="nearfield")
    X0, stats0 = plan.solve_multi(B, tol=1e-9, max_iter=2000, precision="mixed")
    for r in range(2):
        assert stats[r]["residual"] <= 1e-9 and stats0[r]["residual"] <= 1e-9
        assert stats[r]["n_precond"] > 0
        assert _rel(X[r].cpu().numpy(), X0[r].cpu().numpy()) < 1e-7
    plan.close()


def test_solve_multi_rejects_bad_arguments():
    g, mat, plan = _plan(6, 2, False, 300.0)
    B = torch.zeros(2, 2, 6, 6, 9, dtype=torch.complex128, device=plan.device)
    X, stats = plan.solve_multi(B, tol=1e-8, max_iter=10)  # zero right-hand sides: zero fields
    assert torch.count_nonzero(X) == 0 and all(s["residual"] == 0 for s in stats)
    with pytest.raises(ValueError):
        plan.solve_multi(B[0], tol=1e-8, max_iter=10)
    lib = _native.load()
    opts = _native.SolveOpts(1e-8, 10, 30, 0, 0, 0.0, 0, 0)
    for bad in (0, _native.MSC_MAX_RHS + 1):
        assert lib.msc_solve_multi(plan.handle, bad, C.c_void_p(B.data_ptr()), C.c_void_p(X.data_ptr()),
                                   C.byref(opts), None) == _native.MSC_ERR_INVALID
    plan.close()
