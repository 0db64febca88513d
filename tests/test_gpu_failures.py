"""Failure paths on the GPU, made on the host without faulting the device.

* Non-finite input: NaN contrasts make T0 NaN; the solve detects the non-finite
  residual and returns MSC_ERR_NONFINITE through msc_solve, and a batch item with NaN
  contrasts fails alone with that status while its neighbours converge.
* A bounded wait that runs out: the tensor-core stencil waits on mbarriers with the
  plan's limit (msc_plan_set_wait_limit). With inject = 1 it also waits on an mbarrier
  that nothing completes (a flag nothing sets); that wait gives up after the limit, the
  kernel drains its copies and MMAs in flight, frees its tensor memory and returns, the
  timeout reaches the host through the plan's status word (msc_plan_status,
  MSC_ERR_TIMEOUT from msc_solve), and the same plan works again once the injection is
  off and the default limit is back.
"""

import ctypes as C
import warnings

import numpy as np
import pytest
import torch

from oracle import slab_oracle as O

pytestmark = pytest.mark.gpu

if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from multiplescatteringcalculations_b200 import (  # noqa: E402
    BatchProblem,
    MaterialContrast,
    ReferenceMedium,
    SlabGeometry,
    SlabMaterial,
    SlabPlan,
    _native,
    compute_slab_scattering_batch,
    random_slab_material,
)

REF = ReferenceMedium(3000.0, 1732.0, 2500.0)


def _rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


def _material(M, Nz, seed, nan_at=None):
    g = SlabGeometry(M, Nz, 1.0)
    mat = random_slab_material(g, REF, MaterialContrast(2e9, 1e9, 300.0), 0.5, seed=seed)
    if nan_at is not None:
        dl = np.array(mat.Dlambda, copy=True)
        dl[nan_at] = np.nan
        mat = SlabMaterial(dl, mat.Dmu, mat.Drho, REF)
    return g, mat


def _solve_abi(plan, psi0, tol=1e-8, max_iter=200, pc=_native.MSC_PC_NONE):
    lib = _native.load()
    x = torch.empty_like(psi0)
    opts = _native.SolveOpts(tol, max_iter, 30, _native.MSC_SOLVE_MIXED, 0, 0.0, 0, pc)
    st = _native.SolveStats()
    status = lib.msc_solve(plan.handle, C.c_void_p(psi0.data_ptr()), C.c_void_p(x.data_ptr()), C.byref(opts),
                           C.byref(st))
    return status, x, st


def test_nan_contrast_returns_nonfinite():
    g, mat = _material(12, 4, 1, nan_at=(2, 5, 7))
    om = 0.5 * REF.beta
    plan = SlabPlan(g, REF)
    plan.build_t0(mat, om)
    plan.build_g0(om)
    psi0 = plan.incident(om, np.array([1.0, 0.0, 0.0]), "P")
    status, _, st = _solve_abi(plan, psi0)
    assert status == _native.MSC_ERR_NONFINITE, _native.load().msc_status_string(status)
    assert b"NaN" in _native.load().msc_last_error() or b"finite" in _native.load().msc_last_error()
    # the plan is still usable: finite contrasts on the same plan solve
    g2, mat2 = _material(12, 4, 1)
    plan.build_t0(mat2, om)
    status, _, st = _solve_abi(plan, psi0)
    assert status == 0 and st.residual < 1e-8
    plan.close()


def test_nan_contrast_fails_one_batch_item():
    om = 0.5 * REF.beta
    kh = np.array([np.cos(0.2), np.sin(0.2), 0.0])
    probs = []
    for i, nan_at in enumerate((None, (1, 3, 3), None)):
        g, mat = _material(10, 3, 10 + i, nan_at=nan_at)
        probs.append(BatchProblem(g, mat, om, kh, "P"))
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        sols, _ = compute_slab_scattering_batch(probs, gmres_tol=1e-8, max_iter=300, workers=1)
    assert any("did not converge or failed" in str(x.message) for x in w)
    assert [s.status for s in sols] == [0, _native.MSC_ERR_NONFINITE, 0]
    for i in (0, 2):
        assert sols[i].gmres_residual < 1e-8


def test_tensor_core_wait_limit_runs_out_and_recovers():
    lib = _native.load()
    M, Nz, om = 16, 8, 0.7 * REF.beta
    g, mat = _material(M, Nz, 3)
    plan = SlabPlan(g, REF)
    plan.build_t0(mat, om)
    plan.build_g0(om)
    plan.set_nearfield(2, weights="bf16_tc")
    rng = np.random.default_rng(4)
    x = rng.standard_normal((Nz, M, M, 9)) + 1j * rng.standard_normal((Nz, M, M, 9))
    xt = torch.from_numpy(x)
    word = C.c_int32(7)
    assert lib.msc_plan_status(plan.handle, C.byref(word)) == 0 and word.value == 0
    for bad in ((-1, 0), (0, 2)):
        with pytest.raises(ValueError):
            _native.check(lib.msc_plan_set_wait_limit(plan.handle, *bad), "msc_plan_set_wait_limit")

    # a wait on an mbarrier nothing completes, 64 polls: it runs out, the call returns,
    # the status is set
    assert lib.msc_plan_set_wait_limit(plan.handle, 64, 1) == 0
    plan.precondition(xt, "complex64")
    assert lib.msc_plan_status(plan.handle, C.byref(word)) == 0
    assert word.value == 1
    assert lib.msc_plan_status(plan.handle, C.byref(word)) == 0 and word.value == 0  # read clears it
    psi0 = plan.incident(om, np.array([1.0, 0.0, 0.0]), "P")
    status, _, _ = _solve_abi(plan, psi0, max_iter=60, pc=_native.MSC_PC_NEARFIELD)
    assert status == _native.MSC_ERR_TIMEOUT
    assert b"bounded wait" in lib.msc_last_error()

    # no injection, default limit: the same plan gives the oracle's result and solves
    assert lib.msc_plan_set_wait_limit(plan.handle, 0, 0) == 0
    t4 = O.t0_scalars(om, 1.0, REF.alpha, REF.beta, REF.rho, mat.Dlambda, mat.Dmu, mat.Drho)
    want = O.nearfield_precondition_rounded(x.ravel(), t4, plan.nearfield_blocks(), M, Nz)
    got = plan.precondition(xt, "complex64").cpu().numpy().ravel()
    assert lib.msc_plan_status(plan.handle, C.byref(word)) == 0 and word.value == 0
    assert _rel(got, want) < 2e-5
    status, _, st = _solve_abi(plan, psi0, max_iter=400, pc=_native.MSC_PC_NEARFIELD)
    assert status == 0 and st.residual < 1e-8
    plan.close()
