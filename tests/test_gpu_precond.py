"""Near-field polynomial preconditioner and flexible GMRES on the GPU (through the
C-ABI), against the oracle's restatement (oracle/slab_oracle.py, section 9).

The preconditioner is an addition of this library (the reference solves without
one); it is judged by the oracle's stencil on the same inputs and by the FP64
true residual of the preconditioned solve.
"""

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
    compute_slab_scattering_gpu,
    gaussian_random_field_material,
    random_slab_material,
)

REF = ReferenceMedium(3000.0, 1732.0, 2500.0)


def _rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


def _grf_problem(seed, M=16, Nz=8):
    """GRF slab with (correlation length, std, ka, angle, wave) drawn from the seed,
    the distribution of the learned-preconditioner workload at a smaller size."""
    r = np.random.default_rng(seed)
    ell, std, ka = r.uniform(2, 6), r.uniform(0.1, 0.3), r.uniform(0.3, 1.0)
    g = SlabGeometry(M, Nz, 1.0)
    mat = gaussian_random_field_material(g, REF, correlation_length=ell, std=std, seed=seed)
    th = r.uniform(0, np.deg2rad(40))
    kh = np.array([np.cos(th), np.sin(th), 0.0])
    wave = "P" if r.random() < 0.5 else "S"
    return g, mat, ka * REF.beta, kh, wave


@pytest.mark.parametrize("va", [False, True])
def test_nearfield_blocks_match_oracle(va):
    M, Nz, om = 5, 3, 500.0
    g = SlabGeometry(M, Nz, 1.0)
    plan = SlabPlan(g, REF)
    plan.build_t0(random_slab_material(g, REF, MaterialContrast(1e9, 5e8, 100.0), 0.5, seed=1), om)
    plan.build_g0(om, volume_averaged=va)
    want = O.nearfield_blocks(M, Nz, 1.0, om, REF.alpha, REF.beta, REF.rho, volume_averaged=va)
    assert _rel(plan.nearfield_blocks(), want) < 1e-13


@pytest.mark.parametrize("M,Nz", [(16, 8), (7, 5), (33, 2)])
def test_precondition_matches_oracle(M, Nz):
    om = 0.7 * REF.beta
    g = SlabGeometry(M, Nz, 1.0)
    mat = random_slab_material(g, REF, MaterialContrast(2e9, 1e9, 300.0), 0.5, seed=M + Nz)
    plan = SlabPlan(g, REF)
    plan.build_t0(mat, om)
    plan.build_g0(om)
    t4 = O.t0_scalars(om, 1.0, REF.alpha, REF.beta, REF.rho, mat.Dlambda, mat.Dmu, mat.Drho)
    blocks = O.nearfield_blocks(M, Nz, 1.0, om, REF.alpha, REF.beta, REF.rho)
    rng = np.random.default_rng(0)
    x = rng.standard_normal(Nz * M * M * 9) + 1j * rng.standard_normal(Nz * M * M * 9)
    xt = torch.from_numpy(x.reshape(Nz, M, M, 9))
    # default: degree 2, coefficients 1 (truncated Neumann series)
    want = O.nearfield_precondition(x, t4, blocks, M, Nz)
    assert _rel(plan.precondition(xt).cpu().numpy().ravel(), want) < 1e-12
    assert _rel(plan.precondition(xt, "complex64").cpu().numpy().ravel(), want) < 1e-5
    # degree 3 with coefficients and block corrections
    coef = np.array([1.0, 0.8 + 0.1j, 0.5 - 0.2j, 0.1j])
    dbl = (rng.standard_normal((3, 27, 9, 9)) + 1j * rng.standard_normal((3, 27, 9, 9))) * 0.1 * np.abs(blocks).max()
    plan.set_nearfield(3, coef, dbl)
    want = O.nearfield_precondition(x, t4, blocks, M, Nz, coef, dbl)
    assert _rel(plan.precondition(xt).cpu().numpy().ravel(), want) < 1e-12
    assert _rel(plan.precondition(xt, "complex64").cpu().numpy().ravel(), want) < 1e-5
    with pytest.raises(ValueError):
        plan.set_nearfield(7)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_fgmres_nearfield_on_a_hard_slab(precision):
    """A strongly scattering GRF slab on which plain GMRES(30) needs hundreds of
    matvecs: the near-field preconditioned solve reaches the same tolerance with
    several times fewer operator applications and the same field."""
    g, mat, om, kh, wave = _grf_problem(124)
    plain = compute_slab_scattering_gpu(g, mat, om, kh, wave, gmres_tol=1e-8, max_iter=3000, precision=precision)
    pc = compute_slab_scattering_gpu(g, mat, om, kh, wave, gmres_tol=1e-8, max_iter=3000, precision=precision,
                                     preconditioner="nearfield")
    assert plain.gmres_residual < 1e-8 and pc.gmres_residual < 1e-8
    assert not pc.stats["pc_fallback"]
    assert pc.stats["n_precond"] > 0
    assert pc.n_gmres_iter * 2.5 < plain.n_gmres_iter
    assert _rel(pc.psi, plain.psi) < 1e-6


def test_fgmres_falls_back_to_plain_gmres():
    """A preconditioner that maps everything to zero cannot reduce the residual: the
    first cycle stalls, plain GMRES finishes the solve."""
    g, mat, om, kh, wave = _grf_problem(125)
    plan = SlabPlan(g, REF)
    plan.build_t0(mat, om)
    plan.build_g0(om)
    psi0 = plan.incident(om, kh, wave)
    plan.set_nearfield(1, [0.0, 0.0])
    x, st = plan.solve(psi0, tol=1e-8, max_iter=2000, preconditioner="nearfield")
    assert st["pc_fallback"]
    assert st["residual"] < 1e-8
    ref, st0 = plan.solve(psi0, tol=1e-8, max_iter=2000)
    assert _rel(x.cpu().numpy(), ref.cpu().numpy()) < 1e-6
    with pytest.raises(ValueError):
        plan.solve(psi0, tol=1e-8, max_iter=10, preconditioner="bogus")


# Tolerances of the BF16 preconditioner forms:
# * against the oracle in FP64: the BF16 rounding (unit roundoff 2^-9 = 2e-3 per operand)
#   touches only the stencil terms, which are a fraction of P x (the identity term
#   c0 x is exact), so the norm-wise error stays below 1e-3 (observed 1e-4 to 3e-4);
# * against the oracle with the device's roundings restated
#   (nearfield_precondition_rounded): only the FP32 summation order differs, observed
#   about 1e-6; 2e-5 leaves margin while a single wrong tap or operand slot (about 1e-2)
#   fails it by far.
TOL_BF16_EXACT = 1e-3
TOL_BF16_ROUNDED = 2e-5


def _check_bf16_forms(plan, xt, x, t4, blocks, M, Nz, deg, c, d):
    """bf16_tc (tensor cores, BF16 activations) and bf16 (CUDA cores, FP32 activations,
    the same BF16 weights) against the oracle, exact and rounded, and against each
    other: their difference is the activation rounding alone."""
    args = () if c is None else (c, d)
    want = O.nearfield_precondition(x, t4, blocks, M, Nz, *args)
    coef = (1, 1, 1) if c is None else c
    em_tc = O.nearfield_precondition_rounded(x, t4, blocks, M, Nz, coef, d, activations="bf16")
    em_cc = O.nearfield_precondition_rounded(x, t4, blocks, M, Nz, coef, d, activations="fp32")
    plan.set_nearfield(deg, c, d, weights="bf16_tc")
    got_tc = plan.precondition(xt, "complex64").cpu().numpy().ravel()
    plan.set_nearfield(deg, c, d, weights="bf16")
    got_cc = plan.precondition(xt, "complex64").cpu().numpy().ravel()
    assert _rel(got_tc, want) < TOL_BF16_EXACT
    assert _rel(got_tc, em_tc) < TOL_BF16_ROUNDED
    assert _rel(got_cc, em_cc) < TOL_BF16_ROUNDED
    d_dev, d_em = got_tc - got_cc, em_tc - em_cc
    assert np.linalg.norm(d_dev - d_em) < 0.1 * np.linalg.norm(d_em)
    return got_tc


@pytest.mark.parametrize("M,Nz", [(16, 8), (7, 5), (33, 2)])
def test_precondition_bf16_tensor_cores_match_oracle(M, Nz):
    """Weights "bf16_tc" run each stencil layer on the tensor cores (tcgen05: BF16
    operands, FP32 accumulation in tensor memory). Against the oracle in FP64 the
    difference is the BF16 rounding of weights and activations; against the oracle
    with those roundings restated it is the FP32 summation order."""
    om = 0.7 * REF.beta
    g = SlabGeometry(M, Nz, 1.0)
    mat = random_slab_material(g, REF, MaterialContrast(2e9, 1e9, 300.0), 0.5, seed=M + 2 * Nz)
    plan = SlabPlan(g, REF)
    plan.build_t0(mat, om)
    plan.build_g0(om)
    t4 = O.t0_scalars(om, 1.0, REF.alpha, REF.beta, REF.rho, mat.Dlambda, mat.Dmu, mat.Drho)
    blocks = O.nearfield_blocks(M, Nz, 1.0, om, REF.alpha, REF.beta, REF.rho)
    rng = np.random.default_rng(1)
    x = rng.standard_normal(Nz * M * M * 9) + 1j * rng.standard_normal(Nz * M * M * 9)
    xt = torch.from_numpy(x.reshape(Nz, M, M, 9))
    coef = np.array([1.0, 0.8 + 0.1j, 0.5 - 0.2j, 0.1j])
    dbl = (rng.standard_normal((3, 27, 9, 9)) + 1j * rng.standard_normal((3, 27, 9, 9))) * 0.1 * np.abs(blocks).max()
    for deg, c, d in ((2, None, None), (3, coef, dbl)):
        _check_bf16_forms(plan, xt, x, t4, blocks, M, Nz, deg, c, d)
        # the complex128 path keeps FP64 weights
        want = O.nearfield_precondition(x, t4, blocks, M, Nz, *(() if c is None else (c, d)))
        assert _rel(plan.precondition(xt).cpu().numpy().ravel(), want) < 1e-12


def test_precondition_tensor_cores_several_layers_per_block():
    """A 100 x 100 x 7 lattice: 91 tile columns, so on a 148-SM B200 each block sweeps a
    chunk of layers (3, 3 and 1), which exercises the ring of halo planes, the double-
    buffered accumulator and the mbarrier hand-offs between the staging warps and the MMA
    warp; the tiles are ragged in x and y (100 = 6 x 16 + 4 = 12 x 8 + 4). The blocks are
    the plan's own (pinned against the oracle by test_nearfield_blocks_match_oracle); the
    stencil and polynomial are the oracle's."""
    M, Nz = 100, 7
    om = 0.7 * REF.beta
    g = SlabGeometry(M, Nz, 1.0)
    mat = random_slab_material(g, REF, MaterialContrast(2e9, 1e9, 300.0), 0.5, seed=5)
    plan = SlabPlan(g, REF)
    plan.build_t0(mat, om)
    plan.build_g0(om)
    t4 = O.t0_scalars(om, 1.0, REF.alpha, REF.beta, REF.rho, mat.Dlambda, mat.Dmu, mat.Drho)
    blocks = plan.nearfield_blocks()
    rng = np.random.default_rng(2)
    x = rng.standard_normal(Nz * M * M * 9) + 1j * rng.standard_normal(Nz * M * M * 9)
    xt = torch.from_numpy(x.reshape(Nz, M, M, 9))
    coef = np.array([1.0, 0.8 + 0.1j, 0.5 - 0.2j, 0.1j])
    dbl = (rng.standard_normal((3, 27, 9, 9)) + 1j * rng.standard_normal((3, 27, 9, 9))) * 0.1 * np.abs(blocks).max()
    for deg, c, d in ((3, coef, dbl), (4, np.r_[coef, 0.05], np.concatenate([dbl, dbl[:1]]))):
        got = _check_bf16_forms(plan, xt, x, t4, blocks, M, Nz, deg, c, d)
    # two applications in a row give the same result (no state carried between launches)
    plan.set_nearfield(4, np.r_[coef, 0.05], np.concatenate([dbl, dbl[:1]]), weights="bf16_tc")
    assert np.array_equal(plan.precondition(xt, "complex64").cpu().numpy().ravel(), got)
