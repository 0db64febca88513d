"""Learned near-field preconditioner on the GPU (through the C-ABI): the library's
forward and backward kernels against the oracle's restatement
(oracle/slab_oracle.py, section 9), the Adam step, training, and an ablation of what
the trained network gains over the method without it.

The preconditioner is an addition of this library; the reference solves without one.
"""

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
    NearFieldPreconditioner,
    ReferenceMedium,
    SlabGeometry,
    SlabPlan,
    fgmres_matvecs,
    gaussian_random_field_material,
    random_slab_material,
    solver_residuals,
    train_nearfield,
)

REF = ReferenceMedium(3000.0, 1732.0, 2500.0)


def _rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b))


def _bf16(x):
    """Round to bfloat16 as the device does: to float32, then to nearest even."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32).astype(np.uint64)
    r = ((f + 0x7FFF + ((f >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def _setup(M=6, Nz=4, seed=3, om=0.7 * 1732.0):
    g = SlabGeometry(M, Nz, 1.0)
    mat = random_slab_material(g, REF, MaterialContrast(2e9, 1e9, 300.0), 0.5, seed=seed)
    plan = SlabPlan(g, REF)
    plan.build_t0(mat, om)
    plan.build_g0(om)
    t4 = O.t0_scalars(om, 1.0, REF.alpha, REF.beta, REF.rho, mat.Dlambda, mat.Dmu, mat.Drho)
    kh = O.build_slab_kernels(M, Nz, 1.0, om, REF.alpha, REF.beta, REF.rho)
    blocks = O.nearfield_blocks(M, Nz, 1.0, om, REF.alpha, REF.beta, REF.rho)
    return g, plan, t4, kh, blocks


@pytest.mark.parametrize("degree", [1, 2, 3])
def test_loss_and_gradients_match_oracle(degree):
    M, Nz = 6, 4
    g, plan, t4, kh, blocks = _setup(M, Nz)
    rng = np.random.default_rng(degree)
    coef = 1.0 + 0.2 * (rng.standard_normal(degree + 1) + 1j * rng.standard_normal(degree + 1))
    w = 0.05 * (rng.standard_normal((degree, 27, 9, 9)) + 1j * rng.standard_normal((degree, 27, 9, 9)))
    r = rng.standard_normal((Nz, M, M, 9)) + 1j * rng.standard_normal((Nz, M, M, 9))
    want = O.nearfield_residual_loss_grad(r.ravel(), t4, kh, blocks, M, Nz, coef, w)
    assert abs(plan.nearfield_scale() - np.abs(blocks).max()) < 1e-13 * np.abs(blocks).max()
    loss, gc, gw = plan.nf_loss_grad(torch.from_numpy(r), coef, w, "complex128")
    assert abs(loss - want[0]) < 1e-10 * want[0]
    assert _rel(gc, want[1]) < 1e-9
    assert _rel(gw, want[2]) < 1e-9
    # entries outside the mirror-symmetry pattern get no gradient
    assert np.all(gw[:, ~O.nearfield_symmetry_mask()] == 0)
    # complex64 evaluates with the layer blocks G_nn + s w rounded to BF16: against the
    # oracle at those rounded weights, to FP32 accuracy
    s = np.abs(blocks).max()
    lay = blocks[None] + s * w
    wb = (_bf16(lay.real) + 1j * _bf16(lay.imag) - blocks[None]) / s
    want32 = O.nearfield_residual_loss_grad(r.ravel(), t4, kh, blocks, M, Nz, coef, wb)
    loss32, gc32, gw32 = plan.nf_loss_grad(torch.from_numpy(r), coef, w, "complex64")
    assert abs(loss32 - want32[0]) < 1e-3 * want32[0]
    assert _rel(gc32, want32[1]) < 1e-3
    assert _rel(gw32, want32[2]) < 1e-3


def test_adam_step():
    """One training step moves every parameter with a nonzero gradient by lr against
    the sign of its gradient (Adam's first step), others not at all."""
    M, Nz = 6, 4
    g, plan, t4, kh, blocks = _setup(M, Nz, seed=5)
    rng = np.random.default_rng(7)
    r = torch.from_numpy(rng.standard_normal((1, Nz, M, M, 9)) + 1j * rng.standard_normal((1, Nz, M, M, 9)))
    coef, w = np.ones(3, complex), np.zeros((2, 27, 9, 9), complex)
    _, gc, gw = plan.nf_loss_grad(r[0], coef, w, "complex64")
    lr = 1e-3
    c1, w1, adam, losses = plan.nf_train(r, coef, w, None, 1, lr)
    assert adam[-1] == 1 and losses.shape == (1,)
    g = np.concatenate([gc.view(float), gw.ravel().view(float)])
    p0 = np.concatenate([coef.view(float), w.ravel().view(float)])
    p1 = np.concatenate([c1.view(float), w1.ravel().view(float)])
    step = p1 - p0
    want = -lr * g / (np.abs(g) + 1e-8)
    assert np.allclose(step, want, rtol=1e-4, atol=1e-9)
    assert np.all(step[g == 0] == 0) and np.count_nonzero(g) > 1000


def test_training_reduces_the_loss():
    M, Nz = 12, 6
    g = SlabGeometry(M, Nz, 1.0)
    mat = gaussian_random_field_material(g, REF, correlation_length=3.0, std=0.25, seed=11)
    om = 0.8 * REF.beta
    plan = SlabPlan(g, REF)
    plan.build_t0(mat, om)
    plan.build_g0(om)
    b = plan.incident(om, [1.0, 0.0, 0.0], "P")
    res = solver_residuals(plan, b, (2, 5, 10, 20))
    assert res.shape == (4, Nz, M, M, 9) and res.dtype == torch.complex64
    net = NearFieldPreconditioner(2)

    def total(n):
        return sum(plan.nf_loss_grad(res[k], n.coef, n.w, "complex64")[0] for k in range(res.shape[0]))

    before = total(net)
    net.coef, net.w, net.adam, losses = plan.nf_train(res, net.coef, net.w, None, 80, 1e-3)
    after = total(net)
    assert np.all(np.isfinite(losses))
    assert after < 0.9 * before, (before, after)


def _grf(seed, M=16, Nz=8):
    r = np.random.default_rng(seed)
    ell, std, ka = r.uniform(2, 6), r.uniform(0.1, 0.3), r.uniform(0.3, 1.0)
    g = SlabGeometry(M, Nz, 1.0)
    mat = gaussian_random_field_material(g, REF, correlation_length=ell, std=std, seed=seed)
    th = r.uniform(0, np.deg2rad(40))
    return BatchProblem(g, mat, ka * REF.beta, np.array([np.cos(th), np.sin(th), 0.0]),
                        "P" if r.random() < 0.5 else "S")


def test_learned_preconditioner_ablation(capsys):
    """What training adds: FGMRES operator applications to 1e-8 on held-out GRF slabs
    (the learned-preconditioner workload's distribution at 16 x 16 x 8) for plain
    GMRES, the physics polynomial the network starts from (the same degree), and the
    trained network after model selection on validation slabs. Training on the GPU
    with the library's kernels: 48 slabs x 8 epochs x 10 Adam steps."""
    train = [_grf(3000 + i) for i in range(48)]
    val = [_grf(4000 + i) for i in range(12)]
    test = [_grf(5000 + i) for i in range(12)]
    net = train_nearfield(train, val, max_iter=2000)
    assert net.degree == 4 and len(net.history[0]["losses"]) == 48 * 8 * 10
    plain = fgmres_matvecs(test, None, max_iter=2000)
    start = fgmres_matvecs(test, NearFieldPreconditioner(net.degree), max_iter=2000)
    learned = fgmres_matvecs(test, net, max_iter=2000)
    v = net.history[1]
    with capsys.disabled():
        print(f"\nablation (matvecs to 1e-8, 12 held-out slabs): plain {plain} = {sum(plain)}, "
              f"physics {start} = {sum(start)}, learned {learned} = {sum(learned)}; validation "
              f"{sum(v['validation_start'])} -> {sum(v['validation_trained'])}, selected {net.history[-1]}")
    # model selection: never worse than the start on the validation slabs
    if net.history[-1]["selected"] == "trained":
        assert sum(v["validation_trained"]) <= sum(v["validation_start"])
    else:
        assert np.array_equal(net.coef, np.ones(net.degree + 1)) and not net.w.any()
    assert sum(learned) < sum(plain)
    # training earns its place on held-out slabs: no more operator applications than the
    # untrained polynomial of the same degree
    assert sum(learned) <= sum(start)


def test_packaged_network_as_drop_in_option():
    """preconditioner="learned" loads the packaged network (trained on the GPU on GRF
    slabs, data/make_nearfield_weights.py) and solves a hard held-out slab to the same
    field as plain GMRES in fewer operator applications."""
    from multiplescatteringcalculations_b200 import compute_slab_scattering_gpu

    p = _grf(124)
    plain = compute_slab_scattering_gpu(p.geometry, p.material, p.omega, p.k_hat, p.wave_type, gmres_tol=1e-8,
                                        max_iter=3000)
    lrn = compute_slab_scattering_gpu(p.geometry, p.material, p.omega, p.k_hat, p.wave_type, gmres_tol=1e-8,
                                      max_iter=3000, preconditioner="learned")
    assert plain.gmres_residual < 1e-8 and lrn.gmres_residual < 1e-8
    assert lrn.stats["n_precond"] > 0 and not lrn.stats["pc_fallback"]
    assert lrn.n_gmres_iter < plain.n_gmres_iter
    assert _rel(lrn.psi, plain.psi) < 1e-6


def test_packaged_network_beats_its_untrained_polynomial_held_out():
    """The packaged network (streamed training over 20 000 solver residuals on 64 x 64 x 16
    GRF slabs, the checkpoint model selection kept) against the untrained degree-4
    polynomial it starts from, FGMRES with every cycle preconditioned (the counts do not
    depend on the adaptive policy's timings), summed over the six held-out slabs that both
    solve within seven restart cycles (seeds 5003, 5007, 5008, 5010, 5011, 5015: 366 against
    408 matvecs). Counts of slabs that need many restarts move by tens of percent with the
    rounding of the Krylov sums, either way, so no single such slab decides."""
    from multiplescatteringcalculations_b200 import compute_slab_scattering_gpu
    from multiplescatteringcalculations_b200.data.make_nearfield_weights import grf_problem
    from multiplescatteringcalculations_b200.learned import NearFieldPreconditioner

    kw = dict(gmres_tol=1e-8, max_iter=3000, pc_policy="always")
    n_start = n_lrn = 0
    for seed in (5003, 5007, 5008, 5010, 5011, 5015):
        p = grf_problem(seed)
        start = compute_slab_scattering_gpu(p.geometry, p.material, p.omega, p.k_hat, p.wave_type,
                                            preconditioner=NearFieldPreconditioner(4), **kw)
        lrn = compute_slab_scattering_gpu(p.geometry, p.material, p.omega, p.k_hat, p.wave_type,
                                          preconditioner="learned", **kw)
        assert start.gmres_residual < 1e-8 and lrn.gmres_residual < 1e-8
        assert _rel(lrn.psi, start.psi) < 1e-6
        n_start += start.n_gmres_iter
        n_lrn += lrn.n_gmres_iter
    assert n_lrn <= 0.95 * n_start, (n_lrn, n_start)


def test_streamed_training_keeps_the_best_checkpoint():
    """train_nearfield_stream: residuals from a stream of slabs (16 x 16 x 8 here), the
    count it stops at, the validation score of every checkpoint, and the returned network
    is the best-scoring one (the start included)."""
    from multiplescatteringcalculations_b200.learned import fgmres_matvecs, train_nearfield_stream

    val = [_grf(900), _grf(901)]
    gen = (_grf(1000 + i) for i in range(100))
    net = train_nearfield_stream(gen, val, n_pairs=15, degree=2, iterations=(2, 4, 8), check_every=6,
                                 max_iter=600, policy="always")
    assert net.history[0]["pairs"] == 15
    scores = net.history[1]["validation"]
    assert [t for t, _ in scores] == [0, 6, 12, 15]
    best_tag, best = min(scores, key=lambda ts: ts[1])
    assert net.history[2]["selected_at_pairs"] == best_tag
    assert sum(fgmres_matvecs(val, net, max_iter=600, policy="always")) == best
