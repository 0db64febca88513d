"""Learned near-field preconditioner: a network trained on the GPU on residuals the
solver generates, applied as the right preconditioner of flexible GMRES.

The network is the near-field polynomial of the library (``SlabPlan.set_nearfield``)
with learned parameters: degree L layers S_l x = (G_nn + s w_l)(T0 x), each a 27-point
3D convolution over the 9 field components whose 27 x 9 x 9 complex blocks start at
the physical near-field kernel G_nn and carry a learned correction s w_l
(s = max |G_nn|, so w is dimensionless and serves every frequency), followed by the
per-voxel T0 product; the output is P r = sum_l c_l h_l with learned c_l. It starts at
the truncated Neumann series (c = 1, w = 0). Training minimises the residual of one
GMRES step on the preconditioned operator, min_alpha ||alpha A P r^ - r^||^2, over
residuals r^ = r/||r|| of truncated GMRES runs on random contrast slabs, with the
library's forward and backward kernels and Adam on the device (msc_nf_train); the
layer weights are BF16 with FP32 accumulation in training and inference, and inference
runs each layer on the tensor cores (BF16 activations) by default. The
reference solves without a preconditioner; this module has no counterpart there.

Model selection: ``train_nearfield`` keeps the trained parameters only if flexible
GMRES on held-out validation slabs needs no more operator applications than with
the starting parameters, so the network is never worse than the physics polynomial
on the validation set. Plain GMRES remains the solver's fallback when a
preconditioned cycle fails to reduce the residual.
"""

from __future__ import annotations

import copy
from dataclasses import dataclass, field

import numpy as np
import torch

from .slab import BatchProblem, SlabPlan, _cached_plan, compute_slab_scattering_gpu

__all__ = [
    "NearFieldPreconditioner",
    "solver_residuals",
    "train_nearfield",
    "train_nearfield_stream",
    "fgmres_matvecs",
]


@dataclass
class NearFieldPreconditioner:
    """Parameters of the learned near-field preconditioner: ``coef`` (degree + 1
    complex), ``w`` (degree x 27 x 9 x 9 complex, in units of max |G_nn|) and the Adam
    state of its training. ``weights`` is the form of the layer blocks in the complex64
    path: "bf16_tc" (default; BF16 blocks and activations on the tensor cores, FP32
    accumulation), "bf16" (BF16 blocks on the CUDA cores with FP32 activations, the
    training form) or "fp32"."""

    degree: int = 2
    coef: np.ndarray = None
    w: np.ndarray = None
    adam: np.ndarray | None = None
    weights: str = "bf16_tc"
    history: list = field(default_factory=list)

    def __post_init__(self):
        if not 1 <= self.degree <= 6:
            raise ValueError(f"degree must be in [1, 6], got {self.degree}")
        if self.coef is None:
            self.coef = np.ones(self.degree + 1, dtype=np.complex128)
        if self.w is None:
            self.w = np.zeros((self.degree, 27, 9, 9), dtype=np.complex128)
        self.coef = np.asarray(self.coef, dtype=np.complex128).ravel()
        self.w = np.asarray(self.w, dtype=np.complex128).reshape(self.degree, 27, 9, 9)
        if self.coef.size != self.degree + 1:
            raise ValueError(f"coef needs {self.degree + 1} entries, got {self.coef.size}")

    def install(self, plan: SlabPlan) -> None:
        """Set the plan's near-field preconditioner to this network (after build_g0)."""
        s = plan.nearfield_scale()
        plan.set_nearfield(self.degree, self.coef, s * self.w, weights=self.weights)

    def copy(self) -> "NearFieldPreconditioner":
        return copy.deepcopy(self)

    def save(self, path) -> None:
        np.savez(path, degree=self.degree, coef=self.coef, w=self.w,
                 adam=np.zeros(0) if self.adam is None else self.adam, weights=self.weights)

    @classmethod
    def load(cls, path) -> "NearFieldPreconditioner":
        z = np.load(path)
        adam = z["adam"]
        return cls(int(z["degree"]), z["coef"], z["w"], None if adam.size == 0 else adam, str(z["weights"]))


def _plan_for(problem: BatchProblem) -> SlabPlan:
    return _cached_plan(problem.geometry, problem.material.ref, problem.periodic, None)


def solver_residuals(plan: SlabPlan, b: torch.Tensor, iterations=(2, 5, 10, 20, 40),
                     restart: int = 30) -> torch.Tensor:
    """Residuals r_k = b - A x_k of FP64 GMRES stopped after k operator applications,
    for each k in ``iterations``: the residuals a preconditioner meets during a solve.
    Returns a complex64 tensor (len(iterations), N_z, M, M, 9) on the plan's device."""
    out = []
    for k in iterations:
        x, _ = plan.solve(b, tol=1e-15, max_iter=int(k), restart=restart, precision="fp64")
        out.append((b - plan.matvec(x)).to(torch.complex64))
    return torch.stack(out)


def fgmres_matvecs(problems, preconditioner, *, tol: float = 1e-8, max_iter: int = 3000,
                   precision: str = "mixed", policy: str = "adaptive") -> list[int]:
    """Operator applications of the solve of each problem to ``tol`` with the given
    preconditioner (None: plain GMRES; "nearfield": the Neumann polynomial; a
    NearFieldPreconditioner) under the cycle policy ``policy`` ("adaptive", whose choices
    depend on measured cycle times, or "always", deterministic). A solve that does not
    converge counts ``max_iter``."""
    out = []
    for p in problems:
        import warnings

        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            r = compute_slab_scattering_gpu(p.geometry, p.material, p.omega, p.k_hat, p.wave_type, gmres_tol=tol,
                                            max_iter=max_iter, precision=precision, periodic=p.periodic,
                                            preconditioner=preconditioner, pc_policy=policy)
        out.append(int(r.n_gmres_iter) if r.gmres_residual <= tol else int(max_iter))
    return out


def train_nearfield(train, validation=(), *, degree: int = 4, lr: float = 1e-4, epochs: int = 8,
                    steps_per_slab: int = 10, iterations=(2, 5, 10, 20, 40), init: NearFieldPreconditioner | None = None,
                    tol: float = 1e-8, max_iter: int = 3000, verbose: bool = False) -> NearFieldPreconditioner:
    """Train the learned near-field preconditioner on the GPU.

    ``train`` and ``validation`` are sequences of BatchProblem (geometry, material,
    frequency, incidence; no Bloch phase). For each training slab the solver's
    residuals are generated once (``solver_residuals``); each epoch then takes
    ``steps_per_slab`` Adam steps per slab. With a validation set, the returned
    network is the trained one only if its FGMRES operator applications on the
    validation slabs do not exceed those of the starting network (model selection);
    ``history`` records the losses and the validation counts."""
    net = (init or NearFieldPreconditioner(degree)).copy()
    start = net.copy()
    data = []
    for p in train:
        if p.bloch:
            raise ValueError("training slabs must not carry a Bloch phase")
        plan = _plan_for(p)
        plan.build_t0(p.material, p.omega)
        plan.build_g0(p.omega)
        b = plan.incident(p.omega, p.k_hat, p.wave_type)
        data.append((p, solver_residuals(plan, b, iterations)))
    losses = []
    for ep in range(int(epochs)):
        for p, res in data:
            plan = _plan_for(p)
            plan.build_t0(p.material, p.omega)
            plan.build_g0(p.omega)
            net.coef, net.w, net.adam, ls = plan.nf_train(res, net.coef, net.w, net.adam, steps_per_slab, lr)
            losses.extend(ls.tolist())
        if verbose:
            print(f"epoch {ep}: mean loss {np.mean(losses[-len(data) * steps_per_slab:]):.4g}", flush=True)
    net.history = [{"losses": losses}]
    if validation:
        m0 = fgmres_matvecs(validation, start, tol=tol, max_iter=max_iter)
        m1 = fgmres_matvecs(validation, net, tol=tol, max_iter=max_iter)
        net.history.append({"validation_start": m0, "validation_trained": m1})
        if sum(m1) > sum(m0):
            kept = start.copy()
            kept.history = net.history + [{"selected": "start"}]
            return kept
        net.history.append({"selected": "trained"})
    return net


def train_nearfield_stream(problems, validation=(), *, n_pairs: int = 20000, degree: int = 4, lr: float = 3e-5,
                           iterations=(2, 4, 8, 16, 32, 64), steps_per_residual: int = 1, check_every: int = 500,
                           init: NearFieldPreconditioner | None = None, tol: float = 1e-8, max_iter: int = 3000,
                           policy: str = "adaptive", verbose: bool = False) -> NearFieldPreconditioner:
    """Train the learned near-field preconditioner on a stream of solver-generated
    residuals, at a scale whose residuals could not all be held at once (20 000
    residuals of a 64 x 64 x 16 slab are 94 GB in complex64).

    ``problems`` is an iterable of BatchProblem (a generator is fine). For each slab the
    residuals of FP64 GMRES after each count in ``iterations`` are generated on the
    device, ``steps_per_residual`` Adam steps are taken per residual, and the residuals
    are dropped; the stream stops after ``n_pairs`` residuals. Every ``check_every``
    residuals, and at the end, the network is scored on the validation slabs (FGMRES
    operator applications to ``tol`` under the cycle policy ``policy``); the best-scoring network seen,
    the starting one included, is returned (model selection), with ``history`` holding
    the losses and the validation scores."""
    net = (init or NearFieldPreconditioner(degree)).copy()
    best = (None, -1, net.copy())
    scores = []

    def score(tag):
        nonlocal best
        if not validation:
            return
        s = sum(fgmres_matvecs(validation, net, tol=tol, max_iter=max_iter, policy=policy))
        scores.append((tag, s))
        if verbose:
            print(f"pairs {tag}: validation matvecs {s}", flush=True)
        if best[0] is None or s < best[0]:
            best = (s, tag, net.copy())

    score(0)
    losses = []
    seen = 0
    next_check = check_every
    for p in problems:
        if seen >= n_pairs:
            break
        if p.bloch:
            raise ValueError("training slabs must not carry a Bloch phase")
        plan = _plan_for(p)
        plan.build_t0(p.material, p.omega)
        plan.build_g0(p.omega)
        b = plan.incident(p.omega, p.k_hat, p.wave_type)
        res = solver_residuals(plan, b, iterations)
        res = res[: max(0, n_pairs - seen)]
        net.coef, net.w, net.adam, ls = plan.nf_train(res, net.coef, net.w, net.adam,
                                                      int(res.shape[0]) * int(steps_per_residual), lr)
        losses.extend(ls.tolist())
        seen += int(res.shape[0])
        del res
        if seen >= next_check:
            score(seen)
            next_check += check_every
    if not scores or scores[-1][0] != seen:
        score(seen)
    sel = best[2] if validation else net.copy()
    sel.history = [{"losses": losses, "pairs": seen}, {"validation": scores},
                   {"selected_at_pairs": best[1] if validation else seen}]
    return sel
