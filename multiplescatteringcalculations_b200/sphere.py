"""Sphere FFT Foldy-Lax on the GPU: drop-in for the reference's
``compute_sphere_foldy_lax_fft_gpu`` (cubic_scattering/sphere_scattering_fft_gpu.py:131-244)
and its CPU twin ``compute_sphere_foldy_lax_fft`` (sphere_scattering_fft.py:228-330).

The reference decomposes a sphere into the cells of an n_sub^3 cube grid that lie inside
it (sub-cell half-width a_sub = radius / n_sub) and solves (I - P T) psi = psi_inc on
those cells by FFT convolution over the (2 n_sub - 1)^3 separations, for 9 incident
patterns. That operator is the slab operator of this library on the n_sub^3 lattice
(N_z = M = n_sub, aperiodic, the same point propagator P) with the contrast inside the
sphere and none outside: the outside cells carry no source (T = 0 there), so the inside
block of the system is the reference's, and the outside cells only follow. So the sphere
runs on a SlabPlan: T0 from the masked contrast, the G0 spectrum of the cube lattice,
the 9 right-hand sides built on the device, one GMRES solve each (mixed precision with
FP64 refinement, or FP64), and T_comp = sum over cells of T psi_exc (sphere_scattering_fft.py:
309-312) as a device reduction.
"""

from __future__ import annotations

import warnings
from dataclasses import dataclass, field

import numpy as np
import torch

from .slab import ReferenceMedium, SlabGeometry, SlabMaterial, _cached_plan, _host_array

__all__ = ["SphereDecompositionResult", "compute_sphere_foldy_lax_fft_gpu", "sphere_grid"]

# Voigt strain components in the order of the field's DOF 3..8 (resonance_tmatrix.py:141-148)
_VOIGT_PAIRS = ((0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1))


@dataclass
class SphereDecompositionResult:
    """Result of the sphere decomposition (sphere_scattering.py:46-76): the 3x3 effective
    displacement T-matrix, the 9x9 composite T-matrix, the inside cells' centres, the
    exciting field psi_exc (9 N, 9) and the inputs. ``stats`` holds the solver counters of
    the 9 solves (an addition of this library)."""

    T3x3: np.ndarray
    T_comp_9x9: np.ndarray
    centres: np.ndarray
    n_sub: int
    n_cells: int
    a_sub: float
    condition_number: float
    psi_exc: np.ndarray
    omega: float
    radius: float
    ref: ReferenceMedium
    contrast: object
    stats: list = field(default_factory=list)


def sphere_grid(radius: float, n_sub: int):
    """The cells of the n_sub^3 cube grid inside the sphere (sphere_scattering_fft.py:42-80):
    per axis the centre coordinates (-n_sub/2 + 1/2 + i) d, d = 2 a_sub, kept when the
    centre's distance from the origin is below the radius. Returns (mask (n, n, n) bool,
    grid_idx (N, 3), centres (N, 3), a_sub)."""
    a_sub = radius / n_sub
    c1 = (-n_sub / 2.0 + 0.5 + np.arange(n_sub)) * (2.0 * a_sub)
    pos = np.stack(np.meshgrid(c1, c1, c1, indexing="ij"), -1)
    mask = np.linalg.norm(pos, axis=-1) < radius
    grid_idx = np.argwhere(mask)
    return mask, grid_idx, pos[mask], a_sub


def _incident_column(col: int, pos: torch.Tensor, mask: torch.Tensor, phase: torch.Tensor,
                     x_mean: torch.Tensor) -> torch.Tensor:
    """Column ``col`` of the reference's coupled incident patterns
    (resonance_tmatrix.py:526-586) on the whole lattice, zero outside the sphere:
    col < 3 a uniform displacement e_col; col >= 3 the displacement eps(e_a) (x - x_mean)
    with the Voigt strain e_a (off-diagonal tensor entries 1/2), times the phase."""
    n = pos.shape[0]
    b = torch.zeros((n, n, n, 9), dtype=torch.complex128, device=pos.device)
    if col < 3:
        b[..., col] = phase
    else:
        p, q = _VOIGT_PAIRS[col - 3]
        e = torch.zeros((3, 3), dtype=torch.float64, device=pos.device)
        if p == q:
            e[p, p] = 1.0
        else:
            e[p, q] = e[q, p] = 0.5
        b[..., :3] = ((pos - x_mean) @ e.T) * phase[..., None]
        b[..., col] = phase
    return b * mask[..., None]


def _incident_columns(pos: torch.Tensor, mask: torch.Tensor, phase: torch.Tensor,
                      x_mean: torch.Tensor) -> torch.Tensor:
    """All 9 columns of ``_incident_column`` at once, (9, n, n, n, 9): a few batched
    operations instead of nine small sequences."""
    n = pos.shape[0]
    dev = pos.device
    B = torch.zeros((9, n, n, n, 9), dtype=torch.complex128, device=dev)
    idx = torch.arange(9, device=dev)
    B[idx, ..., idx] = phase  # the column's own component: the plane-wave phase
    E = torch.zeros((6, 3, 3), dtype=torch.float64, device=dev)
    for a, (p, q) in enumerate(_VOIGT_PAIRS):
        if p == q:
            E[a, p, p] = 1.0
        else:
            E[a, p, q] = E[a, q, p] = 0.5
    # columns 3..8: the displacement eps(e_a) (x - x_mean), times the phase
    B[3:, ..., :3] = torch.einsum("xyzj,aij->axyzi", pos - x_mean, E) * phase[None, ..., None]
    return B * mask[None, ..., None]


def _t0_apply(t4: torch.Tensor, x: torch.Tensor) -> torch.Tensor:
    """T0 x for the 4-scalar form t4 (4, n, n, n) and a field x (n, n, n, 9)."""
    tau = torch.empty_like(x)
    tau[..., :3] = t4[0][..., None] * x[..., :3]
    tau[..., 3:6] = t4[1][..., None] * x[..., 3:6].sum(-1, keepdim=True) + t4[2][..., None] * x[..., 3:6]
    tau[..., 6:] = t4[3][..., None] * x[..., 6:]
    return tau


def compute_sphere_foldy_lax_fft_gpu(omega: float, radius: float, ref: ReferenceMedium, contrast, n_sub: int,
                                     k_hat=None, wave_type: str = "S", gmres_tol: float = 1e-8,
                                     gmres_maxiter: int = 200, initial_guess: str = "born", device=None, dtype=None,
                                     *, precision: str = "mixed", restart: int = 30,
                                     solver: str = "multi") -> SphereDecompositionResult:
    """Composite T-matrix of a sphere by FFT Foldy-Lax on the GPU (the reference's
    signature, sphere_scattering_fft_gpu.py:131-145). ``contrast`` has Dlambda, Dmu,
    Drho (MaterialContrast); ``k_hat`` defaults to (0, 0, 1) as in the reference.
    Keyword-only additions: ``precision`` ("mixed": complex64 GMRES inside FP64
    refinement; "fp64"), ``restart`` and ``solver`` ("multi", the default: the 9
    incident patterns as one stacked system whose operator applications are the multi-
    RHS matvec, msc_solve_multi; "columns": one GMRES solve per pattern, as the
    reference). ``dtype`` is accepted for compatibility; the
    returned arrays are complex128 with FP64 true residuals. Non-convergence of a column
    warns, as the reference does."""
    if wave_type not in ("S", "P"):
        raise ValueError(f"wave_type must be 'S' or 'P', got '{wave_type}'")
    if not (radius > 0) or not (omega > 0):
        raise ValueError("radius and omega must be positive")
    if int(n_sub) < 1:
        raise ValueError(f"n_sub must be >= 1, got {n_sub}")
    if initial_guess not in ("born", "zero"):
        raise ValueError(f"initial_guess must be 'born' or 'zero', got {initial_guess!r}")
    if solver not in ("multi", "columns"):
        raise ValueError(f"solver must be 'multi' or 'columns', got {solver!r}")
    n = int(n_sub)
    mask, grid_idx, centres, a_sub = sphere_grid(radius, n)
    nC = len(centres)
    geom = SlabGeometry(n, n, a_sub)
    m = mask.astype(np.float64)
    mat = SlabMaterial(Dlambda=contrast.Dlambda * m, Dmu=contrast.Dmu * m, Drho=contrast.Drho * m, ref=ref)
    plan = _cached_plan(geom, ref, False, device)
    plan.build_t0(mat, omega)
    plan.build_g0(omega)
    dev = plan.device
    kh = np.array([0.0, 0.0, 1.0]) if k_hat is None else np.asarray(k_hat, dtype=float).ravel()[:3]
    kh = kh / np.linalg.norm(kh)
    k = omega / (ref.beta if wave_type == "S" else ref.alpha)
    c1 = (-n / 2.0 + 0.5 + np.arange(n)) * (2.0 * a_sub)
    pos = torch.stack(torch.meshgrid(*(torch.tensor(c1, dtype=torch.float64, device=dev),) * 3, indexing="ij"), -1)
    mask_t = torch.from_numpy(mask).to(dev)
    phase = torch.exp(1j * k * (pos @ torch.tensor(kh, dtype=torch.float64, device=dev)))
    x_mean = torch.tensor(centres.mean(axis=0), dtype=torch.float64, device=dev)
    t4 = plan.t0_scalars()
    idx = torch.from_numpy(grid_idx).to(dev)
    psi = torch.empty((nC, 9, 9), dtype=torch.complex128, device=dev)
    tcomp = torch.empty((9, 9), dtype=torch.complex128, device=dev)
    if solver == "multi":
        # the 9 incident patterns as one stacked system: every operator application is the
        # multi-RHS matvec, which reads the G0 spectrum once for the 9 fields
        B = _incident_columns(pos, mask_t, phase, x_mean)
        X, stats = plan.solve_multi(B, tol=gmres_tol, max_iter=gmres_maxiter, restart=restart,
                                    precision=precision, initial_guess=initial_guess)
        cols = [(col, X[col], stats[col]) for col in range(9)]
    else:
        cols, stats = [], []
        for col in range(9):
            b = _incident_column(col, pos, mask_t, phase, x_mean)
            x, st = plan.solve(b, tol=gmres_tol, max_iter=gmres_maxiter, restart=restart, precision=precision,
                               initial_guess=initial_guess)
            stats.append(st)
            cols.append((col, x, st))
    for col, x, st in cols:
        if st["residual"] > gmres_tol:
            warnings.warn(f"GPU GMRES did not converge for column {col}: rel_res={st['residual']:.2e} after "
                          f"{st['n_matvec']} matvecs", UserWarning, stacklevel=2)
        psi[:, :, col] = x[idx[:, 0], idx[:, 1], idx[:, 2]]
        tcomp[:, col] = _t0_apply(t4, x).reshape(-1, 9).sum(0)
    T = tcomp.cpu().numpy()
    # the exciting field (9 nC x 9 complex128, 22 MB at n_sub = 32) into a recycled host
    # array: a page-locked one takes an asynchronous DMA instead of a pageable copy
    psi_h, psi_pin = _host_array((9 * nC, 9))
    if psi_pin is not None:
        psi_pin.copy_(psi.reshape(9 * nC, 9), non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
    else:
        torch.from_numpy(psi_h).copy_(psi.reshape(9 * nC, 9))
    return SphereDecompositionResult(
        T3x3=T[:3, :3].copy(), T_comp_9x9=T, centres=centres, n_sub=n, n_cells=nC, a_sub=a_sub,
        condition_number=float("nan"), psi_exc=psi_h, omega=float(omega),
        radius=float(radius), ref=ref, contrast=contrast, stats=stats)
