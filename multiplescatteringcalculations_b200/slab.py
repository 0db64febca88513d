"""Slab Foldy-Lax solver on B200: the reference-facing Python API.

A drop-in for ``cubic_scattering.slab_scattering_gpu.compute_slab_scattering_gpu``
and the helpers callers use with it (tmnestor/MultipleScatteringCalculations
``cubic_scattering/slab_scattering.py`` and ``slab_scattering_gpu.py``): the same
dataclasses, argument names, conventions and errors, with every numeric step
running in the hand-written sm_100a kernels of ``libmsc_b200.so``. PyTorch
provides device memory and the stream; it computes nothing here.

Conventions (the reference's): axes (z, x, y) with z down; 9 DOF per voxel
[u_z, u_x, u_y, e_zz, e_xx, e_yy, 2e_xy, 2e_zy, 2e_zx]; fields (N_z, M, M, 9);
``SlabGeometry.a`` is the cube half-width, d = 2a.
"""

from __future__ import annotations

import ctypes as C
import sys
import threading
import warnings
from pathlib import Path
from dataclasses import dataclass, field
from typing import Callable

import numpy as np
import torch
from numpy.typing import NDArray

from . import _native as N

__all__ = [
    "MaterialContrast",
    "ReferenceMedium",
    "SlabGeometry",
    "SlabMaterial",
    "SlabPlan",
    "SlabResult",
    "compute_slab_scattering_gpu",
    "clear_plan_cache",
    "compute_slab_tmatrices",
    "gaussian_random_field_material",
    "random_slab_material",
    "slab_reflected_field",
    "slab_rpp_periodic",
    "uniform_slab_material",
]


# ---------------------------------------------------------------------------
# Data types (effective_contrasts.py:40-68, slab_scattering.py:40-161)
# ---------------------------------------------------------------------------


@dataclass
class ReferenceMedium:
    """Isotropic elastic background: P speed alpha, S speed beta, density rho."""

    alpha: float
    beta: float
    rho: float

    @property
    def lam(self) -> float:
        return self.rho * (self.alpha**2 - 2 * self.beta**2)

    @property
    def mu(self) -> float:
        return self.rho * self.beta**2


@dataclass
class MaterialContrast:
    """Isotropic contrast (Delta lambda, Delta mu in Pa; Delta rho in kg/m^3)."""

    Dlambda: float
    Dmu: float
    Drho: float


@dataclass
class SlabGeometry:
    """M x M x N_z lattice of cubes of half-width a (slab_scattering.py:40-99)."""

    M: int
    N_z: int
    a: float

    def __post_init__(self) -> None:
        if self.M < 1:
            raise ValueError(f"M must be >= 1, got {self.M}")
        if self.N_z < 1:
            raise ValueError(f"N_z must be >= 1, got {self.N_z}")
        if self.a <= 0:
            raise ValueError(f"a must be > 0, got {self.a}")

    @property
    def d(self) -> float:
        return 2.0 * self.a

    @property
    def n_cubes(self) -> int:
        return self.M * self.M * self.N_z

    def cube_centre(self, lz: int, i: int, j: int) -> NDArray[np.floating]:
        d = self.d
        return np.array([(lz + 0.5) * d, (i - (self.M - 1) / 2.0) * d, (j - (self.M - 1) / 2.0) * d])

    def all_centres(self) -> NDArray[np.floating]:
        d = self.d
        z = (np.arange(self.N_z) + 0.5) * d
        x = (np.arange(self.M) - (self.M - 1) / 2.0) * d
        zz, xx, yy = np.meshgrid(z, x, x, indexing="ij")
        return np.stack([zz, xx, yy], axis=-1)


@dataclass
class SlabMaterial:
    """Per-cube contrasts, each (N_z, M, M) (slab_scattering.py:102-133)."""

    Dlambda: NDArray
    Dmu: NDArray
    Drho: NDArray
    ref: ReferenceMedium

    def __post_init__(self) -> None:
        if self.Dlambda.shape != self.Dmu.shape or self.Dlambda.shape != self.Drho.shape:
            raise ValueError(
                f"Contrast array shapes must match: Dlambda={self.Dlambda.shape}, "
                f"Dmu={self.Dmu.shape}, Drho={self.Drho.shape}"
            )
        if self.Dlambda.ndim != 3:
            raise ValueError(f"Contrast arrays must be 3D (N_z, M, M), got ndim={self.Dlambda.ndim}")


@dataclass
class SlabResult:
    """Solved slab (slab_scattering.py:136-161). ``t0`` (extra) holds the four
    T0 scalars per voxel (4, N_z, M, M) so callers need not rebuild T0; ``stats``
    (extra) has the solver counters."""

    psi: NDArray
    psi0: NDArray
    geometry: SlabGeometry
    material: SlabMaterial
    omega: float
    k_hat: NDArray
    wave_type: str
    n_gmres_iter: int
    gmres_residual: float
    periodic: bool = False
    t0: NDArray | None = None
    bloch: bool = False
    stats: dict = field(default_factory=dict)


# ---------------------------------------------------------------------------
# Plan: one geometry on one device
# ---------------------------------------------------------------------------


def _device(device) -> torch.device:
    if device is None:
        if not torch.cuda.is_available():
            raise RuntimeError("compute_slab_scattering_gpu needs a CUDA device (sm_100a); none is available")
        return torch.device("cuda", torch.cuda.current_device())
    device = torch.device(device)
    if device.type != "cuda":
        raise ValueError(f"this solver runs on CUDA devices only, got device={device}")
    if device.index is None:
        device = torch.device("cuda", torch.cuda.current_device())
    return device


def _ptr(t: torch.Tensor) -> int:
    return t.data_ptr()


class SlabPlan:
    """Owns a native plan (FFT sizes, T0, G0 spectrum, workspaces) for one slab
    geometry and background medium on one CUDA device. ``Lxy`` (aperiodic only): the
    padded lateral FFT length, 0 for the automatic rule, "auto" (or -1) for the timed
    choice between the smallest 2,3,5,7-smooth length and the next power of two."""

    def __init__(self, geometry: SlabGeometry, ref: ReferenceMedium, *, periodic: bool = False, device=None,
                 Lz: int = 0, Lxy: int | str = 0):
        if Lxy == "auto":
            Lxy = -1
        self.lib = N.load()
        self.geometry = geometry
        self.ref = ref
        self.periodic = bool(periodic)
        self.device = _device(device)
        self._handle = C.c_void_p()
        with torch.cuda.device(self.device):
            self.stream = torch.cuda.current_stream(self.device)
            desc = N.SlabDesc(geometry.M, geometry.N_z, float(geometry.a), float(ref.alpha), float(ref.beta),
                              float(ref.rho), int(self.periodic), int(Lz), int(Lxy))
            N.check(self.lib.msc_plan_create(C.byref(desc), C.c_void_p(self.stream.cuda_stream),
                                             C.byref(self._handle)), "msc_plan_create")
        self.omega: float | None = None
        self.kpar: tuple[float, float] | None = None

    @property
    def handle(self) -> C.c_void_p:
        if not self._handle:
            raise RuntimeError("plan was released")
        return self._handle

    def close(self) -> None:
        if getattr(self, "_handle", None):
            self.lib.msc_plan_destroy(self._handle)
            self._handle = C.c_void_p()

    def __del__(self):  # pragma: no cover - finaliser
        try:
            self.close()
        except Exception:
            pass

    def fft_sizes(self) -> tuple[int, int, int]:
        out = (C.c_int32 * 3)()
        N.check(self.lib.msc_plan_fft_sizes(self.handle, out), "msc_plan_fft_sizes")
        return tuple(out)

    def device_bytes(self) -> int:
        return int(self.lib.msc_plan_device_bytes(self.handle))

    def _dev(self, a, dtype) -> torch.Tensor:
        if isinstance(a, torch.Tensor):
            return a.to(device=self.device, dtype=dtype).contiguous()
        return torch.from_numpy(np.ascontiguousarray(a)).to(device=self.device, dtype=dtype)

    def build_t0(self, material: SlabMaterial, omega: float) -> None:
        g = self.geometry
        shp = (g.N_z, g.M, g.M)
        for arr in (material.Dlambda, material.Dmu, material.Drho):
            if tuple(arr.shape) != shp:
                raise ValueError(f"material arrays must have shape {shp}, got {tuple(arr.shape)}")
        dl = self._dev(material.Dlambda, torch.float64)
        dm = self._dev(material.Dmu, torch.float64)
        dr = self._dev(material.Drho, torch.float64)
        N.check(self.lib.msc_build_t0(self.handle, _ptr(dl), _ptr(dm), _ptr(dr), float(omega)), "msc_build_t0")
        self._keep = (dl, dm, dr)
        self.omega = float(omega)

    def set_t0_scalars(self, t4, omega: float) -> None:
        t = self._dev(t4, torch.complex128)
        N.check(self.lib.msc_set_t0_scalars(self.handle, _ptr(t), float(omega)), "msc_set_t0_scalars")
        self._keep_t4 = t

    def t0_scalars(self) -> torch.Tensor:
        g = self.geometry
        out = torch.empty((4, g.N_z, g.M, g.M), dtype=torch.complex128, device=self.device)
        N.check(self.lib.msc_t0_scalars(self.handle, _ptr(out)), "msc_t0_scalars")
        return out

    def build_g0(self, omega: float, *, kpar=None, volume_averaged: bool = False, n_orders: int = 2) -> None:
        kp = None
        if kpar is not None:
            kp = (C.c_double * 2)(float(kpar[0]), float(kpar[1]))
        N.check(self.lib.msc_build_g0(self.handle, float(omega), kp, int(bool(volume_averaged)), int(n_orders)),
                "msc_build_g0")
        self.kpar = None if kpar is None else (float(kpar[0]), float(kpar[1]))

    def incident(self, omega: float, k_hat, wave_type: str) -> torch.Tensor:
        if wave_type not in ("P", "S"):
            raise ValueError(f"wave_type must be 'P' or 'S', got '{wave_type}'")
        g = self.geometry
        kh = (C.c_double * 3)(*[float(v) for v in np.asarray(k_hat, dtype=float).ravel()[:3]])
        out = torch.empty((g.N_z, g.M, g.M, 9), dtype=torch.complex128, device=self.device)
        N.check(self.lib.msc_incident(self.handle, float(omega), kh, N.MSC_WAVE_P if wave_type == "P" else N.MSC_WAVE_S,
                                      _ptr(out)), "msc_incident")
        return out

    def matvec(self, x: torch.Tensor, precision: str = "complex128") -> torch.Tensor:
        """(I - G0 T0) x for x (N_z, M, M, 9) on the device."""
        dt = torch.complex128 if precision == "complex128" else torch.complex64
        xx = x.to(device=self.device, dtype=dt).contiguous()
        y = torch.empty_like(xx)
        N.check(self.lib.msc_matvec(self.handle, _ptr(xx), _ptr(y),
                                    N.MSC_COMPLEX128 if dt == torch.complex128 else N.MSC_COMPLEX64), "msc_matvec")
        return y

    def solve(self, b: torch.Tensor, *, tol: float, max_iter: int, restart: int = 30, precision: str = "mixed",
              initial_guess: str = "born", inner_tol: float = 0.0, x: torch.Tensor | None = None,
              ortho: str = "auto", preconditioner: str | None = None):
        """Solve (I - G0 T0) x = b; returns (x, stats dict). ``preconditioner="nearfield"``
        runs flexible GMRES with the near-field polynomial on the right (the plan's
        settings from ``set_nearfield``; plain GMRES takes over if it stalls)."""
        if precision not in ("mixed", "fp64"):
            raise ValueError(f"precision must be 'mixed' or 'fp64', got {precision!r}")
        pcs = {None: N.MSC_PC_NONE, "none": N.MSC_PC_NONE, "nearfield": N.MSC_PC_NEARFIELD,
               "nearfield_always": N.MSC_PC_NEARFIELD_ALWAYS}
        if preconditioner not in pcs:
            raise ValueError(f"preconditioner must be None, 'nearfield' or 'nearfield_always', got {preconditioner!r}")
        bb = b.to(device=self.device, dtype=torch.complex128).contiguous()
        xx = torch.empty_like(bb) if x is None else x
        if ortho not in ("auto", "cgs1", "cgs2"):
            raise ValueError(f"ortho must be 'auto', 'cgs1' or 'cgs2', got {ortho!r}")
        opts = N.SolveOpts(float(tol), int(max_iter), int(restart),
                           N.MSC_SOLVE_MIXED if precision == "mixed" else N.MSC_SOLVE_FP64,
                           0 if initial_guess == "born" else 1, float(inner_tol),
                           {"auto": 0, "cgs1": 1, "cgs2": 2}[ortho], pcs[preconditioner])
        st = N.SolveStats()
        status = N.check(self.lib.msc_solve(self.handle, _ptr(bb), _ptr(xx), C.byref(opts), C.byref(st)), "msc_solve")
        stats = {"n_matvec": st.n_matvec, "n_matvec64": st.n_matvec64, "n_outer": st.n_outer, "status": status,
                 "residual": st.residual, "n_precond": st.n_precond, "pc_fallback": bool(st.pc_fallback),
                 "pc_cycles": st.pc_cycles, "plain_cycles": st.plain_cycles}
        return xx, stats

    def solve_multi(self, b: torch.Tensor, *, tol: float, max_iter: int, restart: int = 30, precision: str = "mixed",
                    initial_guess: str = "born", inner_tol: float = 0.0, ortho: str = "auto",
                    preconditioner: str | None = None):
        """Solve (I - G0 T0) x_r = b_r for the R right-hand sides b (R, N_z, M, M, 9) as
        one stacked system (msc_solve_multi): each operator application is the multi-RHS
        matvec, which reads the G0 spectrum once for all R. Returns (x (R, N_z, M, M, 9),
        list of R stats dicts; ``n_matvec`` counts multi-RHS applications and
        ``residual`` is each right-hand side's FP64 relative residual)."""
        if precision not in ("mixed", "fp64"):
            raise ValueError(f"precision must be 'mixed' or 'fp64', got {precision!r}")
        pcs = {None: N.MSC_PC_NONE, "none": N.MSC_PC_NONE, "nearfield": N.MSC_PC_NEARFIELD,
               "nearfield_always": N.MSC_PC_NEARFIELD_ALWAYS}
        if preconditioner not in pcs:
            raise ValueError(f"preconditioner must be None, 'nearfield' or 'nearfield_always', got {preconditioner!r}")
        if ortho not in ("auto", "cgs1", "cgs2"):
            raise ValueError(f"ortho must be 'auto', 'cgs1' or 'cgs2', got {ortho!r}")
        g = self.geometry
        bb = b.to(device=self.device, dtype=torch.complex128).contiguous()
        if bb.dim() != 5 or tuple(bb.shape[1:]) != (g.N_z, g.M, g.M, 9):
            raise ValueError(f"b must have shape (R, {g.N_z}, {g.M}, {g.M}, 9), got {tuple(bb.shape)}")
        R = int(bb.shape[0])
        xx = torch.empty_like(bb)
        opts = N.SolveOpts(float(tol), int(max_iter), int(restart),
                           N.MSC_SOLVE_MIXED if precision == "mixed" else N.MSC_SOLVE_FP64,
                           0 if initial_guess == "born" else 1, float(inner_tol),
                           {"auto": 0, "cgs1": 1, "cgs2": 2}[ortho], pcs[preconditioner])
        st = (N.SolveStats * max(1, R))()
        N.check(self.lib.msc_solve_multi(self.handle, R, _ptr(bb), _ptr(xx), C.byref(opts), st), "msc_solve_multi")
        stats = [{"n_matvec": s.n_matvec, "n_matvec64": s.n_matvec64, "n_outer": s.n_outer, "status": s.status,
                  "residual": s.residual, "n_precond": s.n_precond, "pc_fallback": bool(s.pc_fallback),
                  "pc_cycles": s.pc_cycles, "plain_cycles": s.plain_cycles}
                 for s in st[:R]]
        return xx, stats

    def matvec_multi(self, x: torch.Tensor, precision: str = "complex64") -> torch.Tensor:
        """(I - G0 T0) x_r for R fields x (R, 9, N_z, M, M) in the component-major layout
        (msc_matvec_multi)."""
        dt = torch.complex128 if precision == "complex128" else torch.complex64
        xx = x.to(device=self.device, dtype=dt).contiguous()
        y = torch.empty_like(xx)
        N.check(self.lib.msc_matvec_multi(self.handle, int(xx.shape[0]), _ptr(xx), _ptr(y),
                                          N.MSC_COMPLEX128 if dt == torch.complex128 else N.MSC_COMPLEX64),
                "msc_matvec_multi")
        return y

    def set_nearfield(self, degree: int = 2, coef=None, dblocks=None, weights: str = "fp32") -> None:
        """Near-field polynomial preconditioner P = sum_l c_l S_l ... S_1 with
        S_l x = (G_nn + dG_l)(T0 x): ``coef`` (degree + 1 complex, default all ones:
        the truncated Neumann series), ``dblocks`` (degree x 27 x 9 x 9 complex block
        corrections, default none; entries outside the lattice's mirror-symmetry
        pattern are not applied), ``weights`` the storage of the layer blocks in the
        complex64 preconditioner ("fp32", "bf16", or "bf16_tc": BF16 blocks and
        activations on the tensor cores)."""
        modes = {"fp32": N.MSC_NF_WEIGHTS_FP32, "bf16": N.MSC_NF_WEIGHTS_BF16, "bf16_tc": N.MSC_NF_WEIGHTS_BF16_TC}
        if weights not in modes:
            raise ValueError(f"weights must be 'fp32', 'bf16' or 'bf16_tc', got {weights!r}")
        c = None
        if coef is not None:
            cc = np.asarray(coef, dtype=np.complex128).ravel()
            if cc.size != degree + 1:
                raise ValueError(f"coef needs {degree + 1} entries, got {cc.size}")
            c = np.ascontiguousarray(np.stack([cc.real, cc.imag], -1).ravel())
        d = None
        if dblocks is not None:
            dd = np.asarray(dblocks, dtype=np.complex128)
            if dd.shape != (degree, 27, 9, 9):
                raise ValueError(f"dblocks must have shape ({degree}, 27, 9, 9), got {dd.shape}")
            d = np.ascontiguousarray(np.stack([dd.real, dd.imag], -1).ravel())
        N.check(self.lib.msc_set_nearfield(self.handle, int(degree), None if c is None else c.ctypes.data,
                                           None if d is None else d.ctypes.data), "msc_set_nearfield")
        N.check(self.lib.msc_set_nearfield_weights(self.handle, modes[weights]), "msc_set_nearfield_weights")

    def nearfield_scale(self) -> float:
        """s = max |G_nn| of the last build_g0: the unit of the learned block weights."""
        return float(self.lib.msc_nearfield_scale(self.handle))

    def nf_loss_grad(self, r: torch.Tensor, coef, w, precision: str = "complex128"):
        """Training objective of the learned near-field preconditioner for one residual
        r (N_z, M, M, 9): loss = min_alpha ||alpha A P r^ - r^||^2, r^ = r / ||r|| (one
        GMRES step on the preconditioned operator), with P of degree
        len(coef) - 1, coefficients ``coef`` and block weights ``w`` (degree x 27 x 9 x 9,
        dG_l = nearfield_scale() w_l). Returns (loss, dL/dconj(coef), dL/dconj(w)),
        computed by the library's forward and backward kernels; "complex64" evaluates
        with BF16 layer weights."""
        cc = np.asarray(coef, dtype=np.complex128).ravel()
        L = cc.size - 1
        ww = np.ascontiguousarray(np.asarray(w, dtype=np.complex128).reshape(L, 27, 9, 9))
        dt = torch.complex128 if precision == "complex128" else torch.complex64
        rr = r.to(device=self.device, dtype=dt).contiguous()
        loss = C.c_double()
        gc = np.zeros(L + 1, dtype=np.complex128)
        gw = np.zeros((L, 27, 9, 9), dtype=np.complex128)
        cr = np.ascontiguousarray(cc)
        N.check(self.lib.msc_nf_loss_grad(self.handle, _ptr(rr),
                                          N.MSC_COMPLEX128 if dt == torch.complex128 else N.MSC_COMPLEX64, L,
                                          cr.ctypes.data, ww.ctypes.data, C.byref(loss), gc.ctypes.data,
                                          gw.ctypes.data), "msc_nf_loss_grad")
        return float(loss.value), gc, gw

    def nf_train(self, residuals: torch.Tensor, coef, w, adam, steps: int, lr: float):
        """``steps`` Adam steps of the learned preconditioner over the complex64
        residuals (n, N_z, M, M, 9) on the device, one per step in turn. Returns
        (coef, w, adam, losses); ``adam`` is the optimiser state (None to start)."""
        # copies: the library updates them in place
        cc = np.array(coef, dtype=np.complex128).ravel()
        L = cc.size - 1
        ww = np.array(w, dtype=np.complex128).reshape(L, 27, 9, 9)
        npar = 2 * (L + 1) + 2 * L * 27 * 81
        st = np.zeros(2 * npar + 1) if adam is None else np.array(adam, dtype=np.float64)
        if st.size != 2 * npar + 1:
            raise ValueError(f"adam state needs {2 * npar + 1} entries, got {st.size}")
        rr = residuals.to(device=self.device, dtype=torch.complex64).contiguous()
        if rr.dim() != 5:
            raise ValueError("residuals must have shape (n, N_z, M, M, 9)")
        losses = np.zeros(max(int(steps), 1))
        N.check(self.lib.msc_nf_train(self.handle, _ptr(rr), int(rr.shape[0]), L, int(steps), float(lr),
                                      cc.ctypes.data, ww.ctypes.data, st.ctypes.data, losses.ctypes.data),
                "msc_nf_train")
        return cc, ww, st, losses[: int(steps)]

    def nearfield_blocks(self) -> NDArray:
        """The (27, 9, 9) near-field blocks G_nn of the last build_g0."""
        out = np.empty(2 * 27 * 81)
        N.check(self.lib.msc_nearfield_blocks(self.handle, out.ctypes.data), "msc_nearfield_blocks")
        return (out[0::2] + 1j * out[1::2]).reshape(27, 9, 9)

    def precondition(self, x: torch.Tensor, precision: str = "complex128") -> torch.Tensor:
        """z = P x for a (N_z, M, M, 9) field."""
        dt = torch.complex128 if precision == "complex128" else torch.complex64
        xx = x.to(device=self.device, dtype=dt).contiguous()
        z = torch.empty_like(xx)
        N.check(self.lib.msc_precondition(self.handle, _ptr(xx), _ptr(z),
                                          N.MSC_COMPLEX128 if dt == torch.complex128 else N.MSC_COMPLEX64),
                "msc_precondition")
        return z

    def rpp_periodic(self, psi: torch.Tensor, omega: float, p: float = 0.0, bloch: bool = False,
                     moment: str = "reference") -> complex:
        """Specular R_PP at horizontal slowness p. ``moment="reference"`` is the
        reference's formula (slab_scattering.py:672-735), whose strain-moment term
        carries the vertical wavenumber kz; ``moment="plane_wave"`` uses |k| = omega/alpha,
        the gradient of the reflected plane wave. The two agree at p = 0."""
        if moment not in ("reference", "plane_wave"):
            raise ValueError(f"moment must be 'reference' or 'plane_wave', got {moment!r}")
        flags = (N.MSC_RPP_BLOCH if bloch else 0) | (N.MSC_RPP_PLANE_WAVE_MOMENT if moment == "plane_wave" else 0)
        pp = psi.to(device=self.device, dtype=torch.complex128).contiguous()
        out = (C.c_double * 2)()
        N.check(self.lib.msc_rpp_periodic(self.handle, _ptr(pp), float(omega), float(p), flags, out),
                "msc_rpp_periodic")
        return complex(out[0], out[1])

    def reflected_field(self, psi: torch.Tensor, omega: float, k_hat) -> tuple[complex, complex, complex]:
        pp = psi.to(device=self.device, dtype=torch.complex128).contiguous()
        kh = (C.c_double * 3)(*[float(v) for v in np.asarray(k_hat, dtype=float).ravel()[:3]])
        out = (C.c_double * 6)()
        N.check(self.lib.msc_reflected_field(self.handle, _ptr(pp), float(omega), kh, out), "msc_reflected_field")
        return complex(out[0], out[1]), complex(out[2], out[3]), complex(out[4], out[5])


# ---------------------------------------------------------------------------
# T0 in the reference's (N_z, M, M, 9, 9) form
# ---------------------------------------------------------------------------


def t0_expand(t4: NDArray) -> NDArray:
    """(4, ...) scalars -> (..., 9, 9) T-matrices."""
    t_u, t_l, t_d, t_s = t4
    T = np.zeros(t_u.shape + (9, 9), dtype=complex)
    for i in range(3):
        T[..., i, i] = t_u
        T[..., 6 + i, 6 + i] = t_s
        for j in range(3):
            T[..., 3 + i, 3 + j] = t_l + (t_d if i == j else 0.0)
    return T


def t0_compress(T: NDArray) -> NDArray:
    """(..., 9, 9) T-matrices of the cube form -> (4, ...) scalars."""
    T = np.asarray(T)
    t_l = T[..., 3, 4]
    return np.stack([T[..., 0, 0], t_l, T[..., 3, 3] - t_l, T[..., 6, 6]])


def compute_slab_tmatrices(geometry: SlabGeometry, material: SlabMaterial, omega: float, *, device=None) -> NDArray:
    """Per-cube 9x9 T-matrices (N_z, M, M, 9, 9), built on the GPU (replaces
    ``compute_slab_tmatrices``, slab_scattering.py:169-205)."""
    plan = SlabPlan(geometry, material.ref, device=device)
    try:
        plan.build_t0(material, omega)
        t4 = plan.t0_scalars().cpu().numpy()
    finally:
        plan.close()
    return t0_expand(t4)


# ---------------------------------------------------------------------------
# Solve (slab_scattering_gpu.py:158-266)
# ---------------------------------------------------------------------------


_PLAN_CACHE: dict = {}
_PLAN_CACHE_SIZE = 2


# Result arrays handed out recently. An array whose only remaining reference is this
# list (the caller dropped the result and holds no view of it) is unobserved and is
# filled again instead of a fresh one: new host memory costs its first-touch page
# faults on every call (several milliseconds for the 23 MB of a 64 x 64 x 16 result).
#
# The first _PINNED_MAX arrays of the pool are page-locked (views of pinned torch
# tensors), so a recycled result is filled by an asynchronous DMA copy; later ones are
# pageable, so callers that keep every result never pay more than those few
# page-locked allocations (each a cudaHostAlloc of ~16 ms for 23 MB).
_HOST_POOL: list = []   # entries [ndarray, pinned tensor or None]
_HOST_POOL_SIZE = 8
_PINNED_MAX = 6
_HOST_POOL_LOCK = threading.Lock()
_COPY_STREAMS: dict = {}  # device index -> side stream for result copies that overlap the solve


def _copy_stream(device: torch.device) -> torch.cuda.Stream:
    i = device.index if device.index is not None else torch.cuda.current_device()
    st = _COPY_STREAMS.get(i)
    if st is None:
        st = _COPY_STREAMS[i] = torch.cuda.Stream(device=device)
    return st


def _host_array(shape: tuple):
    """(array, pinned tensor or None) for a complex128 result of ``shape``."""
    with _HOST_POOL_LOCK:  # the returned value holds a reference before the lock is released
        for e in _HOST_POOL:
            # references to the array: the entry, getrefcount's argument
            if e[0].shape == shape and sys.getrefcount(e[0]) <= 2:
                return e[0], e[1]
        pinned = sum(1 for e in _HOST_POOL if e[1] is not None)
        if pinned < _PINNED_MAX and torch.cuda.is_available():
            t = torch.empty(shape, dtype=torch.complex128, pin_memory=True)
            e = [t.numpy(), t]
        else:
            e = [np.empty(shape, dtype=np.complex128), None]
        _HOST_POOL.append(e)
        if len(_HOST_POOL) > _HOST_POOL_SIZE:
            _HOST_POOL.pop(0)
        return e[0], e[1]


_NETWORK = None


def _packaged_network():
    """The packaged learned near-field preconditioner (data/nearfield_grf.npz), loaded once;
    its layers run on the tensor cores."""
    global _NETWORK
    if _NETWORK is None:
        from .learned import NearFieldPreconditioner

        _NETWORK = NearFieldPreconditioner.load(Path(__file__).resolve().parent / "data" / "nearfield_grf.npz")
        _NETWORK.weights = "bf16_tc"
    return _NETWORK


def _cached_plan(geometry: SlabGeometry, ref: ReferenceMedium, periodic: bool, device) -> SlabPlan:
    """Plans are reused across calls with the same geometry, medium, periodicity
    and device (allocations and FFT set-up happen once); the two most recent
    plans are kept."""
    dev = _device(device)
    key = (geometry.M, geometry.N_z, float(geometry.a), float(ref.alpha), float(ref.beta), float(ref.rho),
           bool(periodic), dev.index)
    plan = _PLAN_CACHE.pop(key, None)
    if plan is None:
        plan = SlabPlan(geometry, ref, periodic=periodic, device=dev)
        while len(_PLAN_CACHE) >= _PLAN_CACHE_SIZE:
            _PLAN_CACHE.pop(next(iter(_PLAN_CACHE))).close()
    _PLAN_CACHE[key] = plan
    return plan


def clear_plan_cache() -> None:
    """Release the cached plans (their device memory)."""
    while _PLAN_CACHE:
        _PLAN_CACHE.popitem()[1].close()


def _bloch_kpar(omega: float, ref: ReferenceMedium, k_hat, wave_type: str) -> tuple[float, float]:
    kh = np.asarray(k_hat, dtype=float)
    kh = kh / np.linalg.norm(kh)
    k = omega / (ref.alpha if wave_type == "P" else ref.beta)
    return float(k * kh[1]), float(k * kh[2])


def compute_slab_scattering_gpu(
    geometry: SlabGeometry,
    material: SlabMaterial,
    omega: float,
    k_hat: NDArray,
    wave_type: str = "P",
    gmres_tol: float = 1e-6,
    max_iter: int = 500,
    initial_guess: str = "born",
    device=None,
    dtype=None,
    *,
    volume_averaged: bool = False,
    n_orders: int = 2,
    periodic: bool = False,
    restart: int = 30,
    precision: str = "mixed",
    preconditioner=None,
    bloch: bool = False,
    inner_tol: float = 0.0,
    ortho: str = "auto",
    plan: SlabPlan | None = None,
    pc_policy: str = "adaptive",
) -> SlabResult:
    """Solve (I - G0 T0) psi = psi0 on the GPU.

    Arguments as the reference's ``compute_slab_scattering_gpu``; keyword-only
    additions: ``restart`` (GMRES(m)), ``precision`` ("mixed": complex64 inner
    GMRES inside FP64 iterative refinement, "fp64": plain complex128 GMRES),
    ``bloch`` (periodic only: Bloch-phased lateral fold for oblique incidence;
    False is the reference's phase-free fold), ``inner_tol``, ``ortho`` (Arnoldi
    orthogonalisation: "auto" = one classical Gram-Schmidt pass in the complex64
    inner solves and two in FP64 solves; "cgs1"; "cgs2") and ``plan`` (reuse a
    plan of the same geometry). ``dtype`` is accepted for compatibility
    (complex64 or complex128); the arithmetic is set by ``precision`` and the
    returned field is always complex128 with its FP64 true residual.
    ``preconditioner``: None (plain GMRES), "nearfield" (flexible GMRES with the
    near-field Neumann polynomial of the plan's settings), "learned" (the packaged
    network, trained on the GPU on Gaussian-random-field slabs:
    ``data/make_nearfield_weights.py``), or a ``NearFieldPreconditioner`` (its degree,
    coefficients and learned block corrections). ``pc_policy``: "adaptive" (default:
    after a few preconditioned GMRES cycles one plain cycle is measured, and the form
    that reduces the residual faster per unit of device time runs, measured again now
    and then) or "always" (every cycle preconditioned); under both, plain GMRES
    finishes the solve if a preconditioned cycle makes no progress.
    """
    if pc_policy not in ("adaptive", "always"):
        raise ValueError(f"pc_policy must be 'adaptive' or 'always', got {pc_policy!r}")
    if wave_type not in ("P", "S"):
        raise ValueError(f"wave_type must be 'P' or 'S', got '{wave_type}'")
    if dtype is not None and dtype not in (torch.complex64, torch.complex128):
        raise ValueError(f"dtype must be torch.complex64 or torch.complex128, got {dtype}")
    pc_mode = None
    if isinstance(preconditioner, str) and preconditioner == "learned":
        preconditioner = _packaged_network()
    if preconditioner is not None:
        if isinstance(preconditioner, str):
            if preconditioner not in ("nearfield", "none"):
                raise ValueError(f"preconditioner must be None, 'nearfield', 'learned' or a NearFieldPreconditioner, "
                                 f"got {preconditioner!r}")
            pc_mode = None if preconditioner == "none" else "nearfield"
        elif hasattr(preconditioner, "install"):
            pc_mode = "nearfield"
        else:
            raise ValueError(f"unsupported preconditioner {preconditioner!r}")
    if bloch and not periodic:
        raise ValueError("bloch=True needs periodic=True")
    if plan is None:
        plan = _cached_plan(geometry, material.ref, periodic, device)
    elif plan.periodic != bool(periodic) or plan.geometry != geometry:
        raise ValueError("plan geometry/periodicity does not match the problem")
    kp = _bloch_kpar(omega, material.ref, k_hat, wave_type) if bloch else None
    plan.build_t0(material, omega)
    plan.build_g0(omega, kpar=kp, volume_averaged=volume_averaged, n_orders=n_orders)
    psi0 = plan.incident(omega, k_hat, wave_type)
    t4 = plan.t0_scalars()
    # psi0 and T0 are final before the solve: their device -> host copies into page-locked
    # result arrays run on a side stream while GMRES runs (a result array that is not
    # page-locked is copied after the solve)
    cur = torch.cuda.current_stream(plan.device)
    side = _copy_stream(plan.device)
    side.wait_stream(cur)
    early = [_host_array(tuple(t.shape)) for t in (psi0, t4)]
    with torch.cuda.stream(side):
        for (h, ht), t in zip(early, (psi0, t4)):
            if ht is not None:
                ht.copy_(t, non_blocking=True)
                t.record_stream(side)
    if pc_mode is not None:
        if hasattr(preconditioner, "install"):
            preconditioner.install(plan)
        else:
            plan.set_nearfield()
    if pc_mode is not None and pc_policy == "always":
        pc_mode = "nearfield_always"
    x, st = plan.solve(psi0, tol=gmres_tol, max_iter=max_iter, restart=restart, precision=precision,
                       initial_guess=initial_guess, inner_tol=inner_tol, ortho=ortho, preconditioner=pc_mode)
    if st["residual"] > gmres_tol:
        warnings.warn(
            f"GPU GMRES did not converge: rel_res={st['residual']:.2e} after {st['n_matvec']} matvecs",
            stacklevel=2,
        )
    # device -> host into result arrays from a small recycled pool: the first few are
    # page-locked (asynchronous copies), the others plain numpy arrays, which ask for
    # transparent huge pages, so the first touch costs a few faults per array instead of
    # one per 4 KB page. A result array the caller still holds is never reused.
    host = [_host_array(tuple(x.shape))] + early
    for i, ((h, ht), t) in enumerate(zip(host, (x, psi0, t4))):
        if ht is not None:
            if i == 0:
                ht.copy_(t, non_blocking=True)
        else:
            torch.from_numpy(h).copy_(t)
    cur.synchronize()
    side.synchronize()
    psi_h, psi0_h, t4_h = (h for h, _ in host)
    res = SlabResult(
        psi=psi_h,
        psi0=psi0_h,
        geometry=geometry,
        material=material,
        omega=float(omega),
        k_hat=np.asarray(k_hat, dtype=float),
        wave_type=wave_type,
        n_gmres_iter=int(st["n_matvec"]),
        gmres_residual=float(st["residual"]),
        periodic=bool(periodic),
        t0=t4_h,
        bloch=bool(bloch),
        stats=st,
    )
    return res


# ---------------------------------------------------------------------------
# Batched solves
# ---------------------------------------------------------------------------


@dataclass
class BatchProblem:
    """One slab of a batch: geometry, material, frequency and incidence;
    ``volume_averaged``/``n_orders`` as the reference's solver options; ``rpp_p`` the
    horizontal slowness at which R_PP is evaluated (None: the incidence's slowness for
    ``bloch`` items, normal incidence otherwise)."""

    geometry: SlabGeometry
    material: SlabMaterial
    omega: float
    k_hat: NDArray
    wave_type: str = "P"
    periodic: bool = False
    bloch: bool = False
    volume_averaged: bool = False
    n_orders: int = 2
    rpp_p: float | None = None


@dataclass
class BatchSolution:
    """Result of one batch item: the field (None when not requested), the specular
    R_PP of the solution by the Weyl sum (at the Bloch slowness for ``bloch``
    items, else at normal incidence), and the solver counters."""

    psi: NDArray | None
    rpp: complex
    n_gmres_iter: int
    gmres_residual: float
    status: int
    stats: dict


def compute_slab_scattering_batch(problems, *, gmres_tol: float = 1e-6, max_iter: int = 500, restart: int = 30,
                                  precision: str = "mixed", preconditioner: str | None = None,
                                  initial_guess: str = "born", ortho: str = "auto", workers: int = 0,
                                  return_fields: bool = True):
    """Solve many independent slabs of uneven size, frequency and incidence on the
    current GPU in one call (``msc_batch_solve``): per item the T0 and G0 builds,
    the incident field, the solve and R_PP. ``workers`` host threads (each with its
    own stream and plans) run items concurrently; 0 lets the library choose by
    timing. Returns (list of BatchSolution, info) with info["workers"] the count
    used. Items that fail or do not converge keep their own status; a warning names
    them."""
    if precision not in ("mixed", "fp64"):
        raise ValueError(f"precision must be 'mixed' or 'fp64', got {precision!r}")
    pcs = {None: N.MSC_PC_NONE, "none": N.MSC_PC_NONE, "nearfield": N.MSC_PC_NEARFIELD,
           "nearfield_always": N.MSC_PC_NEARFIELD_ALWAYS}
    if preconditioner not in pcs:
        raise ValueError(f"preconditioner must be None, 'nearfield' or 'nearfield_always', got {preconditioner!r}")
    if ortho not in ("auto", "cgs1", "cgs2"):
        raise ValueError(f"ortho must be 'auto', 'cgs1' or 'cgs2', got {ortho!r}")
    problems = list(problems)
    n = len(problems)
    items = (N.BatchItem * max(1, n))()
    keep, outs = [], []
    for i, pr in enumerate(problems):
        if pr.wave_type not in ("P", "S"):
            raise ValueError(f"item {i}: wave_type must be 'P' or 'S', got '{pr.wave_type}'")
        if pr.bloch and not pr.periodic:
            raise ValueError(f"item {i}: bloch=True needs periodic=True")
        g, ref = pr.geometry, pr.material.ref
        arrs = [np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(g.N_z, g.M, g.M))
                for a in (pr.material.Dlambda, pr.material.Dmu, pr.material.Drho)]
        keep.append(arrs)
        it = items[i]
        it.desc = N.SlabDesc(g.M, g.N_z, float(g.a), float(ref.alpha), float(ref.beta), float(ref.rho),
                             int(bool(pr.periodic)), 0, 0)
        it.dlam, it.dmu, it.drho = (a.ctypes.data for a in arrs)
        it.omega = float(pr.omega)
        kh = np.asarray(pr.k_hat, dtype=float).ravel()
        for j in range(3):
            it.k_hat[j] = float(kh[j])
        it.wave_type = N.MSC_WAVE_P if pr.wave_type == "P" else N.MSC_WAVE_S
        it.bloch = int(bool(pr.bloch))
        it.volume_averaged = int(bool(pr.volume_averaged))
        it.n_orders = int(pr.n_orders)
        if pr.rpp_p is not None and not pr.rpp_p >= 0:
            raise ValueError(f"item {i}: rpp_p must be >= 0, got {pr.rpp_p}")
        it.rpp_p = -1.0 if pr.rpp_p is None else float(pr.rpp_p)
        out = np.empty((g.N_z, g.M, g.M, 9), dtype=np.complex128) if return_fields else None
        outs.append(out)
        it.psi = out.ctypes.data if out is not None else None
    opts = N.SolveOpts(float(gmres_tol), int(max_iter), int(restart),
                       N.MSC_SOLVE_MIXED if precision == "mixed" else N.MSC_SOLVE_FP64,
                       0 if initial_guess == "born" else 1, 0.0, {"auto": 0, "cgs1": 1, "cgs2": 2}[ortho],
                       pcs[preconditioner])
    used = C.c_int(0)
    lib = N.load()
    N.check(lib.msc_batch_solve(items, n, C.byref(opts), int(workers), C.byref(used)), "msc_batch_solve")
    sols, bad = [], []
    for i in range(n):
        it = items[i]
        st = {"n_matvec": it.stats.n_matvec, "n_matvec64": it.stats.n_matvec64, "n_outer": it.stats.n_outer,
              "residual": it.stats.residual, "n_precond": it.stats.n_precond,
              "pc_fallback": bool(it.stats.pc_fallback), "pc_cycles": it.stats.pc_cycles,
              "plain_cycles": it.stats.plain_cycles}
        if it.status != 0:
            bad.append((i, it.status, it.error.decode(errors="replace")))
        sols.append(BatchSolution(psi=outs[i], rpp=complex(it.rpp[0], it.rpp[1]), n_gmres_iter=int(it.stats.n_matvec),
                                  gmres_residual=float(it.stats.residual), status=int(it.status), stats=st))
    if bad:
        warnings.warn(f"{len(bad)} batch item(s) did not converge or failed: {bad[:4]}", stacklevel=2)
    return sols, {"workers": int(used.value)}


@dataclass
class SlabSweepResult:
    """Per-frequency results of ``compute_slab_rpp_sweep``: ``rpp`` (n,) complex, the
    specular R_PP of each frequency's solution at slowness ``p``; ``n_gmres_iter`` and
    ``gmres_residual`` per frequency; ``psi`` the fields (None unless asked for)."""

    omegas: NDArray
    rpp: NDArray
    n_gmres_iter: list
    gmres_residual: NDArray
    status: list
    psi: list | None


def compute_slab_rpp_sweep(geometry: SlabGeometry, material: SlabMaterial, omegas, k_hat, p: float = 0.0, *,
                           wave_type: str = "P", gmres_tol: float = 1e-6, max_iter: int = 500,
                           volume_averaged: bool = False, n_orders: int = 2, bloch: bool = False,
                           precision: str = "mixed", restart: int = 30, workers: int = 0,
                           return_fields: bool = False) -> SlabSweepResult:
    """The frequency loop of the reference's ocean-bottom model
    (ocean_bottom.py:290-307): for every angular frequency w of ``omegas`` one periodic
    slab solve at incidence ``k_hat`` and the specular R_PP of its solution at horizontal
    slowness ``p`` by the reference's Weyl sum (``slab_rpp_periodic(result, T_local,
    p=p)``), T0 built once per frequency. All frequencies go to the GPU in one batch call
    (msc_batch_solve). ``bloch=False`` keeps the reference's fold without a Bloch phase;
    ``bloch=True`` solves with the Bloch-phased fold at the incidence's k_par (R_PP then
    demodulates the sources, as ``slab_rpp_periodic`` with ``bloch``)."""
    om = np.atleast_1d(np.asarray(omegas, dtype=float)).ravel()
    if om.size == 0:
        raise ValueError("omegas is empty")
    if not np.all(om > 0):
        raise ValueError("every omega must be > 0")
    if not p >= 0:
        raise ValueError(f"p must be >= 0, got {p}")
    kh = np.asarray(k_hat, dtype=float).ravel()
    probs = [BatchProblem(geometry, material, float(w), kh, wave_type, periodic=True, bloch=bool(bloch),
                          volume_averaged=bool(volume_averaged), n_orders=int(n_orders), rpp_p=float(p))
             for w in om]
    sols, _ = compute_slab_scattering_batch(probs, gmres_tol=gmres_tol, max_iter=max_iter, restart=restart,
                                            precision=precision, workers=workers, return_fields=return_fields)
    return SlabSweepResult(omegas=om, rpp=np.array([s.rpp for s in sols]),
                           n_gmres_iter=[s.n_gmres_iter for s in sols],
                           gmres_residual=np.array([s.gmres_residual for s in sols]),
                           status=[s.status for s in sols],
                           psi=[s.psi for s in sols] if return_fields else None)


# ---------------------------------------------------------------------------
# Observables (slab_scattering.py:589-735)
# ---------------------------------------------------------------------------


def _observable_plan(result: SlabResult, T_local, device) -> SlabPlan:
    plan = SlabPlan(result.geometry, result.material.ref, periodic=result.periodic, device=device)
    t4 = t0_compress(T_local) if np.ndim(T_local) == 5 else np.asarray(T_local)
    plan.set_t0_scalars(t4, result.omega)
    if result.bloch:
        plan.build_g0(result.omega, kpar=_bloch_kpar(result.omega, result.material.ref, result.k_hat,
                                                     result.wave_type))
    return plan


def slab_rpp_periodic(result: SlabResult, T_local, *, p: float = 0.0, device=None,
                      moment: str = "reference") -> complex:
    """Specular P->P reflection of a periodic slab by the Weyl sum (replaces
    ``slab_rpp_periodic``, slab_scattering.py:672-735). ``T_local`` is the
    (N_z, M, M, 9, 9) T-matrices or the (4, N_z, M, M) scalars. For a result
    solved with ``bloch=True`` the sources are demodulated by the Bloch phase.
    ``moment="plane_wave"`` replaces the reference's kz in the strain-moment term by
    omega/alpha (identical at p = 0; at oblique p it is the form that matches the
    Kennett layer reflectivity)."""
    plan = _observable_plan(result, T_local, device)
    try:
        return plan.rpp_periodic(torch.from_numpy(np.ascontiguousarray(result.psi)), result.omega, p, result.bloch,
                                 moment)
    finally:
        plan.close()


def slab_reflected_field(result: SlabResult, T_local, *, device=None) -> tuple[complex, complex, complex]:
    """(R_PP, R_PS, R_SP) far-field amplitudes per unit area (replaces
    ``slab_reflected_field``, slab_scattering.py:589-669)."""
    plan = _observable_plan(result, T_local, device)
    try:
        return plan.reflected_field(torch.from_numpy(np.ascontiguousarray(result.psi)), result.omega, result.k_hat)
    finally:
        plan.close()


# ---------------------------------------------------------------------------
# Material generators (slab_scattering.py:791-852) and the Gaussian random field
# ---------------------------------------------------------------------------


def random_slab_material(geometry: SlabGeometry, ref: ReferenceMedium, contrast: MaterialContrast,
                         phi: float | Callable[[int], float], seed: int | None = None) -> SlabMaterial:
    """Binary random slab: each cube is an inclusion with probability phi
    (per layer if callable), drawn layer by layer from default_rng(seed) exactly
    as the reference does, so the same seed gives the same material."""
    rng = np.random.default_rng(seed)
    shape = (geometry.N_z, geometry.M, geometry.M)
    dl = np.zeros(shape)
    dm = np.zeros(shape)
    dr = np.zeros(shape)
    for lz in range(geometry.N_z):
        p = phi(lz) if callable(phi) else phi
        mask = rng.random((geometry.M, geometry.M)) < p
        dl[lz, mask] = contrast.Dlambda
        dm[lz, mask] = contrast.Dmu
        dr[lz, mask] = contrast.Drho
    return SlabMaterial(Dlambda=dl, Dmu=dm, Drho=dr, ref=ref)


def uniform_slab_material(geometry: SlabGeometry, ref: ReferenceMedium, contrast: MaterialContrast) -> SlabMaterial:
    """Every cube with the same contrast."""
    shape = (geometry.N_z, geometry.M, geometry.M)
    return SlabMaterial(Dlambda=np.full(shape, contrast.Dlambda), Dmu=np.full(shape, contrast.Dmu),
                        Drho=np.full(shape, contrast.Drho), ref=ref)


def uniform_random_material(geometry: SlabGeometry, ref: ReferenceMedium, fraction: float,
                            seed: int | None = None) -> SlabMaterial:
    """i.i.d. U(-fraction, fraction) relative contrasts of (lambda0, mu0, rho0),
    drawn in that order, each (N_z, M, M), from default_rng(seed)."""
    rng = np.random.default_rng(seed)
    shp = (geometry.N_z, geometry.M, geometry.M)
    dl = rng.uniform(-fraction, fraction, shp) * ref.lam
    dm = rng.uniform(-fraction, fraction, shp) * ref.mu
    dr = rng.uniform(-fraction, fraction, shp) * ref.rho
    return SlabMaterial(Dlambda=dl, Dmu=dm, Drho=dr, ref=ref)


def gaussian_random_field(shape: tuple[int, int, int], correlation_length: float, rng: np.random.Generator,
                          ) -> NDArray:
    """Zero-mean unit-variance Gaussian random field on (N_z, M, M) with
    covariance exp(-r^2 / l^2) (l in cells): white noise filtered by sqrt(S(k)),
    S(k) = exp(-k^2 l^2 / 4); periodic in x and y, z padded by 3 l so the field
    does not wrap vertically."""
    nz, m1, m2 = shape
    pad = int(np.ceil(3.0 * correlation_length))
    Lz = nz + pad
    w = rng.standard_normal((Lz, m1, m2))
    kz = 2 * np.pi * np.fft.fftfreq(Lz)
    kx = 2 * np.pi * np.fft.fftfreq(m1)
    ky = 2 * np.pi * np.fft.fftfreq(m2)
    k2 = kz[:, None, None] ** 2 + kx[None, :, None] ** 2 + ky[None, None, :] ** 2
    f = np.fft.ifftn(np.fft.fftn(w) * np.exp(-k2 * correlation_length**2 / 8.0)).real[:nz]
    f = f - f.mean()
    sd = f.std()
    return f / sd if sd > 0 else f


def gaussian_random_field_material(geometry: SlabGeometry, ref: ReferenceMedium, *, correlation_length: float,
                                   std: float, seed: int | None = None, clip: float = 0.9) -> SlabMaterial:
    """Contrasts Delta lambda, Delta mu, Delta rho as independent Gaussian random
    fields (drawn in that order from default_rng(seed)) of relative standard
    deviation ``std`` and correlation length ``correlation_length`` cells,
    clipped to +-``clip`` of (lambda0, mu0, rho0) so the medium stays positive."""
    rng = np.random.default_rng(seed)
    shp = (geometry.N_z, geometry.M, geometry.M)
    fr = [np.clip(std * gaussian_random_field(shp, correlation_length, rng), -clip, clip) for _ in range(3)]
    return SlabMaterial(Dlambda=fr[0] * ref.lam, Dmu=fr[1] * ref.mu, Drho=fr[2] * ref.rho, ref=ref)
