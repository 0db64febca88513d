"""YAML configuration entry of the slab solver.

Mirrors ``cubic_scattering/solver_config.py`` (tmnestor/MultipleScatteringCalculations,
``:35-475``): the same dataclasses, YAML keys (``configs/example_slab.yml``) and
validation messages, dispatching slab problems to the B200 solver. Added keys:
``solver.restart``, ``solver.precision`` ("mixed" | "fp64"), ``solver.ortho``,
``solver.inner_tol``, ``solver.preconditioner`` (none | nearfield | learned),
``problem.incident.bloch``, ``problem.geometry.periodic``, and the slab material types
``grf`` (``correlation_length``, ``std``, ``seed``) and ``iid`` (``fraction``, ``seed``).
Sphere problems (``problem.sphere``: ``radius``, ``n_sub``) go to the sphere FFT
Foldy-Lax solver on the GPU, as the reference's GPU branch does (solver_config.py:440-458).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
import torch
import yaml

from .slab import (
    MaterialContrast,
    ReferenceMedium,
    SlabGeometry,
    SlabResult,
    compute_slab_scattering_gpu,
    gaussian_random_field_material,
    random_slab_material,
    uniform_random_material,
    uniform_slab_material,
)

__all__ = ["DeviceConfig", "ProblemConfig", "ScatteringConfig", "SolverConfig", "build_material", "load_config",
           "run_from_config", "validate_config"]


@dataclass
class DeviceConfig:
    """Device and dtype (solver_config.py:35-108). Only CUDA devices run this solver."""

    backend: str = "auto"
    dtype: str = "auto"
    memory_limit_gb: float = 8.0

    def resolve_device(self) -> torch.device:
        if self.backend in ("auto", "cuda"):
            if not torch.cuda.is_available():
                raise ValueError("CUDA backend requested but no CUDA GPU found.")
            return torch.device("cuda")
        if self.backend in ("cpu", "mps"):
            raise ValueError(f"backend '{self.backend}' is not served by this B200 solver; use 'cuda' or 'auto'.")
        raise ValueError(f"Invalid backend '{self.backend}'. Valid options: auto, mps, cuda, cpu.")

    def resolve_dtype(self, device: torch.device) -> torch.dtype:
        if self.dtype in ("auto", "complex128"):
            return torch.complex128
        if self.dtype == "complex64":
            return torch.complex64
        raise ValueError(f"Invalid dtype '{self.dtype}'. Valid options: auto, complex64, complex128.")


@dataclass
class SolverConfig:
    """GMRES parameters (solver_config.py:111-124) and the additions of this solver."""

    gmres_tol: float = 1e-6
    max_iter: int = 500
    initial_guess: str = "born"
    restart: int = 30
    precision: str = "mixed"
    ortho: str = "auto"
    inner_tol: float = 0.0
    preconditioner: str = "none"


@dataclass
class ProblemConfig:
    """Problem definition (solver_config.py:127-165)."""

    type: str
    geometry: dict = field(default_factory=dict)
    reference: dict = field(default_factory=dict)
    contrast: dict = field(default_factory=dict)
    frequency: dict = field(default_factory=dict)
    incident: dict = field(default_factory=dict)
    sphere: dict | None = None
    slab: dict | None = None

    def to_reference_medium(self) -> ReferenceMedium:
        return ReferenceMedium(alpha=float(self.reference["alpha"]), beta=float(self.reference["beta"]),
                               rho=float(self.reference["rho"]))

    def to_material_contrast(self) -> MaterialContrast:
        return MaterialContrast(Dlambda=float(self.contrast["Dlambda"]), Dmu=float(self.contrast["Dmu"]),
                                Drho=float(self.contrast["Drho"]))

    def to_slab_geometry(self) -> SlabGeometry:
        return SlabGeometry(M=int(self.geometry["M"]), N_z=int(self.geometry["N_z"]), a=float(self.geometry["a"]))


@dataclass
class ScatteringConfig:
    device: DeviceConfig
    solver: SolverConfig
    problem: ProblemConfig


def load_config(path) -> ScatteringConfig:
    """Load and validate a YAML config (solver_config.py:181-253)."""
    path = Path(path)
    if not path.exists():
        raise FileNotFoundError(
            f"Config file not found: {path}\nExpected a YAML file with device, solver, and problem sections.\n"
            f"See configs/example_slab.yml for a template."
        )
    with path.open() as f:
        raw = yaml.safe_load(f)
    if not isinstance(raw, dict):
        raise ValueError(f"Config file must contain a YAML mapping, got {type(raw).__name__}")
    dev = raw.get("device", {}) or {}
    device_config = DeviceConfig(backend=dev.get("backend", "auto"), dtype=dev.get("dtype", "auto"),
                                 memory_limit_gb=float(dev.get("memory_limit_gb", 8.0)))
    sol = raw.get("solver", {}) or {}
    solver_config = SolverConfig(
        gmres_tol=float(sol.get("gmres_tol", 1e-6)),
        max_iter=int(sol.get("max_iter", 500)),
        initial_guess=sol.get("initial_guess", "born"),
        restart=int(sol.get("restart", 30)),
        precision=sol.get("precision", "mixed"),
        ortho=sol.get("ortho", "auto"),
        inner_tol=float(sol.get("inner_tol", 0.0)),
        preconditioner=str(sol.get("preconditioner", "none")),
    )
    prob = raw.get("problem")
    if prob is None:
        raise ValueError("Config missing required 'problem' section.\n"
                         "Must contain: type, geometry, reference, contrast, frequency, incident.")
    problem_config = ProblemConfig(
        type=prob.get("type", "slab"), geometry=prob.get("geometry", {}), reference=prob.get("reference", {}),
        contrast=prob.get("contrast", {}), frequency=prob.get("frequency", {}), incident=prob.get("incident", {}),
        sphere=prob.get("sphere"), slab=prob.get("slab"),
    )
    cfg = ScatteringConfig(device=device_config, solver=solver_config, problem=problem_config)
    validate_config(cfg)
    return cfg


def validate_config(config: ScatteringConfig) -> None:
    """Validation with the reference's messages (solver_config.py:256-372) plus the added keys."""
    p = config.problem
    if p.type not in ("slab", "sphere"):
        raise ValueError(f"Invalid problem type '{p.type}'. Must be 'slab' or 'sphere'.")
    for key in ("alpha", "beta", "rho"):
        if key not in p.reference:
            raise ValueError(f"Missing 'problem.reference.{key}'. Required fields: alpha (P-velocity m/s), "
                             f"beta (S-velocity m/s), rho (density kg/m³).")
        if float(p.reference[key]) <= 0:
            raise ValueError(f"problem.reference.{key} must be positive, got {p.reference[key]}")
    for key in ("Dlambda", "Dmu", "Drho"):
        if key not in p.contrast:
            raise ValueError(f"Missing 'problem.contrast.{key}'. Required fields: Dlambda (Pa), Dmu (Pa), "
                             f"Drho (kg/m³).")
    if "omega" not in p.frequency:
        raise ValueError("Missing 'problem.frequency.omega'. Must be a positive float (rad/s).")
    if float(p.frequency["omega"]) <= 0:
        raise ValueError(f"problem.frequency.omega must be positive, got {p.frequency['omega']}")
    for key in ("M", "N_z", "a"):
        if key not in p.geometry:
            raise ValueError(f"Missing 'problem.geometry.{key}'. Required: M (int, horizontal grid), "
                             f"N_z (int, vertical layers), a (float, half-width m).")
    if "wave_type" not in p.incident:
        raise ValueError("Missing 'problem.incident.wave_type'. Must be 'P' or 'S'.")
    if p.incident["wave_type"] not in ("P", "S"):
        raise ValueError(f"Invalid wave_type '{p.incident['wave_type']}'. Must be 'P' or 'S'.")
    if "k_hat" not in p.incident:
        raise ValueError("Missing 'problem.incident.k_hat'. Must be a 3-element list [z, x, y] direction.")
    s = config.solver
    if s.initial_guess not in ("born", "zero"):
        raise ValueError(f"Invalid initial_guess '{s.initial_guess}'. Must be 'born' or 'zero'.")
    if s.precision not in ("mixed", "fp64"):
        raise ValueError(f"Invalid precision '{s.precision}'. Must be 'mixed' or 'fp64'.")
    if s.ortho not in ("auto", "cgs1", "cgs2"):
        raise ValueError(f"Invalid ortho '{s.ortho}'. Must be 'auto', 'cgs1' or 'cgs2'.")
    if not (1 <= s.restart <= 32):
        raise ValueError(f"solver.restart must be in [1, 32], got {s.restart}")
    valid_backends = ("auto", "mps", "cuda", "cpu")
    if config.device.backend not in valid_backends:
        raise ValueError(f"Invalid backend '{config.device.backend}'. Valid options: {', '.join(valid_backends)}.")
    valid_dtypes = ("auto", "complex64", "complex128")
    if config.device.dtype not in valid_dtypes:
        raise ValueError(f"Invalid dtype '{config.device.dtype}'. Valid options: {', '.join(valid_dtypes)}.")
    if config.solver.preconditioner not in ("none", "nearfield", "learned"):
        raise ValueError(f"Invalid preconditioner '{config.solver.preconditioner}'. "
                         f"Must be 'none', 'nearfield' or 'learned'.")
    if p.type == "sphere":
        sp = p.sphere
        if sp is None:
            raise ValueError("Problem type 'sphere' requires a 'sphere' section with 'radius' and 'n_sub'.")
        if "radius" not in sp or "n_sub" not in sp:
            raise ValueError(f"Sphere config requires 'radius' (m) and 'n_sub' (int). Got keys: {list(sp.keys())}")
    slab = p.slab or {}
    mt = slab.get("material_type", "uniform")
    if mt not in ("uniform", "random", "grf", "iid"):
        raise ValueError(f"Invalid slab.material_type '{mt}'. Must be 'uniform', 'random', 'grf' or 'iid'.")
    if mt == "grf" and ("correlation_length" not in slab or "std" not in slab):
        raise ValueError("slab.material_type 'grf' requires 'correlation_length' (cells) and 'std' (fraction).")


def build_material(config: ScatteringConfig):
    """The slab material the config describes (solver_config.py:399-410 plus grf/iid)."""
    p = config.problem
    geometry = p.to_slab_geometry()
    ref = p.to_reference_medium()
    slab = p.slab or {}
    mt = slab.get("material_type", "uniform")
    seed = slab.get("seed")
    seed = int(seed) if seed is not None else None
    if mt == "random":
        return random_slab_material(geometry, ref, p.to_material_contrast(), float(slab.get("phi", 0.1)), seed)
    if mt == "grf":
        return gaussian_random_field_material(geometry, ref, correlation_length=float(slab["correlation_length"]),
                                              std=float(slab["std"]), seed=seed)
    if mt == "iid":
        return uniform_random_material(geometry, ref, float(slab.get("fraction", 0.1)), seed)
    return uniform_slab_material(geometry, ref, p.to_material_contrast())


def run_from_config(config: ScatteringConfig):
    """Solve the configured problem on the GPU (solver_config.py:375-475): a slab
    (SlabResult) or a sphere (SphereDecompositionResult).

    The reference sends CPU configs to its numpy path; this package has no CPU
    path and raises for them.
    """
    device = config.device.resolve_device()
    dtype = config.device.resolve_dtype(device)
    p = config.problem
    s = config.solver
    if p.type == "sphere":
        from .sphere import compute_sphere_foldy_lax_fft_gpu

        sp = p.sphere or {}
        return compute_sphere_foldy_lax_fft_gpu(
            float(p.frequency["omega"]), float(sp["radius"]), p.to_reference_medium(), p.to_material_contrast(),
            int(sp["n_sub"]), k_hat=np.array(p.incident["k_hat"], dtype=float), wave_type=p.incident["wave_type"],
            gmres_tol=s.gmres_tol, gmres_maxiter=s.max_iter, initial_guess=s.initial_guess, device=device,
            dtype=dtype, precision=s.precision, restart=s.restart)
    geometry = p.to_slab_geometry()
    material = build_material(config)
    return compute_slab_scattering_gpu(
        geometry, material, float(p.frequency["omega"]), np.array(p.incident["k_hat"], dtype=float),
        p.incident["wave_type"], gmres_tol=s.gmres_tol, max_iter=s.max_iter, initial_guess=s.initial_guess,
        device=device, dtype=dtype, periodic=bool(p.geometry.get("periodic", False)), restart=s.restart,
        precision=s.precision, bloch=bool(p.incident.get("bloch", False)), ortho=s.ortho, inner_tol=s.inner_tol,
        preconditioner=None if s.preconditioner == "none" else s.preconditioner,
    )
