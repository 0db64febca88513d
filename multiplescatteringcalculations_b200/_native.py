"""ctypes binding of the C-ABI library ``libmsc_b200.so`` (declared in include/msc.h).

The library is the only compute path of this package: if it is missing or cannot
be loaded the import of the solver functions raises, there is no fallback.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libmsc_b200.so"

MSC_OK = 0
MSC_NOT_CONVERGED = 1
MSC_BREAKDOWN = 2
MSC_ERR_INVALID = -1
MSC_ERR_UNSUPPORTED = -2
MSC_ERR_CUDA = -3
MSC_ERR_NOMEM = -4
MSC_ERR_STATE = -5
MSC_ERR_NONFINITE = -6
MSC_ERR_TIMEOUT = -7
MSC_MAX_RHS = 64

MSC_COMPLEX64 = 0
MSC_COMPLEX128 = 1
MSC_RPP_BLOCH = 1
MSC_RPP_PLANE_WAVE_MOMENT = 2
MSC_PC_NONE = 0
MSC_PC_NEARFIELD = 1
MSC_PC_NEARFIELD_ALWAYS = 2
MSC_NF_WEIGHTS_FP32 = 0
MSC_NF_WEIGHTS_BF16 = 1
MSC_NF_WEIGHTS_BF16_TC = 2
MSC_SOLVE_MIXED = 0
MSC_SOLVE_FP64 = 1
MSC_WAVE_P = 0
MSC_WAVE_S = 1


class SlabDesc(C.Structure):
    _fields_ = [
        ("M", C.c_int32),
        ("N_z", C.c_int32),
        ("a", C.c_double),
        ("alpha", C.c_double),
        ("beta", C.c_double),
        ("rho", C.c_double),
        ("periodic", C.c_int32),
        ("Lz", C.c_int32),
        ("Lxy", C.c_int32),
    ]


class SolveOpts(C.Structure):
    _fields_ = [
        ("tol", C.c_double),
        ("max_iter", C.c_int32),
        ("restart", C.c_int32),
        ("precision", C.c_int32),
        ("initial_guess", C.c_int32),
        ("inner_tol", C.c_double),
        ("ortho", C.c_int32),
        ("preconditioner", C.c_int32),
    ]


class SolveStats(C.Structure):
    _fields_ = [
        ("n_matvec", C.c_int32),
        ("n_matvec64", C.c_int32),
        ("n_outer", C.c_int32),
        ("status", C.c_int32),
        ("residual", C.c_double),
        ("n_precond", C.c_int32),
        ("pc_fallback", C.c_int32),
        ("pc_cycles", C.c_int32),
        ("plain_cycles", C.c_int32),
    ]


class BatchItem(C.Structure):
    _fields_ = [
        ("desc", SlabDesc),
        ("dlam", C.c_void_p),
        ("dmu", C.c_void_p),
        ("drho", C.c_void_p),
        ("omega", C.c_double),
        ("k_hat", C.c_double * 3),
        ("wave_type", C.c_int32),
        ("bloch", C.c_int32),
        ("volume_averaged", C.c_int32),
        ("n_orders", C.c_int32),
        ("rpp_p", C.c_double),
        ("psi", C.c_void_p),
        ("rpp", C.c_double * 2),
        ("stats", SolveStats),
        ("status", C.c_int32),
        ("error", C.c_char * 160),
    ]


# name -> (restype, argtypes); every entry point that include/msc.h declares
SIGNATURES = {
    "msc_plan_create": (C.c_int, [C.POINTER(SlabDesc), C.c_void_p, C.POINTER(C.c_void_p)]),
    "msc_plan_destroy": (C.c_int, [C.c_void_p]),
    "msc_plan_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "msc_plan_fft_sizes": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "msc_plan_device_bytes": (C.c_int64, [C.c_void_p]),
    "msc_plan_set_wait_limit": (C.c_int, [C.c_void_p, C.c_int64, C.c_int]),
    "msc_plan_status": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "msc_build_t0": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double]),
    "msc_t0_scalars": (C.c_int, [C.c_void_p, C.c_void_p]),
    "msc_set_t0_scalars": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double]),
    "msc_build_g0": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_int, C.c_int]),
    "msc_incident": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_int, C.c_void_p]),
    "msc_matvec": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "msc_matvec_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "msc_matvec_soa": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "msc_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(SolveOpts), C.POINTER(SolveStats)]),
    "msc_solve_multi": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.POINTER(SolveOpts),
                                  C.POINTER(SolveStats)]),
    "msc_matvec_multi": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int]),
    "msc_set_nearfield": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "msc_batch_solve": (C.c_int, [C.POINTER(BatchItem), C.c_int, C.POINTER(SolveOpts), C.c_int,
                                  C.POINTER(C.c_int)]),
    "msc_nearfield_blocks": (C.c_int, [C.c_void_p, C.c_void_p]),
    "msc_set_nearfield_weights": (C.c_int, [C.c_void_p, C.c_int]),
    "msc_nearfield_scale": (C.c_double, [C.c_void_p]),
    "msc_nf_loss_grad": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p]),
    "msc_nf_train": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p,
                               C.c_void_p, C.c_void_p, C.c_void_p]),
    "msc_precondition": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "msc_rpp_periodic": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_int, C.c_void_p]),
    "msc_reflected_field": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p]),
    "msc_status_string": (C.c_char_p, [C.c_int]),
    "msc_last_error": (C.c_char_p, []),
    "msc_version": (C.c_char_p, []),
    "msc_launch_count": (C.c_int64, []),
}

_lib = None


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load (once) and return the library with typed entry points."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"{p} is missing: build it with `python -m multiplescatteringcalculations_b200.build` "
            "(this package has no CPU fallback)"
        )
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


class MscError(RuntimeError):
    """A negative status returned by the native library."""

    def __init__(self, status: int, where: str):
        lib = load()
        self.status = status
        name = lib.msc_status_string(status).decode()
        msg = lib.msc_last_error().decode()
        super().__init__(f"{where}: {name}: {msg}")


def check(status: int, where: str) -> int:
    """Raise on errors (ValueError for invalid arguments); return warning statuses."""
    if status >= 0:
        return status
    if status == MSC_ERR_INVALID:
        lib = load()
        raise ValueError(f"{where}: {lib.msc_last_error().decode()}")
    raise MscError(status, where)
