"""msc_matvec_noalloc: the operator without device allocation on the call path.

Callers whose device memory belongs to another allocator, or real-time loops that
must not risk an allocation's latency or failure mid-run, apply the operator
through this entry point; its scratch is the library's static device array
(64 MiB at most). These tests compare it, through the C-ABI, with msc_matvec on
two calls in a row (the array keeps the first call's contents when the second
starts), and check that a plan too large for the array is refused. The file is
named so that pytest collects it last.
"""

import ctypes as C

import numpy as np
import pytest
import torch

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
OMEGA = 150.0


def _plan(M, Nz, periodic):
    g = SlabGeometry(M, Nz, 1.0)
    mat = random_slab_material(g, REF, MaterialContrast(2e9, 1e9, 100.0), 0.5, seed=M * 10 + Nz)
    plan = SlabPlan(g, REF, periodic=periodic)
    plan.build_t0(mat, OMEGA)
    plan.build_g0(OMEGA)
    return g, plan


def _call(lib, name, plan, x, precision):
    y = torch.empty_like(x)
    st = getattr(lib, name)(plan.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), precision)
    return st, y


@pytest.mark.parametrize("M,Nz,periodic", [(12, 3, False), (10, 4, True), (64, 16, False), (96, 16, False)])
@pytest.mark.parametrize("precision", [_native.MSC_COMPLEX64, _native.MSC_COMPLEX128])
def test_noalloc_matches_matvec_twice(M, Nz, periodic, precision):
    lib = _native.load()
    g, plan = _plan(M, Nz, periodic)
    dt = torch.complex128 if precision == _native.MSC_COMPLEX128 else torch.complex64
    rtol = 1e-10 if precision == _native.MSC_COMPLEX128 else 1e-5
    torch.manual_seed(M + Nz)
    Lz, Lx, Ly = plan.fft_sizes()
    need = (16 if precision else 8) * (9 * Nz * Ly * Lx + 18 * g.n_cubes)  # workspace + two fields
    for _ in range(2):
        x = torch.randn(Nz, M, M, 9, dtype=dt, device=plan.device)
        st_ref, y_ref = _call(lib, "msc_matvec", plan, x, precision)
        assert st_ref == 0
        st, y = _call(lib, "msc_matvec_noalloc", plan, x, precision)
        if need > (64 << 20):
            assert st == _native.MSC_ERR_INVALID
            assert b"static limit" in lib.msc_last_error()
            return
        assert st == 0, lib.msc_last_error()
        torch.cuda.synchronize()
        a, b = y.cpu().numpy(), y_ref.cpu().numpy()
        assert np.linalg.norm(a - b) <= rtol * np.linalg.norm(b)


def test_noalloc_rejects_bad_arguments():
    lib = _native.load()
    g, plan = _plan(4, 2, False)
    x = torch.zeros(2, 4, 4, 9, dtype=torch.complex64, device=plan.device)
    assert lib.msc_matvec_noalloc(plan.handle, C.c_void_p(x.data_ptr()), C.c_void_p(x.data_ptr()), 0) == \
        _native.MSC_ERR_INVALID
    y = torch.empty_like(x)
    assert lib.msc_matvec_noalloc(plan.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), 7) == \
        _native.MSC_ERR_INVALID


def test_noalloc_on_fresh_plan_allocates_nothing():
    """On a plan that has never run msc_matvec, the no-allocation call comes first:
    the plan's device bytes and the device's free memory are the same before and
    after it (the library's kernels and the static array are loaded beforehand by
    calls of both precisions on another plan), and its result then matches
    msc_matvec."""
    lib = _native.load()
    g0, warm = _plan(8, 2, False)
    for prec, dt in ((_native.MSC_COMPLEX64, torch.complex64), (_native.MSC_COMPLEX128, torch.complex128)):
        xw = torch.randn(2, 8, 8, 9, dtype=dt, device=warm.device)
        assert _call(lib, "msc_matvec_noalloc", warm, xw, prec)[0] == 0
    g, plan = _plan(32, 8, False)
    torch.manual_seed(5)
    for precision, dt, rtol in ((_native.MSC_COMPLEX64, torch.complex64, 1e-5),
                                (_native.MSC_COMPLEX128, torch.complex128, 1e-10)):
        x = torch.randn(8, 32, 32, 9, dtype=dt, device=plan.device)
        y = torch.empty_like(x)
        torch.cuda.synchronize()
        plan_bytes = lib.msc_plan_device_bytes(plan.handle)
        free0 = torch.cuda.mem_get_info()[0]
        st = lib.msc_matvec_noalloc(plan.handle, C.c_void_p(x.data_ptr()), C.c_void_p(y.data_ptr()), precision)
        torch.cuda.synchronize()
        assert st == 0, lib.msc_last_error()
        assert lib.msc_plan_device_bytes(plan.handle) == plan_bytes
        assert torch.cuda.mem_get_info()[0] == free0
        st_ref, y_ref = _call(lib, "msc_matvec", plan, x, precision)
        assert st_ref == 0
        assert lib.msc_plan_device_bytes(plan.handle) > plan_bytes  # msc_matvec allocated its field copies
        a, b = y.cpu().numpy(), y_ref.cpu().numpy()
        assert np.linalg.norm(a - b) <= rtol * np.linalg.norm(b)
