"""The C-ABI library loads and exports every entry point include/msc.h declares
(no compute calls: these run without a GPU)."""

import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _declared():
    src = (ROOT / "include" / "msc.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w]+\s*\*?\s*(msc_\w+)\s*\(", src, re.M)))


def test_header_declares_entry_points():
    names = _declared()
    for n in ("msc_plan_create", "msc_build_t0", "msc_build_g0", "msc_matvec", "msc_solve", "msc_rpp_periodic"):
        assert n in names


def test_library_exports_declared_symbols():
    from multiplescatteringcalculations_b200 import _native

    lib = _native.load()
    for n in _declared():
        assert hasattr(lib, n), n
        assert n in _native.SIGNATURES, f"{n} has no ctypes signature"
    out = subprocess.run(["nm", "-D", "--defined-only", str(_native.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (msc_\w+)", out))
    assert set(_declared()) <= exported


def test_status_strings_and_version():
    from multiplescatteringcalculations_b200 import _native

    lib = _native.load()
    assert lib.msc_status_string(0) == b"MSC_OK"
    assert lib.msc_status_string(-1) == b"MSC_ERR_INVALID"
    assert lib.msc_status_string(1) == b"MSC_NOT_CONVERGED"
    assert b"sm_100a" in lib.msc_version()


def test_plan_create_rejects_bad_geometry():
    """Argument checks happen before any device work, so they run on a CPU host."""
    import ctypes as C

    from multiplescatteringcalculations_b200 import _native as N

    lib = N.load()
    h = C.c_void_p()
    for bad in (dict(M=0), dict(N_z=0), dict(a=0.0), dict(beta=4000.0)):
        kw = dict(M=4, N_z=2, a=1.0, alpha=3000.0, beta=1732.0, rho=2500.0, periodic=0, Lz=0, Lxy=0)
        kw.update(bad)
        d = N.SlabDesc(**kw)
        assert lib.msc_plan_create(C.byref(d), None, C.byref(h)) == N.MSC_ERR_INVALID
        assert lib.msc_last_error()
    with pytest.raises(ValueError, match="M must be"):
        N.check(N.MSC_ERR_INVALID, "x") if False else N.check(
            lib.msc_plan_create(C.byref(N.SlabDesc(0, 2, 1.0, 3000.0, 1732.0, 2500.0, 0, 0, 0)), None, C.byref(h)),
            "msc_plan_create")


def test_struct_layouts_match_the_header(tmp_path):
    """The ctypes mirrors have the sizes and field offsets of the C structs."""
    import ctypes as C
    import shutil

    from multiplescatteringcalculations_b200 import _native as N

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "sz.c"
    src.write_text(
        '#include <stdio.h>\n#include <stddef.h>\n#include "msc.h"\n'
        "int main(void) {\n"
        '  printf("%zu %zu %zu %zu %zu %zu %zu\\n", sizeof(msc_slab_desc), sizeof(msc_solve_opts),\n'
        "         sizeof(msc_solve_stats), sizeof(msc_batch_item), offsetof(msc_batch_item, stats),\n"
        "         offsetof(msc_batch_item, status), offsetof(msc_solve_opts, preconditioner));\n"
        "  return 0;\n}\n")
    exe = tmp_path / "sz"
    subprocess.run([cc, "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    got = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [C.sizeof(N.SlabDesc), C.sizeof(N.SolveOpts), C.sizeof(N.SolveStats), C.sizeof(N.BatchItem),
            N.BatchItem.stats.offset, N.BatchItem.status.offset, N.SolveOpts.preconditioner.offset]
    assert got == want
