"""CPU tests of the C-ABI library: it loads, exports every symbol the header declares, and fails loudly."""
import os
import re
import subprocess

import pytest

from bosss_b200 import native as nat

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    text = open(os.path.join(ROOT, "include", "bsgpu.h")).read()
    return sorted(set(re.findall(r"BSGPU_API\s+int\s+(bsgpu_\w+)\s*\(", text)))


def test_header_and_binding_agree():
    assert header_symbols() == sorted(nat.EXPORTS)


def test_library_exports_every_declared_symbol():
    out = subprocess.run(["nm", "-D", "--defined-only", nat.LIB_PATH], capture_output=True, text=True, check=True)
    exported = set(re.findall(r"\sT\s(bsgpu_\w+)", out.stdout))
    missing = [s for s in header_symbols() if s not in exported]
    assert not missing, missing
    lib = nat.lib()
    for s in header_symbols():
        assert getattr(lib, s) is not None


def test_version_and_error_reporting():
    import ctypes as C
    a, b = C.c_int(), C.c_int()
    assert nat.lib().bsgpu_get_version(C.byref(a), C.byref(b)) == 0
    assert (a.value, b.value) >= (0, 1)
    # a null handle is an argument error, reported through bsgpu_last_error
    rc = nat.lib().bsgpu_matrix_get_info(None, None, None, None, None)
    assert rc == nat.ERR_ARGUMENT
    assert "null" in nat.last_error()


def test_no_silent_fallback_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from bosss_b200 import assembly as A
    from bosss_b200.solvers import BlockMsrMatrix
    s = A.poisson_3d(2, 1)
    with pytest.raises(nat.BsgpuError):
        BlockMsrMatrix.from_system(s)


def test_solver_config_defaults_follow_reference():
    import ctypes as C
    c = nat.SolverConfig()
    assert nat.lib().bsgpu_solver_config_default(C.byref(c)) == 0
    # IterativeSolverConfig.cs:19-40, PmgConfig.cs:160, FGMRES MaxKrylovDim
    assert c.tol == 1e-10 and c.max_iter == 300 and c.min_iter == 1
    assert c.post_sweeps == 10 and c.bj_iters == 1 and c.bj_omega == 1.0
    assert c.sub_max_iter == 100 and c.sub_reduction == 0.1


def _c_layout(tmp_path, struct, fields):
    """sizeof and offsetof of `struct` as the C compiler lays it out from include/bsgpu.h."""
    src = tmp_path / "layout.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "bsgpu.h"', 'int main(void) {',
             f'  printf("%zu\\n", sizeof({struct}));']
    lines += [f'  printf("%zu\\n", offsetof({struct}, {f}));' for f in fields]
    lines += ['  return 0;', '}']
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    return vals[0], vals[1:]


@pytest.mark.parametrize("struct,cls", [("bsgpu_solver_config", nat.SolverConfig),
                                        ("bsgpu_solve_stats", nat.SolveStats)])
def test_struct_layouts_match_the_header(tmp_path, struct, cls):
    """The ctypes mirrors (and so the C# binding text built the same way) lay the structs out as the C compiler."""
    import ctypes as C
    names = [f[0] for f in cls._fields_]
    size, offsets = _c_layout(tmp_path, struct, names)
    assert size == C.sizeof(cls)
    assert offsets == [getattr(cls, n).offset for n in names]


def test_argument_errors_need_no_device():
    """Null handles and bad sizes are BSGPU_ERR_ARGUMENT (the reference's ArgumentException), reported before any
    device work; destroying a null handle is a no-op."""
    import ctypes as C
    L = nat.lib()
    h = C.c_void_p()
    assert L.bsgpu_matrix_create(C.byref(h), 4, 2, None, None, None, None, 0) == nat.ERR_ARGUMENT
    assert L.bsgpu_matrix_create(C.byref(h), -1, 2, None, None, None, None, 0) == nat.ERR_ARGUMENT
    assert "nb" in nat.last_error()
    assert L.bsgpu_solver_config_default(None) == nat.ERR_ARGUMENT
    assert L.bsgpu_solver_create(C.byref(h), None, None) == nat.ERR_ARGUMENT
    assert L.bsgpu_solver_solve(None, None, None, None) == nat.ERR_ARGUMENT
    assert L.bsgpu_matrix_spmv(None, 1.0, None, 0.0, None) == nat.ERR_ARGUMENT
    assert L.bsgpu_matrix_spmv_noalloc(None, 1.0, None, 0.0, None) == nat.ERR_ARGUMENT
    assert L.bsgpu_matrix_destroy(None) == 0 and L.bsgpu_solver_destroy(None) == 0 and L.bsgpu_mgop_destroy(None) == 0
    with pytest.raises(ValueError):
        nat.check(nat.ERR_ARGUMENT)
