"""CPU test of the natural-order ILU(0) wavefronts the library builds on the host (bsgpu_ilu_wavefronts: no device
work): 3n - 2 wavefronts on an n^3 Cartesian grid (2n - 1 on n^2), every block row exactly once, each row one
wavefront after the latest of its lower neighbours, so the rows of a wavefront never depend on each other."""
import ctypes as C

import numpy as np
import pytest

from bosss_b200 import assembly as A
from bosss_b200 import native as nat
from bosss_b200 import xdg


def _wavefronts(s):
    rp = np.ascontiguousarray(s.row_ptr, np.int64)
    ci = np.ascontiguousarray(s.col_idx, np.int32)
    nb = len(rp) - 1
    nl = C.c_int64()
    f = nat.lib().bsgpu_ilu_wavefronts
    nat.check(f(nb, nat.ptr(rp), nat.ptr(ci), None, None, C.byref(nl)))
    lptr = np.zeros(nl.value + 1, np.int64)
    rows = np.zeros(max(nb, 1), np.int32)
    nat.check(f(nb, nat.ptr(rp), nat.ptr(ci), nat.ptr(lptr), nat.ptr(rows), None))
    return lptr, rows[:nb]


def _check_levels(s, lptr, rows):
    nb = len(s.row_ptr) - 1
    assert np.array_equal(np.sort(rows), np.arange(nb))
    level = np.empty(nb, np.int64)
    for l in range(len(lptr) - 1):
        seg = rows[lptr[l]:lptr[l + 1]]
        assert np.all(np.diff(seg) > 0)
        level[seg] = l
    for i in range(nb):
        lower = [j for j in s.col_idx[s.row_ptr[i]:s.row_ptr[i + 1]] if j < i]
        assert level[i] == (max(level[j] for j in lower) + 1 if lower else 0)


@pytest.mark.parametrize("n", [1, 2, 5, 8])
def test_cartesian_wavefront_counts(n):
    s3 = A.assemble_sip(A.uniform_grid(3, n), 1)
    lptr, rows = _wavefronts(s3)
    assert len(lptr) - 1 == 3 * n - 2
    _check_levels(s3, lptr, rows)
    s2 = A.assemble_sip(A.uniform_grid(2, n), 1)
    lptr2, rows2 = _wavefronts(s2)
    assert len(lptr2) - 1 == 2 * n - 1
    _check_levels(s2, lptr2, rows2)


def test_xdg_structure_levels():
    s = xdg.xdg_sphere(n=6, p=1, seed=1, mu=(1.0, 10.0))
    lptr, rows = _wavefronts(s)
    _check_levels(s, lptr, rows)
