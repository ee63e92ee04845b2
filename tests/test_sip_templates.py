"""CPU test of the GPU assembly's block templates (bsgpu_sip_templates: host computation in the library, no device
work) against the host assembly's own building blocks (assembly.py: 1-D stiffness by Gauss quadrature, traces and
normal derivatives of the orthonormal Legendre basis, Kronecker expansion over the modes)."""
import ctypes as C

import numpy as np
import pytest

from bosss_b200 import assembly as A
from bosss_b200 import native as nat


def _templates(D, p, h):
    hh = (C.c_double * D)(*h)
    n = C.c_int64()
    nat.check(nat.lib().bsgpu_sip_templates(D, p, hh, None, 0, C.byref(n)))
    out = np.zeros(n.value)
    nat.check(nat.lib().bsgpu_sip_templates(D, p, hh, nat.ptr(out), n.value, None))
    Np = A.np_of(D, p)
    return out.reshape(-1, Np, Np)


def _expected(D, p, h):
    modes = A.dg_modes(D, p)
    Np = len(modes)
    S = A.stiffness_1d(p)
    ex = lambda F, d: A._expand_1d(F[None], modes, d)[0]
    o = np.outer
    T = np.zeros((31, Np, Np))
    for d in range(D):
        T[0] += ex(4.0 / h[d] ** 2 * S, d)
        tL, dL = (v[0] for v in A._face_vectors(p, np.array([h[d]]), +1.0))
        tR, dR = (v[0] for v in A._face_vectors(p, np.array([h[d]]), -1.0))
        b = 1 + 4 * d
        T[b] = ex(-0.5 * (o(tL, dL) + o(dL, tL)), d)
        T[b + 1] = ex(o(tL, tL), d)
        T[b + 2] = ex(0.5 * (o(tR, dR) + o(dR, tR)), d)
        T[b + 3] = ex(o(tR, tR), d)
        ob = 13 + 6 * d
        T[ob] = ex(-0.5 * o(tL, dR), d)
        T[ob + 1] = ex(0.5 * o(dL, tR), d)
        T[ob + 2] = ex(-o(tL, tR), d)
    return T


@pytest.mark.parametrize("D,p,h", [(1, 3, [0.25]), (2, 2, [1 / 64, 1 / 32]), (3, 3, [1 / 64] * 3),
                                   (3, 0, [0.5, 0.25, 0.125]), (3, 2, [0.1, 0.2, 0.3]), (2, 6, [0.5, 0.5])])
def test_templates_match_host_assembly(D, p, h):
    got, want = _templates(D, p, h), _expected(D, p, h)
    assert got.shape == want.shape
    scale = np.abs(want).max()
    assert np.abs(got - want).max() <= 1e-13 * scale


def test_templates_reject_bad_arguments():
    with pytest.raises(nat.BsgpuError):
        _templates(4, 1, [1.0] * 4)
    with pytest.raises(nat.BsgpuError):
        _templates(2, 1, [1.0, -1.0])
