"""GPU test of bsgpu_matrix_spmv_noalloc, the host-vector SpMV that allocates no device memory.

It exists for callers that must not allocate device memory (their GPU memory is committed to their own pool, or
they cannot afford the device-wide synchronisation cudaMalloc/cudaFree may cause).  Its result must equal that
of bsgpu_matrix_spmv, which stages through cudaMalloc'd buffers, within the SpMV tolerance of the other tests,
on consecutive calls (the shared staging array keeps the previous call's contents), and the device's free memory
must not change across its calls.  Collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from bosss_b200 import assembly as A
from bosss_b200 import native as nat
from bosss_b200.solvers import BlockMsrMatrix

pytestmark = pytest.mark.gpu

TOL = 1e-13  # relative, as the other FP64 SpMV tests


def _noalloc(M, alpha, x, beta, y):
    rc = nat.lib().bsgpu_matrix_spmv_noalloc(M._h, C.c_double(alpha), nat.ptr(x), C.c_double(beta), nat.ptr(y))
    nat.check(rc)
    return y


def _alloc(M, alpha, x, beta, y):
    nat.check(nat.lib().bsgpu_matrix_spmv(M._h, C.c_double(alpha), nat.ptr(x), C.c_double(beta), nat.ptr(y)))
    return y


def _free_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


def test_noalloc_spmv_matches_allocating_spmv(cuda):
    s = A.poisson_3d(12, 3)  # 34,560 unknowns
    M = BlockMsrMatrix.from_system(s)
    rng = np.random.default_rng(7)
    for call, (alpha, beta) in enumerate(((1.6, 0.5), (-1.0, 0.0))):  # two calls in a row
        x = rng.standard_normal(s.N)
        y0 = rng.standard_normal(s.N)
        ref = _alloc(M, alpha, x, beta, y0.copy())
        got = _noalloc(M, alpha, x, beta, y0.copy())
        assert np.linalg.norm(got - ref) <= TOL * np.linalg.norm(ref), call


def test_noalloc_spmv_leaves_free_device_memory_unchanged(cuda):
    s = A.poisson_3d(10, 3)
    M = BlockMsrMatrix.from_system(s)
    rng = np.random.default_rng(8)
    x = rng.standard_normal(s.N)
    y = np.zeros(s.N)
    _noalloc(M, 1.0, x, 0.0, y)  # first call: looks up the staging array's address
    free0 = _free_bytes()
    for _ in range(3):
        _noalloc(M, 0.5, x, 1.0, y)
    assert _free_bytes() == free0


def test_noalloc_spmv_rejects_oversized_matrix(cuda):
    s = A.poisson_3d(40, 3)  # 1,280,000 unknowns > 2^20
    M = BlockMsrMatrix.from_system(s)
    x = np.zeros(s.N)
    y = np.zeros(s.N)
    with pytest.raises(nat.BsgpuArgumentError, match="staging array"):
        _noalloc(M, 1.0, x, 0.0, y)
