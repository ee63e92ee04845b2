"""GPU parity of the block-sparse SpMV (BlockMsrMatrix.SpMV) against the oracle, through the C ABI."""
import numpy as np
import pytest

import oracle as O
from bosss_b200 import assembly as A
from bosss_b200.solvers import BlockMsrMatrix
from helpers import random_var_bsr

pytestmark = pytest.mark.gpu

TOL = 1e-13  # relative, FP64 (the SpMV parity criterion)


def _check(system, alpha, beta, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(system.N)
    y0 = rng.standard_normal(system.N)
    ref = O.spmv(O.Bsr.of(system), alpha, x, beta, y0.copy())
    M = BlockMsrMatrix.from_system(system)
    y = y0.copy()
    M.SpMV(alpha, x, beta, y)
    assert np.linalg.norm(y - ref) <= TOL * np.linalg.norm(ref)
    return M


@pytest.mark.parametrize("D,p", [(2, 2), (3, 1), (3, 2), (3, 3), (2, 1), (3, 0)])
def test_spmv_uniform_blocks(cuda, D, p):
    s = A.poisson_3d(5, p) if D == 3 else A.poisson_2d_c1(n=9, p=p)
    for alpha, beta in ((1.0, 0.0), (1.6, 0.5), (-1.0, 1.0)):
        _check(s, alpha, beta)


def test_spmv_uneven_blocks(cuda):
    v = random_var_bsr(300, 10, seed=4, max_spc=2, nnz_per_row=7)
    _check(v, 1.3, -0.7)


def test_spmv_uneven_odd_blocks(cuda):
    v = random_var_bsr(200, 3, seed=5, max_spc=3, nnz_per_row=4, empty_rows=True)
    _check(v, 1.0, 0.0)


def test_spmv_single_block(cuda):
    v = random_var_bsr(1, 20, seed=6, max_spc=1, nnz_per_row=1)
    _check(v, 2.0, 1.0)


def test_spmv_device_vectors_and_fp32(cuda):
    import torch
    s = A.poisson_3d(6, 3)
    M = BlockMsrMatrix.from_system(s)
    x = torch.randn(s.N, dtype=torch.float64, device=cuda)
    y = torch.zeros_like(x)
    M.SpMV(1.0, x, 0.0, y)
    ref = s.to_scipy() @ x.cpu().numpy()
    assert np.linalg.norm(y.cpu().numpy() - ref) <= TOL * np.linalg.norm(ref)
    M32 = M.ToSingle()
    x32 = x.float()
    y32 = torch.zeros_like(x32)
    M32.SpMV(1.0, x32, 0.0, y32)
    assert np.linalg.norm(y32.cpu().numpy() - ref) <= 1e-5 * np.linalg.norm(ref)


def test_spmv_argument_errors(cuda):
    s = A.poisson_3d(2, 1)
    M = BlockMsrMatrix.from_system(s)
    x = np.zeros(s.N)
    with pytest.raises(ValueError):
        M.SpMV(1.0, x, 0.0, x)
    with pytest.raises(ValueError):
        M.SpMV(1.0, np.zeros(s.N + 1), 0.0, np.zeros(s.N))


def test_read_values_roundtrip(cuda):
    v = random_var_bsr(50, 6, seed=8, max_spc=2)
    M = BlockMsrMatrix.from_system(v)
    assert np.array_equal(M.read_values(len(v.values)), v.values)


def test_spmv_full_size_properties(cuda):
    """3-D 64^3 p = 3 (5.24M unknowns, 1.81M 20x20 blocks): linearity, and agreement with the oracle on a
    sample of block rows."""
    import torch
    s = A.poisson_3d(64, 3)
    M = BlockMsrMatrix.from_system(s)
    g = torch.Generator(device="cpu").manual_seed(0)
    x1 = torch.randn(s.N, dtype=torch.float64, generator=g).to(cuda)
    x2 = torch.randn(s.N, dtype=torch.float64, generator=g).to(cuda)
    y1, y2, y3 = (torch.zeros_like(x1) for _ in range(3))
    M.SpMV(1.0, x1, 0.0, y1)
    M.SpMV(1.0, x2, 0.0, y2)
    M.SpMV(1.0, 2.0 * x1 - 3.0 * x2, 0.0, y3)
    lin = torch.linalg.norm(y3 - (2 * y1 - 3 * y2)) / torch.linalg.norm(y3)
    assert lin.item() < 1e-13
    # sampled rows against a CPU product of the same blocks
    rows = np.random.default_rng(1).choice(s.nb, 2000, replace=False)
    xh = x1.cpu().numpy()
    yh = y1.cpu().numpy()
    err = 0.0
    nrm = 0.0
    for i in rows:
        acc = np.zeros(20)
        for k in range(s.row_ptr[i], s.row_ptr[i + 1]):
            j = s.col_idx[k]
            acc += s.values[k] @ xh[j * 20:(j + 1) * 20]
        err += np.sum((yh[i * 20:(i + 1) * 20] - acc) ** 2)
        nrm += np.sum(acc ** 2)
    assert np.sqrt(err / nrm) < TOL


@pytest.mark.parametrize("Np", [1, 4, 10, 20])
def test_spmv_two_species_blocks_all_typed_sizes(cuda, Np):
    """Blocks of one or two species of Np modes (the XDG block types) for every Np the species-count kernels are
    specialised on, FP64 against the oracle and FP32 against the FP64 product, with empty rows."""
    import torch
    v = random_var_bsr(240, Np, seed=20 + Np, max_spc=2, nnz_per_row=6, empty_rows=True)
    M = _check(v, 0.9, -0.4, seed=Np)
    rng = np.random.default_rng(Np)
    x = rng.standard_normal(v.N)
    ref = v.to_scipy() @ x
    M32 = M.ToSingle()
    xt = torch.from_numpy(x).float().cuda()
    yt = torch.zeros_like(xt)
    M32.SpMV(1.0, xt, 0.0, yt)
    assert np.linalg.norm(yt.cpu().numpy() - ref) <= 1e-5 * np.linalg.norm(ref)
