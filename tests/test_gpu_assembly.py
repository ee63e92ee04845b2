"""The SIP operator assembled on the GPU (bsgpu_assemble_sip_cartesian, BlockMsrMatrix.AssembleSIP) against the
host assembly of the same grid (assembly.assemble_sip, the restatement of ipLaplace.cs:95-245): block structure
identical, values to 1e-13 relative; and a solve of the GPU-assembled operator against the direct solve."""
import numpy as np
import pytest

import oracle as O
from bosss_b200 import assembly as A
from bosss_b200.solvers import BlockMsrMatrix, FGMRESConfig, MultigridOperator, PmgConfig

pytestmark = pytest.mark.gpu


def _grid(shape):
    return A.RectilinearGrid(nodes=[np.linspace(0.0, 1.0, n + 1) for n in shape])


def _compare(shape, p, penalty, coeff=None, device_coeff=False):
    s = A.assemble_sip(_grid(shape), p, penalty=penalty, coeff=coeff)
    cf = coeff
    if coeff is not None and device_coeff:
        import torch
        cf = torch.from_numpy(np.asarray(coeff, np.float64)).cuda()
    M = BlockMsrMatrix.AssembleSIP(shape, p, penalty=penalty, coeff=cf)
    rp, ci, _ = M._structure
    assert M.N == s.N and M.Np == s.Np and M.nnzb == s.nnzb
    assert np.array_equal(rp, s.row_ptr) and np.array_equal(ci, s.col_idx)
    vals = M.read_values().reshape(s.values.shape)
    err = np.abs(vals - s.values).max() / np.abs(s.values).max()
    assert err <= 1e-13, err
    return M, s


@pytest.mark.parametrize("shape,p", [((7,), 1), ((6, 5), 2), ((4, 5, 3), 3), ((3, 3, 3), 0), ((5, 4, 6), 2)])
def test_assembly_matches_host_constant_coefficient(cuda, shape, p):
    _compare(shape, p, penalty=(p + 1) * (p + 2))


@pytest.mark.parametrize("device_coeff", [False, True])
def test_assembly_matches_host_variable_coefficient(cuda, device_coeff):
    shape = (5, 4, 6)
    rng = np.random.default_rng(3)
    k = np.exp(rng.standard_normal(int(np.prod(shape))))
    _compare(shape, 2, penalty=12.0, coeff=k, device_coeff=device_coeff)


def test_assembly_default_penalty_and_configured_c2_shape_block(cuda):
    """The reference's default penalty factor 1.3 * max((p+1)(p+D)/D, (p+1)^2) and a 32^3 p=3 operator (0.73 GB):
    the whole matrix against the host assembly."""
    M = BlockMsrMatrix.AssembleSIP((6, 6, 6), 2)
    s = A.assemble_sip(A.uniform_grid(3, 6), 2)
    assert np.abs(M.read_values().reshape(s.values.shape) - s.values).max() <= 1e-13 * np.abs(s.values).max()
    big = A.poisson_3d(32, 3, seed=0)
    Mb = BlockMsrMatrix.AssembleSIP((32, 32, 32), 3, penalty=20.0)
    vals = Mb.read_values().reshape(big.values.shape)
    assert np.abs(vals - big.values).max() <= 1e-13 * np.abs(big.values).max()


def test_solve_on_gpu_assembled_operator(cuda):
    """FlexGMRES + p-multigrid on the GPU-assembled 8^3 p=3 operator with the host right-hand side reaches the
    direct solution of the host-assembled system."""
    s = A.poisson_3d(8, 3, seed=0)
    M = BlockMsrMatrix.AssembleSIP((8, 8, 8), 3, penalty=20.0)
    op = MultigridOperator(M)
    slv = FGMRESConfig(ConvergenceCriterion=1e-12, termination="relative",
                       Preconditioners=[PmgConfig(DegreeHierarchy=(20, 10, 4), CoarseTolerance=1e-4)]
                       ).CreateInstance(op)
    x = np.zeros(s.N)
    slv.Solve(x, s.rhs)
    xd = O.direct_solve(s)
    assert slv.Converged
    assert np.linalg.norm(x - xd) <= 1e-9 * np.linalg.norm(xd)


@pytest.mark.parametrize("shape,p", [((9,), 3), ((6, 5), 3), ((5, 4, 3), 2), ((4, 4, 4), 3)])
def test_load_vector_on_gpu_matches_host(cuda, shape, p):
    """The sine-mode load vector with its products and mode sums on the GPU (bsgpu_project_separable) against the
    host projection (SineModes.project) to 1e-14 relative."""
    g = _grid(shape)
    sm = A.SineModes.seeded(5, len(shape))
    ref = sm.project(g, p).reshape(-1)
    got = sm.project_on_gpu(g, p).cpu().numpy()
    assert got.shape == ref.shape
    assert np.abs(got - ref).max() <= 1e-14 * np.abs(ref).max()
