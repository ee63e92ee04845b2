"""GPU parity of the block ILU(0) smoother (CellILU) against the oracle's ILU(0) in the same cell order."""
import numpy as np
import pytest

import oracle as O
from bosss_b200 import assembly as A
from bosss_b200 import native as nat
from bosss_b200.solvers import BlockMsrMatrix, CellILUConfig, FGMRESConfig, MultigridOperator, PmgConfig
from helpers import greedy_colour_order, random_var_bsr

pytestmark = pytest.mark.gpu

SOL_TOL = 1e-9


@pytest.mark.parametrize("n,p", [(5, 1), (4, 2), (3, 3)])
def test_cell_ilu_matches_oracle(cuda, n, p):
    s = A.poisson_3d(n, p, seed=n)
    order = greedy_colour_order(s.row_ptr, s.col_idx)
    Bo = O.Bsr.of(s)
    F = O.ilu0_factor(Bo, order)
    ref = O.ilu0_solve(Bo, F, s.rhs, order)
    op = MultigridOperator(BlockMsrMatrix.from_system(s), MultigridOperator.Eye)
    x = np.random.default_rng(0).standard_normal(s.N)     # CellILU ignores the initial guess
    CellILUConfig().CreateInstance(op).Solve(x, s.rhs)
    assert np.abs(x - ref).max() <= 1e-11 * np.abs(ref).max()


def test_cell_ilu_needs_uniform_two_colour_blocks(cuda):
    v = random_var_bsr(30, 4, seed=5, max_spc=2, spd=True)
    op = MultigridOperator(BlockMsrMatrix.from_system(v), MultigridOperator.Eye)
    with pytest.raises(nat.BsgpuError):
        CellILUConfig().CreateInstance(op)


@pytest.mark.parametrize("mixed", [False, True])
def test_fgmres_pmg_with_ilu(cuda, mixed):
    s = A.poisson_3d(8, 3)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    pmg = PmgConfig(DegreeHierarchy=(20, 10, 4), UseILU=True, NoOfPostSmootherSweeps=4, CoarseTolerance=1e-1,
                    CoarseMaxIterations=60)
    slv = FGMRESConfig(ConvergenceCriterion=1e-12, termination="relative", Preconditioners=[pmg],
                       MixedPrecision=mixed).CreateInstance(op)
    x = np.zeros(s.N)
    slv.Solve(x, s.rhs)
    xd = O.direct_solve(s)
    assert slv.Converged
    assert np.linalg.norm(x - xd) <= SOL_TOL * np.linalg.norm(xd)
