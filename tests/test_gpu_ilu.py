"""GPU parity of the block ILU(0) smoother (CellILU) against the oracle's ILU(0) in the same cell order: the
reference's natural order (wavefront factorisation and triangular solves) and the two-colour order."""
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
    CellILUConfig(Order="coloured").CreateInstance(op).Solve(x, s.rhs)
    assert np.abs(x - ref).max() <= 1e-11 * np.abs(ref).max()


@pytest.mark.parametrize("n,p", [(5, 1), (4, 2), (3, 3), (7, 2)])
def test_cell_ilu_natural_order_matches_oracle(cuda, n, p):
    """The reference's order (CellILU.cs:1229-1330): factors and x = U^{-1} L^{-1} b against the oracle's
    natural-order ILU(0), on the operator and on its DiagBlockEquilib transform."""
    s = A.poisson_3d(n, p, seed=n + 10)
    Bo = O.Bsr.of(s)
    ref = O.ilu0_solve(Bo, O.ilu0_factor(Bo, None), s.rhs, None)
    op = MultigridOperator(BlockMsrMatrix.from_system(s), MultigridOperator.Eye)
    x = np.random.default_rng(1).standard_normal(s.N)
    CellILUConfig(Order="natural").CreateInstance(op).Solve(x, s.rhs)
    assert np.abs(x - ref).max() <= 1e-11 * np.abs(ref).max()


def test_cell_ilu_needs_uniform_blocks(cuda):
    v = random_var_bsr(30, 4, seed=5, max_spc=2, spd=True)
    op = MultigridOperator(BlockMsrMatrix.from_system(v), MultigridOperator.Eye)
    for order in ("natural", "coloured"):
        with pytest.raises(nat.BsgpuError):
            CellILUConfig(Order=order).CreateInstance(op)


def test_natural_ilu_pmg_iterations_match_oracle(cuda):
    """PmgConfig(UseILU = true) with the reference's natural-order smoother: FlexGMRES iteration count within one
    of the oracle's on the same transformed system, solution against the direct solve."""
    s = A.poisson_3d(6, 2, seed=3)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    pmg = PmgConfig(DegreeHierarchy=(10, 4, 1), UseILU=True, NoOfPostSmootherSweeps=4, CoarseTolerance=1e-1,
                    CoarseMaxIterations=60)
    slv = FGMRESConfig(ConvergenceCriterion=1e-10, termination="relative", Preconditioners=[pmg]).CreateInstance(op)
    x = np.zeros(s.N)
    slv.Solve(x, s.rhs)
    xd = O.direct_solve(s)
    assert slv.Converged
    assert np.linalg.norm(x - xd) <= SOL_TOL * np.linalg.norm(xd)
    vals, Lc = O.change_of_basis(O.Bsr.of(s))

    class T:
        Np, row_ptr, col_idx, values = s.Np, s.row_ptr, s.col_idx, vals
    from helpers import apply_blocks
    r = O.solve(O.Bsr.of(T), apply_blocks(Lc, np.full(s.nb, s.Np), s.rhs),
                O.SolverConfig(solver=O.FGMRES_PMG, tol=1e-10, top_mode=O.TERM_RELATIVE, level_keep=(10, 4, 1),
                               coarse_kind=O.COARSE_PCG, coarse_tol=1e-1, coarse_max_iter=60, post_sweeps=4,
                               smoother=O.SMOOTHER_ILU_NATURAL))
    assert abs(r.iterations - slv.ThisLevelIterations) <= 1, (r.iterations, slv.ThisLevelIterations)


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
