"""GPU parity of the block operations and solvers against the oracle and an FP64 direct solve (C ABI)."""
import numpy as np
import pytest

import oracle as O
from bosss_b200 import assembly as A
from bosss_b200.solvers import (BlockJacobiConfig, BlockMsrMatrix, FGMRESConfig, MultigridOperator, PmgConfig,
                                SoftPCGConfig)
from helpers import random_var_bsr

pytestmark = pytest.mark.gpu

SOL_TOL = 1e-9  # relative L2 error of solutions against the FP64 direct solve (the solution criterion)


def test_change_of_basis_matches_oracle(cuda):
    for s in (A.poisson_3d(5, 3), A.poisson_2d_c1(n=8)):
        ref_vals, ref_L = O.change_of_basis(O.Bsr.of(s))
        M = BlockMsrMatrix.from_system(s)
        op = MultigridOperator(M)
        got = op.OperatorMatrix.read_values()
        assert np.abs(got - ref_vals).max() <= 1e-12 * np.abs(ref_vals).max()
        L = op.LeftChangeOfBasis(len(ref_L))
        assert np.abs(L - ref_L).max() <= 1e-12 * np.abs(ref_L).max()


def test_change_of_basis_uneven_blocks(cuda):
    v = random_var_bsr(60, 10, seed=11, max_spc=2, spd=True)
    ref_vals, _ = O.change_of_basis(O.Bsr.of(v))
    op = MultigridOperator(BlockMsrMatrix.from_system(v))
    got = op.OperatorMatrix.read_values(len(v.values))
    assert np.abs(got - ref_vals).max() <= 1e-11 * np.abs(ref_vals).max()


def test_symminv_rejects_indefinite_zero_pivot(cuda):
    v = random_var_bsr(10, 4, seed=3, max_spc=1, spd=True)
    v.values[:16] = 0.0  # first diagonal block of block row 0 is zero
    M = BlockMsrMatrix.from_system(v)
    with pytest.raises(ArithmeticError):
        MultigridOperator(M)


def test_restriction_matches_oracle(cuda):
    s = A.poisson_3d(4, 3)
    ref, _ = O.restrict(O.Bsr.of(s), 10)
    sub = BlockMsrMatrix.from_system(s).Restrict(10)
    assert np.array_equal(sub.read_values(), ref)
    v = random_var_bsr(40, 10, seed=12, max_spc=2)
    ref2, _ = O.restrict(O.Bsr.of(v), 4)
    sub2 = BlockMsrMatrix.from_system(v).Restrict(4)
    assert np.array_equal(sub2.read_values(len(ref2)), ref2)


@pytest.mark.parametrize("Np,spc", [(4, 1), (10, 1), (20, 1), (10, 2), (1, 2), (4, 2), (20, 2)])
def test_blockjacobi_matches_oracle(cuda, Np, spc):
    v = random_var_bsr(80, Np, seed=Np, max_spc=spc, spd=True)
    ref = O.blockjacobi(O.Bsr.of(v), np.zeros(v.N), v.rhs, iters=1)
    op = MultigridOperator(BlockMsrMatrix.from_system(v), MultigridOperator.Eye)
    bj = BlockJacobiConfig(NoOfIterations=1).CreateInstance(op)
    x = np.zeros(v.N)
    bj.Solve(x, v.rhs)
    assert np.abs(x - ref).max() <= 1e-12 * np.abs(ref).max()


def _direct(s):
    return O.direct_solve(s)


def test_softpcg_c1_small(cuda):
    """C1-shaped: 2-D SIP p = 2, block-Jacobi PCG (SoftPCG) to 1e-12, against the direct solve."""
    s = A.poisson_2d_c1(n=32)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    slv = SoftPCGConfig(ConvergenceCriterion=1e-12, termination="relative", MaxSolverIterations=5000).CreateInstance(op)
    x = np.zeros(s.N)
    slv.Solve(x, s.rhs)
    xd = _direct(s)
    assert slv.Converged
    assert np.linalg.norm(x - xd) <= SOL_TOL * np.linalg.norm(xd)
    # iteration count within a few of the oracle's PCG on the same transformed system
    vals, Lc = O.change_of_basis(O.Bsr.of(s))

    class T:
        Np, row_ptr, col_idx, values = s.Np, s.row_ptr, s.col_idx, vals
    from helpers import apply_blocks
    bl = np.full(s.nb, s.Np)
    r = O.solve(O.Bsr.of(T), apply_blocks(Lc, bl, s.rhs),
                O.SolverConfig(solver=O.PCG, tol=1e-12, top_mode=O.TERM_RELATIVE, bj_iters=0, max_iter=5000))
    assert abs(r.iterations - slv.ThisLevelIterations) <= max(3, 0.02 * r.iterations)


@pytest.mark.parametrize("mixed", [False, True])
def test_fgmres_pmg_3d(cuda, mixed):
    """C2-shaped at 8^3: FGMRES(30) + 3-level p-MG (p = 3 -> 2 -> 1) with block-Jacobi smoothing."""
    s = A.poisson_3d(8, 3)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    cfg = FGMRESConfig(ConvergenceCriterion=1e-12, termination="relative", MaxKrylovDim=30,
                       Preconditioners=[PmgConfig(DegreeHierarchy=(20, 10, 4), CoarseTolerance=1e-4)],
                       MixedPrecision=mixed)
    slv = cfg.CreateInstance(op)
    x = np.zeros(s.N)
    slv.Solve(x, s.rhs)
    xd = _direct(s)
    assert slv.Converged
    assert np.linalg.norm(x - xd) <= SOL_TOL * np.linalg.norm(xd)
    # the same configuration in the oracle needs a similar number of outer iterations
    vals, Lc = O.change_of_basis(O.Bsr.of(s))

    class T:
        Np, row_ptr, col_idx, values = s.Np, s.row_ptr, s.col_idx, vals
    from helpers import apply_blocks
    bl = np.full(s.nb, s.Np)
    r = O.solve(O.Bsr.of(T), apply_blocks(Lc, bl, s.rhs),
                O.SolverConfig(solver=O.FGMRES_PMG, tol=1e-12, top_mode=O.TERM_RELATIVE, level_keep=(20, 10, 4),
                               coarse_kind=O.COARSE_PCG, coarse_tol=1e-4))
    assert abs(r.iterations - slv.ThisLevelIterations) <= (3 if not mixed else 5)


@pytest.mark.parametrize("mixed", [False, True])
def test_fgmres_pmg_with_h_levels(cuda, mixed):
    """p-levels 3 -> 2 -> 1 -> 0, then aggregation h-levels on p = 0 down to a dense direct solve."""
    s = A.poisson_3d(10, 3)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    pmg = PmgConfig(DegreeHierarchy=(20, 10, 4, 1), HLevels=4, HSweeps=3, DenseLimit=40)
    slv = FGMRESConfig(ConvergenceCriterion=1e-12, termination="relative", Preconditioners=[pmg],
                       MixedPrecision=mixed).CreateInstance(op)
    x = np.zeros(s.N)
    slv.Solve(x, s.rhs)
    xd = _direct(s)
    assert slv.Converged and slv.ThisLevelIterations < 40
    assert np.linalg.norm(x - xd) <= SOL_TOL * np.linalg.norm(xd)


@pytest.mark.parametrize("mixed", [False, True])
def test_fgmres_pmg_with_amg_coarse(cuda, mixed):
    """p-levels 3 -> 2 -> 1; the p = 1 level solved by CG + smoothed-aggregation AMG."""
    s = A.poisson_3d(10, 3)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    pmg = PmgConfig(DegreeHierarchy=(20, 10, 4), CoarseSolver="amg", HLevels=4, HSweeps=2, DenseLimit=64,
                    CoarseTolerance=1e-1, CoarseMaxIterations=30)
    slv = FGMRESConfig(ConvergenceCriterion=1e-12, termination="relative", Preconditioners=[pmg],
                       MixedPrecision=mixed).CreateInstance(op)
    x = np.zeros(s.N)
    slv.Solve(x, s.rhs)
    xd = _direct(s)
    assert slv.Converged and slv.ThisLevelIterations < 40
    assert np.linalg.norm(x - xd) <= SOL_TOL * np.linalg.norm(xd)


@pytest.mark.parametrize("mixed", [False, True])
def test_fgmres_pmg_with_h_multigrid_coarse(cuda, mixed):
    """p-levels 3 -> 2 -> 1; the p = 1 level solved by h-multigrid on 2x2x2 agglomerations (16^3 -> 8^3 -> 4^3)."""
    s = A.poisson_3d(16, 3)
    hl = A.h_hierarchy(s.grid, 1)
    assert [P.nb_coarse for P in hl] == [512, 64]
    op = MultigridOperator(BlockMsrMatrix.from_system(s), h_levels=hl)
    pmg = PmgConfig(DegreeHierarchy=(20, 10, 4), CoarseSolver="hmg", HSweeps=2, HCycle=1, CoarseTolerance=1e-1,
                    CoarseMaxIterations=20, DenseLimit=256, HSmoother="blockgs")
    slv = FGMRESConfig(ConvergenceCriterion=1e-12, termination="relative", Preconditioners=[pmg],
                       MixedPrecision=mixed).CreateInstance(op)
    x = np.zeros(s.N)
    slv.Solve(x, s.rhs)
    xd = _direct(s)
    assert slv.Converged and slv.ThisLevelIterations < 40
    assert np.linalg.norm(x - xd) <= SOL_TOL * np.linalg.norm(xd)


def test_h_multigrid_needs_prolongations(cuda):
    s = A.poisson_3d(4, 3)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    pmg = PmgConfig(DegreeHierarchy=(20, 10, 4), CoarseSolver="hmg")
    with pytest.raises(ValueError):
        FGMRESConfig(Preconditioners=[pmg]).CreateInstance(op)


def test_dense_coarse_solve(cuda):
    s = A.poisson_3d(4, 2)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    pmg = PmgConfig(DegreeHierarchy=(10, 4, 1), CoarseSolver="dense")
    slv = FGMRESConfig(ConvergenceCriterion=1e-12, termination="relative", Preconditioners=[pmg]).CreateInstance(op)
    x = np.zeros(s.N)
    slv.Solve(x, s.rhs)
    xd = _direct(s)
    assert slv.Converged
    assert np.linalg.norm(x - xd) <= SOL_TOL * np.linalg.norm(xd)


def test_orthomg_pmg_3d(cuda):
    s = A.poisson_3d(6, 2)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    slv = PmgConfig(ConvergenceCriterion=1e-11, termination="relative", DegreeHierarchy=(10, 4),
                    CoarseTolerance=1e-4).CreateInstance(op)
    x = np.zeros(s.N)
    slv.Solve(x, s.rhs)
    xd = _direct(s)
    assert slv.Converged
    assert np.linalg.norm(x - xd) <= SOL_TOL * np.linalg.norm(xd)


def test_nonzero_initial_guess(cuda):
    s = A.poisson_3d(5, 2)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    slv = FGMRESConfig(ConvergenceCriterion=1e-12, termination="relative",
                       Preconditioners=[PmgConfig(DegreeHierarchy=(10, 4), CoarseTolerance=1e-4)]).CreateInstance(op)
    xd = _direct(s)
    x = xd + 1e-3 * np.random.default_rng(0).standard_normal(s.N)
    slv.Solve(x, s.rhs)
    assert np.linalg.norm(x - xd) <= SOL_TOL * np.linalg.norm(xd)


def test_solver_argument_errors(cuda):
    s = A.poisson_3d(3, 1)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    slv = SoftPCGConfig().CreateInstance(op)
    with pytest.raises(ValueError):
        slv.Solve(np.zeros(s.N + 1), s.rhs)


def test_nan_rhs_raises_arithmetic_error(cuda):
    s = A.poisson_3d(4, 2)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    slv = FGMRESConfig(Preconditioners=[PmgConfig(DegreeHierarchy=(10, 4))]).CreateInstance(op)
    b = s.rhs.copy()
    b[5] = np.nan
    with pytest.raises(ArithmeticError):
        slv.Solve(np.zeros(s.N), b)


@pytest.mark.parametrize("mixed", [False, True])
def test_block_gauss_seidel_smoother(cuda, mixed):
    """Symmetric multicolour block Gauss-Seidel on the p-levels, capped PCG coarse solve."""
    s = A.poisson_3d(8, 3)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    pmg = PmgConfig(DegreeHierarchy=(20, 10, 4), Smoother="blockgs", CoarseTolerance=1e-1, CoarseMaxIterations=40)
    slv = FGMRESConfig(ConvergenceCriterion=1e-12, termination="relative", Preconditioners=[pmg],
                       MixedPrecision=mixed).CreateInstance(op)
    x = np.zeros(s.N)
    slv.Solve(x, s.rhs)
    xd = _direct(s)
    assert slv.Converged
    assert np.linalg.norm(x - xd) <= SOL_TOL * np.linalg.norm(xd)


@pytest.mark.parametrize("mode", ["fgmres", "presmooth", "both"])
def test_learned_stage_trains_and_solves(cuda, mode):
    """Learned preconditioner stage: trains on solver-generated residuals (energy loss below that of a zero
    correction) and FGMRES still converges to the direct solution with the stage in place."""
    s = A.poisson_3d(8, 3)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    op.SetCellGraph(s.grid.face_neighbours())
    pmg = PmgConfig(DegreeHierarchy=(20, 10, 4), CoarseTolerance=1e-1, CoarseMaxIterations=60)
    slv = FGMRESConfig(ConvergenceCriterion=1e-12, termination="relative", Preconditioners=[pmg],
                       MixedPrecision=True, Learned=mode).CreateInstance(op)
    loss = slv.TrainLearned(n_rhs=1, steps=60, lr=2e-3, seed=3)
    assert loss < 0.0
    x = np.zeros(s.N)
    slv.Solve(x, s.rhs)
    xd = _direct(s)
    assert slv.Converged
    assert np.linalg.norm(x - xd) <= SOL_TOL * np.linalg.norm(xd)


def test_learned_stage_needs_cell_graph(cuda):
    s = A.poisson_3d(4, 2)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    with pytest.raises(ValueError):
        FGMRESConfig(Preconditioners=[PmgConfig(DegreeHierarchy=(10, 4))], Learned="fgmres").CreateInstance(op)


@pytest.mark.parametrize("precond", [None, "blockjacobi", "ilu"])
def test_softgmres(cuda, precond):
    """SoftGMRES (left-preconditioned restarted GMRES) against the direct solve."""
    from bosss_b200.solvers import SoftGMRESConfig
    s = A.poisson_3d(5, 2)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    slv = SoftGMRESConfig(ConvergenceCriterion=1e-13, termination="relative", MaxKrylovDim=40,
                          MaxSolverIterations=3000, Precond=precond).CreateInstance(op)
    x = np.zeros(s.N)
    slv.Solve(x, s.rhs)
    xd = _direct(s)
    assert slv.Converged
    assert np.linalg.norm(x - xd) <= SOL_TOL * np.linalg.norm(xd)


def test_softgmres_rejects_pmg(cuda):
    from bosss_b200.solvers import SoftGMRESConfig
    op = MultigridOperator(BlockMsrMatrix.from_system(A.poisson_3d(3, 2)))
    with pytest.raises(ValueError):
        SoftGMRESConfig(Precond=PmgConfig(DegreeHierarchy=(10, 4))).CreateInstance(op)


@pytest.mark.parametrize("mixed", [False, True])
def test_recalc_resi_period(cuda, mixed):
    """RecalcResiPeriod > 1: the OrthoMG residual is updated and recomputed every 40 history entries."""
    s = A.poisson_3d(8, 3)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    pmg = PmgConfig(DegreeHierarchy=(20, 10, 4), CoarseTolerance=1e-1, CoarseMaxIterations=60, RecalcResiPeriod=40)
    slv = FGMRESConfig(ConvergenceCriterion=1e-12, termination="relative", Preconditioners=[pmg],
                       MixedPrecision=mixed).CreateInstance(op)
    x = np.zeros(s.N)
    slv.Solve(x, s.rhs)
    xd = _direct(s)
    assert slv.Converged
    assert np.linalg.norm(x - xd) <= SOL_TOL * np.linalg.norm(xd)
