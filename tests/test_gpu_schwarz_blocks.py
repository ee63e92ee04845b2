"""Additive Schwarz with multi-cell blocks (Schwarz.cs:56: METIS blocks, overlap growth, overlap scaling) on the GPU
against the oracle's restatement with the same partition, through the C ABI."""
import numpy as np
import pytest

import oracle as O
from bosss_b200 import assembly as A
from bosss_b200 import xdg
from bosss_b200.solvers import BlockMsrMatrix, FGMRESConfig, MultigridOperator, PmgConfig, SchwarzConfig
from helpers import random_var_bsr

pytestmark = pytest.mark.gpu

SOL_TOL = 1e-9


def _gpu(v, x0, parts, overlap, scaling, iters):
    op = MultigridOperator(BlockMsrMatrix.from_system(v), MultigridOperator.Eye)
    x = x0.copy()
    SchwarzConfig(FixedNoOfIterations=iters, NoOfParts=parts, Overlap=overlap,
                  EnableOverlapScaling=scaling).CreateInstance(op).Solve(x, v.rhs)
    return x


@pytest.mark.parametrize("parts,overlap,scaling,iters", [(12, 0, False, 1), (12, 1, False, 1), (12, 1, True, 2),
                                                         (7, 2, True, 1), (0, 1, False, 3)])
def test_block_schwarz_matches_oracle_uneven_blocks(cuda, parts, overlap, scaling, iters):
    """Blocks of one- and two-species cells (XDG block types), from a zero and from a nonzero initial guess."""
    v = random_var_bsr(60, 4, seed=40 + overlap, max_spc=2, nnz_per_row=3, spd=True)
    Bo = O.Bsr.of(v)
    for x0 in (np.zeros(v.N), np.random.default_rng(3).standard_normal(v.N)):
        ref = O.block_schwarz(Bo, x0, v.rhs, parts=parts, overlap=overlap, scaling=scaling, iters=iters)
        got = _gpu(v, x0, parts, overlap, scaling, iters)
        assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max(), (parts, overlap, scaling, iters)


def test_block_schwarz_matches_oracle_poisson(cuda):
    s = A.poisson_3d(4, 2, seed=5)
    Bo = O.Bsr.of(s)
    ref = O.block_schwarz(Bo, np.zeros(s.N), s.rhs, parts=10, overlap=1, scaling=True, iters=1)
    got = _gpu(s, np.zeros(s.N), 10, 1, True, 1)
    assert np.abs(got - ref).max() <= 1e-11 * np.abs(ref).max()


def test_block_schwarz_single_block_is_exact(cuda):
    """As addSchwarzTest.Test_Solution_IsCorrect (addSchwarzTest.cs:186-202): one block covering the whole system
    makes one application an exact solve."""
    s = A.poisson_3d(4, 1, seed=6)   # 256 unknowns: one dense block
    got = _gpu(s, np.zeros(s.N), 1, 0, False, 1)
    xs = np.linalg.solve(s.to_scipy().toarray(), s.rhs)
    assert np.linalg.norm(got - xs) <= 1e-12 * np.linalg.norm(xs)


def test_block_schwarz_rejects_oversized_blocks(cuda):
    from bosss_b200 import native as nat
    s = A.poisson_3d(6, 2)   # 2,160 unknowns in one block > 1024
    op = MultigridOperator(BlockMsrMatrix.from_system(s), MultigridOperator.Eye)
    with pytest.raises(nat.BsgpuError):
        SchwarzConfig(NoOfParts=1, Overlap=0).CreateInstance(op)


@pytest.mark.parametrize("mixed", [False, True])
def test_pmg_with_block_schwarz_smoother(cuda, mixed):
    """p-multigrid with the multi-cell Schwarz smoother on a two-species XDG system: solution against the direct
    solve; FP64 iteration count within one of the oracle's p-multigrid with the same smoother."""
    s = xdg.xdg_sphere(n=8, p=2, seed=1, mu=(1.0, 10.0))
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    pmg = PmgConfig(DegreeHierarchy=(10, 4, 1), Smoother="schwarz_blocks", SchwarzOverlap=1, SchwarzOverlapScaling=True,
                    NoOfPostSmootherSweeps=2, BlockJacobiIterations=0, CoarseTolerance=1e-2, CoarseMaxIterations=200)
    slv = FGMRESConfig(ConvergenceCriterion=1e-12, termination="relative", Preconditioners=[pmg],
                       MixedPrecision=mixed).CreateInstance(op)
    x = np.zeros(s.N)
    slv.Solve(x, s.rhs)
    xd = O.direct_solve(s)
    assert slv.Converged
    assert np.linalg.norm(x - xd) <= SOL_TOL * np.linalg.norm(xd)
    if not mixed:
        vals, Lc = O.change_of_basis(O.Bsr.of(s))

        class T:
            Np, row_ptr, col_idx, values, nspc = s.Np, s.row_ptr, s.col_idx, vals, s.nspc
        from helpers import apply_blocks
        bl = s.nspc.astype(np.int64) * s.Np
        r = O.solve(O.Bsr.of(T), apply_blocks(Lc, bl, s.rhs),
                    O.SolverConfig(solver=O.FGMRES_PMG, tol=1e-12, top_mode=O.TERM_RELATIVE, level_keep=(10, 4, 1),
                                   coarse_kind=O.COARSE_PCG, coarse_tol=1e-2, coarse_max_iter=200, post_sweeps=2,
                                   bj_iters=0, smoother=O.SMOOTHER_SCHWARZ_BLOCKS, schwarz_overlap=1,
                                   schwarz_scaling=True))
        assert abs(r.iterations - slv.ThisLevelIterations) <= 1, (r.iterations, slv.ThisLevelIterations)
