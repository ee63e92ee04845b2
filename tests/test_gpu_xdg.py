"""GPU parity of the Schwarz smoother and of solves on XDG (two-species, cut-cell) systems (C ABI)."""
import numpy as np
import pytest

import oracle as O
from bosss_b200 import assembly as A
from bosss_b200 import xdg
from bosss_b200.solvers import (BlockMsrMatrix, FGMRESConfig, MultigridOperator, PmgConfig, SchwarzConfig)
from helpers import random_var_bsr

pytestmark = pytest.mark.gpu

SOL_TOL = 1e-9  # relative L2 error of solutions against the FP64 direct solve


@pytest.mark.parametrize("Np,spc", [(4, 1), (4, 2), (10, 2)])
def test_schwarz_block_rows_match_oracle(cuda, Np, spc):
    """One Schwarz update from a zero guess is X = M B, M = centre rows of every patch inverse."""
    v = random_var_bsr(60, Np, seed=20 + Np, max_spc=spc, nnz_per_row=3, spd=True)
    Bo = O.Bsr.of(v)
    ref = O.spmv(O.Bsr.of(v, values=O.schwarz_rows(Bo)), 1.0, v.rhs, 0.0, np.zeros(v.N))
    op = MultigridOperator(BlockMsrMatrix.from_system(v), MultigridOperator.Eye)
    sw = SchwarzConfig(FixedNoOfIterations=1, Blocking="cell").CreateInstance(op)
    x = np.zeros(v.N)
    sw.Solve(x, v.rhs)
    assert np.abs(x - ref).max() <= 1e-10 * np.abs(ref).max()


def test_schwarz_iterations_match_oracle(cuda):
    """FixedNoOfIterations updates x <- x + M (b - A x) (Schwarz.cs:1027-1047, restricted form) against the same
    recursion on the oracle's patch inverses."""
    v = random_var_bsr(50, 4, seed=31, max_spc=2, nnz_per_row=3, spd=True)
    Bo = O.Bsr.of(v)
    Mo = O.Bsr.of(v, values=O.schwarz_rows(Bo))
    x = np.zeros(v.N)
    for _ in range(3):
        r = O.spmv(Bo, -1.0, x, 1.0, v.rhs.copy())
        x = O.spmv(Mo, 1.0, r, 1.0, x.copy())
    op = MultigridOperator(BlockMsrMatrix.from_system(v), MultigridOperator.Eye)
    got = np.zeros(v.N)
    SchwarzConfig(FixedNoOfIterations=3, Blocking="cell").CreateInstance(op).Solve(got, v.rhs)
    assert np.abs(got - x).max() <= 1e-10 * np.abs(x).max()


def test_schwarz_rejects_unsupported_overlap(cuda):
    op = MultigridOperator(BlockMsrMatrix.from_system(A.poisson_3d(3, 1)))
    with pytest.raises(NotImplementedError):
        SchwarzConfig(Overlap=2, Blocking="cell").CreateInstance(op)
    with pytest.raises(ValueError):
        SchwarzConfig(Overlap=3).CreateInstance(op)


@pytest.mark.parametrize("mixed", [False, True])
def test_fgmres_pmg_schwarz_smoother(cuda, mixed):
    s = A.poisson_3d(8, 3)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    pmg = PmgConfig(DegreeHierarchy=(20, 10, 4), Smoother="schwarz", NoOfPostSmootherSweeps=2,
                    CoarseTolerance=1e-1, CoarseMaxIterations=60)
    slv = FGMRESConfig(ConvergenceCriterion=1e-12, termination="relative", Preconditioners=[pmg],
                       MixedPrecision=mixed).CreateInstance(op)
    x = np.zeros(s.N)
    slv.Solve(x, s.rhs)
    xd = O.direct_solve(s)
    assert slv.Converged
    assert np.linalg.norm(x - xd) <= SOL_TOL * np.linalg.norm(xd)


@pytest.mark.parametrize("smoother,mixed,jump", [("blockjacobi", False, 10.0), ("schwarz", False, 10.0),
                                                 ("schwarz", True, 10.0), ("blockjacobi", False, 1000.0),
                                                 ("schwarz", True, 1000.0)])
def test_xdg_sphere_solve(cuda, smoother, mixed, jump):
    """Two species with a diffusivity jump across a sphere; blocks of 10 (uncut) and 20 (cut) rows.  With the
    1:1000 jump the system's condition number is ~5e9 (n = 8), and FP64 bounds the attainable solution accuracy:
    the tolerance there is 1e-8 (1e-9 for 1:10)."""
    s = xdg.xdg_sphere(n=8, p=2, seed=1, mu=(1.0, jump))
    tol = SOL_TOL if jump <= 10 else 1e-8
    assert set(np.unique(s.nspc)) == {1, 2}
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    pmg = PmgConfig(DegreeHierarchy=(10, 4, 1), Smoother=smoother,
                    NoOfPostSmootherSweeps=4 if smoother == "schwarz" else 10,
                    CoarseTolerance=1e-2, CoarseMaxIterations=200)
    slv = FGMRESConfig(ConvergenceCriterion=1e-12, termination="relative", Preconditioners=[pmg],
                       MixedPrecision=mixed).CreateInstance(op)
    x = np.zeros(s.N)
    slv.Solve(x, s.rhs)
    xd = O.direct_solve(s)
    assert slv.Converged
    assert np.linalg.norm(x - xd) <= tol * np.linalg.norm(xd)


def test_xdg_spmv_matches_oracle(cuda):
    s = xdg.xdg_sphere(n=6, p=3, seed=2)
    rng = np.random.default_rng(0)
    xv = rng.standard_normal(s.N)
    yv = rng.standard_normal(s.N)
    ref = O.spmv(O.Bsr.of(s), 0.7, xv, -0.3, yv.copy())
    M = BlockMsrMatrix.from_system(s)
    got = yv.copy()
    M.SpMV(0.7, xv, -0.3, got)
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()


def test_batch_of_independent_xdg_problems(cuda):
    """Waves of concurrently solved problems (one handle and stream each) give the same solutions as the direct
    solve of every problem."""
    from bosss_b200.batch import BatchSolver
    specs = [dict(n=n, p=1, seed=i, mu=(1.0, J), radius=r, centre=(0.5, 0.48, 0.52))
             for i, (n, J, r) in enumerate([(6, 10.0, 0.3), (8, 100.0, 0.25), (6, 1000.0, 0.2), (7, 10.0, 0.33),
                                            (8, 1000.0, 0.3)])]
    systems = [xdg.xdg_sphere(**sp) for sp in specs]
    pmg = PmgConfig(DegreeHierarchy=(4, 1), Smoother="schwarz", NoOfPostSmootherSweeps=2, CoarseTolerance=1e-2,
                    CoarseMaxIterations=200)
    make = lambda op, mixed: FGMRESConfig(ConvergenceCriterion=1e-12, termination="relative",
                                          Preconditioners=[pmg], MixedPrecision=mixed).CreateInstance(op)
    sols = {}
    out = BatchSolver(lambda op: {"mixed": make(op, True), "fp64": make(op, False)}, concurrency=2).run(
        systems, on_result=lambda name, r, w: sols.__setitem__((name, r.index), w["X"][name].cpu().numpy()))
    assert set(out) == {"mixed", "fp64"}
    for summary in out.values():
        assert len(summary.results) == 5 and summary.as_dict()["all_converged"]
    for i, s in enumerate(systems):
        xd = O.direct_solve(s)
        tol = SOL_TOL if specs[i]["mu"][1] <= 10 else 1e-8     # conditioning bound of the larger jumps
        for name in out:
            assert np.linalg.norm(sols[(name, i)] - xd) <= tol * np.linalg.norm(xd)


def test_schwarz_block_covering_everything_is_exact(cuda):
    """As addSchwarzTest.Test_Solution_IsCorrect (addSchwarzTest.cs:186-202): patches that cover the whole system
    (complete block graph) make one Schwarz application an exact solve."""
    from helpers import dense_block_system
    v = dense_block_system(6, 4, seed=5)
    op = MultigridOperator(BlockMsrMatrix.from_system(v), MultigridOperator.Eye)
    x = np.zeros(v.N)
    SchwarzConfig(FixedNoOfIterations=1, Blocking="cell").CreateInstance(op).Solve(x, v.rhs)
    xs = np.linalg.solve(v.to_scipy().toarray(), v.rhs)
    assert np.linalg.norm(x - xs) <= 1e-13 * np.linalg.norm(xs)
