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
    sw = SchwarzConfig(FixedNoOfIterations=1).CreateInstance(op)
    x = np.zeros(v.N)
    sw.Solve(x, v.rhs)
    assert np.abs(x - ref).max() <= 1e-10 * np.abs(ref).max()


def test_schwarz_iterations_reduce_residual(cuda):
    s = A.poisson_3d(5, 2)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    r = []
    for it in (1, 4):
        x = np.zeros(s.N)
        SchwarzConfig(FixedNoOfIterations=it).CreateInstance(op).Solve(x, s.rhs)
        r.append(np.linalg.norm(s.rhs - s.to_scipy() @ x))
    assert r[1] < 0.5 * r[0]


def test_schwarz_rejects_unsupported_overlap(cuda):
    op = MultigridOperator(BlockMsrMatrix.from_system(A.poisson_3d(3, 1)))
    with pytest.raises(NotImplementedError):
        SchwarzConfig(Overlap=2).CreateInstance(op)


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


@pytest.mark.parametrize("smoother,mixed", [("blockjacobi", False), ("schwarz", False), ("schwarz", True)])
def test_xdg_sphere_solve(cuda, smoother, mixed):
    """Two species with a 1:1000 diffusivity jump across a sphere; blocks of 10 (uncut) and 20 (cut) rows."""
    s = xdg.xdg_sphere(n=8, p=2, seed=1)
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
    assert np.linalg.norm(x - xd) <= SOL_TOL * np.linalg.norm(xd)


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
