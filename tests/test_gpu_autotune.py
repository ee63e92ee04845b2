"""The launch-shape autotuner: it times the candidate CTA sizes of the block kernels on the matrix itself, records
its decisions, and a solver set up with it gives the solution of the untuned solver."""
import numpy as np
import pytest

import oracle as O
from bosss_b200 import assembly as A
from bosss_b200 import native as nat
from bosss_b200 import xdg
from bosss_b200.solvers import BlockMsrMatrix, FGMRESConfig, MultigridOperator, PmgConfig

pytestmark = pytest.mark.gpu


def test_autotuned_matrix_product_matches_oracle(cuda):
    for s in (A.poisson_3d(6, 3, seed=2), xdg.xdg_sphere(n=6, p=2, seed=3)):
        M = BlockMsrMatrix.from_system(s)
        M.Autotune()
        rng = np.random.default_rng(1)
        x = rng.standard_normal(s.N)
        y0 = rng.standard_normal(s.N)
        ref = O.spmv(O.Bsr.of(s), 0.8, x, 0.3, y0.copy())
        y = y0.copy()
        M.SpMV(0.8, x, 0.3, y)
        assert np.linalg.norm(y - ref) <= 1e-13 * np.linalg.norm(ref)
    rep = nat.autotune_report()
    assert len(rep) >= 2
    for r in rep:
        assert r["threads_per_cta"] in (64, 128, 256)
        assert str(r["threads_per_cta"]) in r["times_ms"]
        assert all(t > 0 for t in r["times_ms"].values())


@pytest.mark.parametrize("graph", [False, True])
def test_autotuned_solver_matches_untuned(cuda, graph):
    s = A.poisson_3d(8, 3, seed=4)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    pmg = PmgConfig(DegreeHierarchy=(20, 10, 4), CoarseTolerance=0.1, CoarseMaxIterations=60)
    out = []
    for tune in (False, True):
        slv = FGMRESConfig(ConvergenceCriterion=1e-12, termination="relative", Preconditioners=[pmg],
                           MixedPrecision=True, Graph=graph, Autotune=tune).CreateInstance(op)
        x = np.zeros(s.N)
        slv.Solve(x, s.rhs)
        assert slv.Converged
        out.append((x, slv.ThisLevelIterations))
    xd = O.direct_solve(s)
    for x, _ in out:
        assert np.linalg.norm(x - xd) <= 1e-9 * np.linalg.norm(xd)
    assert abs(out[0][1] - out[1][1]) <= 1
