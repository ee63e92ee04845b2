"""The p-multigrid V-cycle recorded as one CUDA graph with its decisions on the device (FGMRESConfig.Graph)
against the host-driven V-cycle and the FP64 direct solve."""
import numpy as np
import pytest

import oracle as O
from bosss_b200 import assembly as A
from bosss_b200 import native as nat
from bosss_b200 import xdg
from bosss_b200.solvers import BlockMsrMatrix, FGMRESConfig, MultigridOperator, PmgConfig

pytestmark = pytest.mark.gpu

SOL_TOL = 1e-9


def _solve(op, s, graph, mixed, **pmg):
    slv = FGMRESConfig(ConvergenceCriterion=1e-12, termination="relative", MaxKrylovDim=30, Graph=graph,
                       Preconditioners=[PmgConfig(**pmg)], MixedPrecision=mixed).CreateInstance(op)
    x = np.zeros(s.N)
    n0 = nat.launch_count()
    slv.Solve(x, s.rhs)
    return slv, x, nat.launch_count() - n0


@pytest.mark.parametrize("mixed", [False, True])
def test_graph_vcycle_poisson(cuda, mixed):
    s = A.poisson_3d(8, 3)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    pmg = dict(DegreeHierarchy=(20, 10, 4), CoarseTolerance=0.1, CoarseMaxIterations=60, RecalcResiPeriod=40)
    host, xh, nh = _solve(op, s, False, mixed, **pmg)
    graph, xg, ng = _solve(op, s, True, mixed, **pmg)
    xd = O.direct_solve(s)
    assert host.Converged and graph.Converged
    assert np.linalg.norm(xg - xd) <= SOL_TOL * np.linalg.norm(xd)
    assert abs(graph.ThisLevelIterations - host.ThisLevelIterations) <= 1
    # the replayed kernels are counted: the same order of magnitude as the host-driven solve
    assert 0.5 * nh <= ng <= 2.0 * nh, (nh, ng)
    # a second solve with the same handle replays the recorded graph
    x2 = np.zeros(s.N)
    graph.Solve(x2, s.rhs)
    assert np.linalg.norm(x2 - xg) <= 1e-12 * np.linalg.norm(xg)


@pytest.mark.parametrize("smoother", ["schwarz", "blockgs", "ilu"])
def test_graph_vcycle_smoothers(cuda, smoother):
    s = A.poisson_3d(6, 2)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    pmg = dict(DegreeHierarchy=(10, 4, 1), Smoother=smoother, NoOfPostSmootherSweeps=4, CoarseTolerance=0.1,
               CoarseMaxIterations=60)
    host, xh, _ = _solve(op, s, False, True, **pmg)
    graph, xg, _ = _solve(op, s, True, True, **pmg)
    xd = O.direct_solve(s)
    assert graph.Converged
    assert np.linalg.norm(xg - xd) <= SOL_TOL * np.linalg.norm(xd)
    assert abs(graph.ThisLevelIterations - host.ThisLevelIterations) <= 1


def test_graph_vcycle_xdg_uneven_blocks(cuda):
    s = xdg.xdg_sphere(n=8, p=2, seed=1, mu=(1.0, 10.0))
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    pmg = dict(DegreeHierarchy=(10, 4, 1), Smoother="schwarz", NoOfPostSmootherSweeps=4, CoarseTolerance=1e-2,
               CoarseMaxIterations=200)
    host, xh, _ = _solve(op, s, False, True, **pmg)
    graph, xg, _ = _solve(op, s, True, True, **pmg)
    xd = O.direct_solve(s)
    assert graph.Converged
    assert np.linalg.norm(xg - xd) <= SOL_TOL * np.linalg.norm(xd)
    assert abs(graph.ThisLevelIterations - host.ThisLevelIterations) <= 1


def test_graph_vcycle_short_history_restarts(cuda):
    """A history of 4 entries per level forces the device-side restart of the minimisation (history full at the
    start of a sub-level iteration) and the full-history guard of the post-smoother sweeps."""
    s = A.poisson_3d(8, 3)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    pmg = dict(DegreeHierarchy=(20, 10, 4), CoarseTolerance=0.1, CoarseMaxIterations=60, OrthoMaxKrylovDim=4,
               NoOfPostSmootherSweeps=6)
    host, xh, _ = _solve(op, s, False, True, **pmg)
    graph, xg, _ = _solve(op, s, True, True, **pmg)
    xd = O.direct_solve(s)
    assert host.Converged and graph.Converged
    assert np.linalg.norm(xg - xd) <= SOL_TOL * np.linalg.norm(xd)
    assert abs(graph.ThisLevelIterations - host.ThisLevelIterations) <= 2


def test_graph_vcycle_rejects_unrecordable_coarse_solver(cuda):
    s = A.poisson_3d(4, 1)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    with pytest.raises(nat.BsgpuError):
        FGMRESConfig(Graph=True, Preconditioners=[PmgConfig(DegreeHierarchy=(4, 1), CoarseSolver="amg")]
                     ).CreateInstance(op)


@pytest.mark.parametrize("graph", [False, True])
def test_fp16_level_matrices(cuda, graph):
    """FP16 level matrices (FP32 arithmetic) in the mixed-precision V-cycle, host-driven and recorded: the solution to
    the direct solve's 1e-9.  (The preconditioner is weaker: FP16 values cost FlexGMRES iterations.)"""
    s = A.poisson_3d(8, 3)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    pmg = dict(DegreeHierarchy=(20, 10, 4), CoarseTolerance=0.1, CoarseMaxIterations=60, RecalcResiPeriod=40)
    ref, _, _ = _solve(op, s, graph, True, **pmg)
    half, xh, _ = _solve(op, s, graph, True, MatrixFP16=True, **pmg)
    xd = O.direct_solve(s)
    assert half.Converged and ref.Converged
    assert np.linalg.norm(xh - xd) <= SOL_TOL * np.linalg.norm(xd)


def test_graph_vcycles_in_a_concurrent_batch(cuda):
    """Independent systems, each with its own recorded V-cycle (recorded at set-up on the calling thread), solved
    concurrently from host threads: every solution against its direct solve."""
    from bosss_b200.batch import BatchSolver
    specs = [dict(n=n, p=1, seed=i, mu=(1.0, 10.0), radius=r, centre=(0.5, 0.48, 0.52))
             for i, (n, r) in enumerate([(6, 0.3), (8, 0.25), (7, 0.33), (6, 0.2)])]
    systems = [xdg.xdg_sphere(**sp) for sp in specs]
    pmg = PmgConfig(DegreeHierarchy=(4, 1), Smoother="schwarz", NoOfPostSmootherSweeps=2, CoarseTolerance=1e-2,
                    CoarseMaxIterations=200)
    make = lambda op: {"graph": FGMRESConfig(ConvergenceCriterion=1e-12, termination="relative",
                                             Preconditioners=[pmg], MixedPrecision=True, Graph=True,
                                             Autotune=True).CreateInstance(op)}
    sols = {}
    out = BatchSolver(make, concurrency=2).run(
        systems, on_result=lambda name, r, w: sols.__setitem__(r.index, w["X"][name].cpu().numpy()))
    assert out["graph"].as_dict()["all_converged"]
    for i, s in enumerate(systems):
        xd = O.direct_solve(s)
        assert np.linalg.norm(sols[i] - xd) <= SOL_TOL * np.linalg.norm(xd)
