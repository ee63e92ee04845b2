"""The whole FlexGMRES solve recorded as one CUDA graph (FGMRESConfig(Graph="solve"): restart and Arnoldi loops,
Givens rotations, the preconditioners' round-robin and every termination test on the device) against the
host-driven FlexGMRES (FlexGMRES.cs:144-277) and the FP64 direct solve, and batches of independent systems run from
one graph launch (GpuBatch, bsgpu_batch_*)."""
import numpy as np
import pytest

import oracle as O
from bosss_b200 import assembly as A
from bosss_b200 import native as nat
from bosss_b200 import xdg
from bosss_b200.solvers import BlockMsrMatrix, FGMRESConfig, GpuBatch, MultigridOperator, PmgConfig

pytestmark = pytest.mark.gpu

SOL_TOL = 1e-9


def _solver(op, graph, mixed, krylov=30, tol=1e-12, learned="off", **pmg):
    return FGMRESConfig(ConvergenceCriterion=tol, termination="relative", MaxKrylovDim=krylov, Graph=graph,
                        Learned=learned, Preconditioners=[PmgConfig(**pmg)],
                        MixedPrecision=mixed).CreateInstance(op)


def _solve(slv, s):
    x = np.zeros(s.N)
    n0 = nat.launch_count()
    slv.Solve(x, s.rhs)
    return x, nat.launch_count() - n0


POISSON_PMG = dict(DegreeHierarchy=(20, 10, 4), CoarseTolerance=0.1, CoarseMaxIterations=60, RecalcResiPeriod=40)


@pytest.mark.parametrize("mixed", [False, True])
def test_recorded_solve_matches_host_flexgmres(cuda, mixed):
    s = A.poisson_3d(8, 3)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    host = _solver(op, False, mixed, **POISSON_PMG)
    rec = _solver(op, "solve", mixed, **POISSON_PMG)
    xh, nh = _solve(host, s)
    xr, nr = _solve(rec, s)
    xd = O.direct_solve(s)
    assert host.Converged and rec.Converged
    assert np.linalg.norm(xr - xd) <= SOL_TOL * np.linalg.norm(xd)
    assert abs(rec.ThisLevelIterations - host.ThisLevelIterations) <= 1
    # the residual history: one entry per restart plus one estimate per Arnoldi step, as the host loop writes it
    hh, hr = host.History(), rec.History()
    assert abs(len(hr) - len(hh)) <= 1
    assert abs(hr[0] - hh[0]) <= 1e-12 * hh[0]
    # the last entry is the true residual of the final restart test: below tol * r0 or the absolute floor 2.2e-13
    # of DefaultTermination (IterativeSolverConfig.cs:48-62)
    assert hr[-1] <= max(1e-12 * hr[0], 2.2205e-13)
    # replayed kernels are counted (the same order as the host-driven solve)
    assert 0.5 * nh <= nr <= 2.0 * nh, (nh, nr)
    # a second solve replays the recording; device vectors take the same path
    import torch
    B = torch.from_numpy(s.rhs).cuda()
    X = torch.zeros_like(B)
    rec.Solve(X, B)
    assert np.linalg.norm(X.cpu().numpy() - xr) <= 1e-12 * np.linalg.norm(xr)


def test_recorded_solve_restart_cycles(cuda):
    """MaxKrylovDim = 3 forces several restart cycles: the device-side back substitution, the cycle's update and the
    restart test run many times; the iteration count follows the host-driven solve."""
    s = A.poisson_3d(6, 2)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    pmg = dict(DegreeHierarchy=(10, 4, 1), NoOfPostSmootherSweeps=1, CoarseTolerance=0.5, CoarseMaxIterations=2,
               SubLevelMaxIterations=1)
    host = _solver(op, False, False, krylov=3, tol=1e-10, **pmg)
    rec = _solver(op, "solve", False, krylov=3, tol=1e-10, **pmg)
    xh, _ = _solve(host, s)
    xr, _ = _solve(rec, s)
    xd = O.direct_solve(s)
    assert host.Converged and rec.Converged
    assert host.ThisLevelIterations > 3  # more than one cycle of 3
    assert abs(rec.ThisLevelIterations - host.ThisLevelIterations) <= 1
    assert np.linalg.norm(xr - xd) <= 1e-8 * np.linalg.norm(xd)


def test_recorded_solve_iteration_limit(cuda):
    """MaxSolverIterations ends the recorded loops without convergence, as in the host loop."""
    s = A.poisson_3d(6, 2)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    pmg = dict(DegreeHierarchy=(10, 4, 1), NoOfPostSmootherSweeps=1, CoarseTolerance=0.5, CoarseMaxIterations=2)
    cfgs = [FGMRESConfig(ConvergenceCriterion=1e-14, termination="relative", MaxKrylovDim=4, MaxSolverIterations=5,
                         Graph=g, Preconditioners=[PmgConfig(**pmg)]).CreateInstance(op) for g in (False, "solve")]
    for slv in cfgs:
        _solve(slv, s)
        assert not slv.Converged
    assert cfgs[1].ThisLevelIterations == cfgs[0].ThisLevelIterations


def test_recorded_solve_tracing_runs_host_driven(cuda):
    """With tracing on, a Graph="solve" handle runs host-driven (per-block timings need the host); the two give the
    same iteration count and solution."""
    s = A.poisson_3d(6, 2)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    rec = _solver(op, "solve", True, DegreeHierarchy=(10, 4, 1), CoarseTolerance=0.1, CoarseMaxIterations=60)
    xr, _ = _solve(rec, s)
    it = rec.ThisLevelIterations
    rec.SetTracing(True)
    xt, _ = _solve(rec, s)
    trace = rec.Trace()
    rec.SetTracing(False)
    assert abs(rec.ThisLevelIterations - it) <= 1
    assert np.linalg.norm(xt - xr) <= 1e-9 * np.linalg.norm(xr)
    assert any(t["name"] == "FlexGMRES" and t["calls"] > 0 for t in trace)


def test_recorded_solve_learned_round_robin(cuda):
    """The learned stage as FlexGMRES's second preconditioner: the recording holds both preconditioners behind IF
    nodes switched by the device's round-robin and stall test.  Trained once, the handle solves recorded (tracing off)
    and host-driven (tracing on) with the same weights: same solution, iteration counts within one."""
    s = A.poisson_3d(6, 2)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    op.SetCellGraph(s.grid.face_neighbours())
    rec = _solver(op, "solve", True, learned="fgmres", DegreeHierarchy=(10, 4, 1), CoarseTolerance=0.1,
                  CoarseMaxIterations=60, NoOfPostSmootherSweeps=2)
    rec.TrainLearned(n_rhs=2, steps=50, seed=3)
    xr, _ = _solve(rec, s)  # re-recorded with the stage switched on
    it = rec.ThisLevelIterations
    rec.SetTracing(True)
    xt, _ = _solve(rec, s)
    assert rec.Converged
    trace = {t["name"]: t for t in rec.Trace()}
    rec.SetTracing(False)
    assert abs(rec.ThisLevelIterations - it) <= 1
    xd = O.direct_solve(s)
    assert np.linalg.norm(xr - xd) <= SOL_TOL * np.linalg.norm(xd)
    assert np.linalg.norm(xt - xd) <= SOL_TOL * np.linalg.norm(xd)
    assert trace["LearnedStage"]["calls"] >= 1


def test_recorded_solve_nan_rhs_raises(cuda):
    """A NaN right-hand side raises ArithmeticException in both forms (the recorded loops end on the device)."""
    s = A.poisson_3d(4, 1)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    b = s.rhs.copy()
    b[3] = np.nan
    for g in (False, "solve"):
        slv = _solver(op, g, False, DegreeHierarchy=(4, 1), CoarseTolerance=0.1, CoarseMaxIterations=20)
        with pytest.raises(nat.BsgpuArithmeticError):
            slv.Solve(np.zeros(s.N), b)


def _xdg_systems():
    specs = [dict(n=n, p=1, seed=i, mu=(1.0, 10.0), radius=r, centre=(0.5, 0.48, 0.52))
             for i, (n, r) in enumerate([(6, 0.3), (8, 0.25), (7, 0.33), (6, 0.2), (5, 0.3)])]
    return [xdg.xdg_sphere(**sp) for sp in specs]


XDG_PMG = dict(DegreeHierarchy=(4, 1), Smoother="schwarz", NoOfPostSmootherSweeps=2, CoarseTolerance=1e-2,
               CoarseMaxIterations=200)


def test_batch_one_graph_launch(cuda):
    """Five XDG systems of different sizes in one graph: every solution against its direct solve, every member's
    iteration count equal to its own recorded solve, latencies from the launch positive and at most the batch's."""
    import torch
    systems = _xdg_systems()
    ops = [MultigridOperator(BlockMsrMatrix.from_system(s)) for s in systems]
    slvs = [_solver(op, "solve", True, **XDG_PMG) for op in ops]
    alone = []
    for slv, s in zip(slvs, systems):
        _solve(slv, s)
        alone.append(slv.ThisLevelIterations)
    Bs = [torch.from_numpy(s.rhs).cuda() for s in systems]
    Xs = [torch.zeros_like(b) for b in Bs]
    gb = GpuBatch(slvs)
    n0 = nat.launch_count()
    gb.Solve(Xs, Bs)
    launched = nat.launch_count() - n0
    lat = gb.Latencies()
    for slv, s, X, it in zip(slvs, systems, Xs, alone):
        assert slv.Converged
        assert slv.ThisLevelIterations == it
        xd = O.direct_solve(s)
        assert np.linalg.norm(X.cpu().numpy() - xd) <= SOL_TOL * np.linalg.norm(xd)
    assert all(0 < t for t in lat)
    assert launched > 100 * len(systems)
    # a second batch solve replays the same graph: same solutions
    Xs2 = [torch.zeros_like(b) for b in Bs]
    gb.Solve(Xs2, Bs)
    for X, X2 in zip(Xs, Xs2):
        assert torch.allclose(X, X2, rtol=0, atol=1e-13 * float(X.abs().max()))
    gb.Dispose()


def test_batch_rejects_members_without_recorded_solve(cuda):
    s = _xdg_systems()[0]
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    rec = _solver(op, "solve", True, **XDG_PMG)
    vcyc = _solver(op, True, True, **XDG_PMG)
    with pytest.raises(nat.BsgpuError):
        GpuBatch([rec, vcyc])
    with pytest.raises(nat.BsgpuError):
        GpuBatch([rec, rec])


def test_batch_solver_one_graph_waves(cuda):
    """BatchSolver with one_graph: waves of two systems, each wave one graph launch; solutions against the direct
    solve and against the host-thread waves of the same problems."""
    from bosss_b200.batch import BatchSolver
    systems = _xdg_systems()
    make = lambda op: {"one_graph": _solver(op, "solve", True, **XDG_PMG),
                       "threads": _solver(op, True, True, **XDG_PMG)}
    sols = {}
    out = BatchSolver(make, concurrency=2, one_graph=["one_graph"]).run(
        systems, on_result=lambda name, r, w: sols.__setitem__((name, r.index), w["X"][name].cpu().numpy()))
    assert out["one_graph"].as_dict()["all_converged"] and out["threads"].as_dict()["all_converged"]
    for i, s in enumerate(systems):
        xd = O.direct_solve(s)
        for name in ("one_graph", "threads"):
            assert np.linalg.norm(sols[(name, i)] - xd) <= SOL_TOL * np.linalg.norm(xd)


def test_batch_with_learned_stage_in_one_graph(cuda):
    """Uniform systems, each with its trained learned stage as FlexGMRES's second preconditioner (IF nodes of the
    round-robin inside every branch), solved from one graph launch: solutions against the direct solves.  A member
    whose X and B are the same vector is rejected."""
    import torch
    systems = [A.poisson_3d(n, 2, seed=i) for i, n in enumerate((5, 6, 4))]
    slvs = []
    for s in systems:
        op = MultigridOperator(BlockMsrMatrix.from_system(s))
        op.SetCellGraph(s.grid.face_neighbours())
        slv = _solver(op, "solve", True, learned="fgmres", DegreeHierarchy=(10, 4, 1), CoarseTolerance=0.1,
                      CoarseMaxIterations=60, NoOfPostSmootherSweeps=2)
        slv.TrainLearned(n_rhs=2, steps=30, seed=1)
        slvs.append(slv)
    Bs = [torch.from_numpy(s.rhs).cuda() for s in systems]
    Xs = [torch.zeros_like(b) for b in Bs]
    gb = GpuBatch(slvs)
    gb.Solve(Xs, Bs)
    for slv, s, X in zip(slvs, systems, Xs):
        assert slv.Converged
        xd = O.direct_solve(s)
        assert np.linalg.norm(X.cpu().numpy() - xd) <= SOL_TOL * np.linalg.norm(xd)
    with pytest.raises(nat.BsgpuError):
        gb.Solve([Bs[0]] + Xs[1:], Bs)
    gb.Dispose()
