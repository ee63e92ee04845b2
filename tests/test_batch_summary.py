"""CPU tests of the batch runner's bookkeeping: per-configuration summaries (aggregate DOF/s, latency percentiles,
set-up phases) from per-problem results, without a GPU."""
import pytest

from bosss_b200.batch import BatchResult, BatchSolver, BatchSummary


def _results():
    out = []
    for i, (dof, t, it) in enumerate([(1000, 1.0, 10), (3000, 2.0, 20), (6000, 4.0, 40), (2000, 1.5, 15)]):
        out.append(BatchResult(index=i, dof=dof, setup_s=0.5, solve_s=t, iterations=it, converged=True,
                               relres=1e-11 * (i + 1),
                               info={"matrix_s": 0.1, "change_of_basis_s": 0.05, "solvers_s": 0.35}))
    return out


def test_summary_aggregates():
    s = BatchSummary(results=_results(), solve_wall_s=4.0, setup_wall_s=2.0)
    d = s.as_dict()
    assert d["problems"] == 4 and d["dof"] == 12000
    assert d["dof_per_s_solve"] == pytest.approx(3000.0)
    assert d["dof_per_s_with_setup"] == pytest.approx(2000.0)
    assert d["latency_p50_s"] == pytest.approx(1.75) and 2.0 < d["latency_p99_s"] <= 4.0
    assert d["iterations_max"] == 40 and d["all_converged"]
    assert d["relres_max"] == pytest.approx(4e-11)
    assert d["setup_phases_s"] == pytest.approx({"matrix_s": 0.4, "change_of_basis_s": 0.2, "solvers_s": 1.4})


def test_summary_flags_non_convergence():
    r = _results()
    r[2].converged = False
    assert not BatchSummary(results=r, solve_wall_s=1.0, setup_wall_s=1.0).as_dict()["all_converged"]


def test_solver_rejects_zero_concurrency():
    with pytest.raises(ValueError):
        BatchSolver(lambda op: None, concurrency=0)
