"""CPU tests of the configuration mirrors: field mapping onto the C struct and the reference's argument errors."""
import pytest

from bosss_b200 import native as nat
from bosss_b200.solvers import FGMRESConfig, PmgConfig, SoftGMRESConfig, SoftPCGConfig


def test_fgmres_pmg_fields_reach_the_c_struct():
    pmg = PmgConfig(DegreeHierarchy=(20, 10, 4), NoOfPostSmootherSweeps=7, CoarseTolerance=0.1,
                    CoarseMaxIterations=60, UseILU=True, OrthoMaxKrylovDim=48, RecalcResiPeriod=40)
    c = FGMRESConfig(ConvergenceCriterion=1e-9, termination="relative", MaxKrylovDim=25, Preconditioners=[pmg],
                     MixedPrecision=True, Learned="both", LearnedStall=0.8)._config()
    assert c.solver == nat.SOLVER_FGMRES_PMG and c.termination == nat.TERM_RELATIVE and c.tol == 1e-9
    assert c.max_krylov == 25 and c.n_levels == 3 and list(c.level_keep)[:3] == [20, 10, 4]
    assert c.post_sweeps == 7 and c.coarse_tol == 0.1 and c.coarse_max_iter == 60
    assert c.smoother == nat.SMOOTHER_ILU_NATURAL and c.precision == nat.PRECISION_MIXED
    assert c.learned == nat.LEARNED_BOTH and c.learned_stall == 0.8
    assert c.ortho_max_krylov == 48 and c.recalc_resi_period == 40


@pytest.mark.parametrize("kw", [dict(Smoother="jacobi"), dict(CoarseSolver="pardiso"), dict(OrthoMaxKrylovDim=1),
                                dict(RecalcResiPeriod=0)])
def test_pmg_rejects_bad_values(kw):
    with pytest.raises(ValueError):
        FGMRESConfig(Preconditioners=[PmgConfig(**kw)])._config()


def test_fgmres_rejects_unknown_learned_mode_and_several_preconditioners():
    with pytest.raises(ValueError):
        FGMRESConfig(Learned="sometimes")._config()
    with pytest.raises(NotImplementedError):
        FGMRESConfig(Preconditioners=[PmgConfig(), PmgConfig()])._config()


def test_softgmres_and_softpcg_mapping():
    c = SoftGMRESConfig(MaxKrylovDim=12, Precond="schwarz", BlockJacobiIterations=2)._config()
    assert c.solver == nat.SOLVER_SOFTGMRES and c.n_levels == 1 and c.smoother == nat.SMOOTHER_SCHWARZ
    assert c.bj_iters == 2 and c.max_krylov == 12
    assert SoftGMRESConfig(Precond=None)._config().bj_iters == -1
    with pytest.raises(ValueError):
        SoftGMRESConfig(Precond=PmgConfig())._config()
    with pytest.raises(ValueError):
        SoftGMRESConfig(Precond="amg")._config()
    assert SoftPCGConfig(BlockJacobiPrecond=False)._config().bj_iters == -1


@pytest.mark.parametrize("graph,value", [(False, 0), (True, 1), ("vcycle", 1), ("solve", 2)])
def test_fgmres_graph_modes(graph, value):
    assert FGMRESConfig(Graph=graph)._config().graph == value


def test_fgmres_rejects_unknown_graph_mode():
    with pytest.raises(ValueError):
        FGMRESConfig(Graph="always")._config()


def test_assemble_sip_rejects_bad_shapes_before_the_library():
    from bosss_b200.solvers import BlockMsrMatrix
    with pytest.raises(ValueError):
        BlockMsrMatrix.AssembleSIP((2, 2, 2, 2), 1)
    with pytest.raises(ValueError):
        BlockMsrMatrix.AssembleSIP((3, 3), 1, coeff=[1.0, 2.0])
