"""CPU tests: the oracle (CPU restatement) pinned against the reference's own known-answer tests.

The reference ships no golden vectors; its solver-path tests pin tolerances (see the citations per test).
"""
import math

import numpy as np
import pytest

import oracle as O
from bosss_b200 import assembly as A
from helpers import apply_blocks, l2_error, random_var_bsr, sip_cartesian1


def test_testcartesian1_exactness():
    """ipPoisson TestProgram.TestCartesian (Tests/TestProgram.cs:47-73): L2 error <= 5e-9 for a quadratic."""
    g, s, exact = sip_cartesian1()
    u = O.direct_solve(s)
    assert l2_error(g, 2, u, exact) <= 5.0e-9


@pytest.mark.parametrize("D,p", [(2, 2), (3, 2)])
def test_convergence_slope(D, p):
    """TestOperatorConvergence2D/3D (Tests/TestProgram.cs:321-406): slope >= p + 0.5."""
    errs, hs = [], []
    for n in ((4, 8) if D == 3 else (4, 8, 16)):
        g = A.uniform_grid(D, n)
        ex = lambda X: np.prod([np.sin(math.pi * x) for x in X], axis=0)
        f = lambda X: D * math.pi ** 2 * ex(X)
        s = A.assemble_sip(g, p, penalty=(p + 1) * (p + 2), rhs_f=f, quad=p + 4)
        errs.append(l2_error(g, p, O.direct_solve(s), ex))
        hs.append(1.0 / n)
    slope = np.polyfit(np.log(hs), np.log(errs), 1)[0]
    assert slope >= p + 0.5


def test_spmv_matches_csr():
    """Matrix_MPItest AllUpTest.SpMVTest (AllUpTest.cs:475-590): |err| <= 1e-10 |B| for SpMV(1.6, X, 0.5, B)."""
    for s in (A.poisson_3d(6, 3), A.poisson_2d_c1(n=8)):
        B = O.Bsr.of(s)
        rng = np.random.default_rng(3)
        X, Bv = rng.standard_normal(s.N), rng.standard_normal(s.N)
        ref = 0.5 * Bv + 1.6 * (s.to_scipy() @ X)
        out = O.spmv(B, 1.6, X, 0.5, Bv.copy())
        assert np.linalg.norm(out - ref) <= 1e-10 * np.linalg.norm(ref)


def test_spmv_uneven_blocks():
    v = random_var_bsr(40, 10, seed=1)
    B = O.Bsr.of(v)
    x = np.random.default_rng(0).standard_normal(v.N)
    ref = v.to_scipy() @ x
    out = O.spmv(B, 1.0, x, 0.0, np.zeros(v.N))
    assert np.linalg.norm(out - ref) <= 1e-13 * np.linalg.norm(ref)


def test_symminv_equilibrates():
    """SymmInv (MultigridOperator_ChangeOfBasis.cs:624): L M L^T = I for an SPD block, L lower triangular."""
    rng = np.random.default_rng(0)
    for n in (4, 10, 20):
        Q = rng.standard_normal((n, n))
        M = Q @ Q.T + n * np.eye(n)
        L = O.symminv(M)
        assert np.allclose(np.triu(L, 1), 0)
        assert np.abs(L @ M @ L.T - np.eye(n)).max() < 1e-12


def test_change_of_basis_and_restriction_consistency():
    """The leading p-sub-block of L A L^T equals the transform of the restricted operator (lower-triangular L)."""
    s = A.poisson_3d(4, 3)
    B = O.Bsr.of(s)
    vals, Lcat = O.change_of_basis(B)
    rows = np.repeat(np.arange(s.nb), np.diff(s.row_ptr))
    diag = vals.reshape(-1, 20, 20)[rows == s.col_idx]
    assert np.abs(diag - np.eye(20)).max() < 1e-12
    sub, _ = O.restrict(B, 10)

    class S:  # restricted raw operator
        Np, row_ptr, col_idx, values = 10, s.row_ptr, s.col_idx, sub
    sub_t, _ = O.change_of_basis(O.Bsr.of(S))
    lead = vals.reshape(-1, 20, 20)[:, :10, :10].reshape(-1)
    assert np.abs(lead - sub_t).max() < 1e-10 * np.abs(lead).max()


def test_restriction_is_polynomial_exact():
    """MultigridTest (TestProgramLinearMG.cs:131-360): transfer of a degree-p' polynomial is exact (1e-10)."""
    g = A.uniform_grid(3, 3)
    f = lambda X: 1 + X[0] - 2 * X[1] * X[2] + X[2] ** 2
    full = A.project_function(g, 3, f, q=6).reshape(-1)
    low = A.project_function(g, 2, f, q=6).reshape(-1)
    # the leading 10 of 20 modes hold the P2 projection
    assert np.abs(full.reshape(-1, 20)[:, :10].reshape(-1) - low).max() < 1e-10
    assert np.abs(full.reshape(-1, 20)[:, 10:]).max() < 1e-10


def _transformed(s):
    B = O.Bsr.of(s)
    vals, Lcat = O.change_of_basis(B)

    class T:
        Np, row_ptr, col_idx, values = s.Np, s.row_ptr, s.col_idx, vals
    Bt = O.Bsr.of(T)
    bl = np.full(s.nb, s.Np)
    return Bt, Lcat, bl


def test_pcg_solves_c1_small():
    """Block-Jacobi PCG (SoftPCG.cs:113-194) on the transformed 2-D operator reaches the direct solution."""
    s = A.poisson_2d_c1(n=16)
    Bt, Lcat, bl = _transformed(s)
    bt = apply_blocks(Lcat, bl, s.rhs)
    r = O.solve(Bt, bt, O.SolverConfig(solver=O.PCG, tol=1e-12, top_mode=O.TERM_RELATIVE, bj_iters=0))
    x = apply_blocks(Lcat, bl, r.x, transpose=True)
    xd = O.direct_solve(s)
    assert r.converged
    assert np.linalg.norm(x - xd) <= 1e-9 * np.linalg.norm(xd)


@pytest.mark.parametrize("kind", [O.FGMRES_PMG, O.ORTHOMG])
def test_pmg_solvers_small(kind):
    """FGMRES(30) with a 3-level p-MG V-cycle, and OrthoMG p-MG (PmgConfig.cs:80-245), 3-D p = 3."""
    s = A.poisson_3d(6, 3)
    Bt, Lcat, bl = _transformed(s)
    bt = apply_blocks(Lcat, bl, s.rhs)
    cfg = O.SolverConfig(solver=kind, tol=1e-11, top_mode=O.TERM_RELATIVE, level_keep=(20, 10, 4),
                         coarse_kind=O.COARSE_PCG, coarse_tol=1e-4)
    r = O.solve(Bt, bt, cfg)
    x = apply_blocks(Lcat, bl, r.x, transpose=True)
    xd = O.direct_solve(s)
    assert r.converged and r.iterations < 40
    assert np.linalg.norm(x - xd) <= 1e-9 * np.linalg.norm(xd)


def test_reference_fgmres_defect_is_richardson():
    """FlexGMRES.cs:259-260 discards the least-squares solution: with the flag the method needs far more
    iterations than Saad's FGMRES on the same system."""
    s = A.poisson_3d(4, 2)
    Bt, Lcat, bl = _transformed(s)
    bt = apply_blocks(Lcat, bl, s.rhs)
    base = dict(solver=O.FGMRES_PMG, tol=1e-8, top_mode=O.TERM_RELATIVE, level_keep=(10, 4), max_iter=60,
                coarse_kind=O.COARSE_PCG, coarse_tol=1e-2, max_krylov=10)
    good = O.solve(Bt, bt, O.SolverConfig(**base))
    bad = O.solve(Bt, bt, O.SolverConfig(**base, reference_fgmres_defect=True))
    assert good.converged
    assert bad.iterations > good.iterations


def test_blockjacobi_two_updates():
    """BlockJacobi with NoOfIterations = 1 performs two updates x <- x + D^-1 (b - A x) from x = 0."""
    v = random_var_bsr(30, 4, seed=2, spd=True)
    B = O.Bsr.of(v)
    x = O.blockjacobi(B, np.zeros(v.N), v.rhs, iters=1)
    M = v.to_scipy().toarray()
    D = np.zeros_like(M)
    i0 = np.concatenate([[0], np.cumsum(v.block_len)])
    for i in range(v.nb):
        sl = slice(i0[i], i0[i + 1])
        D[sl, sl] = M[sl, sl]
    Di = np.linalg.inv(D)
    x1 = Di @ v.rhs
    x2 = x1 + Di @ (v.rhs - M @ x1)
    assert np.abs(x - x2).max() < 1e-12 * np.abs(x2).max()


@pytest.mark.parametrize("ordered", [False, True])
def test_ilu0_reproduces_the_matrix_on_its_pattern(ordered):
    """Defining property of ILU(0) (CellILU.ComputeILU, Saad's in-place form): (L U)_ij = A_ij on every occupied
    block, L unit lower and U upper in the factorisation order; the solve applies (L U)^{-1}."""
    from helpers import greedy_colour_order
    s = A.poisson_3d(3, 1, seed=4)
    order = greedy_colour_order(s.row_ptr, s.col_idx) if ordered else np.arange(s.nb, dtype=np.int32)
    Bo = O.Bsr.of(s)
    F = O.ilu0_factor(Bo, order if ordered else None).reshape(-1, s.Np, s.Np)
    pos = np.empty(s.nb, np.int64)
    pos[order] = np.arange(s.nb)
    Np, N = s.Np, s.N
    L, U = np.eye(N), np.zeros((N, N))
    pattern = np.zeros((N, N), bool)
    for i in range(s.nb):
        for q in range(s.row_ptr[i], s.row_ptr[i + 1]):
            j = s.col_idx[q]
            sl = np.s_[i * Np:(i + 1) * Np, j * Np:(j + 1) * Np]
            pattern[sl] = True
            if pos[j] < pos[i]:
                L[sl] = F[q]
            else:
                U[sl] = F[q]
    Ad = s.to_scipy().toarray()
    assert np.abs((L @ U - Ad)[pattern]).max() <= 1e-12 * np.abs(Ad).max()
    b = np.random.default_rng(1).standard_normal(N)
    x = O.ilu0_solve(Bo, F.reshape(-1), b, order if ordered else None)
    assert np.abs(L @ U @ x - b).max() <= 1e-10 * np.abs(b).max()


def test_recalc_resi_period_keeps_the_solution():
    """RecalcResiPeriod > 1 (OrthonormalizationMultigrid.cs:179-211) changes only how the OrthoMG residual is kept."""
    s = A.poisson_3d(4, 2, seed=2)
    xd = O.direct_solve(s)
    for period in (1, 5):
        cfg = O.SolverConfig(solver=O.FGMRES_PMG, tol=1e-12, level_keep=(10, 4), recalc_resi_period=period,
                             coarse_tol=1e-2)
        r = O.solve(O.Bsr.of(s), s.rhs, cfg)
        assert r.converged
        assert np.linalg.norm(r.x - xd) <= 1e-9 * np.linalg.norm(xd)


def test_schwarz_block_covering_everything_is_exact():
    """addSchwarzTest.Test_Solution_IsCorrect (AdvancedSolverTestsMPI/Solver/addSchwarzTest.cs:186-202): when a
    Schwarz block covers the whole system, one application solves it (|x - x*| < 1e-14 there).  With a complete
    block graph every cell's patch is the whole system, so the restricted factors are the rows of A^{-1}."""
    from helpers import dense_block_system
    v = dense_block_system(6, 4, seed=5)
    M = O.schwarz_rows(O.Bsr.of(v))
    x = O.spmv(O.Bsr.of(v, values=M), 1.0, v.rhs, 0.0, np.zeros(v.N))
    xs = np.linalg.solve(v.to_scipy().toarray(), v.rhs)
    assert np.linalg.norm(x - xs) < 1e-14


def test_log_coeff_features():
    """Learned-stage features: log k of the cell and its six face neighbours (the cell's own value at walls)."""
    s = A.variable_coeff_3d(4, 1, seed=1)
    f = A.log_coeff_features(s)
    assert f.shape == (s.nb, 7) and f.dtype == np.float32
    lk = np.log(s.coeff)
    nbr = s.grid.face_neighbours()
    for c in (0, 21, s.nb - 1):
        assert np.isclose(f[c, 0], lk[c])
        for q in range(6):
            assert np.isclose(f[c, 1 + q], lk[nbr[c, q]] if nbr[c, q] >= 0 else lk[c])


@pytest.mark.parametrize("bj", [-1, 0])
def test_softgmres_restatement(bj):
    """SoftGMRES (SoftGMRES.cs:227-460) restated: left-preconditioned GMRES(m), without a preconditioner and with
    block Jacobi, reaches the direct solution.  As in the solver path, it runs on the DiagBlockEquilib operator
    L A L^T (its termination test compares the preconditioned residual estimate with the unpreconditioned
    initial residual, which is only meaningful when M^{-1} is of unit scale)."""
    from helpers import apply_blocks
    s = A.poisson_3d(4, 2, seed=3)
    vals, Lc = O.change_of_basis(O.Bsr.of(s))

    class T:
        Np, row_ptr, col_idx, values = s.Np, s.row_ptr, s.col_idx, vals
    bl = np.full(s.nb, s.Np)
    r = O.solve(O.Bsr.of(T), apply_blocks(Lc, bl, s.rhs),
                O.SolverConfig(solver=O.SOFTGMRES, tol=1e-13, max_krylov=40, max_iter=5000, bj_iters=bj))
    x = apply_blocks(Lc, bl, r.x, transpose=True)
    xd = O.direct_solve(s)
    assert r.converged
    assert np.linalg.norm(x - xd) <= 1e-9 * np.linalg.norm(xd)


@pytest.mark.parametrize("smoother", [O.SMOOTHER_SCHWARZ, O.SMOOTHER_ILU_COLOURED, O.SMOOTHER_ILU_NATURAL])
def test_pmg_with_schwarz_and_ilu_smoothers(smoother):
    """p-multigrid post-smoothing with restricted Schwarz and with block ILU(0) (natural and two-colour order):
    FlexGMRES reaches the direct solution on the equilibrated operator."""
    from helpers import apply_blocks
    s = A.poisson_3d(4, 2, seed=6)
    vals, Lc = O.change_of_basis(O.Bsr.of(s))

    class T:
        Np, row_ptr, col_idx, values = s.Np, s.row_ptr, s.col_idx, vals
    bl = np.full(s.nb, s.Np)
    cfg = O.SolverConfig(solver=O.FGMRES_PMG, tol=1e-12, level_keep=(10, 4), post_sweeps=4, coarse_tol=1e-2,
                         smoother=smoother)
    r = O.solve(O.Bsr.of(T), apply_blocks(Lc, bl, s.rhs), cfg)
    x = apply_blocks(Lc, bl, r.x, transpose=True)
    xd = O.direct_solve(s)
    assert r.converged
    assert np.linalg.norm(x - xd) <= 1e-9 * np.linalg.norm(xd)


@pytest.mark.parametrize("D,p", [(2, 2), (3, 1)])
def test_h_prolongation_is_polynomial_exact(D, p):
    """Agglomeration prolongation (the h-levels of the coarse solver): a degree-p polynomial's coarse projection,
    prolongated, is its fine projection (the MG transfer exactness of TestProgramLinearMG.cs:166,308-309)."""
    g = A.uniform_grid(D, 4)
    P = A.h_prolongation(g, p)
    f = lambda X: 1.0 + 0.5 * X[0] - 0.3 * X[-1] + (0.7 * X[0] * X[-1] if p >= 2 else 0.0)
    cf = A.project_function(g, p, f, q=p + 3)
    cc = A.project_function(P.coarse_grid, p, f, q=p + 3)
    vals = np.asarray(P.values).reshape(P.nb_fine, P.Np, P.Np)
    got = np.stack([vals[i] @ cc[P.col_idx[i]] for i in range(P.nb_fine)])
    assert np.abs(got - cf).max() <= 1e-12 * np.abs(cf).max()


def test_sip_operators_are_symmetric_and_coefficient_scaled():
    """The SIP operators are symmetric; a constant diffusivity k scales the operator by k (ipLaplace.cs:95-245)."""
    s = A.poisson_3d(3, 2)
    M = s.to_scipy()
    assert abs(M - M.T).max() <= 1e-12 * abs(M).max()
    g = A.uniform_grid(3, 3)
    k = A.assemble_sip(g, 2, penalty=12.0, coeff=np.full(g.ncells, 2.5)).to_scipy()
    assert abs(k - 2.5 * M).max() <= 1e-12 * abs(M).max()


def test_natural_order_ilu_parallelises_by_wavefronts():
    """Block ILU(0) in the reference's natural order depends only on lower neighbours, so the rows of one wavefront
    (level = 1 + max level of the lower neighbours) can be factored together: any order inside a wavefront gives the
    same factors up to the order in which a diagonal block receives its updates (rounding only), and an n^3
    Cartesian grid has 3n - 2 wavefronts."""
    s = A.poisson_3d(4, 1, seed=7)
    nb = s.nb
    level = np.zeros(nb, np.int64)
    for i in range(nb):
        lower = [j for j in s.col_idx[s.row_ptr[i]:s.row_ptr[i + 1]] if j < i]
        level[i] = 1 + max((level[j] for j in lower), default=-1)
    assert level.max() + 1 == 3 * 4 - 2
    Bo = O.Bsr.of(s)
    F_nat = O.ilu0_factor(Bo)
    # wavefront order with each wavefront reversed: a different sequential order with the same dependencies
    order = np.concatenate([np.nonzero(level == L)[0][::-1] for L in range(level.max() + 1)]).astype(np.int32)
    F_wave = O.ilu0_factor(Bo, order)
    assert np.abs(F_nat - F_wave).max() <= 1e-14 * np.abs(F_nat).max()
    b = np.random.default_rng(0).standard_normal(s.N)
    x1, x2 = O.ilu0_solve(Bo, F_nat, b), O.ilu0_solve(Bo, F_wave, b, order)
    assert np.abs(x1 - x2).max() <= 1e-12 * np.abs(x1).max()


def test_block_schwarz_single_block_is_exact_and_overlap_sums():
    """Oracle multi-cell Schwarz: one block covering the system is an exact solve (addSchwarzTest.cs:186-202); with
    every cell its own block and no overlap it is block Jacobi."""
    from bosss_b200 import assembly as A
    s = A.poisson_3d(3, 1, seed=2)
    Bo = O.Bsr.of(s)
    x = O.block_schwarz(Bo, np.zeros(s.N), s.rhs, parts=1, overlap=0, iters=1)
    xs = np.linalg.solve(s.to_scipy().toarray(), s.rhs)
    assert np.linalg.norm(x - xs) <= 1e-12 * np.linalg.norm(xs)
    bj = O.block_schwarz(Bo, np.zeros(s.N), s.rhs, parts=s.nb, overlap=0, iters=1)
    ref = O.blockjacobi(Bo, np.zeros(s.N), s.rhs, iters=0)
    assert np.linalg.norm(bj - ref) <= 1e-12 * np.linalg.norm(ref)


def test_fgmres_restart_cycles_and_iteration_limit():
    """FlexGMRES with a Krylov dimension of 3 (restart cycles every 3 steps) still reaches the direct solution; with
    MaxSolverIterations = 4 it stops unconverged after at most 4 preconditioner applications (the limit test of
    IterativeSolverConfig.cs:55)."""
    s = A.poisson_3d(4, 2)
    Bt, Lcat, bl = _transformed(s)
    bt = apply_blocks(Lcat, bl, s.rhs)
    base = dict(solver=O.FGMRES_PMG, top_mode=O.TERM_RELATIVE, level_keep=(10, 4, 1), coarse_kind=O.COARSE_PCG,
                coarse_tol=0.5, coarse_max_iter=2, post_sweeps=1, sub_max_iter=1)
    r = O.solve(Bt, bt, O.SolverConfig(tol=1e-11, max_krylov=3, **base))
    x = apply_blocks(Lcat, bl, r.x, transpose=True)
    xd = O.direct_solve(s)
    assert r.converged and r.iterations > 3
    assert np.linalg.norm(x - xd) <= 1e-8 * np.linalg.norm(xd)
    lim = O.solve(Bt, bt, O.SolverConfig(tol=1e-14, max_krylov=3, max_iter=4, **base))
    assert not lim.converged and lim.iterations <= 5


def test_default_termination_absolute_floor():
    """DefaultTermination (IterativeSolverConfig.cs:48-62): R < R0 tol + tol.  For a right-hand side of norm 1e-9
    the absolute part (1e-10) ends the solve after a reduction of about 10, the relative form continues to its own
    tolerance or the machine-precision floor 2.2e-13."""
    s = A.poisson_3d(4, 1)
    Bt, Lcat, bl = _transformed(s)
    bt = apply_blocks(Lcat, bl, s.rhs)
    bt = bt / np.linalg.norm(bt) * 1e-9
    # a weak preconditioner (one sweep, two coarse CG steps), so that the residual falls gradually
    cfg = dict(solver=O.FGMRES_PMG, tol=1e-10, level_keep=(4, 1), coarse_kind=O.COARSE_PCG, coarse_tol=0.5,
               coarse_max_iter=2, post_sweeps=1, sub_max_iter=1)
    absolute = O.solve(Bt, bt, O.SolverConfig(top_mode=O.TERM_DEFAULT, **cfg))
    relative = O.solve(Bt, bt, O.SolverConfig(top_mode=O.TERM_RELATIVE, **cfg))
    assert absolute.converged and relative.converged
    assert absolute.res < absolute.res0 * 1e-10 + 1e-10
    assert relative.res < max(relative.res0 * 1e-10, 2.2205e-13)
    assert relative.iterations > absolute.iterations
