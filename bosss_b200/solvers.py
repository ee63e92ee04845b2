"""Host-side mirror of the BoSSS solver-path API over the C ABI.

Names, argument meaning and error behaviour follow the reference:

* ``BlockMsrMatrix`` -- ``src/L1-platform/BoSSS.Platform/BlockMsrMatrix.cs:191``; ``SpMV(alpha, a, beta, acc)``
  (``:2970``) raises ``ValueError`` (the reference's ``ArgumentException``) on length mismatch or aliasing.
* ``MultigridOperator`` -- ``src/L3-solution/BoSSS.Solution.AdvancedSolvers/MultigridOperator.cs:37`` with the
  ``DiagBlockEquilib`` change of basis (``MultigridOperator_ChangeOfBasis.cs:624``).
* Solver configurations implement ``ISolverFactory.CreateInstance(MultigridOperator)``
  (``ISmootherTemplate.cs:136-152``): ``FGMRESConfig`` (``FlexGMRES.cs:35``), ``PmgConfig`` (``PmgConfig.cs:80``),
  ``SoftPCGConfig`` (``SoftPCG.cs:37``), ``SoftGMRESConfig`` (``SoftGMRES.cs:75``), ``BlockJacobiConfig``
  (``BlockJacobi.cs:35``), ``SchwarzConfig`` (``Schwarz.cs:424``), ``CellILUConfig`` (``CellILU.cs:22``).  The returned solver
  implements ``ISolverSmootherTemplate`` (``ISmootherTemplate.cs:29-83``): ``Solve(X, B)`` with X the initial
  guess in and the solution out, ``ThisLevelIterations``, ``IterationsInNested``, ``Converged``, ``ResetStat``,
  ``Dispose``.  Non-convergence is not an exception; NaN/Inf or breakdown raise ``ArithmeticError``.

Vectors may be numpy arrays (host; copied to and from the device by the library) or CUDA torch tensors
(device-resident; no copies).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import native as nat


def _is_device(a) -> bool:
    return hasattr(a, "is_cuda") and a.is_cuda


class BlockMsrMatrix:
    """Device-resident block-sparse matrix with dense Np x Np (or nspc*Np) blocks."""

    def __init__(self, handle: C.c_void_p, owner: bool = True, single: bool = False):
        self._h = handle
        self._owner = owner
        self.single = single
        n, nb, nnzb, Np = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int32()
        nat.check(nat.lib().bsgpu_matrix_get_info(self._h, C.byref(n), C.byref(nb), C.byref(nnzb), C.byref(Np)))
        self.N, self.NoOfBlocks, self.nnzb, self.Np = n.value, nb.value, nnzb.value, Np.value

    @classmethod
    def from_bsr(cls, Np: int, row_ptr, col_idx, values, nspc=None) -> "BlockMsrMatrix":
        """values: row-major blocks concatenated in block-CSR order (numpy on the host or CUDA tensors)."""
        dev = _is_device(values)
        if dev:
            import torch
            row_ptr = row_ptr.to(torch.int64).contiguous()
            col_idx = col_idx.to(torch.int32).contiguous()
            values = values.to(torch.float64).contiguous()
            nspc = None if nspc is None else nspc.to(torch.int32).contiguous()
        else:
            row_ptr = np.ascontiguousarray(row_ptr, np.int64)
            col_idx = np.ascontiguousarray(col_idx, np.int32)
            values = np.ascontiguousarray(values, np.float64)
            nspc = None if nspc is None else np.ascontiguousarray(nspc, np.int32)
        nb = (row_ptr.shape[0] if dev else len(row_ptr)) - 1
        h = C.c_void_p()
        nat.check(nat.lib().bsgpu_matrix_create(
            C.byref(h), nb, int(Np), None if nspc is None else nat.ptr(nspc), nat.ptr(row_ptr), nat.ptr(col_idx),
            nat.ptr(values), nat.DEVICE_POINTERS if dev else nat.HOST_POINTERS))
        M = cls(h)
        host = (lambda a: a.cpu().numpy()) if dev else (lambda a: a)
        M._structure = (host(row_ptr), host(col_idx), None if nspc is None else host(nspc))
        return M

    @classmethod
    def AssembleSIP(cls, shape, p: int, penalty: Optional[float] = None, coeff=None, lo: float = 0.0,
                    hi: float = 1.0) -> "BlockMsrMatrix":
        """The SIP operator of -div(nu grad u) on a uniform Cartesian grid of ``shape`` cells over [lo, hi]^D,
        degree ``p``, homogeneous Dirichlet boundaries, assembled on the GPU (bsgpu_assemble_sip_cartesian): the
        matrix ``assembly.assemble_sip`` builds on the host (ipLaplace.cs:95-245).  ``penalty`` defaults to
        1.3 * max((p+1)(p+D)/D, (p+1)^2); ``coeff``: per-cell diffusivity (numpy or CUDA tensor, cells x fastest)."""
        shape = [int(n) for n in shape]
        D = len(shape)
        if not 1 <= D <= 3:
            raise ValueError("shape must have 1, 2 or 3 entries")
        if penalty is None:
            penalty = 1.3 * max((p + 1) * (p + D) / D, (p + 1) ** 2)
        nc = int(np.prod(shape))
        flags, nu = nat.HOST_POINTERS, None
        if coeff is not None:
            if _is_device(coeff):
                import torch
                nu = coeff.to(torch.float64).contiguous()
                flags = nat.DEVICE_POINTERS
            else:
                nu = np.ascontiguousarray(coeff, np.float64)
            if (nu.numel() if _is_device(nu) else nu.size) != nc:
                raise ValueError("coeff must hold one value per cell")
        dims = (C.c_int32 * D)(*shape)
        h = C.c_void_p()
        nat.check(nat.lib().bsgpu_assemble_sip_cartesian(C.byref(h), D, dims, float(lo), float(hi), int(p),
                                                         float(penalty), None if nu is None else nat.ptr(nu),
                                                         flags))
        M = cls(h)
        # host copy of the block structure: block columns ascending (-z, -y, -x, self, +x, +y, +z as present)
        ids = np.arange(nc, dtype=np.int64)
        idx = np.unravel_index(ids, tuple(reversed(shape)))[::-1]   # per direction, x first
        strides = [int(np.prod(shape[:d])) for d in range(D)]
        cand = [np.where(idx[d] > 0, ids - strides[d], -1) for d in reversed(range(D))] + [ids] + \
               [np.where(idx[d] < shape[d] - 1, ids + strides[d], -1) for d in range(D)]
        cand = np.stack(cand, axis=1)
        keep = cand >= 0
        rp = np.zeros(nc + 1, np.int64)
        np.cumsum(keep.sum(axis=1), out=rp[1:])
        M._structure = (rp, cand[keep].astype(np.int32), None)
        return M

    @classmethod
    def from_system(cls, s) -> "BlockMsrMatrix":
        return cls.from_bsr(s.Np, s.row_ptr, s.col_idx, s.values, getattr(s, "nspc", None))

    # --- reference API -------------------------------------------------------------------------------------------
    def SpMV(self, alpha: float, a, beta: float, acc):
        """acc = alpha*A*a + beta*acc (BlockMsrMatrix.SpMV)."""
        if a is acc:
            raise ValueError("In-Place computation is not supported.")
        na = a.numel() if _is_device(a) else len(a)
        nacc = acc.numel() if _is_device(acc) else len(acc)
        if na != self.N:
            raise ValueError("Mismatch in number of columns.")
        if nacc != self.N:
            raise ValueError("Mismatch in number of rows.")
        if _is_device(a) != _is_device(acc):
            raise ValueError("a and acc must both live on the host or both on the device")
        if self.single:
            if not _is_device(a):
                raise ValueError("single-precision matrices take device vectors")
            nat.check(nat.lib().bsgpu_matrix_spmv_device_f32(self._h, float(alpha), nat.ptr(a), float(beta),
                                                             nat.ptr(acc), None))
            return acc
        if _is_device(a):
            import torch
            stream = torch.cuda.current_stream().cuda_stream
            nat.check(nat.lib().bsgpu_matrix_spmv_device(self._h, float(alpha), nat.ptr(a), float(beta), nat.ptr(acc),
                                                         C.c_void_p(stream)))
        else:
            if acc.dtype != np.float64 or not acc.flags.c_contiguous:
                raise ValueError("acc must be a contiguous float64 array")
            a = np.ascontiguousarray(a, np.float64)
            nat.check(nat.lib().bsgpu_matrix_spmv(self._h, float(alpha), nat.ptr(a), float(beta), nat.ptr(acc)))
        return acc

    def ToSingle(self) -> "BlockMsrMatrix":
        h = C.c_void_p()
        nat.check(nat.lib().bsgpu_matrix_create_single(self._h, C.byref(h)))
        return BlockMsrMatrix(h, single=True)

    def Autotune(self):
        """Picks the launch shape of this matrix's FP64 product by timing the candidates (autotune_report)."""
        nat.check(nat.lib().bsgpu_matrix_autotune(self._h))

    def Restrict(self, keep: int) -> "BlockMsrMatrix":
        """Sub-matrix of the leading ``keep`` modes per species (GridAndDegRestriction's coarse operator)."""
        h = C.c_void_p()
        nat.check(nat.lib().bsgpu_matrix_restrict(self._h, int(keep), C.byref(h)))
        return BlockMsrMatrix(h)

    def SaveToTextFileSparse(self, path: str) -> int:
        """Writes the matrix in the text format of BoSSS's SaveToTextFileSparse (IMutuableMatrixEx_Extensions.cs:517);
        returns the number of non-zero entries.  Available for matrices created with ``from_bsr``."""
        from .matrixio import save_text_sparse
        st = getattr(self, "_structure", None)
        if st is None:
            raise ValueError("the block structure of this matrix is not known on the host")
        rp, ci, nspc = st
        L = (np.ones(self.NoOfBlocks, np.int64) if nspc is None else np.asarray(nspc, np.int64)) * self.Np
        rows = np.repeat(np.arange(self.NoOfBlocks), np.diff(rp))
        nvals = int((L[rows] * L[np.asarray(ci)]).sum())
        return save_text_sparse(path, self.Np, rp, ci, self.read_values(nvals), nspc)

    def read_values(self, nvals: Optional[int] = None) -> np.ndarray:
        """All blocks, row-major, in block-CSR order (the layout of ReadBlock).

        ``nvals`` (the total number of block entries) is needed for blocks of uneven size."""
        if nvals is None:
            if self.N != self.NoOfBlocks * self.Np:
                raise ValueError("uneven block sizes: pass nvals")
            nvals = self.nnzb * self.Np * self.Np
        out = np.empty(nvals)
        nat.check(nat.lib().bsgpu_matrix_read_values(self._h, nat.ptr(out), nat.HOST_POINTERS))
        return out

    def Dispose(self):
        if self._h is not None and self._owner:
            nat.lib().bsgpu_matrix_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.Dispose()
        except Exception:
            pass


class MultigridOperator:
    """Operator as seen by the solvers: L*A*L^T with L from SymmInv of each diagonal block."""

    Eye, DiagBlockEquilib = nat.COB_EYE, nat.COB_DIAG_BLOCK_EQUILIB

    def __init__(self, A: BlockMsrMatrix, mode: int = nat.COB_DIAG_BLOCK_EQUILIB, h_levels=()):
        """``h_levels``: prolongations of the agglomeration levels below the coarsest p-level, finest first
        (objects with Np, nb_fine, nb_coarse, row_ptr, col_idx, values -- e.g. ``assembly.h_hierarchy``)."""
        self.BaseMatrix = A
        self.mode = mode
        h = C.c_void_p()
        nat.check(nat.lib().bsgpu_mgop_create(C.byref(h), A._h, int(mode)))
        self._h = h
        oh = C.c_void_p()
        nat.check(nat.lib().bsgpu_mgop_get_operator(self._h, C.byref(oh)))
        self.OperatorMatrix = BlockMsrMatrix(oh, owner=False)
        for P in h_levels:
            self.AddHLevel(P)

    def SetCellGraph(self, neighbours, features=None):
        """Face neighbours per cell ([cells, faces], -1 = none) and optional per-cell features for the learned
        stage."""
        nb = np.ascontiguousarray(neighbours, np.int32)
        nat.check(nat.lib().bsgpu_mgop_set_cell_neighbours(self._h, int(nb.shape[1]), nat.ptr(nb)))
        if features is not None:
            ft = np.ascontiguousarray(features, np.float32)
            if ft.ndim == 1:
                ft = ft[:, None]
            nat.check(nat.lib().bsgpu_mgop_set_cell_features(self._h, int(ft.shape[1]), nat.ptr(ft)))

    def AddHLevel(self, P):
        rp = np.ascontiguousarray(P.row_ptr, np.int64)
        ci = np.ascontiguousarray(P.col_idx, np.int32)
        v = np.ascontiguousarray(P.values, np.float64)
        nat.check(nat.lib().bsgpu_mgop_add_h_level(self._h, int(P.Np), int(P.nb_fine), int(P.nb_coarse),
                                                   nat.ptr(rp), nat.ptr(ci), nat.ptr(v)))

    def LeftChangeOfBasis(self, total_len: int) -> np.ndarray:
        out = np.empty(total_len)
        nat.check(nat.lib().bsgpu_mgop_read_left_cob(self._h, nat.ptr(out)))
        return out

    def Dispose(self):
        if self._h is not None:
            nat.lib().bsgpu_mgop_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.Dispose()
        except Exception:
            pass


@dataclass
class IterativeSolverConfig:
    """IterativeSolverConfig.cs:19-62.  termination: 'default' (R < R0*tol + tol) or 'relative' (R < R0*tol)."""
    ConvergenceCriterion: float = 1e-10
    MaxSolverIterations: int = 300
    MinSolverIterations: int = 1
    termination: str = "default"

    def _base(self) -> nat.SolverConfig:
        c = nat.SolverConfig()
        nat.check(nat.lib().bsgpu_solver_config_default(C.byref(c)))
        c.tol = self.ConvergenceCriterion
        c.max_iter = self.MaxSolverIterations
        c.min_iter = self.MinSolverIterations
        c.termination = nat.TERM_RELATIVE if self.termination == "relative" else nat.TERM_DEFAULT
        return c

    def CreateInstance(self, op: MultigridOperator) -> "GpuSolver":
        return GpuSolver(op, self._config())


@dataclass
class PmgConfig(IterativeSolverConfig):
    """PmgConfig.CreateInstanceImpl__Kummer (PmgConfig.cs:80-245).

    Post-smoother of every p-level: ``UseILU = True`` selects block ILU(0) in the natural cell order (CellILU, as
    PmgConfig.cs:124-141 does for the levels it creates), otherwise ``Smoother``: "blockjacobi" (BlockJacobi with
    ``BlockJacobiIterations``), "blockgs" (symmetric multicolour block Gauss-Seidel), "schwarz" (restricted
    additive Schwarz, one patch per cell), "schwarz_blocks" (additive Schwarz with multi-cell blocks:
    ``SchwarzParts``, ``SchwarzOverlap``, ``SchwarzOverlapScaling``), "ilu_natural" or "ilu" (block ILU(0) with the
    cells ordered by the two colours of the block graph).

    ``DegreeHierarchy``: modes per species kept on each level, finest first (e.g. (20, 10, 4) for p = 3 -> 2 -> 1
    in 3-D).  The coarsest level is solved by block-Jacobi PCG to ``CoarseTolerance`` (relative), by CG
    preconditioned with a smoothed-aggregation AMG V-cycle (``CoarseSolver = "amg"``: ``HLevels`` AMG levels,
    ``HSweeps`` Jacobi sweeps, dense below ``DenseLimit``), or densely (``CoarseSolver = "dense"``, p = 0 levels
    up to 4096 unknowns), or by h-multigrid on the agglomeration levels given to the ``MultigridOperator``
    (``CoarseSolver = "hmg"``: OrthoMG to ``CoarseTolerance`` with ``HSweeps`` block-Jacobi sweeps,
    ``HCycle`` iterations per coarser h-level, dense below ``DenseLimit``).
    With ``HLevels > 0``, ``CoarseSolver = "pcg"`` and a p = 0 last level
    (DegreeHierarchy ending in 1), up to ``HLevels`` aggregation h-levels follow, each an OrthoMG with
    ``HCycle`` iterations and ``HSweeps`` post-smoother sweeps, down to ``DenseLimit`` unknowns.
    """
    DegreeHierarchy: tuple = (20, 10, 4)
    NoOfPostSmootherSweeps: int = 10
    BlockJacobiIterations: int = 1
    BlockJacobiOmega: float = 1.0
    CoarseTolerance: float = 1e-3
    CoarseMaxIterations: int = 2000
    CoarseSolver: str = "pcg"
    SubLevelMaxIterations: int = 100
    SubLevelReduction: float = 0.1
    HLevels: int = 0
    HSweeps: int = 3
    HCycle: int = 1
    DenseLimit: int = 1024
    Smoother: str = "blockjacobi"
    HSmoother: str = "blockjacobi"
    OrthoMaxKrylovDim: int = 96     # OrthonormalizationMultigrid.Config.MaxKrylovDim: history length per level
    RecalcResiPeriod: int = 1       # OrthonormalizationMultigrid.RecalcResiPeriod: full residual every n updates
    UseILU: bool = False
    SchwarzParts: int = 0           # Smoother "schwarz_blocks": number of blocks (0: blocks of 8 cells)
    SchwarzOverlap: int = 1         # ... layers of overlap (0, 1, 2)
    SchwarzOverlapScaling: bool = False
    MatrixFP16: bool = False        # FP16 level matrices in the FP32 V-cycle (FGMRESConfig MixedPrecision)

    def _fill(self, c):
        c.n_levels = len(self.DegreeHierarchy)
        for i, k in enumerate(self.DegreeHierarchy):
            c.level_keep[i] = int(k)
        c.post_sweeps = self.NoOfPostSmootherSweeps
        c.bj_iters = self.BlockJacobiIterations
        c.bj_omega = self.BlockJacobiOmega
        kinds = {"dense": nat.COARSE_DENSE, "pcg": nat.COARSE_PCG, "amg": nat.COARSE_AMG, "hmg": nat.COARSE_HMG}
        if self.CoarseSolver not in kinds:
            raise ValueError(f"CoarseSolver must be one of {sorted(kinds)}")
        c.coarse_kind = kinds[self.CoarseSolver]
        c.coarse_tol = self.CoarseTolerance
        c.coarse_max_iter = self.CoarseMaxIterations
        c.sub_max_iter = self.SubLevelMaxIterations
        c.sub_reduction = self.SubLevelReduction
        c.h_levels = self.HLevels
        c.h_sweeps = self.HSweeps
        c.h_cycle = self.HCycle
        c.dense_limit = self.DenseLimit
        sm = {"blockjacobi": nat.SMOOTHER_BLOCKJACOBI, "blockgs": nat.SMOOTHER_BLOCKGS,
              "schwarz": nat.SMOOTHER_SCHWARZ, "ilu": nat.SMOOTHER_ILU, "ilu_natural": nat.SMOOTHER_ILU_NATURAL,
              "schwarz_blocks": nat.SMOOTHER_SCHWARZ_BLOCKS}
        if self.Smoother not in sm or self.HSmoother not in sm:
            raise ValueError(f"Smoother / HSmoother must be one of {sorted(sm)}")
        c.smoother = nat.SMOOTHER_ILU_NATURAL if self.UseILU else sm[self.Smoother]
        c.h_smoother = sm[self.HSmoother]
        if self.OrthoMaxKrylovDim < 2:
            raise ValueError("OrthoMaxKrylovDim must be at least 2")
        c.ortho_max_krylov = self.OrthoMaxKrylovDim
        if self.RecalcResiPeriod < 1:
            raise ValueError("RecalcResiPeriod must be at least 1")
        c.recalc_resi_period = self.RecalcResiPeriod
        c.fp16_storage = nat.FP16_MATRICES if self.MatrixFP16 else 0
        if self.SchwarzOverlap < 0 or self.SchwarzOverlap > 2:
            raise ValueError("SchwarzOverlap must be 0, 1 or 2")
        c.schwarz_parts = self.SchwarzParts
        c.schwarz_overlap = self.SchwarzOverlap
        c.schwarz_scaling = 1 if self.SchwarzOverlapScaling else 0

    def _config(self):
        c = self._base()
        c.solver = nat.SOLVER_ORTHOMG
        self._fill(c)
        return c


@dataclass
class FGMRESConfig(IterativeSolverConfig):
    """FGMRESConfig (FlexGMRES.cs:35) with one p-multigrid V-cycle (a PmgConfig) as preconditioner.

    ``MixedPrecision``: the preconditioner runs in FP32 (matrices, block-Jacobi factors and vectors); the outer
    residual, the Arnoldi process and the solution update stay FP64.
    """
    MaxKrylovDim: int = 30
    Preconditioners: List[PmgConfig] = field(default_factory=lambda: [PmgConfig()])
    MixedPrecision: bool = False
    Learned: str = "off"            # "off" | "fgmres" | "presmooth" | "both"; needs MultigridOperator.SetCellGraph
    LearnedHidden: int = 64
    LearnedStall: float = 0.99
    LearnedPairs: int = 0           # training residuals collected in total (0: 12 per right-hand side)
    # True / "vcycle": record the V-cycle once as a CUDA graph with device-side decisions; "solve": record the
    # whole solve (FlexGMRES loops included) as one graph, one launch per solve, usable in a GpuBatch
    Graph: object = False
    Autotune: bool = False          # time the launch shapes of the level matrices' kernels at set-up

    def _config(self):
        if len(self.Preconditioners) != 1:
            raise NotImplementedError("exactly one PmgConfig preconditioner is supported")
        c = self._base()
        c.solver = nat.SOLVER_FGMRES_PMG
        c.max_krylov = self.MaxKrylovDim
        self.Preconditioners[0]._fill(c)
        c.precision = nat.PRECISION_MIXED if self.MixedPrecision else nat.PRECISION_FP64
        modes = {"off": nat.LEARNED_OFF, "fgmres": nat.LEARNED_FGMRES, "presmooth": nat.LEARNED_PRESMOOTH,
                 "both": nat.LEARNED_BOTH}
        if self.Learned not in modes:
            raise ValueError(f"Learned must be one of {sorted(modes)}")
        c.learned = modes[self.Learned]
        c.learned_hidden = self.LearnedHidden
        c.learned_stall = self.LearnedStall
        if self.LearnedPairs < 0:
            raise ValueError("LearnedPairs must be >= 0")
        c.learned_pairs = self.LearnedPairs
        graph_modes = {False: 0, None: 0, "off": 0, True: 1, "vcycle": 1, "solve": 2}
        if self.Graph not in graph_modes:
            raise ValueError("Graph must be False, True / 'vcycle' or 'solve'")
        c.graph = graph_modes[self.Graph]
        c.autotune = 1 if self.Autotune else 0
        return c


@dataclass
class SoftGMRESConfig(IterativeSolverConfig):
    """SoftGMRES (SoftGMRES.cs:75,227-460): restarted GMRES(MaxKrylovDim) with left preconditioning.

    ``Precond``: one of the block smoothers "blockjacobi", "schwarz", "ilu" (``BlockJacobiIterations`` sweeps for
    block Jacobi / Schwarz), or None.  Left preconditioning needs the same M^{-1} in every application, so the
    p-multigrid V-cycle (which varies between calls) belongs in ``FGMRESConfig``; a ``PmgConfig`` is rejected.
    The termination test compares the preconditioned residual estimate with the unpreconditioned initial
    residual, as the reference does; that comparison is meaningful when the preconditioner is of unit scale, as
    block Jacobi is on the DiagBlockEquilib operator (the ``MultigridOperator`` default).  On an unscaled operator
    with large diagonal blocks the preconditioned estimate falls below the absolute machine-precision floor early.
    """
    MaxKrylovDim: int = 80
    Precond: object = None
    BlockJacobiIterations: int = 1

    def _config(self):
        c = self._base()
        c.solver = nat.SOLVER_SOFTGMRES
        c.max_krylov = self.MaxKrylovDim
        if isinstance(self.Precond, PmgConfig):
            raise ValueError("SoftGMRES takes a block-smoother preconditioner; use FGMRESConfig for p-multigrid")
        c.n_levels = 1
        kinds = {"blockjacobi": nat.SMOOTHER_BLOCKJACOBI, "schwarz": nat.SMOOTHER_SCHWARZ, "ilu": nat.SMOOTHER_ILU}
        if self.Precond is None:
            c.bj_iters = -1
        elif self.Precond in kinds:
            c.smoother = kinds[self.Precond]
            c.bj_iters = self.BlockJacobiIterations
        else:
            raise ValueError(f"Precond must be a PmgConfig, one of {sorted(kinds)} or None")
        return c


@dataclass
class SoftPCGConfig(IterativeSolverConfig):
    """SoftPCG (SoftPCG.cs:37) preconditioned by the inverse block diagonal (``BlockJacobiPrecond``)."""
    BlockJacobiPrecond: bool = True

    def _config(self):
        c = self._base()
        c.solver = nat.SOLVER_SOFTPCG
        c.bj_iters = 0 if self.BlockJacobiPrecond else -1
        return c


@dataclass
class BlockJacobiConfig:
    """BlockJacobi (BlockJacobi.cs:35): NoOfIterations, omega."""
    NoOfIterations: int = 1
    omega: float = 1.0

    def CreateInstance(self, op: MultigridOperator) -> "GpuSolver":
        c = nat.SolverConfig()
        nat.check(nat.lib().bsgpu_solver_config_default(C.byref(c)))
        c.solver = nat.SOLVER_BLOCKJACOBI
        c.bj_iters = self.NoOfIterations
        c.bj_omega = self.omega
        return GpuSolver(op, c)


@dataclass
class CellILUConfig:
    """CellILU (CellILU.cs:22) with ILU_level = 0 as a stand-alone solver: X = U^{-1} L^{-1} B per call.

    ``Order``: "natural" (the reference's cell order, factored and applied wavefront by wavefront) or "coloured"
    (the cells ordered by the two colours of the block graph: one launch per triangular solve, a different ILU(0)).
    Blocks must be uniform of size 4, 6, 10 or 20."""
    ILU_level: int = 0
    Order: str = "natural"

    def CreateInstance(self, op: MultigridOperator) -> "GpuSolver":
        if self.ILU_level != 0:
            raise NotImplementedError("only ILU_level = 0 is available")
        orders = {"natural": nat.SMOOTHER_ILU_NATURAL, "coloured": nat.SMOOTHER_ILU}
        if self.Order not in orders:
            raise ValueError(f"Order must be one of {sorted(orders)}")
        c = nat.SolverConfig()
        nat.check(nat.lib().bsgpu_solver_config_default(C.byref(c)))
        c.solver = nat.SOLVER_BLOCKJACOBI
        c.smoother = orders[self.Order]
        return GpuSolver(op, c)


@dataclass
class SchwarzConfig:
    """Schwarz.Config (Schwarz.cs:424) as a stand-alone solver: FixedNoOfIterations (Schwarz.cs:979) updates of
    additive Schwarz.

    ``Blocking = "parts"`` (the reference's form): ``NoOfParts`` blocks (METISBlockingStrategy
    NoOfPartsOnCurrentProcess, Schwarz.cs:195; here a greedy breadth-first partition of the cell graph; 0: blocks of
    8 cells) grown by ``Overlap`` in {0, 1, 2} layers of neighbours, dense block inverses (at most 1024 unknowns per
    block), block solutions added, scaled by one over the multiplicity with ``EnableOverlapScaling``.
    ``Blocking = "cell"``: one block per cell plus its face neighbours with the correction kept on the centre cell
    (restricted additive Schwarz, Overlap = 1, no scaling): the same sparsity as the operator, applied as one
    block-sparse product.
    """
    FixedNoOfIterations: int = 1
    Overlap: int = 1
    Blocking: str = "parts"
    NoOfParts: int = 0
    EnableOverlapScaling: bool = False

    def CreateInstance(self, op: MultigridOperator) -> "GpuSolver":
        if self.FixedNoOfIterations < 1:
            raise ValueError("FixedNoOfIterations must be at least 1")
        if self.Overlap < 0 or self.Overlap > 2:
            raise ValueError("Overlap must be 0, 1 or 2 (Schwarz.cs:501-516)")
        if self.Blocking not in ("parts", "cell"):
            raise ValueError("Blocking must be 'parts' or 'cell'")
        if self.Blocking == "cell" and (self.Overlap != 1 or self.EnableOverlapScaling):
            raise NotImplementedError("cell blocks are one cell plus its face neighbours (Overlap = 1, no scaling)")
        c = nat.SolverConfig()
        nat.check(nat.lib().bsgpu_solver_config_default(C.byref(c)))
        c.solver = nat.SOLVER_BLOCKJACOBI
        c.smoother = nat.SMOOTHER_SCHWARZ_BLOCKS if self.Blocking == "parts" else nat.SMOOTHER_SCHWARZ
        c.bj_iters = self.FixedNoOfIterations - 1
        c.schwarz_parts = self.NoOfParts
        c.schwarz_overlap = self.Overlap
        c.schwarz_scaling = 1 if self.EnableOverlapScaling else 0
        return GpuSolver(op, c)


class GpuSolver:
    """ISolverSmootherTemplate backed by a bsgpu solver handle."""

    def __init__(self, op: MultigridOperator, cfg: nat.SolverConfig):
        self.op = op
        self.cfg = cfg
        h = C.c_void_p()
        nat.check(nat.lib().bsgpu_solver_create(C.byref(h), op._h, C.byref(cfg)))
        self._h = h
        self.stats = nat.SolveStats()

    def Solve(self, X, B):
        """X: initial guess in, solution out; B: right-hand side (original basis)."""
        N = self.op.BaseMatrix.N
        nx = X.numel() if _is_device(X) else len(X)
        nb = B.numel() if _is_device(B) else len(B)
        if nx != N:
            raise ValueError("Wrong length of unknowns vector.")
        if nb != N:
            raise ValueError("Wrong length of RHS vector.")
        if _is_device(X):
            nat.check(nat.lib().bsgpu_solver_solve_device(self._h, nat.ptr(X), nat.ptr(B), C.byref(self.stats)))
        else:
            if X.dtype != np.float64 or not X.flags.c_contiguous:
                raise ValueError("X must be a contiguous float64 array")
            B = np.ascontiguousarray(B, np.float64)
            nat.check(nat.lib().bsgpu_solver_solve(self._h, nat.ptr(X), nat.ptr(B), C.byref(self.stats)))
        return X

    @property
    def ThisLevelIterations(self) -> int:
        return self.stats.iterations

    @property
    def IterationsInNested(self) -> int:
        return self.stats.nested

    @property
    def Converged(self) -> bool:
        return bool(self.stats.converged)

    @property
    def SolveSeconds(self) -> float:
        return self.stats.seconds

    def ResetStat(self):
        self.stats = nat.SolveStats()

    def History(self) -> np.ndarray:
        n = C.c_int32()
        nat.check(nat.lib().bsgpu_solver_get_history(self._h, None, 0, C.byref(n)))
        out = np.zeros(max(n.value, 1))
        nat.check(nat.lib().bsgpu_solver_get_history(self._h, nat.ptr(out), n.value, C.byref(n)))
        return out[:n.value]

    def TrainLearned(self, n_rhs: int = 2, steps: int = 200, lr: float = 1e-3, seed: int = 0) -> float:
        """Trains the learned stage on residuals this solver generates; returns the final mean energy loss."""
        loss = C.c_double()
        nat.check(nat.lib().bsgpu_solver_train_learned(self._h, int(n_rhs), int(steps), float(lr), int(seed),
                                                       C.byref(loss)))
        return loss.value

    def LearnedInfo(self) -> dict:
        d = (C.c_int32 * 8)()
        nat.check(nat.lib().bsgpu_solver_learned_info(self._h, d))
        return dict(zip(("Np", "nfaces", "nextra", "F", "Fp", "H", "Op", "pairs"), list(d)))

    def LearnedWeights(self):
        """(W1 [Fp x H], W2 [H x H], W3 [H x Op]): the BF16 weights of the learned stage as float32."""
        i = self.LearnedInfo()
        w = [np.zeros((i["Fp"], i["H"]), np.float32), np.zeros((i["H"], i["H"]), np.float32),
             np.zeros((i["H"], i["Op"]), np.float32)]
        nat.check(nat.lib().bsgpu_solver_learned_get_weights(self._h, *(nat.ptr(a) for a in w)))
        return w

    def SetLearnedWeights(self, w1, w2, w3):
        w = [np.ascontiguousarray(a, np.float32) for a in (w1, w2, w3)]
        i = self.LearnedInfo()
        if [a.shape for a in w] != [(i["Fp"], i["H"]), (i["H"], i["H"]), (i["H"], i["Op"])]:
            raise ValueError("learned-stage weight shapes do not match")
        nat.check(nat.lib().bsgpu_solver_learned_set_weights(self._h, *(nat.ptr(a) for a in w)))

    def ApplyLearned(self, r) -> np.ndarray:
        """One application of the learned stage to r (operator basis, host vector)."""
        r = np.ascontiguousarray(r, np.float64)
        z = np.zeros_like(r)
        nat.check(nat.lib().bsgpu_solver_learned_apply(self._h, nat.ptr(r), nat.ptr(z)))
        return z

    def LearnedGradient(self, r):
        """(loss, [dL/dW1, dL/dW2, dL/dW3]) of the training loss for one residual r; no update."""
        i = self.LearnedInfo()
        r = np.ascontiguousarray(r, np.float64)
        g = [np.zeros((i["Fp"], i["H"]), np.float32), np.zeros((i["H"], i["H"]), np.float32),
             np.zeros((i["H"], i["Op"]), np.float32)]
        loss = C.c_double()
        nat.check(nat.lib().bsgpu_solver_learned_gradient(self._h, nat.ptr(r), *(nat.ptr(a) for a in g),
                                                          C.byref(loss)))
        return loss.value, g

    def SetTracing(self, on: bool = True):
        nat.check(nat.lib().bsgpu_solver_set_tracing(self._h, 1 if on else 0))

    def Trace(self):
        """Per-solver-block calls / inclusive seconds / iterations recorded while tracing was on."""
        import json
        buf = C.create_string_buffer(1 << 16)
        nat.check(nat.lib().bsgpu_solver_get_trace(self._h, buf, len(buf)))
        return json.loads(buf.value.decode())

    def Dispose(self):
        if self._h is not None:
            nat.lib().bsgpu_solver_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.Dispose()
        except Exception:
            pass


class GpuBatch:
    """Independent systems solved together from ONE CUDA graph (bsgpu_batch_*): every member's whole solve
    (``FGMRESConfig(Graph="solve")``) is one branch of the graph, all branches run concurrently from one launch.
    The reference solves independent systems one after another (``UniSolver.cs:588,623``)."""

    def __init__(self, solvers: List["GpuSolver"]):
        if not solvers:
            raise ValueError("empty batch")
        self.solvers = list(solvers)
        arr = (C.c_void_p * len(self.solvers))(*[s._h.value for s in self.solvers])
        h = C.c_void_p()
        nat.check(nat.lib().bsgpu_batch_create(C.byref(h), arr, len(self.solvers)))
        self._h = h
        self.stats = (nat.SolveStats * len(self.solvers))()

    def Solve(self, Xs, Bs):
        """Xs: initial guesses in, solutions out; Bs: right-hand sides (device tensors, original basis)."""
        n = len(self.solvers)
        if len(Xs) != n or len(Bs) != n:
            raise ValueError("one X and one B per batch member")
        for s, X, B in zip(self.solvers, Xs, Bs):
            if not (_is_device(X) and _is_device(B)):
                raise ValueError("batch vectors must be device tensors")
            N = s.op.BaseMatrix.N
            if X.numel() != N or B.numel() != N:
                raise ValueError("Wrong length of unknowns or RHS vector.")
        xp = (C.c_void_p * n)(*[nat.ptr(X) for X in Xs])
        bp = (C.c_void_p * n)(*[nat.ptr(B) for B in Bs])
        rc = nat.lib().bsgpu_batch_solve_device(self._h, xp, bp, self.stats)
        for s, st in zip(self.solvers, self.stats):  # results are written even when a member raised
            C.memmove(C.byref(s.stats), C.byref(st), C.sizeof(st))
        nat.check(rc)
        return Xs

    def Latencies(self) -> List[float]:
        """Device seconds from the batch launch to the end of each member's solve."""
        return [st.seconds for st in self.stats]

    def Dispose(self):
        if getattr(self, "_h", None):
            nat.lib().bsgpu_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.Dispose()
        except Exception:
            pass
