/*
 * bsgpu -- B200-native (sm_100a) library for the BoSSS linear-solver hot path.
 *
 * C ABI for P/Invoke (C#), ctypes (Python) or plain C/C++.  All handles are opaque; every function returns an
 * int status (BSGPU_OK = 0).  Host arrays are plain pointers + sizes; functions ending in _device take device
 * pointers and an optional cudaStream_t passed as void* (NULL = the handle's own stream).
 *
 * Reference interfaces replaced (paths relative to the BoSSS source tree):
 *   BlockMsrMatrix            src/L1-platform/BoSSS.Platform/BlockMsrMatrix.cs:191 (SpMV :2970, ReadBlock :1743)
 *   MultigridOperator         src/L3-solution/BoSSS.Solution.AdvancedSolvers/MultigridOperator.cs:37
 *                             (change of basis :650-700, UseSolver :1213-1262)
 *   ISolverSmootherTemplate   src/L3-solution/BoSSS.Solution.AdvancedSolvers/ISmootherTemplate.cs:29-83
 *   ISolverFactory            ISmootherTemplate.cs:136-152 (configs: PmgConfig.cs:80, FlexGMRES.cs:35,
 *                             SoftPCG.cs:37, BlockJacobi.cs:35)
 *   native binding precedent  src/ilPSP/ExtBinding/ilPSP.ExternalBinding/ExternalBinding.cs:15-75 (int ierr)
 *
 * Threading: a handle is not thread-safe; use one handle per host thread.  Each solver handle owns one CUDA
 * stream; host-pointer calls are synchronous with respect to the caller.
 */
#ifndef BSGPU_H
#define BSGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define BSGPU_API __declspec(dllexport)
#else
#define BSGPU_API __attribute__((visibility("default")))
#endif

/* ---- status codes (ISmootherTemplate / LAPACK-info conventions mapped to ints) --------------------------- */
enum {
  BSGPU_OK = 0,
  BSGPU_ERR_ARGUMENT = 1,      /* ArgumentException: length / partition mismatch, bad handle, bad config   */
  BSGPU_ERR_CUDA = 2,          /* CUDA runtime error (see bsgpu_last_error)                                */
  BSGPU_ERR_ARITHMETIC = 3,    /* ArithmeticException: NaN/Inf, zero pivot, residual increase, breakdown    */
  BSGPU_ERR_NOMEM = 4,         /* device allocation failed                                                 */
  BSGPU_ERR_UNSUPPORTED = 5,   /* feature/size not supported by this library                               */
  BSGPU_ERR_TIMEOUT = 6        /* a bounded device-side wait gave up                                       */
};

/* pointer-kind flag for creation functions */
enum { BSGPU_HOST_POINTERS = 0, BSGPU_DEVICE_POINTERS = 1 };

typedef struct bsgpu_matrix_s* bsgpu_matrix_t;
typedef struct bsgpu_mgop_s* bsgpu_mgop_t;
typedef struct bsgpu_solver_s* bsgpu_solver_t;

/* ---- library ------------------------------------------------------------------------------------------- */
BSGPU_API int bsgpu_get_version(int* major, int* minor);
/* Copies the message of the last failed call on this host thread into buf (NUL-terminated). */
BSGPU_API int bsgpu_last_error(char* buf, size_t len);
/* Number of kernels this library has launched in this process (tracing; FuncTrace/BlockTrace counterpart,
 * src/ilPSP/layer_1.2-ilPSP/ilPSP/Tracing.cs:703,806). */
BSGPU_API int bsgpu_get_launch_count(uint64_t* n);
/* Selects the CUDA device used by handles created afterwards on this host thread. */
BSGPU_API int bsgpu_set_device(int device);
/* Launch-shape autotuner (no counterpart in the reference; BoSSS has no GPU kernels to tune): tunes the FP64
 * product of A on the current device, and reports every decision taken in this process (solvers created with
 * cfg.autotune = 1 tune their level matrices) as a JSON array of {matrix, times_ms per candidate, threads_per_cta}. */
BSGPU_API int bsgpu_matrix_autotune(bsgpu_matrix_t A);
BSGPU_API int bsgpu_autotune_report(char* buf, size_t len);

/* ---- BlockMsrMatrix (BlockMsrMatrix.cs:191) ------------------------------------------------------------ *
 * nb block rows/columns; block i has nspc[i]*Np rows (nspc == NULL: one species); row_ptr[nb+1] and
 * col_idx[nnzb] are the block-CSR structure with block columns ascending inside a block row (the
 * SortedDictionary order of BlockMsrMatrix.cs:315); values holds the blocks row-major and concatenated in that
 * order (the layout ReadBlock, BlockMsrMatrix.cs:1743, returns).  The library re-packs them into its own
 * device layout.  flags: BSGPU_HOST_POINTERS or BSGPU_DEVICE_POINTERS for all four arrays. */
BSGPU_API int bsgpu_matrix_create(bsgpu_matrix_t* A, int64_t nb, int32_t Np, const int32_t* nspc,
                                  const int64_t* row_ptr, const int32_t* col_idx, const double* values,
                                  int32_t flags);
/* SIP (symmetric interior penalty) DG operator of -div(nu grad u) on a uniform Cartesian grid of shape[0] x ... x
 * shape[D-1] cells over [lo, hi]^D (D = 1, 2, 3; cells numbered x fastest), polynomial degree p (orthonormal
 * Legendre products of total degree <= p, modes ordered by total degree, then lexicographically), homogeneous
 * Dirichlet boundaries, assembled on the GPU into a new matrix handle: the matrix the host assembly of ipLaplace.cs
 * (:95-245) produces for this grid.  Inner faces: penalty * max(cj) * max(nu) of the two cells; boundary faces:
 * 2 * penalty * cj * nu; cj = 0.5 * (surface + boundary area) / volume (GridData_CellData.cs:681-687).  nu: per-cell
 * diffusivity (NULL: 1), a host or device array per flags (BSGPU_HOST_POINTERS / BSGPU_DEVICE_POINTERS). */
BSGPU_API int bsgpu_assemble_sip_cartesian(bsgpu_matrix_t* A, int32_t D, const int32_t* shape, double lo, double hi,
                                           int32_t p, double penalty, const double* nu, int32_t flags);
/* Load vector of a separable right-hand side f(x) = sum_m coef[m] prod_d f_{m,d}(x_d) on the same grid and basis:
 * tables holds, per term m and direction d, the 1-D projections of f_{m,d} onto the 1-D basis of every cell
 * interval, [M][D][shape[d]][p + 1] (the integral over the interval of f_{m,d} times the scaled 1-D Legendre
 * function); out[c * Np + a] = sum_m coef[m] prod_d tables[m][d][i_d(c)][mode_a[d]], a host or device array per
 * flags.  (The benchmark's sine-mode right-hand sides are of this form.) */
BSGPU_API int bsgpu_project_separable(int32_t D, const int32_t* shape, int32_t p, int32_t M, const double* coef,
                                      const double* tables, double* out, int32_t flags);
/* The block templates of that assembly for cell sizes h[0..D) (host computation, no device work): 31 row-major
 * Np x Np matrices (0: volume term; 1+4d .. 4+4d: consistency and penalty terms of the +d and -d faces of
 * direction d; 13+6d .. 15+6d: the off-diagonal terms of direction d).  n (may be NULL): entries; out (may be NULL
 * to query n) holds cap entries. */
BSGPU_API int bsgpu_sip_templates(int32_t D, int32_t p, const double* h, double* out, int64_t cap, int64_t* n);
/* The cell blocks of BSGPU_SMOOTHER_SCHWARZ_BLOCKS for a block structure (host computation, no device work): the
 * partition into `parts` blocks (0: blocks of 8 cells; greedy breadth-first aggregation of the block graph, the
 * stand-in for METISBlockingStrategy, Schwarz.cs:190-320) grown by `overlap` layers (Schwarz.cs:690-735), each
 * block's cells ascending.  ptr[nblocks + 1] and cells[total] (both NULL: sizes only). */
BSGPU_API int bsgpu_schwarz_blocks(int64_t nb, const int64_t* row_ptr, const int32_t* col_idx, int64_t parts,
                                   int32_t overlap, int64_t* ptr, int32_t* cells, int64_t* nblocks, int64_t* total);
/* The wavefronts of BSGPU_SMOOTHER_ILU_NATURAL for a block structure (host computation, no device work): a block
 * row's wavefront is one more than the largest of its lower neighbours' (the dependency levels of CellILU's natural
 * order, CellILU.cs:1229-1330).  level_ptr[nlevels + 1] offsets into rows[nb] (ascending within a wavefront); pass
 * NULL outputs to query nlevels. */
BSGPU_API int bsgpu_ilu_wavefronts(int64_t nb, const int64_t* row_ptr, const int32_t* col_idx, int64_t* level_ptr,
                                   int32_t* rows, int64_t* nlevels);
BSGPU_API int bsgpu_matrix_destroy(bsgpu_matrix_t A);
BSGPU_API int bsgpu_matrix_get_info(bsgpu_matrix_t A, int64_t* nrows, int64_t* nb, int64_t* nnzb, int32_t* Np);
/* Copies the values back in the creation layout (row-major blocks) to a host or device buffer. */
BSGPU_API int bsgpu_matrix_read_values(bsgpu_matrix_t A, double* values, int32_t flags);
/* BlockMsrMatrix.SpMV (BlockMsrMatrix.cs:2970): y = alpha*A*x + beta*y on host vectors of length nrows.
 * x and y must not alias (ArgumentException in the reference).  beta == 0: y is not read. */
BSGPU_API int bsgpu_matrix_spmv(bsgpu_matrix_t A, double alpha, const double* x, double beta, double* y);
/* Same as bsgpu_matrix_spmv but allocates no device memory, for callers that must not (a host program whose
 * device memory is already committed to its own pool, or one that cannot afford the device-wide synchronisation
 * cudaMalloc/cudaFree may cause).  No counterpart in the reference.  x and y are staged in a fixed array of
 * 2 x 2^20 doubles (16 MiB) that a GPU holds from the moment the library's module is loaded on it (its first use
 * there, under CUDA's lazy loading) until exit, whether or not this function is called; nrows must be
 * <= 1,048,576 (BSGPU_ERR_ARGUMENT otherwise).  The first call on a device looks up that array's device address,
 * so make it before any stream capture; a reset of the device's primary context invalidates the cached address
 * (as it does every handle).  All calls share the array: calls that overlap on the GPU (several host threads)
 * race. */
BSGPU_API int bsgpu_matrix_spmv_noalloc(bsgpu_matrix_t A, double alpha, const double* x, double beta, double* y);
/* Same on device vectors, asynchronous on `stream` (NULL = the legacy default stream). */
BSGPU_API int bsgpu_matrix_spmv_device(bsgpu_matrix_t A, double alpha, const double* x, double beta, double* y,
                                       void* stream);
/* FP32 copy of the values (for the single-precision preconditioner path) and its SpMV on float vectors. */
BSGPU_API int bsgpu_matrix_create_single(bsgpu_matrix_t A, bsgpu_matrix_t* A32);
BSGPU_API int bsgpu_matrix_spmv_device_f32(bsgpu_matrix_t A32, float alpha, const float* x, float beta, float* y,
                                           void* stream);
/* Sub-matrix of the leading `keep` modes of every species in every block (GridAndDegRestriction.cs:47-99). */
BSGPU_API int bsgpu_matrix_restrict(bsgpu_matrix_t A, int32_t keep, bsgpu_matrix_t* Asub);

/* ---- MultigridOperator change of basis (MultigridOperator.cs:650-700) ---------------------------------- *
 * mode 0 = Eye, 1 = DiagBlockEquilib (SymmInv per diagonal block, MultigridOperator_ChangeOfBasis.cs:624).
 * The operator seen by the solvers is L*A*L^T; B~ = L*B, X = L^T*X~. */
enum { BSGPU_COB_EYE = 0, BSGPU_COB_DIAG_BLOCK_EQUILIB = 1 };
BSGPU_API int bsgpu_mgop_create(bsgpu_mgop_t* op, bsgpu_matrix_t A, int32_t mode);
BSGPU_API int bsgpu_mgop_destroy(bsgpu_mgop_t op);
/* Borrowed handle of the transformed operator (owned by op). */
BSGPU_API int bsgpu_mgop_get_operator(bsgpu_mgop_t op, bsgpu_matrix_t* Aop);
/* Adds one h-level below the coarsest p-level, finest first: the prolongation from the agglomerated (coarser)
 * grid to the current one, in the untransformed orthonormal DG basis of that p-level, as block-CSR with
 * nb_fine block rows, nb_coarse block columns and Np x Np row-major blocks (host pointers).  The counterpart of
 * the prolongation operators of the reference's multigrid hierarchy on aggregation grids
 * (MultigridOperator.cs:774,815; AggregationGridBasis.cs); used by BSGPU_COARSE_HMG. */
BSGPU_API int bsgpu_mgop_add_h_level(bsgpu_mgop_t op, int32_t Np, int64_t nb_fine, int64_t nb_coarse,
                                     const int64_t* row_ptr, const int32_t* col_idx, const double* values);
/* Cell graph for the learned stage: nb x nfaces face-neighbour indices (-1 where a face has no neighbour), and
 * optional per-cell input features (nb x nfeat floats, e.g. log of the diffusivity of the cell and its
 * neighbours).  Host pointers; copied. */
BSGPU_API int bsgpu_mgop_set_cell_neighbours(bsgpu_mgop_t op, int32_t nfaces, const int32_t* nbr);
BSGPU_API int bsgpu_mgop_set_cell_features(bsgpu_mgop_t op, int32_t nfeat, const float* feats);
/* Per-block L factors, row-major, concatenated in block order (host buffer). */
BSGPU_API int bsgpu_mgop_read_left_cob(bsgpu_mgop_t op, double* L);

/* ---- solvers (ISolverSmootherTemplate / ISolverFactory) ------------------------------------------------ */
enum {
  BSGPU_SOLVER_SOFTPCG = 0,     /* SoftPCG.cs:113 with a block-Jacobi preconditioner (or none)              */
  BSGPU_SOLVER_FGMRES_PMG = 1,  /* FlexGMRES.cs:144 (Saad FGMRES(m)) preconditioned by one p-MG V-cycle     */
  BSGPU_SOLVER_ORTHOMG = 2,     /* PmgConfig.cs:80 OrthonormalizationMultigrid p-multigrid as the solver    */
  BSGPU_SOLVER_BLOCKJACOBI = 3, /* the smoother cfg.smoother selects (BlockJacobi.cs:35, Schwarz.cs:56) alone */
  BSGPU_SOLVER_SOFTGMRES = 4    /* SoftGMRES.cs:227 left-preconditioned GMRES(m) with the cfg.smoother block
                                   preconditioner (n_levels <= 1; none if bj_iters < 0) */
};
enum { BSGPU_TERM_DEFAULT = 0 /* R < R0*tol + tol */, BSGPU_TERM_RELATIVE = 1 /* R < R0*tol */ };
/* coarsest-level solver: dense inverse (p = 0, <= 4096 unknowns), block-Jacobi PCG, or PCG preconditioned by a
 * smoothed-aggregation AMG V-cycle (h_levels levels, h_sweeps Jacobi sweeps, dense below dense_limit) */
enum { BSGPU_COARSE_DENSE = 0, BSGPU_COARSE_PCG = 1, BSGPU_COARSE_AMG = 2,
       BSGPU_COARSE_HMG = 3 /* h-multigrid on the caller's agglomeration levels (bsgpu_mgop_add_h_level):
                               OrthoMG to coarse_tol with h_sweeps block-Jacobi sweeps, h_cycle iterations on the
                               coarser h-levels, dense below dense_limit */ };
enum { BSGPU_PRECISION_FP64 = 0, BSGPU_PRECISION_MIXED = 1 /* preconditioner in FP32, outer FP64 */ };
/* FP16 storage inside the FP32 preconditioner: the level matrices (uniform blocks of 4, 10 or 20; not with the
 * Gauss-Seidel smoother).  Bit 1 is reserved (FP16 OrthoMG histories lost the minimisation's consistency). */
enum { BSGPU_FP16_MATRICES = 2 };
/* post-smoother of the OrthoMG levels: BlockJacobi (BlockJacobi.cs:35; NoOfIterations = bj_iters), symmetric
 * multicolour block Gauss-Seidel (max(1, bj_iters) symmetric sweeps; uniform blocks of 4, 6, 10 or 20), or
 * restricted additive Schwarz with one overlapping block per cell (Schwarz.cs:56; bj_iters + 1 updates; blocks
 * of up to ~160 unknowns, uneven sizes allowed), factors in FP32 for the mixed-precision preconditioner */
enum { BSGPU_SMOOTHER_BLOCKJACOBI = 0, BSGPU_SMOOTHER_BLOCKGS = 1, BSGPU_SMOOTHER_SCHWARZ = 2,
       BSGPU_SMOOTHER_ILU = 3 /* block ILU(0) (CellILU.cs:22), cells ordered by the two colours of the block graph
                                 (one launch per triangular solve); uniform blocks of 4, 6, 10 or 20 */,
       BSGPU_SMOOTHER_ILU_NATURAL = 4 /* block ILU(0) in the reference's natural cell order (CellILU.cs:1229-1330,
                                         PmgConfig UseILU), factored and applied wavefront by wavefront; uniform
                                         blocks of 4, 6, 10 or 20 */,
       BSGPU_SMOOTHER_SCHWARZ_BLOCKS = 5 /* additive Schwarz with multi-cell blocks (Schwarz.cs:56, METIS blocking
                                            :190-320): cfg.schwarz_parts blocks from a greedy breadth-first
                                            partition of the cell graph, grown by cfg.schwarz_overlap layers, dense
                                            block inverses (at most 1024 unknowns per block), optional overlap
                                            scaling; bj_iters + 1 updates */ };
/* learned preconditioner stage (no counterpart in the reference): a one-hop message-passing MLP over the cell
 * graph, BF16 weights, FP32 accumulation.  FGMRES: an extra FlexGMRES preconditioner used in turn with the
 * p-multigrid V-cycle (FlexGMRES.cs:196-199 round-robin); PRESMOOTH: pre-smoother of the finest OrthoMG level
 * (OrthonormalizationMultigrid.cs:899); plain p-multigrid takes over when the stage stalls. */
enum { BSGPU_LEARNED_OFF = 0, BSGPU_LEARNED_FGMRES = 1, BSGPU_LEARNED_PRESMOOTH = 2, BSGPU_LEARNED_BOTH = 3 };

typedef struct {
  int32_t solver;           /* BSGPU_SOLVER_*                                                   */
  int32_t termination;      /* BSGPU_TERM_*                                                     */
  double tol;               /* ConvergenceCriterion (IterativeSolverConfig.cs:40), default 1e-10 */
  int32_t max_iter;         /* MaxSolverIterations, default 300                                 */
  int32_t min_iter;         /* MinSolverIterations, default 1                                   */
  int32_t max_krylov;       /* FGMRESConfig.MaxKrylovDim                                        */
  int32_t n_levels;         /* p-levels including the coarsest                                  */
  int32_t level_keep[8];    /* modes per species kept on each level (level_keep[0] = Np)        */
  int32_t post_sweeps;      /* NoOfPostSmootherSweeps (PmgConfig: 10)                           */
  int32_t bj_iters;         /* BlockJacobi.NoOfIterations (<0: no preconditioner for SoftPCG)   */
  double bj_omega;          /* BlockJacobi.omega                                                */
  int32_t coarse_kind;      /* BSGPU_COARSE_*                                                   */
  double coarse_tol;        /* relative tolerance of the PCG coarse solve                       */
  int32_t coarse_max_iter;
  int32_t sub_max_iter;     /* intermediate-level OrthoMG iteration limit (PmgConfig: 100)      */
  double sub_reduction;     /* intermediate-level residual reduction (PmgConfig: 0.1)           */
  int32_t precision;        /* BSGPU_PRECISION_*                                                */
  int32_t h_levels;         /* aggregation h-levels below a p = 0 last p-level (0: none)        */
  int32_t h_sweeps;         /* post-smoother sweeps on the h-levels                             */
  int32_t h_cycle;          /* OrthoMG iterations per call on the h-levels (1 = V-cycle)        */
  int32_t dense_limit;      /* levels with at most this many unknowns are solved densely        */
  int32_t smoother;         /* BSGPU_SMOOTHER_* on the p-levels                                 */
  int32_t h_smoother;       /* BSGPU_SMOOTHER_* on the h-levels (aggregation / h-multigrid)     */
  int32_t learned;          /* BSGPU_LEARNED_* (needs cell neighbours on the operator)          */
  int32_t learned_hidden;   /* hidden width of the learned stage (multiple of 16, default 64)   */
  double learned_stall;     /* a learned step reducing the residual by less than this factor
                               switches the stage off for the rest of the solve (default 0.99)  */
  int32_t ortho_max_krylov; /* OrthoMG history length (OrthonormalizationMultigrid.Config.MaxKrylovDim,
                               OrthonormalizationMultigrid.cs:486); when full, the minimisation restarts from
                               the current iterate (default 96)                                  */
  int32_t recalc_resi_period; /* OrthoMG RecalcResiPeriod (OrthonormalizationMultigrid.cs:211): the residual is
                                 recomputed from scratch every this many history entries, else updated (default 1) */
  int32_t learned_pairs;    /* training residuals bsgpu_solver_train_learned collects in total, spread over its
                               n_rhs solves (0: 12 per right-hand side)                           */
  int32_t graph;            /* 1: record the p-multigrid V-cycle of BSGPU_SOLVER_FGMRES_PMG once as a CUDA graph
                               with its decisions (termination tests, re-orthonormalisation, residual checks) taken
                               on the device, and replay it per application; 2: record the whole solve (change of
                               basis, FlexGMRES restart and Arnoldi loops, Givens rotations, preconditioner
                               round-robin, V-cycle) as one graph, replayed by one launch per solve and usable in a
                               bsgpu_batch; 0: host-driven (default).  Tracing and training run host-driven. */
  int32_t autotune;         /* 1: pick the launch shape (threads per CTA) of every level matrix's product and
                               block-Jacobi kernels by timing the candidates at set-up (bsgpu_autotune_report) */
  int32_t fp16_storage;     /* BSGPU_FP16_* bits, with BSGPU_PRECISION_MIXED: parts of the FP32 preconditioner
                               stored in FP16, arithmetic staying FP32 (0: none)                     */
  int32_t schwarz_parts;    /* BSGPU_SMOOTHER_SCHWARZ_BLOCKS: number of blocks (METISBlockingStrategy
                               NoOfPartsOnCurrentProcess, Schwarz.cs:195); 0: blocks of 8 cells      */
  int32_t schwarz_overlap;  /* Schwarz.Config.Overlap (Schwarz.cs:501): 0, 1 (default) or 2 layers   */
  int32_t schwarz_scaling;  /* Schwarz.Config.EnableOverlapScaling (Schwarz.cs:524): 1 scales by 1/multiplicity */
  int32_t reserved[5];
} bsgpu_solver_config;

typedef struct {
  int32_t iterations;       /* ThisLevelIterations                                              */
  int32_t nested;           /* IterationsInNested                                               */
  int32_t converged;        /* Converged                                                        */
  int32_t n_history;        /* entries written to the history buffer                            */
  double res0, res;         /* initial and final residual norms (transformed basis)             */
  double seconds;           /* device time of the solve                                         */
} bsgpu_solve_stats;

BSGPU_API int bsgpu_solver_config_default(bsgpu_solver_config* cfg);
BSGPU_API int bsgpu_solver_create(bsgpu_solver_t* s, bsgpu_mgop_t op, const bsgpu_solver_config* cfg);
BSGPU_API int bsgpu_solver_destroy(bsgpu_solver_t s);
/* ISolverSmootherTemplate.Solve via MultigridOperator.UseSolver: X (initial guess in, solution out) and B in the
 * original basis, host vectors.  Non-convergence is not an error (stats->converged = 0). */
BSGPU_API int bsgpu_solver_solve(bsgpu_solver_t s, double* X, const double* B, bsgpu_solve_stats* stats);
/* Same with device vectors; synchronous on return.  The solve is ordered after work already queued on the legacy
 * default stream; work on other streams that writes X or B must be complete before the call.  Handles are not
 * thread-safe, but different handles may be driven from different host threads at the same time. */
BSGPU_API int bsgpu_solver_solve_device(bsgpu_solver_t s, double* X, const double* B, bsgpu_solve_stats* stats);
/* Residual-norm history of the last solve (outer iterations), up to cap entries. */
BSGPU_API int bsgpu_solver_get_history(bsgpu_solver_t s, double* hist, int32_t cap, int32_t* n);
/* Per-block tracing (FuncTrace counterpart, Tracing.cs:703): when on, every solver of the tree records calls,
 * inclusive seconds and iterations (the stream is synchronised at block boundaries, so leave it off when timing
 * the whole solve).  Also switched on by the environment variable BSGPU_TRACE=1.  get_trace writes a JSON array. */
BSGPU_API int bsgpu_solver_set_tracing(bsgpu_solver_t s, int32_t on);
/* Trains the learned stage (cfg.learned != 0) on residuals the solver itself generates: the Arnoldi vectors of
 * n_rhs solves with seeded random right-hand sides (learned stage off), then `steps` Adam steps at learning rate
 * lr on the energy-norm loss.  Switches the stage on.  loss (may be NULL): final mean loss. */
BSGPU_API int bsgpu_solver_train_learned(bsgpu_solver_t s, int32_t n_rhs, int32_t steps, double lr, uint64_t seed,
                                         double* loss);
BSGPU_API int bsgpu_solver_get_trace(bsgpu_solver_t s, char* buf, size_t len);

/* ---- batches of independent systems (no counterpart in the reference, which solves them one after another,
 * UniSolver.cs:588,623) ----------------------------------------------------------------------------------------- *
 * create records the whole solves of n handles (each created with cfg.graph = 2, each at most once in the batch) as
 * the branches of ONE CUDA graph; solve_device stages B[i] and the initial guess X[i] (device vectors) into handle
 * i's buffers, runs every member concurrently from one graph launch, writes the solutions to X[i] and returns when
 * all are done.  stats (n entries, may be NULL): per member as bsgpu_solver_solve_device, with seconds = device time
 * from the launch to the end of that member's branch (its latency inside the batch).  The member handles must not
 * be used elsewhere while a batch solve runs, and the batch must be destroyed before its members (its graph uses
 * their device memory); a batch whose member had its learned stage switched since create is rejected (create it
 * again).  All members live on the current device.  Errors a member's solve records are raised after all results
 * were written. */
typedef struct bsgpu_batch_s* bsgpu_batch_t;
BSGPU_API int bsgpu_batch_create(bsgpu_batch_t* b, const bsgpu_solver_t* solvers, int32_t n);
BSGPU_API int bsgpu_batch_solve_device(bsgpu_batch_t b, double* const* X, const double* const* B,
                                       bsgpu_solve_stats* stats);
BSGPU_API int bsgpu_batch_destroy(bsgpu_batch_t b);

/* ---- learned stage access (no counterpart in the reference) --------------------------------------------- *
 * For checking and exchanging the trained network.  dims[8]: Np, nfaces, nextra, F (input width), Fp (F padded
 * to 16), H (hidden width), Op (Np padded to 16), residuals collected by the last training.  Weights are the
 * padded row-major matrices W1 [Fp x H], W2 [H x H], W3 [H x Op] of z_c = W3^T relu(W2^T relu(W1^T f_c)), f_c =
 * [r_c, r of the face neighbours in table order (0 where none), cell features, 0 padding]; get returns the BF16
 * values the kernels use, set stores FP32 masters and their BF16 roundings.  apply evaluates the stage once on a
 * host vector r in the operator's (transformed) basis: z = s NN(r / s), s = |r| / sqrt(n).  gradient evaluates the
 * training loss (z^T A z - 2 z^T r) / |r|^2 for one r and its gradient with respect to W1, W2, W3 (host buffers of
 * the padded shapes) without updating the weights. */
BSGPU_API int bsgpu_solver_learned_info(bsgpu_solver_t s, int32_t* dims);
BSGPU_API int bsgpu_solver_learned_get_weights(bsgpu_solver_t s, float* w1, float* w2, float* w3);
BSGPU_API int bsgpu_solver_learned_set_weights(bsgpu_solver_t s, const float* w1, const float* w2, const float* w3);
BSGPU_API int bsgpu_solver_learned_apply(bsgpu_solver_t s, const double* r, double* z);
BSGPU_API int bsgpu_solver_learned_gradient(bsgpu_solver_t s, const double* r, float* g1, float* g2, float* g3,
                                            double* loss);

#ifdef __cplusplus
}
#endif
#endif /* BSGPU_H */
