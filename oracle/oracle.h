/* ORACLE -- test infrastructure only (CPU restatement of the BoSSS solver path; see oracle.cpp). */
#ifndef BOSSS_ORACLE_H
#define BOSSS_ORACLE_H
#include <stdint.h>

enum { OR_OK = 0, OR_ERR_ARGUMENT = 1, OR_ERR_ARITHMETIC = 3 };
enum { OR_SOLVER_PCG = 0, OR_SOLVER_FGMRES_PMG = 1, OR_SOLVER_ORTHOMG = 2, OR_SOLVER_SOFTGMRES = 3 };
enum { OR_COARSE_DENSE = 0, OR_COARSE_PCG = 1 };
enum { OR_SMOOTHER_BLOCKJACOBI = 0, OR_SMOOTHER_SCHWARZ = 1, OR_SMOOTHER_ILU_COLOURED = 2, OR_SMOOTHER_ILU_NATURAL = 3,
       OR_SMOOTHER_SCHWARZ_BLOCKS = 4 };

/* Block-sparse matrix: block i has nspc[i]*Np rows (nspc NULL: 1 species); blocks row-major, concatenated in
 * BSR order (block rows ascending, block columns ascending). */
typedef struct {
  int64_t nb;
  int32_t Np;
  const int32_t* nspc;
  const int64_t* row_ptr;
  const int32_t* col_idx;
  const double* values;
} or_bsr;

typedef struct {
  int32_t solver;
  int32_t top_mode; /* 0: R < R0*tol + tol (IterativeSolverConfig.DefaultTermination), 1: R < R0*tol */
  double tol;
  int32_t max_iter, min_iter;
  int32_t max_krylov;
  int32_t n_levels;
  int32_t level_keep[8]; /* modes per species kept on each level; level_keep[0] = Np */
  int32_t post_sweeps, bj_iters;
  double bj_omega;
  int32_t coarse_kind;
  double coarse_tol;
  int32_t coarse_max_iter;
  int32_t sub_max_iter;
  double sub_reduction;
  int32_t reference_fgmres_defect;
  int32_t recalc_resi_period; /* OrthoMG RecalcResiPeriod (OrthonormalizationMultigrid.cs:211); <= 1: every update */
  int32_t smoother;           /* OR_SMOOTHER_*: post-smoother of the p-levels */
  int32_t schwarz_parts, schwarz_overlap, schwarz_scaling; /* OR_SMOOTHER_SCHWARZ_BLOCKS (0 parts: 8 cells each) */
} or_solver_cfg;

typedef struct {
  int32_t iterations, nested, converged, n_hist;
  double res0, res;
} or_stats;

const char* or_last_error(void);
int or_set_threads(int n);
int or_spmv(const or_bsr* m, double alpha, const double* x, double beta, double* y);
int or_symminv(int n, double* M, double* L);
int or_invert(int n, double* A);
int or_change_of_basis(const or_bsr* m, double* values_out, double* L_out);
int or_restrict(const or_bsr* m, int keep, double* values_out, int64_t* map_out);
int or_blockjacobi(const or_bsr* m, int iters, double omega, double* x, const double* b);
/* additive Schwarz with multi-cell blocks: `parts` greedy breadth-first blocks (0: 8 cells each) grown by
 * `overlap` layers, dense block solves, optional overlap scaling; `iters` updates of x */
int or_block_schwarz(const or_bsr* m, int64_t parts, int overlap, int scaling, int iters, double* x, const double* b);
/* the cell lists of the multi-cell Schwarz blocks (partition into `parts` blocks, 0: blocks of 8 cells; grown by
   `overlap` layers): ptr[nblocks + 1], cells[total]; null ptr/cells: sizes only */
int or_schwarz_blocks(const or_bsr* m, int64_t parts, int overlap, int64_t* ptr, int32_t* cells, int64_t* nblocks,
                      int64_t* total);
int or_schwarz_rows(const or_bsr* m, double* values_out);
/* block ILU(0) over the block rows in `order` (NULL: natural order); factors in the matrix layout */
int or_ilu0_factor(const or_bsr* m, const int32_t* order, double* factor_out);
int or_ilu0_solve(const or_bsr* m, const int32_t* order, const double* factor, const double* b, double* x);
int or_solve(const or_bsr* m, const or_solver_cfg* c, const double* b, double* x, or_stats* stats, double* hist,
             int hist_cap);
/* persistent solver (set-up once, many solves); the matrix arrays must outlive it */
typedef struct or_solver_s* or_solver_t;
or_solver_t or_solver_create(const or_bsr* m, const or_solver_cfg* c);
int or_solver_solve(or_solver_t h, const double* b, double* x, or_stats* stats);
void or_solver_destroy(or_solver_t h);
#endif
