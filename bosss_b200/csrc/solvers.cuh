// Solver tree of the hot path: BlockJacobi, GridAndDegRestriction, OrthonormalizationMultigrid (p-multigrid),
// FlexGMRES, SoftPCG and the coarsest-level solve.  Host C++ drives the kernels of matrix.cu / blas1.cu on one
// CUDA stream; scalars (norms, projection coefficients) stay in device memory and the host reads back only the
// values its control flow branches on.
#pragma once
#include <memory>

#include "aggregation.cuh"
#include "amg.cuh"
#include "blas1.cuh"
#include "blockops.cuh"
#include "learned.cuh"
#include "matrix.cuh"

namespace bsgpu {

// Per-solver-tree execution context.
struct Ctx {
  cudaStream_t st = nullptr;
  ReduceScratch red;
  DBuf<double> dscal;   // device scalars
  double* hscal = nullptr;  // pinned mirror
  DBuf<int> dflag;      // device error flags
  int nscal = 0, nflag = 0;
  int scal_cap = 4096;
  uint64_t seed = 12345;
  Ctx();
  ~Ctx();
  double* scal(int n);  // allocate n device scalars
  int* flag();
  // copy device scalars to the host mirror and wait
  void fetch(const double* d, int n);
  double get(const double* d) {
    fetch(d, 1);
    return hscal[d - dscal.p];
  }
  void check_flag(const int* f, const char* what);

  // Tracing (counterpart of ilPSP FuncTrace/BlockTrace, Tracing.cs:703,806): per named block, the number of
  // calls, inclusive wall time (the stream is synchronised at block exit when tracing is on) and iterations.
  struct TraceEntry {
    std::string name;
    long calls = 0;
    double seconds = 0;
    long iterations = 0;
  };
  bool tracing = false;
  std::vector<TraceEntry> trace;
  int trace_id(const std::string& name);
};

// Scoped trace block; no-op unless ctx.tracing.
struct TraceScope {
  Ctx& c;
  int id;
  double t0 = 0;
  long* iters_out = nullptr;
  TraceScope(Ctx& ctx, int id_);
  ~TraceScope();
};

template <typename T>
struct Solver {
  virtual ~Solver() {}
  // X: initial guess in, solution out (device); B: right-hand side (device).  zero_guess: X is known to be 0.
  virtual void solve(Ctx& c, T* X, const T* B, bool zero_guess) = 0;
  virtual int nested() const { return 0; }
  int this_level_iterations = 0;
  bool converged = false;
  std::vector<double> history;
  int trace = -1;  // trace entry of this solver
};

// Termination criteria (IterativeSolverConfig.cs:48-62, PmgConfig.cs:202-215).
struct Term {
  int mode = 0;  // 0: R < R0*tol + tol, 1: R < R0*tol, 2: fixed iteration count, 3: sub-level (reduction)
  double tol = 1e-10;
  int max_iter = 300, min_iter = 1;
  double reduction = 0.1;
  std::pair<bool, bool> operator()(int iter, double R0, double R) const;
};

// What the MultigridOperator holds beyond the transformed matrix: the untransformed finest matrix, its left
// change of basis and the caller's h-level prolongations (used by the h-multigrid coarse solve).
struct OperatorInfo {
  const Matrix* top = nullptr;
  const double* L = nullptr;  // device, per block row I x I row-major; nullptr for Eye
  const std::vector<HostBsr>* hprol = nullptr;
  // cell graph for the learned stage: face neighbours per cell (-1 = none) and optional per-cell features
  int nfaces = 0;
  const std::vector<int32_t>* nbr = nullptr;
  int nfeat = 0;
  const std::vector<float>* feats = nullptr;
};

// Builds the solver tree for `cfg` on the (transformed) operator A (FP64).  For BSGPU_PRECISION_MIXED the
// preconditioner runs on FP32 copies of the level matrices.
struct Tree {
  std::unique_ptr<Ctx> ctx;
  std::vector<std::unique_ptr<Matrix>> owned;
  std::vector<std::unique_ptr<Aggregation>> aggs;
  std::vector<std::unique_ptr<AmgHierarchy>> amgs;
  std::vector<std::unique_ptr<HmgHierarchy>> hmgs;
  std::unique_ptr<Solver<double>> top;
  const Matrix* A = nullptr;
  bsgpu_solver_config cfg{};
  OperatorInfo info;
  std::unique_ptr<LearnedNet> net;  // learned preconditioner stage (cfg.learned != 0)
  bool learned_on = false;          // switched on once trained
  // hooks used while generating training data: the outer FGMRES copies its Arnoldi vectors here
  std::vector<DBuf<double>>* collect = nullptr;
  size_t collect_cap = 0;
  int learned_stalls = 0;           // solves in which the learned stage stalled and was switched off
  int learned_pool = 0;             // training residuals collected by the last train_learned
};
Tree* build_tree(const Matrix* A, const bsgpu_solver_config& cfg, const OperatorInfo& info);
// Generates training residuals with the solver itself (FGMRES Arnoldi vectors of solves with seeded random
// right-hand sides, learned stage off) and trains the learned stage; returns the final mean loss.
double train_learned(Tree& t, int n_rhs, int steps, double lr, uint64_t seed);

}  // namespace bsgpu
