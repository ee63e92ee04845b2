// Solver tree of the hot path: BlockJacobi, GridAndDegRestriction, OrthonormalizationMultigrid (p-multigrid),
// FlexGMRES, SoftPCG and the coarsest-level solve.  Host C++ drives the kernels of matrix.cu / blas1.cu on one
// CUDA stream; scalars (norms, projection coefficients) stay in device memory and the host reads back only the
// values its control flow branches on.
#pragma once
#include <map>
#include <memory>

#include "aggregation.cuh"
#include "amg.cuh"
#include "blas1.cuh"
#include "blockops.cuh"
#include "bschwarz.cuh"
#include "devctl.cuh"
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
  bool autotune = false;  // tune the launch shapes of the level matrices' kernels at set-up
  void tune(const Matrix& A, int mode, const void* dinv = nullptr) {
    if (autotune) bsgpu::autotune(A, mode, dinv, st);
  }
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

  // Graph capture with device-side control flow (devctl.cuh).  While `capturing`, solvers record their kernels
  // into the graph being captured on `st`; cond_begin adds a conditional node (IF or WHILE) after the work
  // recorded so far and redirects `st` to a stream that captures the node's body until cond_end.  Kernels are
  // counted per body at capture time; the device counts how often each body runs (cond_set), so the launch
  // counter can add the kernels a replay actually ran (flush_graph_counts).
  bool capturing = false;
  std::vector<cudaStream_t> body_streams;
  std::vector<cudaStream_t> st_stack;
  std::vector<int> body_stack;
  std::vector<long long> body_kernels;  // kernels recorded directly in each body (0: the top level)
  int cur_body = 0;
  unsigned long long mark = 0;
  DBuf<unsigned int> d_exec;            // executions of each conditional body
  std::vector<unsigned int> h_exec;
  int* d_err = nullptr;                 // error word of captured solves (kDevErr* bits)
  int* h_err = nullptr;                 // pinned mirror
  bool err_pending = false;             // a copy of the error word is queued behind a graph launch
  bool graph_ran = false;
  void graph_init();
  void capture_begin();
  long long capture_end(cudaGraph_t* g);  // returns the kernels recorded at the top level
  // recording into a graph whose capture another stream began (st joined it through an event): the same
  // bookkeeping without beginning or ending the capture of st
  void capture_join();
  long long capture_leave();
  int first_body = 1;                   // first conditional body of the current recording
  long long recorded_total() const;     // kernels recorded by the current recording
  // after an exception inside a recording: ends the open conditional bodies and leaves capturing mode
  void capture_abort();
  int new_body(const std::string& name);
  std::vector<std::string> body_names;
  std::map<std::string, unsigned long long> graph_counts;  // executions of the conditional bodies, by name
  unsigned int* exec_of(int body) { return d_exec.p + body; }
  cudaGraphConditionalHandle cond_handle();
  void cond_begin(cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type, int body);
  void cond_end();
  void check_graph_errors();  // after a synchronisation: raises the pending device error, if any
  void flush_graph_counts();  // synchronises; adds the kernels of the conditional bodies that ran
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
  // Graph capture (Ctx::capturing): whether solve_graph can be recorded into a CUDA graph, the buffers it needs
  // (allocated before the capture), and the recorded form of solve, whose decisions are taken on the device.
  // Solvers without host decisions record solve itself.
  virtual bool graphable() const { return false; }
  virtual void prepare_graph(Ctx&) {}
  virtual void solve_graph(Ctx& c, T* X, const T* B, bool zero) { solve(c, X, B, zero); }
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
  TermParams params() const { return TermParams{mode, max_iter, min_iter, tol, reduction}; }
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
// wavefronts of the natural-order block ILU(0) from the host block structure (lptr offsets into order)
void ilu_wavefronts(const Matrix& A, std::vector<int64_t>& lptr, std::vector<int32_t>& order);

// The whole FlexGMRES solve recorded into a CUDA graph (cfg.graph == 2): restart and Arnoldi loops as WHILE nodes,
// the preconditioners' round-robin as IF nodes, every decision on the device (devctl.cuh FgState), the V-cycle
// recorded inline.  Used by the solver handle (one graph per handle) and by batches (one graph for many handles).
struct RecordedSolve {
  virtual ~RecordedSolve() {}
  virtual void prepare(Ctx& c) = 0;                           // buffers and the preconditioners' recorded forms
  virtual void record(Ctx& c, double* X, const double* B) = 0;  // emits the solve into the capture on c.st
  virtual int key() const = 0;                                // changes when the recording must be redone
  virtual void queue_result(Ctx& c, cudaStream_t st) = 0;     // device state -> pinned host memory on st
  virtual void take_result(Ctx& c) = 0;                       // after st synchronised: iterations, history, ...
};
// the recorded form of the tree's top solver, or nullptr (not FlexGMRES, or cfg.graph != 2)
RecordedSolve* recorded_form(Tree& t);
// Generates training residuals with the solver itself (FGMRES Arnoldi vectors of solves with seeded random
// right-hand sides, learned stage off) and trains the learned stage; returns the final mean loss.
double train_learned(Tree& t, int n_rhs, int steps, double lr, uint64_t seed);

}  // namespace bsgpu
