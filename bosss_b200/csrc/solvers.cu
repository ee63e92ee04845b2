// Solver tree of the hot path (see solvers.cuh).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "solvers.cuh"

namespace bsgpu {

// Wavefronts of the natural-order block ILU(0) (CellILU.cs:1229-1330): a block row's wavefront is one more than the
// largest wavefront of its lower neighbours, so the rows of one wavefront depend only on earlier ones.  lptr: offsets
// of the wavefronts in `order` (rows ascending within a wavefront).
void ilu_wavefronts(const Matrix& A, std::vector<int64_t>& lptr, std::vector<int32_t>& order) {
  const int64_t nb = A.nb;
  std::vector<int32_t> lev(nb, 0);
  int nlev = nb ? 1 : 0;
  for (int64_t i = 0; i < nb; ++i) {
    for (int64_t k = A.h_rp[i]; k < A.h_rp[i + 1]; ++k) {
      const int32_t j = A.h_ci[k];
      if (j < i) lev[i] = std::max(lev[i], lev[j] + 1);
    }
    nlev = std::max(nlev, lev[i] + 1);
  }
  lptr.assign(nlev + 1, 0);
  for (int64_t i = 0; i < nb; ++i) lptr[lev[i] + 1]++;
  for (int l = 0; l < nlev; ++l) lptr[l + 1] += lptr[l];
  order.assign(nb, 0);
  std::vector<int64_t> fillp(lptr.begin(), lptr.end() - 1);
  for (int64_t i = 0; i < nb; ++i) order[fillp[lev[i]]++] = (int32_t)i;
}

// ---------------------------------------------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------------------------------------------
Ctx::Ctx() {
  BSGPU_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  dscal.alloc(scal_cap);
  BSGPU_CUDA(cudaMallocHost(&hscal, scal_cap * sizeof(double)));
  dflag.alloc(256);
  BSGPU_CUDA(cudaMemset(dflag.p, 0, 256 * sizeof(int)));
  BSGPU_CUDA(cudaMemset(dscal.p, 0, scal_cap * sizeof(double)));
  red.init();
}
Ctx::~Ctx() {
  if (hscal) cudaFreeHost(hscal);
  if (h_err) cudaFreeHost(h_err);
  for (cudaStream_t b : body_streams) cudaStreamDestroy(b);
  if (st) cudaStreamDestroy(st);
}

namespace {
constexpr int kMaxBodies = 32768;
constexpr int kMaxDepth = 16;
}  // namespace

void Ctx::graph_init() {
  if (h_err) return;
  d_err = flag();
  BSGPU_CUDA(cudaMallocHost(&h_err, sizeof(int)));
  *h_err = 0;
  d_exec.alloc(kMaxBodies);
  BSGPU_CUDA(cudaMemset(d_exec.p, 0, kMaxBodies * sizeof(unsigned int)));
  h_exec.assign(kMaxBodies, 0);
  for (int i = 0; i < kMaxDepth; ++i) {
    cudaStream_t b = nullptr;
    BSGPU_CUDA(cudaStreamCreateWithFlags(&b, cudaStreamNonBlocking));
    body_streams.push_back(b);
  }
}

// Conditional bodies keep their numbers across recordings (every recording appends its own), so that the execution
// counters of a graph recorded earlier stay meaningful; body 0 counts the top level of the current recording.
void Ctx::capture_join() {
  graph_init();
  if (body_kernels.empty()) {
    body_kernels.assign(1, 0);
    body_names.assign(1, "top");
  }
  body_kernels[0] = 0;
  first_body = (int)body_kernels.size();
  body_stack.clear();
  st_stack.clear();
  cur_body = 0;
  capturing = true;
  mark = launches_now();
}

long long Ctx::recorded_total() const {
  long long total = body_kernels[0];
  for (size_t b = (size_t)first_body; b < body_kernels.size(); ++b) total += body_kernels[b];
  return total;
}

long long Ctx::capture_leave() {
  require(st_stack.empty(), "graph capture: unbalanced conditional bodies");
  body_kernels[cur_body] += (long long)(launches_now() - mark);
  capturing = false;
  add_launches(-recorded_total());  // recorded, not launched: replays add what they run
  return body_kernels[0];
}

void Ctx::capture_begin() {
  graph_init();  // allocations before the capture (capture_join finds them made)
  BSGPU_CUDA(cudaStreamSynchronize(st));
  BSGPU_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
  capture_join();
}

long long Ctx::capture_end(cudaGraph_t* g) {
  const long long top = capture_leave();
  BSGPU_CUDA(cudaStreamEndCapture(st, g));
  return top;
}

void Ctx::capture_abort() {
  while (!st_stack.empty()) {
    cudaGraph_t b = nullptr;
    cudaStreamEndCapture(st, &b);
    st = st_stack.back();
    st_stack.pop_back();
  }
  body_kernels[cur_body] += (long long)(launches_now() - mark);
  add_launches(-recorded_total());
  body_stack.clear();
  cur_body = 0;
  capturing = false;
}

int Ctx::new_body(const std::string& name) {
  require(capturing, "conditional body outside a graph capture");
  require((int)body_kernels.size() < kMaxBodies, "graph capture: too many conditional bodies",
          BSGPU_ERR_UNSUPPORTED);
  body_kernels.push_back(0);
  body_names.push_back(name);
  return (int)body_kernels.size() - 1;
}

cudaGraphConditionalHandle Ctx::cond_handle() {
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  BSGPU_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, nullptr, nullptr));
  require(cs == cudaStreamCaptureStatusActive, "conditional handle outside a graph capture");
  cudaGraphConditionalHandle h;
  BSGPU_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
  return h;
}

void Ctx::cond_begin(cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type, int body) {
  require((int)st_stack.size() < kMaxDepth, "graph capture: conditional bodies nested too deeply",
          BSGPU_ERR_UNSUPPORTED);
  cudaStreamCaptureStatus cs;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  BSGPU_CUDA(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &ndeps));
  require(cs == cudaStreamCaptureStatusActive, "conditional node outside a graph capture");
  cudaGraphNodeParams p{};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = type;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  BSGPU_CUDA(cudaGraphAddNode(&node, g, deps, ndeps, &p));
  cudaGraph_t body_graph = p.conditional.phGraph_out[0];
  BSGPU_CUDA(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
  body_kernels[cur_body] += (long long)(launches_now() - mark);
  body_stack.push_back(cur_body);
  cur_body = body;
  st_stack.push_back(st);
  st = body_streams[st_stack.size() - 1];
  BSGPU_CUDA(cudaStreamBeginCaptureToGraph(st, body_graph, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  mark = launches_now();
}

void Ctx::cond_end() {
  require(!st_stack.empty(), "graph capture: no open conditional body");
  body_kernels[cur_body] += (long long)(launches_now() - mark);
  cudaGraph_t g = nullptr;
  BSGPU_CUDA(cudaStreamEndCapture(st, &g));
  st = st_stack.back();
  st_stack.pop_back();
  cur_body = body_stack.back();
  body_stack.pop_back();
  mark = launches_now();
}

void Ctx::check_graph_errors() {
  if (!err_pending) return;
  err_pending = false;
  const int e = *h_err;
  if (e == 0) return;
  *h_err = 0;
  BSGPU_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), st));
  BSGPU_CUDA(cudaStreamSynchronize(st));
  if (e & kDevErrSlots) throw Error(BSGPU_ERR_ARITHMETIC, "Orthonormalization: history slots exhausted");
  if (e & kDevErrKrylovNaN) throw Error(BSGPU_ERR_ARITHMETIC, "FlexGMRES: residual is NaN/Inf");
  if (e & kDevErrResidualIncrease) throw Error(BSGPU_ERR_ARITHMETIC, "Orthonormalization: residual increase");
  throw Error(BSGPU_ERR_ARITHMETIC, "Orthonormalization: NaN/Inf in the preconditioner");
}

void Ctx::flush_graph_counts() {
  if (!graph_ran) return;
  graph_ran = false;
  const size_t nb = body_kernels.size();
  BSGPU_CUDA(cudaMemcpyAsync(h_exec.data(), d_exec.p, nb * sizeof(unsigned int), cudaMemcpyDeviceToHost, st));
  BSGPU_CUDA(cudaMemsetAsync(d_exec.p, 0, nb * sizeof(unsigned int), st));
  BSGPU_CUDA(cudaStreamSynchronize(st));
  long long n = 0;
  for (size_t b = 1; b < nb; ++b) {
    n += body_kernels[b] * (long long)h_exec[b];
    graph_counts[body_names[b]] += h_exec[b];
  }
  add_launches(n);
  check_graph_errors();
}
double* Ctx::scal(int n) {
  require(nscal + n <= scal_cap, "solver tree needs too many device scalars", BSGPU_ERR_UNSUPPORTED);
  double* p = dscal.p + nscal;
  nscal += n;
  return p;
}
int* Ctx::flag() {
  require(nflag < 256, "solver tree needs too many device flags", BSGPU_ERR_UNSUPPORTED);
  return dflag.p + nflag++;
}
void Ctx::fetch(const double* d, int n) {
  require(!capturing, "host read of a device scalar inside a graph capture");
  BSGPU_CUDA(cudaMemcpyAsync(hscal + (d - dscal.p), d, n * sizeof(double), cudaMemcpyDeviceToHost, st));
  BSGPU_CUDA(cudaStreamSynchronize(st));
  check_graph_errors();
}
void Ctx::check_flag(const int* f, const char* what) {
  int h = 0;
  BSGPU_CUDA(cudaMemcpyAsync(&h, f, sizeof(int), cudaMemcpyDeviceToHost, st));
  BSGPU_CUDA(cudaStreamSynchronize(st));
  if (h) {
    BSGPU_CUDA(cudaMemsetAsync(const_cast<int*>(f), 0, sizeof(int), st));
    throw Error(BSGPU_ERR_ARITHMETIC, what);
  }
}

int Ctx::trace_id(const std::string& name) {
  for (size_t i = 0; i < trace.size(); ++i)
    if (trace[i].name == name) return (int)i;
  trace.push_back(TraceEntry{name});
  return (int)trace.size() - 1;
}

static double wall_now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

TraceScope::TraceScope(Ctx& ctx, int id_) : c(ctx), id(id_) {
  if (c.tracing && id >= 0) {
    cudaStreamSynchronize(c.st);
    t0 = wall_now();
  }
}
TraceScope::~TraceScope() {
  if (c.tracing && id >= 0) {
    cudaStreamSynchronize(c.st);
    c.trace[id].seconds += wall_now() - t0;
    c.trace[id].calls += 1;
  }
}

std::pair<bool, bool> Term::operator()(int iter, double R0, double R) const {
  const double eps = 2.2204460492503131e-16 * 1000;  // IterativeSolverConfig.MachineEpsilon
  if (mode == 2) return {iter <= max_iter, true};
  if (mode == 3) {
    if (iter <= 1) return {true, false};
    if (R < R0 * reduction) return {false, true};
    if (iter > max_iter) return {false, false};
    return {true, false};
  }
  if (iter <= min_iter) return {true, false};
  const bool ok = (mode == 0) ? (R < R0 * tol + tol) : (R < R0 * tol);
  if (ok) return {false, true};
  if (iter > max_iter) return {false, false};
  if (R0 < eps || R < eps) return {false, true};
  return {true, false};
}

namespace {

template <typename T>
void copy_vec(T* dst, const T* src, int64_t n, cudaStream_t st) {
  if (n && dst != src) BSGPU_CUDA(cudaMemcpyAsync(dst, src, n * sizeof(T), cudaMemcpyDeviceToDevice, st));
}

int elt_grid(int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 8));
}

// ---------------------------------------------------------------------------------------------------------------
// BlockJacobi (BlockJacobi.cs:68-266).  NoOfIterations = n gives n+1 updates x <- x + omega*Dinv*(b - A*x)
// (the default termination `iter <= NoOfIterations` is tested before each update, :171-173).  Updates are fused
// with the SpMV; the first update from a zero guess is a block-diagonal solve.  The reference's final SpMV,
// whose residual only feeds that count-based test, is not performed.
// ---------------------------------------------------------------------------------------------------------------
template <typename T>
struct BlockJacobiT : Solver<T> {
  bool graphable() const override { return true; }
  const Matrix* A;
  DBuf<T> dinv;
  DBuf<T> tmp;
  int updates;
  T omega;
  BlockJacobiT(Ctx& c, const Matrix* A64, const Matrix* AT, int iters, double om)
      : A(AT), updates(iters + 1), omega((T)om) {
    std::vector<int64_t> o = diag_offsets(*A64);
    dinv.alloc(std::max<int64_t>(o.back(), 1));
    int* err = c.flag();
    if constexpr (sizeof(T) == 8)
      invert_diag_blocks(*A64, dinv.p, nullptr, err, c.st);
    else
      invert_diag_blocks(*A64, nullptr, dinv.p, err, c.st);
    c.check_flag(err, "BlockJacobi: singular diagonal block");
    tmp.alloc(std::max<int64_t>(A->N, 1));
    c.tune(*A, 1, dinv.p);
    c.tune(*A, 0);
  }
  void solve(Ctx& c, T* X, const T* B, bool zero) override {
    TraceScope ts(c, this->trace);
    const int n = updates;
    const T* src = X;
    for (int s = 0; s < n; ++s) {
      T* dst = ((n - 1 - s) % 2 == 0) ? X : tmp.p;
      if (s == 0 && zero) {
        blockdiag_apply(*A, dinv.p, omega, B, dst, c.st);
      } else {
        if (s == 0 && dst == X) {
          copy_vec(tmp.p, X, A->N, c.st);
          src = tmp.p;
        }
        bj_update(*A, dinv.p, omega, src, B, dst, c.st);
      }
      src = dst;
    }
    this->converged = true;
  }
};

// Symmetric multicolour block Gauss-Seidel: per sweep the colours of a greedy colouring of the cell graph are
// relaxed forwards and then backwards with in-place block updates x_i += omega*D_i^-1*(b - A x)_i.  A stronger
// smoother than block Jacobi at the same memory traffic per sweep; the GPU form of the cell-wise ILU/GS
// smoothing BoSSS uses on its low p-levels (CellILU, PmgConfig.cs:124-141).
template <typename T>
struct BlockGST : Solver<T> {
  bool graphable() const override { return true; }
  const Matrix* A;
  DBuf<T> dinv;
  std::vector<DBuf<int32_t>> rows;
  std::vector<int64_t> counts;
  int sweeps;
  T omega;
  BlockGST(Ctx& c, const Matrix* A64, const Matrix* AT, int sweeps_, double om)
      : A(AT), sweeps(std::max(1, sweeps_)), omega((T)om) {
    std::vector<int64_t> o = diag_offsets(*A64);
    dinv.alloc(std::max<int64_t>(o.back(), 1));
    int* err = c.flag();
    if constexpr (sizeof(T) == 8)
      invert_diag_blocks(*A64, dinv.p, nullptr, err, c.st);
    else
      invert_diag_blocks(*A64, nullptr, dinv.p, err, c.st);
    c.check_flag(err, "block Gauss-Seidel: singular diagonal block");
    for (auto& l : greedy_colouring(*A64)) {
      rows.emplace_back(std::max<size_t>(l.size(), 1));
      counts.push_back((int64_t)l.size());
      BSGPU_CUDA(cudaMemcpy(rows.back().p, l.data(), l.size() * 4, cudaMemcpyHostToDevice));
    }
  }
  void solve(Ctx& c, T* X, const T* B, bool zero) override {
    TraceScope ts(c, this->trace);
    if (zero) fill(T(0), X, A->N, c.st);
    const int nc = (int)rows.size();
    for (int s = 0; s < sweeps; ++s) {
      for (int k = 0; k < nc; ++k) gs_update_rows(*A, dinv.p, omega, rows[k].p, counts[k], B, X, c.st);
      for (int k = nc - 1; k >= 0; --k) gs_update_rows(*A, dinv.p, omega, rows[k].p, counts[k], B, X, c.st);
    }
    this->converged = true;
  }
};

// Block ILU(0) smoother (CellILU, CellILU.cs:22; factorisation :1229-1330, Solve :182-250 with the
// single-precision back substitution of BackSubs_Optimized_SinglePrec :914).  The reference factors the cells in
// their natural order, a chain of dependencies as long as the grid is wide; here the cells are ordered by the two
// colours of the block graph (faces of a Cartesian or cut-cell grid: parity of the cell index), which makes the
// factorisation one launch and x = U^{-1} L^{-1} b two block Gauss-Seidel-type launches over the colours:
//   x <- b;  x_b <- U_bb^{-1} (b_b - sum_r L_br x_r)  (colour 1);  x_r <- A_rr^{-1} (b_r - sum_b A_rb x_b)  (colour 0)
// (with M_ii = U_ii the in-place update x_i + U_ii^{-1}(b_i - sum_j M_ij x_j) is exactly that).  Factors in FP32
// for the mixed-precision preconditioner.
template <typename T>
struct ILU0T : Solver<T> {
  bool graphable() const override { return true; }
  std::unique_ptr<Matrix> M64, M32;
  const Matrix* M = nullptr;
  DBuf<T> uinv;
  DBuf<int32_t> rows[2];
  int64_t cnt[2] = {0, 0};
  ILU0T(Ctx& c, const Matrix* A64) {
    require(A64->uniform && (A64->Np == 4 || A64->Np == 6 || A64->Np == 10 || A64->Np == 20),
            "ILU smoother needs uniform blocks of 4, 6, 10 or 20", BSGPU_ERR_UNSUPPORTED);
    auto cols = greedy_colouring(*A64);
    require(cols.size() <= 2, "ILU smoother needs a two-colour block graph (" + std::to_string(cols.size()) +
                                  " colours)", BSGPU_ERR_UNSUPPORTED);
    for (size_t k = 0; k < cols.size(); ++k) {
      cnt[k] = (int64_t)cols[k].size();
      rows[k].alloc(std::max<int64_t>(cnt[k], 1));
      if (cnt[k]) BSGPU_CUDA(cudaMemcpy(rows[k].p, cols[k].data(), cnt[k] * 4, cudaMemcpyHostToDevice));
    }
    std::vector<int64_t> o = diag_offsets(*A64);
    DBuf<double> dinv(std::max<int64_t>(o.back(), 1));
    int* err = c.flag();
    invert_diag_blocks(*A64, dinv.p, nullptr, err, c.st);
    c.check_flag(err, "ILU: singular diagonal block");
    M64.reset(matrix_like(*A64, false));
    err = c.flag();
    ilu0_two_colour(*A64, dinv.p, rows[1].p, cnt[1], *M64, err, c.st);
    c.check_flag(err, "ILU: block pattern is not structurally symmetric");
    uinv.alloc(std::max<int64_t>(o.back(), 1));
    err = c.flag();
    if constexpr (sizeof(T) == 8)
      invert_diag_blocks(*M64, uinv.p, nullptr, err, c.st);
    else
      invert_diag_blocks(*M64, nullptr, uinv.p, err, c.st);
    c.check_flag(err, "ILU: singular pivot block");
    if constexpr (sizeof(T) == 4) {
      M32.reset(matrix_to_single(*M64, c.st));
      BSGPU_CUDA(cudaStreamSynchronize(c.st));
      M64.reset();
      M = M32.get();
    } else {
      M = M64.get();
    }
  }
  void solve(Ctx& c, T* X, const T* B, bool zero) override {
    (void)zero;  // CellILU overwrites X
    TraceScope ts(c, this->trace);
    copy_vec(X, B, M->N, c.st);
    if (cnt[1]) gs_update_rows(*M, uinv.p, T(1), rows[1].p, cnt[1], B, X, c.st);
    if (cnt[0]) gs_update_rows(*M, uinv.p, T(1), rows[0].p, cnt[0], B, X, c.st);
    this->this_level_iterations++;
    this->converged = true;
  }
};

// Block ILU(0) smoother in the reference's natural cell order (CellILU.cs:22; ComputeILU :1229-1330, Solve
// :182-250).  The dependency chain of the natural order is cut into wavefronts (block rows whose lower neighbours
// all lie in earlier wavefronts; 3n-2 of them on an n^3 Cartesian grid): the factorisation is one launch per
// wavefront (ilu0_levels), and x = U^{-1} L^{-1} b is one launch per wavefront and pass: the forward pass
// y_i = b_i - sum_{k<i} L_ik y_k over the wavefronts in order, the backward pass x_i = U_ii^{-1} (y_i - sum_{j>i}
// U_ij x_j) in reverse order, both as in-place row updates on zero-initialised vectors (rows not yet visited are
// zero, so the full row product only sees the finished neighbours).  Factors computed in FP64, stored and applied
// in FP32 for the mixed-precision preconditioner (the reference's single-precision back substitution,
// CellILU.cs:914).
template <typename T>
struct ILUNaturalT : Solver<T> {
  bool graphable() const override { return true; }
  std::unique_ptr<Matrix> M64, M32;
  const Matrix* M = nullptr;
  DBuf<double> uinv64;
  DBuf<float> uinv32;
  DBuf<int32_t> rows;
  std::vector<int64_t> lptr;
  DBuf<T> y;
  ILUNaturalT(Ctx& c, const Matrix* A64) {
    require(A64->uniform && (A64->Np == 4 || A64->Np == 6 || A64->Np == 10 || A64->Np == 20),
            "natural-order ILU needs uniform blocks of 4, 6, 10 or 20", BSGPU_ERR_UNSUPPORTED);
    const int64_t nb = A64->nb;
    std::vector<int32_t> order;
    ilu_wavefronts(*A64, lptr, order);
    rows.alloc(std::max<int64_t>(nb, 1));
    if (nb) BSGPU_CUDA(cudaMemcpy(rows.p, order.data(), nb * 4, cudaMemcpyHostToDevice));
    const std::vector<int64_t> o = diag_offsets(*A64);
    uinv64.alloc(std::max<int64_t>(o.back(), 1));
    if constexpr (sizeof(T) == 4) uinv32.alloc(std::max<int64_t>(o.back(), 1));
    M64.reset(matrix_like(*A64, false));
    int* err = c.flag();
    ilu0_levels(*A64, rows.p, lptr, *M64, uinv64.p, sizeof(T) == 4 ? uinv32.p : nullptr, err, c.st);
    c.check_flag(err, "ILU: singular pivot block");
    if constexpr (sizeof(T) == 4) {
      M32.reset(matrix_to_single(*M64, c.st));
      BSGPU_CUDA(cudaStreamSynchronize(c.st));
      M64.reset();
      uinv64.release();
      M = M32.get();
    } else {
      M = M64.get();
    }
    y.alloc(std::max<int64_t>(M->N, 1));
  }
  const T* uinv() const {
    if constexpr (sizeof(T) == 4)
      return uinv32.p;
    else
      return uinv64.p;
  }
  int wavefronts() const { return (int)lptr.size() - 1; }
  void solve(Ctx& c, T* X, const T* B, bool zero) override {
    (void)zero;  // CellILU overwrites X
    TraceScope ts(c, this->trace);
    const int L = wavefronts();
    fill(T(0), y.p, M->N, c.st);
    for (int l = 0; l < L; ++l) unit_update_rows(*M, rows.p + lptr[l], lptr[l + 1] - lptr[l], B, y.p, c.st);
    fill(T(0), X, M->N, c.st);
    for (int l = L - 1; l >= 0; --l)
      gs_update_rows(*M, uinv(), T(1), rows.p + lptr[l], lptr[l + 1] - lptr[l], y.p, X, c.st);
    this->this_level_iterations++;
    this->converged = true;
  }
};

// Additive Schwarz smoother (Schwarz.cs:56; Init :623-840, Solve :996-1147) in restricted form with one
// overlapping block per cell (schwarz_factor in blockops.cu): x <- x + M (b - A x), M holding the centre rows of
// the block inverses, stored in FP32 for the mixed-precision preconditioner.  bj_iters + 1 updates per call, as
// for BlockJacobi.
template <typename T>
struct SchwarzT : Solver<T> {
  bool graphable() const override { return true; }
  const Matrix* A;
  std::unique_ptr<Matrix> M;
  DBuf<T> r;
  int updates;
  SchwarzT(Ctx& c, const Matrix* A64, const Matrix* AT, int iters) : A(AT), updates(iters + 1) {
    M.reset(matrix_like(*A64, sizeof(T) == 4));
    int* err = c.flag();
    schwarz_factor(*A64, *M, err, c.st);
    c.check_flag(err, "Schwarz: singular block");
    r.alloc(std::max<int64_t>(A->N, 1));
    c.tune(*A, 0);
    c.tune(*M, 0);
  }
  void solve(Ctx& c, T* X, const T* B, bool zero) override {
    TraceScope ts(c, this->trace);
    for (int s = 0; s < updates; ++s) {
      if (s == 0 && zero) {
        spmv(*M, T(1), B, T(0), (const T*)nullptr, X, c.st);
      } else {
        spmv(*A, T(-1), X, T(1), B, r.p, c.st);
        spmv(*M, T(1), r.p, T(1), X, X, c.st);
      }
    }
    this->converged = true;
  }
};

// Additive Schwarz with multi-cell blocks (Schwarz.cs:56; blocking :190-320, overlap :690-735, Solve :996-1147):
// per update r = b - A x (skipped from a zero guess, as the reference skips the product for X = 0), x += sum over
// the blocks of R_b^T A_b^{-1} R_b r, then x *= 1/multiplicity with overlap scaling.  Blocks from
// schwarz_partition (parts blocks; 0: blocks of 8 cells) grown by `overlap` layers; inverses FP32 in the mixed
// preconditioner.  bj_iters + 1 updates per call (FixedNoOfIterations), as for the one-cell-patch form.
template <typename T>
struct BlockSchwarzT : Solver<T> {
  bool graphable() const override { return true; }
  const Matrix* A;
  std::unique_ptr<SchwarzBlocks> S;
  DBuf<T> r;
  int updates;
  bool scaling;
  BlockSchwarzT(Ctx& c, const Matrix* A64, const Matrix* AT, int iters, int64_t parts, int overlap, bool scale)
      : A(AT), updates(iters + 1), scaling(scale && overlap > 0) {
    auto blocks = schwarz_partition(*A64, parts > 0 ? parts : std::max<int64_t>(1, (A64->nb + 7) / 8));
    schwarz_extend(*A64, blocks, overlap);
    int* err = c.flag();
    S.reset(schwarz_blocks_setup(*A64, blocks, scaling, sizeof(T) == 4, err, c.st));
    c.check_flag(err, "Schwarz: singular block");
    r.alloc(std::max<int64_t>(A->N, 1));
  }
  void solve(Ctx& c, T* X, const T* B, bool zero) override {
    TraceScope ts(c, this->trace);
    if (zero) fill(T(0), X, A->N, c.st);
    for (int s = 0; s < updates; ++s) {
      if (s == 0 && zero)
        copy_vec(r.p, B, A->N, c.st);
      else
        spmv(*A, T(-1), X, T(1), B, r.p, c.st);
      schwarz_blocks_add(*S, r.p, X, c.st);
      if (scaling) schwarz_blocks_scale(*S, X, c.st);
    }
    this->converged = true;
  }
};

// ---------------------------------------------------------------------------------------------------------------
// PCG with a block-diagonal preconditioner (SoftPCG.cs:113-194; also the coarsest-level solve).  The iteration
// runs on device scalars; its kernels are predicated on a device flag that the convergence test clears, so the
// host launches batches of iterations and reads the state once per batch (the iterate equals that of a test
// after every iteration).
// scalars: s[0] rz, s[1] pq, s[2] rz_new, s[3] rr, s[4] rr0, s[5] iterations, s[6] beta, s[7] alpha
// ---------------------------------------------------------------------------------------------------------------
__global__ void pcg_alpha_kernel(double* s, const int* active) {
  if (*active == 0) return;
  s[7] = s[0] / s[1];
}

__global__ void pcg_beta_kernel(double* s, int* active, int mode, double tol, int max_iter, int min_iter) {
  if (*active == 0) return;
  pcg_beta_step(s, active, mode, tol, max_iter, min_iter);
}

template <typename T>
__global__ void xpby_kernel(const T* __restrict__ z, const double* __restrict__ beta, T* __restrict__ p, int64_t n,
                            const int* __restrict__ active) {
  if (*active == 0) return;
  const double b = *beta;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = (T)((double)z[i] + b * (double)p[i]);
}

__global__ void pcg_init_kernel(double* s, int* active) {
  s[0] = s[2];  // rz
  s[4] = s[3];  // rr0
  s[5] = 0.0;
  *active = 1;
}

template <typename T>
struct PCGT : Solver<T> {
  const Matrix* A;
  DBuf<T> dinv;
  DBuf<T> r, z, p, q;
  double* s;
  int* active;
  Term term;
  int batch = 8;
  bool precond;
  bool use_graph = true;
  cudaGraphExec_t graph_exec = nullptr;
  const T* graph_X = nullptr;
  long graph_kernels = 0;  // kernels per captured batch (counted at capture time)
  ~PCGT() override {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
  }
  void launches_in_graph(Ctx&) { add_launches(graph_kernels); }  // kernels of one replayed batch
  PCGT(Ctx& c, const Matrix* A64, const Matrix* AT, bool use_pc, Term t) : A(AT), term(t), precond(use_pc) {
    const int64_t N = std::max<int64_t>(A->N, 1);
    r.alloc(N); z.alloc(N); p.alloc(N); q.alloc(N);
    s = c.scal(8);
    active = c.flag();
    if (precond) {
      std::vector<int64_t> o = diag_offsets(*A64);
      dinv.alloc(std::max<int64_t>(o.back(), 1));
      int* err = c.flag();
      if constexpr (sizeof(T) == 8)
        invert_diag_blocks(*A64, dinv.p, nullptr, err, c.st);
      else
        invert_diag_blocks(*A64, nullptr, dinv.p, err, c.st);
      c.check_flag(err, "PCG: singular diagonal block");
    }
    c.tune(*A, 0);
  }
  void apply_pc(Ctx& c, const T* in, T* out, const int* act) {
    if (precond)
      blockdiag_apply(*A, dinv.p, T(1), in, out, c.st, act);
    else
      copy_vec(out, in, A->N, c.st);
  }
  void solve(Ctx& c, T* X, const T* B, bool zero) override {
    TraceScope ts(c, this->trace);
    const int64_t N = A->N;
    cudaStream_t st = c.st;
    if (zero)
      copy_vec(r.p, B, N, st);
    else
      spmv(*A, T(-1), X, T(1), B, r.p, st);
    apply_pc(c, r.p, z.p, nullptr);
    copy_vec(p.p, z.p, N, st);
    {
      const T* a[2] = {r.p, r.p};
      const T* b[2] = {z.p, r.p};
      dots(c.red, 2, a, b, N, s + 2, 0, st);
    }
    pcg_init_kernel<<<1, 1, 0, st>>>(s, active);
    BSGPU_CHECK_LAUNCH();
    c.fetch(s, 8);
    const double* hs = c.hscal + (s - c.dscal.p);
    const double R0 = std::sqrt(hs[4]);
    this->history.assign(1, R0);
    auto st0 = term(0, R0, R0);
    int it = 0;
    double R = R0;
    if (!std::isfinite(R0)) throw Error(BSGPU_ERR_ARITHMETIC, "PCG: NaN/Inf in the initial residual");
    if (st0.first) {
      const int grid = elt_grid(N);
      const bool fused = precond && A->uniform && A->nb > 0 &&
                         (A->Np == 4 || A->Np == 6 || A->Np == 10 || A->Np == 20);
      const T* px[1] = {p.p};
      const T* qx[1] = {q.p};
      auto batch_kernels = [&]() {
        for (int bi = 0; bi < batch; ++bi) {
          spmv(*A, T(1), p.p, T(0), (const T*)nullptr, q.p, st, active);
          dots(c.red, 1, px, qx, N, s + 1, 0, st, active);
          if (fused) {
            // alpha, x and r updates, z = Dinv r, r.z, r.r and the beta / termination step in one launch
            pcg_update(c.red, A->Np, s, active, X, p.p, q.p, r.p, z.p, dinv.p, A->nb, term.mode, term.tol,
                       term.max_iter, term.min_iter, st);
            xpby_kernel<T><<<grid, 256, 0, st>>>(z.p, s + 6, p.p, N, active);
            BSGPU_CHECK_LAUNCH();
            continue;
          }
          pcg_alpha_kernel<<<1, 1, 0, st>>>(s, active);
          BSGPU_CHECK_LAUNCH();
          axpys(1, s + 7, nullptr, 1.0, px, X, N, st, active);
          axpys(1, s + 7, nullptr, -1.0, qx, r.p, N, st, active);
          apply_pc(c, r.p, z.p, active);
          {
            const T* a[2] = {r.p, r.p};
            const T* b[2] = {z.p, r.p};
            dots(c.red, 2, a, b, N, s + 2, 0, st, active);
          }
          pcg_beta_kernel<<<1, 1, 0, st>>>(s, active, term.mode, term.tol, term.max_iter, term.min_iter);
          xpby_kernel<T><<<grid, 256, 0, st>>>(z.p, s + 6, p.p, N, active);
          BSGPU_CHECK_LAUNCH();
        }
      };
      // the batch is captured once per solution vector and replayed as one CUDA graph launch (its kernels,
      // predicated on `active`, become no-ops once converged)
      if (use_graph && (graph_exec == nullptr || graph_X != X)) {
        if (graph_exec) cudaGraphExecDestroy(graph_exec);
        graph_exec = nullptr;
        cudaGraph_t g = nullptr;
        BSGPU_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        try {
          const unsigned long long n0 = launches_now();
          batch_kernels();
          graph_kernels = (long)(launches_now() - n0);
          add_launches(-(long long)graph_kernels);
        } catch (...) {
          cudaStreamEndCapture(st, &g);
          if (g) cudaGraphDestroy(g);
          throw;
        }
        BSGPU_CUDA(cudaStreamEndCapture(st, &g));
        BSGPU_CUDA(cudaGraphInstantiate(&graph_exec, g, 0));
        cudaGraphDestroy(g);
        graph_X = X;
      }
      while (true) {
        if (use_graph) {
          BSGPU_CUDA(cudaGraphLaunch(graph_exec, st));
          launches_in_graph(c);
        } else {
          batch_kernels();
        }
        int h_active = 0;
        BSGPU_CUDA(cudaMemcpyAsync(&h_active, active, sizeof(int), cudaMemcpyDeviceToHost, st));
        c.fetch(s, 8);
        it = (int)hs[5];
        R = std::sqrt(hs[3]);
        this->history.push_back(R);
        if (!std::isfinite(hs[3]) || !std::isfinite(hs[2])) throw Error(BSGPU_ERR_ARITHMETIC, "PCG: NaN/Inf");
        if (!h_active) break;
      }
      auto fin = term(it, R0, R);
      this->converged = fin.second;
    } else {
      this->converged = st0.second;
    }
    this->this_level_iterations = it;
    if (c.tracing && this->trace >= 0) c.trace[this->trace].iterations += it;
  }
  bool graphable() const override { return term.max_iter <= kMaxRecordedIterations && term.min_iter <= term.max_iter; }
  // Recorded form: the initialisation, then a WHILE node whose body is one CG iteration; the fused update's
  // termination step clears `active` (at the latest when the iteration count passes max_iter), which ends the loop.
  void solve_graph(Ctx& c, T* X, const T* B, bool zero) override {
    require(graphable(), "coarse CG: iteration limits cannot be recorded");
    const int64_t N = A->N;
    if (zero)
      copy_vec(r.p, B, N, c.st);
    else
      spmv(*A, T(-1), X, T(1), B, r.p, c.st);
    apply_pc(c, r.p, z.p, nullptr);
    copy_vec(p.p, z.p, N, c.st);
    {
      const T* a[2] = {r.p, r.p};
      const T* b[2] = {z.p, r.p};
      dots(c.red, 2, a, b, N, s + 2, 0, c.st);
    }
    pcg_init_kernel<<<1, 1, 0, c.st>>>(s, active);
    BSGPU_CHECK_LAUNCH();
    const cudaGraphConditionalHandle h = c.cond_handle();
    const int body = c.new_body((this->trace >= 0 ? c.trace[this->trace].name + ": " : std::string()) + "CG iteration");
    cond_set(h, active, nullptr, nullptr, 0, c.exec_of(body), c.st);
    c.cond_begin(h, cudaGraphCondTypeWhile, body);
    iteration_kernels(c, X);
    cond_set(h, active, nullptr, nullptr, 0, c.exec_of(body), c.st);
    c.cond_end();
  }
  // one CG iteration on c.st, every kernel predicated on `active`
  void iteration_kernels(Ctx& c, T* X) {
    const int64_t N = A->N;
    const int grid = elt_grid(N);
    const bool fused = precond && A->uniform && A->nb > 0 && (A->Np == 4 || A->Np == 6 || A->Np == 10 || A->Np == 20);
    const T* px[1] = {p.p};
    const T* qx[1] = {q.p};
    spmv(*A, T(1), p.p, T(0), (const T*)nullptr, q.p, c.st, active);
    dots(c.red, 1, px, qx, N, s + 1, 0, c.st, active);
    if (fused) {
      pcg_update(c.red, A->Np, s, active, X, p.p, q.p, r.p, z.p, dinv.p, A->nb, term.mode, term.tol, term.max_iter,
                 term.min_iter, c.st);
    } else {
      pcg_alpha_kernel<<<1, 1, 0, c.st>>>(s, active);
      BSGPU_CHECK_LAUNCH();
      axpys(1, s + 7, nullptr, 1.0, px, X, N, c.st, active);
      axpys(1, s + 7, nullptr, -1.0, qx, r.p, N, c.st, active);
      apply_pc(c, r.p, z.p, active);
      const T* a[2] = {r.p, r.p};
      const T* b[2] = {z.p, r.p};
      dots(c.red, 2, a, b, N, s + 2, 0, c.st, active);
      pcg_beta_kernel<<<1, 1, 0, c.st>>>(s, active, term.mode, term.tol, term.max_iter, term.min_iter);
      BSGPU_CHECK_LAUNCH();
    }
    xpby_kernel<T><<<grid, 256, 0, c.st>>>(z.p, s + 6, p.p, N, active);
    BSGPU_CHECK_LAUNCH();
  }
};

// ---------------------------------------------------------------------------------------------------------------
// CoreOrthonormalizationProcedure (OrthonormalizationMultigrid.cs:58-445).
// AddSol A-orthonormalises a new correction against the history.  The reference uses modified Gram-Schmidt;
// here the projections of one sweep are computed together (classical Gram-Schmidt: one multi-dot launch, one
// multi-axpy launch per vector set) and repeated once when the norm drops below 1/2 ("twice is enough"), which
// restores the orthogonality MGS provides.  The reference's cancellation branch (norm <= 1e-5, up to 10
// re-orthonormalisation sweeps, random restart) is kept as is.
// MinimizeResidual uses RecalcResiPeriod = 1: the residual is recomputed from scratch after each update.
// ---------------------------------------------------------------------------------------------------------------
template <typename T>
struct OrthoT {
  const Matrix* A;
  int64_t N;
  std::vector<DBuf<T>> Sol, Mxx;
  int k = 0;
  int cap = 96;
  double* d_proj;   // [0] |M| after a projection sweep, [1] |M|^2 before it, [2..] projection coefficients
  double* d_beta;   // = d_proj + 2
  double* d_norm;   // [2]
  double* d_alpha;  // [1]
  bool cancellation = false;
  OrthoT(Ctx& c, const Matrix* A_) : A(A_), N(A_->N) {
    d_proj = c.scal(kMaxDots + 2);
    d_beta = d_proj + 2;
    d_norm = c.scal(2);
    d_alpha = c.scal(1);
  }
  int recalc_period = 1;        // RecalcResiPeriod (OrthonormalizationMultigrid.cs:211)
  bool used_more_cycles = false;  // m_UsedMoreThanOneOrthoCycle: the last AddSol needed more than one sweep
  void clear() { k = 0; }
  bool full() const { return k >= cap; }
  T* next_sol(Ctx& c) {
    if ((int)Sol.size() <= k) {
      Sol.emplace_back(std::max<int64_t>(N, 1));
      Mxx.emplace_back(std::max<int64_t>(N, 1));
    }
    fill(T(0), Sol[k].p, N, c.st);
    return Sol[k].p;
  }
  double norm(Ctx& c, const T* v) {
    const T* a[1] = {v};
    dots(c.red, 1, a, a, N, d_norm, 1, c.st);
    return c.get(d_norm);
  }
  // One classical Gram-Schmidt sweep of (X, M) against the history, launched without a host round trip:
  // d_proj[0] = |M| after the sweep and, with `self`, d_proj[1] = |M|^2 before it (one more product in the
  // first multi-dot launch).  History chunks of kMaxDots - 1 vectors; later chunks project the already-updated M
  // (block MGS).
  void cgs_launch(Ctx& c, T* X, T* M, bool self) {
    const int chunk = kMaxDots - 1;
    for (int i0 = 0; i0 < k; i0 += chunk) {
      const int kc = std::min(chunk, k - i0);
      const bool withself = self && i0 == 0;
      const T* a[kMaxDots];
      const T* b[kMaxDots];
      int K = 0;
      if (withself) {
        a[K] = M;
        b[K++] = M;
      }
      for (int i = 0; i < kc; ++i) {
        a[K] = Mxx[i0 + i].p;
        b[K++] = M;
      }
      dots(c.red, K, a, b, N, withself ? d_proj + 1 : d_beta, 0, c.st);
      const T* sx[kMaxDots];
      const T* mx[kMaxDots];
      for (int i = 0; i < kc; ++i) {
        sx[i] = Sol[i0 + i].p;
        mx[i] = Mxx[i0 + i].p;
      }
      axpys2(kc, d_beta, -1.0, sx, X, mx, M, N, c.st);
    }
    const T* a[1] = {M};
    dots(c.red, 1, a, a, N, d_proj, 1, c.st);
  }
  void random_restart(Ctx& c, T* X, T* M) {
    fill_random(X, N, c.seed++, c.st);
    spmv(*A, T(1), X, T(0), (const T*)nullptr, M, c.st);
    const double nm = norm(c, M);
    if (nm == 0 || !std::isfinite(nm))
      throw Error(BSGPU_ERR_ARITHMETIC, "Orthonormalization: breakdown with a random vector");
  }
  // AddSol: Sol[k] holds the new correction; computes Mxx[k] = A Sol[k], A-orthonormalises both against the
  // history and appends.  The normalisation by |M| that the reference applies before the projection
  // (OrthonormalizationMultigrid.cs:263-337) is folded into the final scaling (the projection is linear), so the
  // common case costs one SpMV, one multi-dot, one dual multi-axpy, one norm, one scaling and one host round trip.
  void add_sol(Ctx& c) {
    T* X = Sol[k].p;
    T* M = Mxx[k].p;
    spmv(*A, T(1), X, T(0), (const T*)nullptr, M, c.st);
    if (k > 0) {
      cgs_launch(c, X, M, true);
      c.fetch(d_proj, 2);
      const double nA = c.hscal[d_proj - c.dscal.p];
      const double nM = std::sqrt(c.hscal[d_proj + 1 - c.dscal.p]);
      if (!std::isfinite(nM)) throw Error(BSGPU_ERR_ARITHMETIC, "Orthonormalization: norm of matrix*solution is NaN/Inf");
      if (nM > 0) {
        double rel = nA / nM;
        if (rel > 1e-5 && rel < 0.5) {
          cgs_launch(c, X, M, false);
          rel = c.get(d_proj) / nM;
        }
        if (rel > 1e-5) {
          scale_inv2(d_proj, X, M, N, nullptr, c.st);
          cancellation = false;
          used_more_cycles = false;
          ++k;
          return;
        }
        // cancellation: continue in the reference's order from the state it would have (normalised by |M|)
        axpby(T(1.0 / nM), M, T(0), M, N, c.st);
        axpby(T(1.0 / nM), X, T(0), X, N, c.st);
        add_sol_tail(c, X, M, rel);
        return;
      }
      // X == 0: random restart below (M is zero as well)
    }
    double nM = norm(c, M);
    if (!std::isfinite(nM)) throw Error(BSGPU_ERR_ARITHMETIC, "Orthonormalization: norm of matrix*solution is NaN/Inf");
    if (nM == 0) {
      random_restart(c, X, M);
      nM = c.hscal[d_norm - c.dscal.p];
    }
    axpby(T(1.0 / nM), M, T(0), M, N, c.st);
    axpby(T(1.0 / nM), X, T(0), X, N, c.st);
    add_sol_tail(c, X, M, -1.0);
  }
  // the re-orthonormalisation loop of AddSol on normalised (X, M); nn0 >= 0: result of the first sweep
  void add_sol_tail(Ctx& c, T* X, T* M, double nn0) {
    const int MaxOrtho = 10;
    bool canc = false;
    for (int jj = 0; jj <= MaxOrtho; ++jj) {
      double nn;
      if (jj == 0 && nn0 >= 0) {
        nn = nn0;
      } else {
        nn = 1.0;
        if (k > 0) {
          cgs_launch(c, X, M, false);
          nn = c.get(d_proj);
          if (nn > 1e-5 && nn < 0.5) {
            cgs_launch(c, X, M, false);
            nn = c.get(d_proj);
          }
        }
      }
      if (nn <= 1e-5) {
        canc = true;
        if (jj < MaxOrtho) {
          const double Xn = norm(c, X);
          if (Xn < 1e-200 || jj == MaxOrtho - 1) {
            random_restart(c, X, M);
          } else {
            axpby(T(1.0 / Xn), X, T(0), X, N, c.st);
            spmv(*A, T(1), X, T(0), (const T*)nullptr, M, c.st);
            if (norm(c, M) == 0) random_restart(c, X, M);
          }
          axpby(T(1.0 / nn), M, T(0), M, N, c.st);
          axpby(T(1.0 / nn), X, T(0), X, N, c.st);
        } else {
          throw Error(BSGPU_ERR_ARITHMETIC, "Orthonormalization: numerical breakdown");
        }
      } else {
        if (nn != 1.0) {
          axpby(T(1.0 / nn), M, T(0), M, N, c.st);
          axpby(T(1.0 / nn), X, T(0), X, N, c.st);
        }
        break;
      }
    }
    cancellation = canc;
    used_more_cycles = canc;
    ++k;
  }
  // MinimizeResidual: X += alpha*Sol[k-1], alpha = <Mxx[k-1], Res0>; Res = B - A*X; returns |Res|.
  // With RecalcResiPeriod > 1 the residual is updated as Res -= alpha Mxx[k-1] and recomputed from scratch only
  // when the history length is a multiple of the period or after a re-orthonormalisation
  // (OrthonormalizationMultigrid.cs:171-190).
  double minimize(Ctx& c, T* X, const T* B, const T* Res0, T* Res, double oldN) {
    const int i = k - 1;
    const T* a[1] = {Mxx[i].p};
    const T* b[1] = {Res0};
    dots(c.red, 1, a, b, N, d_alpha, 0, c.st);
    const T* sx[1] = {Sol[i].p};
    axpys(1, d_alpha, nullptr, 1.0, sx, X, N, c.st);
    if (recalc_period <= 1 || used_more_cycles || k % recalc_period == 0) {
      spmv(*A, T(-1), X, T(1), B, Res, c.st);
    } else {
      const T* mx[1] = {Mxx[i].p};
      axpys(1, d_alpha, nullptr, -1.0, mx, Res, N, c.st);
    }
    const double rn = norm(c, Res);
    if (!std::isfinite(rn)) throw Error(BSGPU_ERR_ARITHMETIC, "Orthonormalization: residual is NaN/Inf");
    const double tol = std::max(std::max(rn, oldN) * 0.2, 1.0e-7);
    if (rn > oldN + tol) throw Error(BSGPU_ERR_ARITHMETIC, "Orthonormalization: residual increase");
    return rn;
  }

  // ---- recorded form (graph capture): the history length lives on the device ----------------------------------
  // A new correction is built in the fixed buffers W (correction) and MW (its image), projected against the
  // history by the device-count kernels, normalised and copied into history slot k; MinimizeResidual then uses
  // W and MW.  A correction with nothing independent of the history left is stored as zero (devctl.cu).
  int nslots = 0;
  DBuf<T> W, MW;
  DBuf<T*> d_sol, d_mxx;
  DBuf<OrthoState> state;
  HistScratch hs;
  double* d_hbeta = nullptr;  // projection coefficients of the recorded form [nslots]
  double* d_rn = nullptr;     // residual norm after MinimizeResidual
  OrthoState* dev() { return state.p; }
  std::string tag;  // owner's trace name, for the graph statistics
  void prepare_dev(Ctx& c, int slots) {
    slots = std::max(1, std::min(slots, cap));
    require(slots <= kHistMax, "recorded OrthoMG: history longer than 128", BSGPU_ERR_UNSUPPORTED);
    if (nslots >= slots) return;
    W.alloc(std::max<int64_t>(N, 1));
    MW.alloc(std::max<int64_t>(N, 1));
    while ((int)Sol.size() < slots) {
      Sol.emplace_back(std::max<int64_t>(N, 1));
      Mxx.emplace_back(std::max<int64_t>(N, 1));
    }
    std::vector<T*> ps(slots), pm(slots);
    for (int j = 0; j < slots; ++j) {
      ps[j] = Sol[j].p;
      pm[j] = Mxx[j].p;
    }
    d_sol.alloc(slots);
    d_mxx.alloc(slots);
    BSGPU_CUDA(cudaMemcpy(d_sol.p, ps.data(), slots * sizeof(T*), cudaMemcpyHostToDevice));
    BSGPU_CUDA(cudaMemcpy(d_mxx.p, pm.data(), slots * sizeof(T*), cudaMemcpyHostToDevice));
    if (!state.p) {
      state.alloc(1);
      BSGPU_CUDA(cudaMemset(state.p, 0, sizeof(OrthoState)));
      d_rn = c.scal(1);
    }
    hs.init(slots);
    d_hbeta = c.scal(slots);
    nslots = slots;
  }
  T* next_sol_dev(Ctx& c) {
    fill(T(0), W.p, N, c.st);
    return W.p;
  }
  // one projection sweep of (W, MW) against the first k history entries; |MW| after it into d_proj[0] and, with
  // `self`, |MW|^2 before it into d_proj[1]
  void cgs_dev(Ctx& c, bool self) {
    hist_dots(hs, d_mxx.p, &state.p->k, MW.p, N, d_hbeta, self ? d_proj + 1 : nullptr, c.st);
    hist_axpy2(d_sol.p, d_mxx.p, &state.p->k, nslots, d_hbeta, W.p, MW.p, N, c.st);
    const T* a[1] = {MW.p};
    dots(c.red, 1, a, a, N, d_proj, 1, c.st);
  }
  void add_sol_dev(Ctx& c) {
    spmv(*A, T(1), W.p, T(0), (const T*)nullptr, MW.p, c.st);
    cgs_dev(c, true);
    ortho_decide1(state.p, d_proj, c.d_err, c.st);
    const cudaGraphConditionalHandle h = c.cond_handle();
    const int body = c.new_body(tag + "second Gram-Schmidt sweep");
    cond_set(h, &state.p->second, nullptr, nullptr, 0, c.exec_of(body), c.st);
    c.cond_begin(h, cudaGraphCondTypeIf, body);
    cgs_dev(c, false);
    ortho_decide2(state.p, d_proj, c.st);
    c.cond_end();
    ortho_final(state.p, d_proj, c.st);
    ortho_store(state.p, W.p, MW.p, d_sol.p, d_mxx.p, nslots, N, c.d_err, c.st);
    ortho_advance(state.p, recalc_period, nslots, c.st);
  }
  void minimize_dev(Ctx& c, T* X, const T* B, const T* Res0, T* Res, const TermParams& tp) {
    const T* a[1] = {MW.p};
    const T* b[1] = {Res0};
    dots(c.red, 1, a, b, N, d_alpha, 0, c.st);
    const T* sx[1] = {W.p};
    axpys(1, d_alpha, nullptr, 1.0, sx, X, N, c.st);
    spmv(*A, T(-1), X, T(1), B, Res, c.st, &state.p->recalc);
    const T* mx[1] = {MW.p};
    axpys(1, d_alpha, nullptr, -1.0, mx, Res, N, c.st, &state.p->update);
    const T* r[1] = {Res};
    dots(c.red, 1, r, r, N, d_rn, 1, c.st);
    minimize_check(state.p, d_rn, tp, c.d_err, c.st);
  }
};

// ---------------------------------------------------------------------------------------------------------------
// OrthonormalizationMultigrid.Solve (OrthonormalizationMultigrid.cs:797-1104) as configured by PmgConfig
// (PmgConfig.cs:80-245): no pre-smoother, m_omega = 1, coarse correction on the same level through
// GridAndDegRestriction (CoarseOnLowerLevel = false), NoOfPostSmootherSweeps post-smoother calls, each followed
// by orthonormalisation and residual minimisation.
// ---------------------------------------------------------------------------------------------------------------
template <typename T>
struct OrthoMGT : Solver<T> {
  const Matrix* A;
  int64_t N;
  std::unique_ptr<Solver<T>> coarse, post, pre;
  const bool* pre_on = nullptr;  // the pre-smoother runs only while *pre_on (learned stage trained)
  int sweeps = 10;
  Term term;
  OrthoT<T> ortho;
  DBuf<T> Res0, Res;
  OrthoMGT(Ctx& c, const Matrix* A_, Term t) : A(A_), N(A_->N), term(t), ortho(c, A_) {
    Res0.alloc(std::max<int64_t>(N, 1));
    Res.alloc(std::max<int64_t>(N, 1));
  }
  int nested() const override {
    int s = 0;
    if (coarse) s += coarse->this_level_iterations + coarse->nested();
    if (post) s += post->this_level_iterations + post->nested();
    return s;
  }
  void solve(Ctx& c, T* X, const T* B, bool zero) override {
    TraceScope ts(c, this->trace);
    if (zero)
      copy_vec(Res0.p, B, N, c.st);
    else
      spmv(*A, T(-1), X, T(1), B, Res0.p, c.st);
    copy_vec(Res.p, Res0.p, N, c.st);
    const double r0 = ortho.norm(c, Res0.p);
    double rn = r0;
    this->history.assign(1, r0);
    ortho.clear();
    this->converged = false;
    for (int iIter = 1;; ++iIter) {
      auto st = term(iIter, r0, rn);
      if (!st.first) {
        this->converged = st.second;
        break;
      }
      if (ortho.full() ) {
        // history capacity reached: restart the minimisation from the current iterate
        copy_vec(Res0.p, Res.p, N, c.st);
        ortho.clear();
      }
      if (pre && (pre_on == nullptr || *pre_on)) {
        // pre-smoother (OrthonormalizationMultigrid.cs:893-915)
        T* pc = ortho.next_sol(c);
        pre->solve(c, pc, Res.p, true);
        ortho.add_sol(c);
        rn = ortho.minimize(c, X, B, Res0.p, Res.p, rn);
        st = term(iIter, r0, rn);
        if (!st.first) {
          this->converged = st.second;
          break;
        }
      }
      if (coarse) {
        T* vl = ortho.next_sol(c);
        coarse->solve(c, vl, Res.p, true);
        ortho.add_sol(c);
        rn = ortho.minimize(c, X, B, Res0.p, Res.p, rn);
        st = term(iIter, r0, rn);
        if (!st.first) {
          this->converged = st.second;
          break;
        }
      }
      bool termPost = false;
      if (post) {
        for (int g = 0; g < sweeps; ++g) {
          if (ortho.full()) break;
          T* pc = ortho.next_sol(c);
          post->solve(c, pc, Res.p, true);
          ortho.add_sol(c);
          rn = ortho.minimize(c, X, B, Res0.p, Res.p, rn);
          st = term(iIter, r0, rn);
          if (!st.first) {
            this->converged = st.second;
            termPost = true;
            break;
          }
          if (ortho.cancellation) break;
        }
      }
      if (termPost) break;
      this->this_level_iterations++;
      this->history.push_back(rn);
      if (c.tracing && this->trace >= 0) c.trace[this->trace].iterations += 1;
    }
  }

  // ---- recorded form --------------------------------------------------------------------------------------------
  // The loop above with its decisions on the device: iterations in a WHILE node (inline for a fixed single
  // iteration, the p-multigrid preconditioner's top level), each correction after the first of an iteration in an
  // IF node on (level active, no cancellation, history not full).
  bool graphable() const override {
    return (!coarse || coarse->graphable()) && (!post || post->graphable()) && (!pre || pre->graphable()) &&
           ortho.cap <= kHistMax;
  }
  int corrections_per_iteration() const {
    return (coarse ? 1 : 0) + (post ? sweeps : 0) + ((pre && (pre_on == nullptr || *pre_on)) ? 1 : 0);
  }
  void prepare_graph(Ctx& c) override {
    if (this->trace >= 0) ortho.tag = c.trace[this->trace].name + ": ";
    const int per = std::max(1, corrections_per_iteration());
    const long long most = (long long)std::max(1, term.max_iter) * per;
    ortho.prepare_dev(c, (int)std::min<long long>(most, ortho.cap));
    if (coarse) coarse->prepare_graph(c);
    if (post) post->prepare_graph(c);
    if (pre) pre->prepare_graph(c);
  }
  void correction_dev(Ctx& c, Solver<T>* sv, T* X, const T* B, const TermParams& tp) {
    T* w = ortho.next_sol_dev(c);
    sv->solve_graph(c, w, Res.p, true);
    ortho.add_sol_dev(c);
    ortho.minimize_dev(c, X, B, Res0.p, Res.p, tp);
  }
  // a correction recorded inside an IF node on (active && !cancel && k < cap) (post-smoother sweeps) or on
  // `active` alone
  void guarded_correction_dev(Ctx& c, Solver<T>* sv, T* X, const T* B, const TermParams& tp, bool post_sweep,
                              int cap_eff) {
    OrthoState* st = ortho.dev();
    const cudaGraphConditionalHandle h = c.cond_handle();
    const int body = c.new_body((this->trace >= 0 ? c.trace[this->trace].name + ": " : std::string()) + "correction");
    cond_set(h, &st->active, post_sweep ? &st->cancel : nullptr, post_sweep ? &st->k : nullptr, cap_eff,
             c.exec_of(body), c.st);
    c.cond_begin(h, cudaGraphCondTypeIf, body);
    correction_dev(c, sv, X, B, tp);
    c.cond_end();
  }
  void iteration_dev(Ctx& c, T* X, const T* B, const TermParams& tp) {
    OrthoState* st = ortho.dev();
    const int cap_eff = ortho.nslots;
    iter_begin(st, cap_eff, c.st);
    copy_if(Res.p, Res0.p, N, &st->restart, c.st);
    bool first = true;
    auto run = [&](Solver<T>* sv, bool post_sweep) {
      if (first)
        correction_dev(c, sv, X, B, tp);
      else
        guarded_correction_dev(c, sv, X, B, tp, post_sweep, cap_eff);
      first = false;
    };
    if (pre && (pre_on == nullptr || *pre_on)) run(pre.get(), false);
    if (coarse) run(coarse.get(), false);
    if (post)
      for (int g = 0; g < sweeps; ++g) run(post.get(), true);
  }
  void solve_graph(Ctx& c, T* X, const T* B, bool zero) override {
    if (zero)
      copy_vec(Res0.p, B, N, c.st);
    else
      spmv(*A, T(-1), X, T(1), B, Res0.p, c.st);
    copy_vec(Res.p, Res0.p, N, c.st);
    const T* a[1] = {Res0.p};
    dots(c.red, 1, a, a, N, ortho.d_norm, 1, c.st);
    const TermParams tp = term.params();
    OrthoState* st = ortho.dev();
    level_begin(st, ortho.d_norm, tp, c.st);
    if (term.mode == 2 && term.max_iter == 1) {
      iteration_dev(c, X, B, tp);
      iter_end(st, tp, c.st);
      return;
    }
    const cudaGraphConditionalHandle h = c.cond_handle();
    const int body = c.new_body((this->trace >= 0 ? c.trace[this->trace].name + ": " : std::string()) + "iteration");
    cond_set(h, &st->active, nullptr, nullptr, 0, c.exec_of(body), c.st);
    c.cond_begin(h, cudaGraphCondTypeWhile, body);
    iteration_dev(c, X, B, tp);
    iter_end(st, tp, c.st);
    cond_set(h, &st->active, nullptr, nullptr, 0, c.exec_of(body), c.st);
    c.cond_end();
  }
};

// ---------------------------------------------------------------------------------------------------------------
// GridAndDegRestriction.Solve (GridAndDegRestriction.cs:379-439): solve on the leading modes, add back.
// ---------------------------------------------------------------------------------------------------------------
template <typename T>
struct GridAndDegT : Solver<T> {
  const Matrix* A;    // level operator
  const Matrix* sub;  // restricted operator (same precision)
  int keep;
  std::unique_ptr<Solver<T>> lower;
  DBuf<T> xLo, bLo;
  DBuf<int64_t> map;  // sub -> full index (non-uniform blocks only)
  double* d_norm;
  GridAndDegT(Ctx& c, const Matrix* A_, const Matrix* sub_, int keep_) : A(A_), sub(sub_), keep(keep_) {
    xLo.alloc(std::max<int64_t>(sub->N, 1));
    bLo.alloc(std::max<int64_t>(sub->N, 1));
    d_norm = c.scal(1);
    if (!A->uniform) {
      std::vector<int64_t> m(sub->N);
      for (int64_t i = 0; i < A->nb; ++i)
        for (int s = 0; s < A->h_nspc[i]; ++s)
          for (int q = 0; q < keep; ++q) m[sub->h_i0[i] + s * keep + q] = A->h_i0[i] + s * A->Np + q;
      map.alloc(std::max<int64_t>(sub->N, 1));
      if (sub->N) BSGPU_CUDA(cudaMemcpy(map.p, m.data(), sub->N * 8, cudaMemcpyHostToDevice));
    }
  }
  int nested() const override { return lower ? lower->this_level_iterations + lower->nested() : 0; }
  void solve(Ctx& c, T* X, const T* B, bool zero) override {
    TraceScope ts(c, this->trace);
    restrict_gather(B, bLo.p, sub->N, A->Np, keep, map.p, c.st);
    const T* a[1] = {bLo.p};
    dots(c.red, 1, a, a, sub->N, d_norm, 1, c.st);
    if (!(c.get(d_norm) > 0)) {
      this->converged = true;
      return;
    }
    if (zero)
      fill(T(0), xLo.p, sub->N, c.st);
    else
      restrict_gather(X, xLo.p, sub->N, A->Np, keep, map.p, c.st);
    lower->solve(c, xLo.p, bLo.p, zero);
    this->converged = lower->converged;
    restrict_scatter_add(xLo.p, X, sub->N, A->Np, keep, map.p, c.st);
  }
  // recorded form: the zero-right-hand-side return becomes an IF node on |b_lo| > 0
  int* nonzero = nullptr;
  bool graphable() const override { return lower && lower->graphable(); }
  void prepare_graph(Ctx& c) override {
    if (!nonzero) nonzero = c.flag();
    lower->prepare_graph(c);
  }
  void solve_graph(Ctx& c, T* X, const T* B, bool zero) override {
    restrict_gather(B, bLo.p, sub->N, A->Np, keep, map.p, c.st);
    const T* a[1] = {bLo.p};
    dots(c.red, 1, a, a, sub->N, d_norm, 1, c.st);
    positive_flag(d_norm, nonzero, c.st);
    const cudaGraphConditionalHandle h = c.cond_handle();
    const int body = c.new_body((this->trace >= 0 ? c.trace[this->trace].name + ": " : std::string()) + "coarse correction");
    cond_set(h, nonzero, nullptr, nullptr, 0, c.exec_of(body), c.st);
    c.cond_begin(h, cudaGraphCondTypeIf, body);
    if (zero)
      fill(T(0), xLo.p, sub->N, c.st);
    else
      restrict_gather(X, xLo.p, sub->N, A->Np, keep, map.p, c.st);
    lower->solve_graph(c, xLo.p, bLo.p, zero);
    restrict_scatter_add(xLo.p, X, sub->N, A->Np, keep, map.p, c.st);
    c.cond_end();
  }
};

// h-coarse correction: restrict by aggregate sums, solve the Galerkin operator, prolongate by injection.
template <typename T>
struct AggregationT : Solver<T> {
  const Aggregation* g;
  std::unique_ptr<Solver<T>> lower;
  DBuf<T> xc, bc;
  double* d_norm;
  AggregationT(Ctx& c, const Aggregation* g_) : g(g_) {
    xc.alloc(std::max<int64_t>(g->nc, 1));
    bc.alloc(std::max<int64_t>(g->nc, 1));
    d_norm = c.scal(1);
  }
  int nested() const override { return lower ? lower->this_level_iterations + lower->nested() : 0; }
  void solve(Ctx& c, T* X, const T* B, bool zero) override {
    TraceScope ts(c, this->trace);
    (void)zero;
    agg_restrict(*g, B, bc.p, c.st);
    const T* a[1] = {bc.p};
    dots(c.red, 1, a, a, g->nc, d_norm, 1, c.st);
    if (!(c.get(d_norm) > 0)) {
      this->converged = true;
      return;
    }
    fill(T(0), xc.p, g->nc, c.st);
    lower->solve(c, xc.p, bc.p, true);
    this->converged = lower->converged;
    agg_prolong_add(*g, xc.p, X, c.st);
  }
  // recorded form: the zero-right-hand-side return becomes an IF node
  int* nonzero = nullptr;
  bool graphable() const override { return lower && lower->graphable(); }
  void prepare_graph(Ctx& c) override {
    if (!nonzero) nonzero = c.flag();
    lower->prepare_graph(c);
  }
  void solve_graph(Ctx& c, T* X, const T* B, bool zero) override {
    (void)zero;
    agg_restrict(*g, B, bc.p, c.st);
    const T* a[1] = {bc.p};
    dots(c.red, 1, a, a, g->nc, d_norm, 1, c.st);
    positive_flag(d_norm, nonzero, c.st);
    const cudaGraphConditionalHandle h = c.cond_handle();
    const int body = c.new_body((this->trace >= 0 ? c.trace[this->trace].name + ": " : std::string()) + "aggregation coarse correction");
    cond_set(h, nonzero, nullptr, nullptr, 0, c.exec_of(body), c.st);
    c.cond_begin(h, cudaGraphCondTypeIf, body);
    fill(T(0), xc.p, g->nc, c.st);
    lower->solve_graph(c, xc.p, bc.p, true);
    agg_prolong_add(*g, xc.p, X, c.st);
    c.cond_end();
  }
};

// Direct solve of the coarsest level by a dense inverse computed once in FP64 (DirectSolver, DirectSolver.cs:43).
template <typename T>
struct DenseDirectT : Solver<T> {
  int n;
  DBuf<T> inv;
  DenseDirectT(Ctx& c, const Matrix* A64) : n((int)A64->N) {
    std::vector<double> h;
    dense_inverse(*A64, h, c.st);
    upload(h);
  }
  DenseDirectT(const std::vector<double>& h, int64_t n_) : n((int)n_) { upload(h); }
  void upload(const std::vector<double>& h) {
    inv.alloc(std::max<size_t>(h.size(), 1));
    std::vector<T> ht(h.begin(), h.end());
    if (!ht.empty()) BSGPU_CUDA(cudaMemcpy(inv.p, ht.data(), ht.size() * sizeof(T), cudaMemcpyHostToDevice));
  }
  void solve(Ctx& c, T* X, const T* B, bool zero) override {
    TraceScope ts(c, this->trace);
    (void)zero;
    dense_gemv(inv.p, B, X, n, c.st);
    this->converged = true;
    this->this_level_iterations = 1;
  }
  bool graphable() const override { return true; }
};

// Coarse correction through explicit restriction / prolongation matrices (MultigridOperator.Restrict /
// Prolongate, MultigridOperator.cs:774,815): b_c = R b, solve on the coarser h-level, X += P x_c.
template <typename T>
struct TransferT : Solver<T> {
  const Csr* P;
  const Csr* R;
  std::unique_ptr<Solver<T>> lower;
  DBuf<T> xc, bc;
  double* d_norm;
  TransferT(Ctx& c, const Csr* P_, const Csr* R_) : P(P_), R(R_) {
    xc.alloc(std::max<int64_t>(P->cols, 1));
    bc.alloc(std::max<int64_t>(P->cols, 1));
    d_norm = c.scal(1);
  }
  int nested() const override { return lower ? lower->this_level_iterations + lower->nested() : 0; }
  void solve(Ctx& c, T* X, const T* B, bool zero) override {
    TraceScope ts(c, this->trace);
    (void)zero;
    csr_spmv(*R, T(1), B, T(0), bc.p, c.st);
    const T* a[1] = {bc.p};
    dots(c.red, 1, a, a, R->rows, d_norm, 1, c.st);
    if (!(c.get(d_norm) > 0)) {
      this->converged = true;
      return;
    }
    fill(T(0), xc.p, P->cols, c.st);
    lower->solve(c, xc.p, bc.p, true);
    this->converged = lower->converged;
    csr_spmv(*P, T(1), xc.p, T(1), X, c.st);
  }
  // recorded form: the zero-right-hand-side return becomes an IF node
  int* nonzero = nullptr;
  bool graphable() const override { return lower && lower->graphable(); }
  void prepare_graph(Ctx& c) override {
    if (!nonzero) nonzero = c.flag();
    lower->prepare_graph(c);
  }
  void solve_graph(Ctx& c, T* X, const T* B, bool zero) override {
    (void)zero;
    csr_spmv(*R, T(1), B, T(0), bc.p, c.st);
    const T* a[1] = {bc.p};
    dots(c.red, 1, a, a, R->rows, d_norm, 1, c.st);
    positive_flag(d_norm, nonzero, c.st);
    const cudaGraphConditionalHandle h = c.cond_handle();
    const int body = c.new_body((this->trace >= 0 ? c.trace[this->trace].name + ": " : std::string()) + "transfer coarse correction");
    cond_set(h, nonzero, nullptr, nullptr, 0, c.exec_of(body), c.st);
    c.cond_begin(h, cudaGraphCondTypeIf, body);
    fill(T(0), xc.p, P->cols, c.st);
    lower->solve_graph(c, xc.p, bc.p, true);
    csr_spmv(*P, T(1), xc.p, T(1), X, c.st);
    c.cond_end();
  }
};

// Coarsest p-level: CG preconditioned by one smoothed-aggregation V-cycle (amg.cu) per iteration, to a relative
// tolerance.  Stand-in for the reference's direct solve of this level (PmgConfig.cs:167-177).
template <typename T>
struct AmgPcgT : Solver<T> {
  const AmgHierarchy* H;
  std::vector<const Matrix*> Al;  // level operators in precision T
  std::vector<DBuf<T>> lx, lb, lr;
  DBuf<T> dense, r, z, p, q;
  int nu;
  Term term;
  double* d_s;  // [0] rr, [1] rz, [2] pq
  AmgPcgT(Tree& t, const AmgHierarchy* H_, const Matrix* AT, int sweeps, Term tm) : H(H_), nu(sweeps), term(tm) {
    Ctx& c = *t.ctx;
    const size_t nl = H->levels.size();
    for (size_t l = 0; l < nl; ++l) {
      const Matrix* A64 = H->levels[l].Aref;
      if (l == 0)
        Al.push_back(AT);
      else if (sizeof(T) == 8)
        Al.push_back(A64);
      else {
        t.owned.emplace_back(matrix_to_single(*A64, c.st));
        Al.push_back(t.owned.back().get());
      }
      const int64_t n = std::max<int64_t>(H->levels[l].n, 1);
      lx.emplace_back(n);
      lb.emplace_back(n);
      lr.emplace_back(n);
    }
    if (H->n_dense) {
      dense.alloc(H->dense_inv.size());
      std::vector<T> h(H->dense_inv.begin(), H->dense_inv.end());
      BSGPU_CUDA(cudaMemcpy(dense.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
    }
    const int64_t N = std::max<int64_t>(H->levels[0].n, 1);
    r.alloc(N); z.alloc(N); p.alloc(N); q.alloc(N);
    d_s = c.scal(3);
  }
  const T* dinv(int l) const {
    if constexpr (sizeof(T) == 8) return H->levels[l].dinv64.p;
    else return H->levels[l].dinv32.p;
  }
  void smooth(Ctx& c, int l, T* X, const T* B, bool zero, int sweeps) {
    const Matrix& A = *Al[l];
    const T w = (T)H->levels[l].omega;
    const int64_t n = H->levels[l].n;
    for (int s = 0; s < sweeps; ++s) {
      if (s == 0 && zero) {
        jacobi_update(dinv(l), w, B, (const T*)nullptr, X, n, c.st);
      } else {
        spmv(A, T(1), X, T(0), (const T*)nullptr, lr[l].p, c.st);
        jacobi_update(dinv(l), w, B, lr[l].p, X, n, c.st);
      }
    }
  }
  std::vector<int> tr_smooth, tr_transfer;
  void trace_ids(Ctx& c) {
    for (size_t l = 0; l < H->levels.size(); ++l) {
      tr_smooth.push_back(c.trace_id("AMG" + std::to_string(l) + ".smooth(n=" + std::to_string(H->levels[l].n) + ")"));
      tr_transfer.push_back(c.trace_id("AMG" + std::to_string(l) + ".transfer"));
    }
  }
  void vcycle(Ctx& c, int l, T* X, const T* B, bool zero) {
    const int last = (int)H->levels.size() - 1;
    const AmgLevel& L = H->levels[l];
    if (tr_smooth.empty()) trace_ids(c);
    if (l == last) {
      TraceScope ts(c, tr_smooth[l]);
      if (H->n_dense)
        dense_gemv(dense.p, B, X, (int)H->n_dense, c.st);
      else
        smooth(c, l, X, B, zero, 2 * nu);
      return;
    }
    {
      TraceScope ts(c, tr_smooth[l]);
      smooth(c, l, X, B, zero, nu);
    }
    {
      TraceScope ts(c, tr_transfer[l]);
      spmv(*Al[l], T(-1), X, T(1), B, lr[l].p, c.st);
      csr_spmv(*L.R, T(1), lr[l].p, T(0), lb[l + 1].p, c.st);
    }
    vcycle(c, l + 1, lx[l + 1].p, lb[l + 1].p, true);
    {
      TraceScope ts(c, tr_transfer[l]);
      csr_spmv(*L.P, T(1), lx[l + 1].p, T(1), X, c.st);
    }
    TraceScope ts(c, tr_smooth[l]);
    smooth(c, l, X, B, false, nu);
  }
  void solve(Ctx& c, T* X, const T* B, bool zero) override {
    TraceScope ts(c, this->trace);
    const Matrix& A = *Al[0];
    const int64_t N = A.N;
    if (zero)
      copy_vec(r.p, B, N, c.st);
    else
      spmv(A, T(-1), X, T(1), B, r.p, c.st);
    const T* rv[1] = {r.p};
    dots(c.red, 1, rv, rv, N, d_s, 0, c.st);
    const double rr0 = c.get(d_s);
    if (!std::isfinite(rr0)) throw Error(BSGPU_ERR_ARITHMETIC, "AMG-PCG: NaN/Inf in the right-hand side");
    this->history.assign(1, std::sqrt(rr0));
    int it = 0;
    if (rr0 > 0) {
      vcycle(c, 0, z.p, r.p, true);
      copy_vec(p.p, z.p, N, c.st);
      const T* zv[1] = {z.p};
      dots(c.red, 1, rv, zv, N, d_s + 1, 0, c.st);
      double rz = c.get(d_s + 1);
      const T* pv[1] = {p.p};
      const T* qv[1] = {q.p};
      for (it = 1; it <= term.max_iter; ++it) {
        spmv(A, T(1), p.p, T(0), (const T*)nullptr, q.p, c.st);
        dots(c.red, 1, pv, qv, N, d_s + 2, 0, c.st);
        const double pq = c.get(d_s + 2);
        const double alpha = rz / pq;
        if (!std::isfinite(alpha)) throw Error(BSGPU_ERR_ARITHMETIC, "AMG-PCG: breakdown");
        const double ha[1] = {alpha}, hm[1] = {-alpha};
        axpys(1, nullptr, ha, 1.0, pv, X, N, c.st);
        axpys(1, nullptr, hm, 1.0, qv, r.p, N, c.st);
        dots(c.red, 1, rv, rv, N, d_s, 0, c.st);
        const double rr = c.get(d_s);
        this->history.push_back(std::sqrt(rr));
        if (rr <= term.tol * term.tol * rr0) break;
        vcycle(c, 0, z.p, r.p, true);
        dots(c.red, 1, rv, zv, N, d_s + 1, 0, c.st);
        const double rz_new = c.get(d_s + 1);
        axpby(T(1), z.p, T(rz_new / rz), p.p, N, c.st);
        rz = rz_new;
      }
      if (it > term.max_iter) it = term.max_iter;
    }
    this->converged = this->history.back() <= term.tol * this->history.front() || rr0 == 0;
    this->this_level_iterations = it;
    if (c.tracing && this->trace >= 0) c.trace[this->trace].iterations += it;
  }
};

// The learned stage as a preconditioner / smoother: X = NN(B) (learned.cu); inputs normalised by the RMS of B.
template <typename T>
struct LearnedPrecondT : Solver<T> {
  bool graphable() const override { return true; }
  const LearnedNet* net;
  int64_t N;
  double* d_s;  // [0] |B|, [1] scale
  LearnedPrecondT(Ctx& c, const LearnedNet* n_) : net(n_), N(n_->ncells * n_->Np) { d_s = c.scal(2); }
  void solve(Ctx& c, T* X, const T* B, bool zero) override {
    TraceScope ts(c, this->trace);
    (void)zero;
    const T* a[1] = {B};
    dots(c.red, 1, a, a, N, d_s, 1, c.st);
    learned_scale(d_s, d_s + 1, N, c.st);
    learned_apply(*net, B, X, d_s + 1, c.st);
    this->converged = true;
    this->this_level_iterations = 1;
  }
};

// FP64 interface around an FP32 solver (mixed-precision preconditioner).
struct MixedAdapter : Solver<double> {
  std::unique_ptr<Solver<float>> inner;
  DBuf<float> x32, b32;
  int64_t N;
  explicit MixedAdapter(int64_t n) : N(n) {
    x32.alloc(std::max<int64_t>(n, 1));
    b32.alloc(std::max<int64_t>(n, 1));
  }
  int nested() const override { return inner->this_level_iterations + inner->nested(); }
  void solve(Ctx& c, double* X, const double* B, bool zero) override {
    convert(B, b32.p, N, c.st);
    if (zero)
      fill(0.0f, x32.p, N, c.st);
    else
      convert(X, x32.p, N, c.st);
    inner->solve(c, x32.p, b32.p, zero);
    convert(x32.p, X, N, c.st);
    this->converged = inner->converged;
    this->this_level_iterations = inner->this_level_iterations;
  }
  bool graphable() const override { return inner->graphable(); }
  void prepare_graph(Ctx& c) override { inner->prepare_graph(c); }
  void solve_graph(Ctx& c, double* X, const double* B, bool zero) override {
    convert(B, b32.p, N, c.st);
    if (zero)
      fill(0.0f, x32.p, N, c.st);
    else
      convert(X, x32.p, N, c.st);
    inner->solve_graph(c, x32.p, b32.p, zero);
    convert(x32.p, X, N, c.st);
  }
};

// The p-multigrid V-cycle recorded once as a CUDA graph (device-side control flow, devctl.cuh) and replayed by one
// graph launch per application.  The graph reads and writes fixed buffers: the owner's (MixedAdapter's FP32
// vectors, which it fills before and reads after the call) or this wrapper's own (the right-hand side is copied in,
// the result out).  Recorded again when the learned pre-smoother is switched on or off.
template <typename T>
struct GraphedT : Solver<T> {
  std::unique_ptr<Solver<T>> inner;
  int64_t N;
  T* Xs = nullptr;          // owner's buffers (X is zero on entry), or null: own buffers
  const T* Bs = nullptr;
  DBuf<T> xin, bin;
  const bool* key_src = nullptr;
  int key = -1;
  cudaGraphExec_t exec = nullptr;
  long long top_kernels = 0;
  GraphedT(int64_t n, std::unique_ptr<Solver<T>> in) : inner(std::move(in)), N(n) {}
  ~GraphedT() override {
    if (exec) cudaGraphExecDestroy(exec);
  }
  int nested() const override { return inner->this_level_iterations + inner->nested(); }
  // inside a larger recording (the whole FlexGMRES solve) the V-cycle is recorded inline
  bool graphable() const override { return inner->graphable(); }
  void prepare_graph(Ctx& c) override { inner->prepare_graph(c); }
  void solve_graph(Ctx& c, T* X, const T* B, bool zero) override { inner->solve_graph(c, X, B, zero); }
  void capture(Ctx& c, T* X, const T* B) {
    if (exec) {
      cudaGraphExecDestroy(exec);
      exec = nullptr;
    }
    inner->prepare_graph(c);
    c.capture_begin();
    cudaGraph_t g = nullptr;
    try {
      inner->solve_graph(c, X, B, true);
    } catch (...) {
      c.capture_abort();
      cudaStreamEndCapture(c.st, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    top_kernels = c.capture_end(&g);
    const cudaError_t e = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    BSGPU_CUDA(e);
  }
  T* graph_x() { return Xs ? Xs : xin.p; }
  const T* graph_b() { return Xs ? Bs : bin.p; }
  // records the graph if there is none yet or the learned pre-smoother was switched since (set-up time)
  void ensure(Ctx& c) {
    if (!Xs && !xin.p) {
      xin.alloc(std::max<int64_t>(N, 1));
      bin.alloc(std::max<int64_t>(N, 1));
    }
    const int k = key_src ? (*key_src ? 1 : 0) : 0;
    if (!exec || k != key) {
      capture(c, graph_x(), graph_b());
      key = k;
    }
  }
  void solve(Ctx& c, T* X, const T* B, bool zero) override {
    if (!zero || c.tracing || (Xs && (X != Xs || B != Bs))) {
      inner->solve(c, X, B, zero);
      this->this_level_iterations = inner->this_level_iterations;
      this->converged = inner->converged;
      return;
    }
    ensure(c);
    if (!Xs) {
      copy_vec(bin.p, B, N, c.st);
      fill(T(0), xin.p, N, c.st);
    }
    BSGPU_CUDA(cudaGraphLaunch(exec, c.st));
    add_launches(top_kernels);
    c.graph_ran = true;
    BSGPU_CUDA(cudaMemcpyAsync(c.h_err, c.d_err, sizeof(int), cudaMemcpyDeviceToHost, c.st));
    c.err_pending = true;
    if (!Xs) copy_vec(X, (const T*)xin.p, N, c.st);
    this->converged = true;
    this->this_level_iterations = 1;
  }
};

// ---------------------------------------------------------------------------------------------------------------
// FlexGMRES (FlexGMRES.cs:144-277), Saad-1993 FGMRES(m): the minimal-residual combination of the preconditioned
// vectors Z_j is formed from the least-squares solution of the Hessenberg system (Givens rotations, the dgelsy
// solution for full-rank H).  The reference overwrites that solution with (beta, 0, ..., 0) at :259-260, which
// reduces it to preconditioned Richardson; this implementation does not.  The implicit residual |g_{j+1}| is
// tested after every Arnoldi step; the true residual is recomputed at every restart.  Arnoldi uses classical
// Gram-Schmidt applied twice (one multi-dot and one multi-axpy launch per sweep) instead of MGS.
// ---------------------------------------------------------------------------------------------------------------
struct FlexGMRES : Solver<double>, RecordedSolve {
  const Matrix* A;
  int64_t N;
  int m;
  Term term;
  bool whole = false;  // cfg.graph == 2: the handle records the whole solve (RecordedSolve)
  std::unique_ptr<Solver<double>> pc;
  // second preconditioner used in turn with pc (FlexGMRES.cs:196-199 cycles PrecondS); switched off for the rest
  // of a solve when one of its steps reduces the residual estimate by less than the factor `stall`
  std::unique_ptr<Solver<double>> pc2;
  Tree* tree = nullptr;
  double stall = 0.99;
  std::vector<DBuf<double>> V, Z;
  DBuf<double> R0;
  double* d_h;     // [2*(m+1)] projections of both sweeps
  double* d_norm;  // [1]
  FlexGMRES(Ctx& c, const Matrix* A_, int m_, Term t) : A(A_), N(A_->N), m(m_), term(t) {
    for (int j = 0; j <= m; ++j) V.emplace_back(std::max<int64_t>(N, 1));
    for (int j = 0; j < m; ++j) Z.emplace_back(std::max<int64_t>(N, 1));
    R0.alloc(std::max<int64_t>(N, 1));
    d_h = c.scal(2 * (m + 1));
    d_norm = c.scal(1);
  }
  int nested() const override { return pc ? pc->this_level_iterations + pc->nested() : 0; }
  double norm(Ctx& c, const double* v) {
    const double* a[1] = {v};
    dots(c.red, 1, a, a, N, d_norm, 1, c.st);
    return c.get(d_norm);
  }
  // W -= sum_i h_i V_i for i <= j; projections into d_h[off..off+j]
  void project(Ctx& c, int j, double* W, int off) {
    for (int i0 = 0; i0 <= j; i0 += kMaxDots) {
      const int kc = std::min(kMaxDots, j + 1 - i0);
      const double* a[kMaxDots];
      const double* b[kMaxDots];
      for (int i = 0; i < kc; ++i) {
        a[i] = V[i0 + i].p;
        b[i] = W;
      }
      dots(c.red, kc, a, b, N, d_h + off + i0, 0, c.st);
    }
    std::vector<const double*> vx(j + 1);
    for (int i = 0; i <= j; ++i) vx[i] = V[i].p;
    axpys(j + 1, d_h + off, nullptr, -1.0, vx.data(), W, N, c.st);
  }
  void solve(Ctx& c, double* X, const double* B, bool zero) override {
    TraceScope ts(c, this->trace);
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
    bool nn_active = pc2 && tree && tree->learned_on;
    int turn = 0;
    int iIter = 0;
    double r0 = 0;
    this->history.clear();
    bool first = true;
    while (true) {
      if (first && zero)
        copy_vec(R0.p, B, N, c.st);
      else
        spmv(*A, -1.0, X, 1.0, B, R0.p, c.st);
      first = false;
      const double r = norm(c, R0.p);
      if (!std::isfinite(r)) throw Error(BSGPU_ERR_ARITHMETIC, "FlexGMRES: residual is NaN/Inf");
      if (iIter == 0) r0 = r;
      this->history.push_back(r);
      auto st = term(iIter, r0, r);
      if (!st.first || st.second) {
        this->converged = st.second;
        this->this_level_iterations = iIter;
        if (c.tracing && this->trace >= 0) c.trace[this->trace].iterations += iIter;
        return;
      }
      axpby(1.0 / r, R0.p, 0.0, V[0].p, N, c.st);
      std::fill(g.begin(), g.end(), 0.0);
      g[0] = r;
      int j;
      for (j = 0; j < m; ++j) {
        fill(0.0, Z[j].p, N, c.st);
        const bool use2 = pc2 && nn_active && (turn++ % 2 == 1);
        const double g_before = std::fabs(g[j]);
        if (use2)
          pc2->solve(c, Z[j].p, V[j].p, true);
        else
          pc->solve(c, Z[j].p, V[j].p, true);
        iIter++;
        double* W = V[j + 1].p;
        spmv(*A, 1.0, Z[j].p, 0.0, (const double*)nullptr, W, c.st);
        project(c, j, W, 0);
        project(c, j, W, m + 1);
        const double* a[1] = {W};
        dots(c.red, 1, a, a, N, d_norm, 1, c.st);
        c.fetch(d_h, 2 * (m + 1) + 1);
        const double* hh = c.hscal + (d_h - c.dscal.p);
        const double wn = hh[2 * (m + 1)];
        if (!std::isfinite(wn)) throw Error(BSGPU_ERR_ARITHMETIC, "FlexGMRES: Arnoldi vector is NaN/Inf");
        for (int i = 0; i <= j; ++i) H[i * m + j] = hh[i] + hh[m + 1 + i];
        H[(j + 1) * m + j] = wn;
        if (wn > 0) axpby(1.0 / wn, W, 0.0, W, N, c.st);
        if (tree && tree->collect && tree->collect->size() < tree->collect_cap && wn > 0) {
          tree->collect->emplace_back(N);
          copy_vec(tree->collect->back().p, (const double*)W, N, c.st);
        }
        for (int i = 0; i < j; ++i) {
          const double a0 = H[i * m + j], b0 = H[(i + 1) * m + j];
          H[i * m + j] = cs[i] * a0 + sn[i] * b0;
          H[(i + 1) * m + j] = -sn[i] * a0 + cs[i] * b0;
        }
        const double a0 = H[j * m + j], b0 = H[(j + 1) * m + j];
        const double den = std::hypot(a0, b0);
        cs[j] = a0 / den;
        sn[j] = b0 / den;
        H[j * m + j] = den;
        H[(j + 1) * m + j] = 0.0;
        g[j + 1] = -sn[j] * g[j];
        g[j] = cs[j] * g[j];
        const double est = std::fabs(g[j + 1]);
        this->history.push_back(est);
        if (use2 && est > stall * g_before) {
          nn_active = false;  // the learned stage stalls: plain p-multigrid for the rest of this solve
          if (tree) tree->learned_stalls++;
        }
        auto st2 = term(iIter, r0, est);
        if (!st2.first || st2.second || wn == 0.0) {
          ++j;
          break;
        }
      }
      const int kk = j;
      for (int i = kk - 1; i >= 0; --i) {
        double s = g[i];
        for (int q = i + 1; q < kk; ++q) s -= H[i * m + q] * y[q];
        y[i] = s / H[i * m + i];
      }
      std::vector<const double*> zx(kk);
      for (int i = 0; i < kk; ++i) zx[i] = Z[i].p;
      axpys(kk, nullptr, y.data(), 1.0, zx.data(), X, N, c.st);
    }
  }

  // ---- the recorded whole solve (RecordedSolve) ----
  // Same steps as solve() with the host's scalars and branches moved to FgState: the basis vectors and the
  // preconditioned vectors are addressed through device pointer tables by the device's Arnoldi index (slot_load /
  // slot_store), the Gram-Schmidt sweeps project against the first j + 1 basis vectors with hist_dots /
  // hist_axpy1, and the cycle's update X += Z y is one hist_axpy1 with the negated back-substitution.
  DBuf<double> vin, zf, Wf, farr;
  DBuf<double*> dV, dZ;
  HistScratch hsV;
  DBuf<FgState> fst;
  FgArrays fa{};
  double *d_h1 = nullptr, *d_h2 = nullptr, *d_wn = nullptr, *d_rn = nullptr;
  FgState* h_fst = nullptr;
  double* h_hist = nullptr;
  ~FlexGMRES() override {
    if (h_fst) cudaFreeHost(h_fst);
    if (h_hist) cudaFreeHost(h_hist);
  }
  void norm_dev(Ctx& c, const double* v, double* out) {
    const double* a[1] = {v};
    dots(c.red, 1, a, a, N, out, 1, c.st);
  }
  void prepare(Ctx& c) override {
    if (!fst.p) {
      require(m + 1 <= kHistMax, "recorded FlexGMRES: MaxKrylovDim above 127", BSGPU_ERR_UNSUPPORTED);
      const int64_t n1 = std::max<int64_t>(N, 1);
      vin.alloc(n1);
      zf.alloc(n1);
      Wf.alloc(n1);
      std::vector<double*> pv(m + 1), pz(m);
      for (int j = 0; j <= m; ++j) pv[j] = V[j].p;
      for (int j = 0; j < m; ++j) pz[j] = Z[j].p;
      dV.alloc(m + 1);
      dZ.alloc(m);
      BSGPU_CUDA(cudaMemcpy(dV.p, pv.data(), (m + 1) * sizeof(double*), cudaMemcpyHostToDevice));
      BSGPU_CUDA(cudaMemcpy(dZ.p, pz.data(), m * sizeof(double*), cudaMemcpyHostToDevice));
      hsV.init(m + 1);
      fst.alloc(1);
      BSGPU_CUDA(cudaMemset(fst.p, 0, sizeof(FgState)));
      fa.m = m;
      fa.hcap = 2 * std::max(term.max_iter, 1) + 16;
      const size_t nH = (size_t)(m + 1) * m;
      farr.alloc(nH + 3 * (size_t)m + (m + 1) + fa.hcap);
      BSGPU_CUDA(cudaMemset(farr.p, 0, (nH + 3 * (size_t)m + (m + 1) + fa.hcap) * sizeof(double)));
      fa.H = farr.p;
      fa.cs = fa.H + nH;
      fa.sn = fa.cs + m;
      fa.ny = fa.sn + m;
      fa.g = fa.ny + m;
      fa.hist = fa.g + (m + 1);
      d_h1 = c.scal(m + 1);
      d_h2 = c.scal(m + 1);
      d_wn = c.scal(1);
      d_rn = c.scal(1);
      BSGPU_CUDA(cudaMallocHost(&h_fst, sizeof(FgState)));
      BSGPU_CUDA(cudaMallocHost(&h_hist, fa.hcap * sizeof(double)));
    }
    c.graph_init();
    require(pc && pc->graphable() && (!pc2 || pc2->graphable()),
            "the FlexGMRES solve cannot be recorded as a graph with this preconditioner", BSGPU_ERR_UNSUPPORTED);
    pc->prepare_graph(c);
    if (pc2) pc2->prepare_graph(c);
  }
  // the learned stage (second preconditioner or pre-smoother inside the V-cycle) switched on or off
  int key() const override { return (tree && tree->net && tree->learned_on) ? 1 : 0; }
  void precondition_dev(Ctx& c, Solver<double>* p) {
    fill(0.0, zf.p, N, c.st);
    p->solve_graph(c, zf.p, vin.p, true);
  }
  void record(Ctx& c, double* X, const double* B) override {
    const TermParams tp = term.params();
    FgState* s = fst.p;
    const std::string tag = this->trace >= 0 ? c.trace[this->trace].name + ": " : std::string("FlexGMRES: ");
    fg_begin(s, (pc2 && key()) ? 1 : 0, pc2 ? 1 : 0, c.st);
    spmv(*A, -1.0, X, 1.0, B, R0.p, c.st);
    norm_dev(c, R0.p, d_rn);
    fg_restart(s, fa, d_rn, tp, c.d_err, c.st);
    const cudaGraphConditionalHandle h_outer = c.cond_handle();
    const int b_outer = c.new_body(tag + "restart cycle");
    cond_set(h_outer, &s->outer, nullptr, nullptr, 0, c.exec_of(b_outer), c.st);
    c.cond_begin(h_outer, cudaGraphCondTypeWhile, b_outer);
    {
      slot_store(R0.p, &s->inv, dV.p, nullptr, m + 1, N, c.d_err, c.st);
      const cudaGraphConditionalHandle h_inner = c.cond_handle();
      const int b_inner = c.new_body(tag + "Arnoldi step");
      cond_set(h_inner, &s->inner, nullptr, nullptr, 0, c.exec_of(b_inner), c.st);
      c.cond_begin(h_inner, cudaGraphCondTypeWhile, b_inner);
      {
        fg_step_begin(s, fa, c.st);
        slot_load(dV.p, &s->j, vin.p, N, c.st);
        if (pc2) {
          const cudaGraphConditionalHandle h1 = c.cond_handle();
          const int b1 = c.new_body(tag + "first preconditioner");
          cond_set(h1, nullptr, &s->use2, nullptr, 0, c.exec_of(b1), c.st);
          c.cond_begin(h1, cudaGraphCondTypeIf, b1);
          precondition_dev(c, pc.get());
          c.cond_end();
          const cudaGraphConditionalHandle h2 = c.cond_handle();
          const int b2 = c.new_body(tag + "second preconditioner");
          cond_set(h2, &s->use2, nullptr, nullptr, 0, c.exec_of(b2), c.st);
          c.cond_begin(h2, cudaGraphCondTypeIf, b2);
          precondition_dev(c, pc2.get());
          c.cond_end();
        } else {
          precondition_dev(c, pc.get());
        }
        slot_store(zf.p, nullptr, dZ.p, &s->j, m, N, c.d_err, c.st);
        spmv(*A, 1.0, zf.p, 0.0, (const double*)nullptr, Wf.p, c.st);
        hist_dots(hsV, dV.p, &s->k1, Wf.p, N, d_h1, nullptr, c.st);
        hist_axpy1(dV.p, &s->k1, m + 1, d_h1, Wf.p, N, c.st);
        hist_dots(hsV, dV.p, &s->k1, Wf.p, N, d_h2, nullptr, c.st);
        hist_axpy1(dV.p, &s->k1, m + 1, d_h2, Wf.p, N, c.st);
        norm_dev(c, Wf.p, d_wn);
        fg_step_end(s, fa, d_h1, d_h2, d_wn, tp, stall, c.d_err, c.st);
        slot_store(Wf.p, &s->inv, dV.p, &s->j, m + 1, N, c.d_err, c.st);
        cond_set(h_inner, &s->inner, nullptr, nullptr, 0, c.exec_of(b_inner), c.st);
      }
      c.cond_end();
      fg_backsub(s, fa, c.st);
      hist_axpy1(dZ.p, &s->kk, m, fa.ny, X, N, c.st);
      spmv(*A, -1.0, X, 1.0, B, R0.p, c.st);
      norm_dev(c, R0.p, d_rn);
      fg_restart(s, fa, d_rn, tp, c.d_err, c.st);
      cond_set(h_outer, &s->outer, nullptr, nullptr, 0, c.exec_of(b_outer), c.st);
    }
    c.cond_end();
  }
  void queue_result(Ctx& c, cudaStream_t st) override {
    BSGPU_CUDA(cudaMemcpyAsync(h_fst, fst.p, sizeof(FgState), cudaMemcpyDeviceToHost, st));
    BSGPU_CUDA(cudaMemcpyAsync(h_hist, fa.hist, fa.hcap * sizeof(double), cudaMemcpyDeviceToHost, st));
    BSGPU_CUDA(cudaMemcpyAsync(c.h_err, c.d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    c.err_pending = true;
  }
  void take_result(Ctx& c) override {
    (void)c;
    const FgState& s = *h_fst;
    this->history.assign(h_hist, h_hist + std::min(std::max(s.nhist, 0), fa.hcap));
    this->this_level_iterations = s.iter;
    this->converged = s.converged != 0;
    if (s.stalled && tree) tree->learned_stalls++;
  }
};


// ---------------------------------------------------------------------------------------------------------------
// SoftGMRES.Solve (SoftGMRES.cs:227-460): restarted GMRES(m) with left preconditioning, r = M^{-1}(b - A x),
// Arnoldi on M^{-1} A, Givens rotations, x += V y at convergence and at every restart.  As in the reference, the
// termination test compares the preconditioned residual estimate |s_i| against the unpreconditioned initial
// residual |b - A x0|.  Gram-Schmidt: classical, one multi-dot and one multi-axpy launch per sweep, two sweeps
// (the reference uses one modified sweep).  When the iteration limit is reached at the end of a cycle the update of
// that cycle is applied (the reference leaves x at the start of the cycle).
// ---------------------------------------------------------------------------------------------------------------
struct SoftGMRES : Solver<double> {
  const Matrix* A;
  int64_t N;
  int m;
  Term term;
  std::unique_ptr<Solver<double>> pc;
  std::vector<DBuf<double>> V;
  DBuf<double> Z;
  double* d_h;     // [2*(m+1)] projections of both sweeps
  double* d_norm;  // [1]
  SoftGMRES(Ctx& c, const Matrix* A_, int m_, Term t) : A(A_), N(A_->N), m(m_), term(t) {
    for (int j = 0; j <= m; ++j) V.emplace_back(std::max<int64_t>(N, 1));
    Z.alloc(std::max<int64_t>(N, 1));
    d_h = c.scal(2 * (m + 1));
    d_norm = c.scal(1);
  }
  int nested() const override { return pc ? pc->this_level_iterations + pc->nested() : 0; }
  double norm(Ctx& c, const double* v) {
    const double* a[1] = {v};
    dots(c.red, 1, a, a, N, d_norm, 1, c.st);
    return c.get(d_norm);
  }
  void project(Ctx& c, int j, double* W, int off) {
    for (int i0 = 0; i0 <= j; i0 += kMaxDots) {
      const int kc = std::min(kMaxDots, j + 1 - i0);
      const double* a[kMaxDots];
      const double* b[kMaxDots];
      for (int i = 0; i < kc; ++i) {
        a[i] = V[i0 + i].p;
        b[i] = W;
      }
      dots(c.red, kc, a, b, N, d_h + off + i0, 0, c.st);
    }
    std::vector<const double*> vx(j + 1);
    for (int i = 0; i <= j; ++i) vx[i] = V[i].p;
    axpys(j + 1, d_h + off, nullptr, -1.0, vx.data(), W, N, c.st);
  }
  void precondition(Ctx& c, const double* in, double* out) {
    if (pc) {
      fill(0.0, out, N, c.st);
      pc->solve(c, out, in, true);
    } else {
      copy_vec(out, in, N, c.st);
    }
  }
  void solve(Ctx& c, double* X, const double* B, bool zero) override {
    TraceScope ts(c, this->trace);
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1), y(m);
    this->history.clear();
    int tot = 0;
    if (zero)
      copy_vec(Z.p, B, N, c.st);
    else
      spmv(*A, -1.0, X, 1.0, B, Z.p, c.st);
    const double r0 = norm(c, Z.p);
    if (!std::isfinite(r0)) throw Error(BSGPU_ERR_ARITHMETIC, "SoftGMRES: residual is NaN/Inf");
    this->history.push_back(r0);
    auto st0 = term(0, r0, r0);
    if (!st0.first) {
      this->converged = st0.second;
      this->this_level_iterations = 0;
      return;
    }
    bool first = true;
    while (true) {
      if (!first) spmv(*A, -1.0, X, 1.0, B, Z.p, c.st);
      first = false;
      precondition(c, Z.p, V[0].p);
      const double beta = norm(c, V[0].p);
      if (!std::isfinite(beta)) throw Error(BSGPU_ERR_ARITHMETIC, "SoftGMRES: preconditioned residual is NaN/Inf");
      if (beta == 0.0) {
        this->converged = true;
        break;
      }
      axpby(1.0 / beta, V[0].p, 0.0, V[0].p, N, c.st);
      std::fill(g.begin(), g.end(), 0.0);
      g[0] = beta;
      int j;
      bool stop = false;
      double err = beta;
      for (j = 0; j < m; ++j) {
        spmv(*A, 1.0, V[j].p, 0.0, (const double*)nullptr, Z.p, c.st);
        double* W = V[j + 1].p;
        precondition(c, Z.p, W);
        project(c, j, W, 0);
        project(c, j, W, m + 1);
        const double* a[1] = {W};
        dots(c.red, 1, a, a, N, d_norm, 1, c.st);
        c.fetch(d_h, 2 * (m + 1) + 1);
        const double* hh = c.hscal + (d_h - c.dscal.p);
        const double wn = hh[2 * (m + 1)];
        if (!std::isfinite(wn)) throw Error(BSGPU_ERR_ARITHMETIC, "SoftGMRES: Arnoldi vector is NaN/Inf");
        for (int i = 0; i <= j; ++i) H[i * m + j] = hh[i] + hh[m + 1 + i];
        H[(j + 1) * m + j] = wn;
        if (wn > 0) axpby(1.0 / wn, W, 0.0, W, N, c.st);
        for (int i = 0; i < j; ++i) {
          const double a0 = H[i * m + j], b0 = H[(i + 1) * m + j];
          H[i * m + j] = cs[i] * a0 + sn[i] * b0;
          H[(i + 1) * m + j] = -sn[i] * a0 + cs[i] * b0;
        }
        const double a0 = H[j * m + j], b0 = H[(j + 1) * m + j];
        const double den = std::hypot(a0, b0);
        cs[j] = a0 / den;
        sn[j] = b0 / den;
        H[j * m + j] = den;
        H[(j + 1) * m + j] = 0.0;
        g[j + 1] = -sn[j] * g[j];
        g[j] = cs[j] * g[j];
        err = std::fabs(g[j + 1]);
        this->history.push_back(err);
        auto st1 = term(tot, r0, err);
        ++tot;
        if (!st1.first || wn == 0.0) {
          stop = true;
          this->converged = st1.second || wn == 0.0;
          ++j;
          break;
        }
      }
      const int kk = j;
      for (int i = kk - 1; i >= 0; --i) {
        double s = g[i];
        for (int q = i + 1; q < kk; ++q) s -= H[i * m + q] * y[q];
        y[i] = s / H[i * m + i];
      }
      std::vector<const double*> vx(kk);
      for (int i = 0; i < kk; ++i) vx[i] = V[i].p;
      axpys(kk, nullptr, y.data(), 1.0, vx.data(), X, N, c.st);
      if (stop) break;
      auto st2 = term(tot, r0, err);
      if (!st2.first) {
        this->converged = st2.second;
        break;
      }
    }
    this->this_level_iterations = tot;
    if (c.tracing && this->trace >= 0) c.trace[this->trace].iterations += tot;
  }
};

// ---------------------------------------------------------------------------------------------------------------
// tree construction (PmgConfig.CreateInstanceImpl__Kummer, PmgConfig.cs:80-245, with UseILU = false)
// ---------------------------------------------------------------------------------------------------------------
template <typename T>
const Matrix* level_matrix(Tree& t, const Matrix* A64) {
  if constexpr (sizeof(T) == 8) {
    return A64;
  } else {
    if (t.cfg.fp16_storage & BSGPU_FP16_MATRICES)
      t.owned.emplace_back(matrix_to_half(*A64, t.ctx->st));
    else
      t.owned.emplace_back(matrix_to_single(*A64, t.ctx->st));
    return t.owned.back().get();
  }
}

template <typename T>
std::unique_ptr<Solver<T>> make_smoother(Ctx& c, const Matrix* A64, const Matrix* AT, int kind,
                                         const bsgpu_solver_config& cfg, const std::string& name);

// Aggregation levels below the last (p = 0) p-level: OrthoMG with h_cycle iterations per call, h_sweeps
// block-Jacobi post-smoother sweeps and an aggregation coarse correction; the last level is solved densely.
template <typename T>
std::unique_ptr<Solver<T>> build_hlevel(Tree& t, const Matrix* A64, const Matrix* AT, int hl) {
  const bsgpu_solver_config& cfg = t.cfg;
  Ctx& c = *t.ctx;
  const std::string lv = "H" + std::to_string(hl);
  if (A64->N <= cfg.dense_limit) {
    auto d = std::make_unique<DenseDirectT<T>>(c, A64);
    d->trace = c.trace_id(lv + ".DenseDirect");
    return d;
  }
  if (hl >= cfg.h_levels) {
    Term ct;
    ct.mode = 1;
    ct.tol = cfg.coarse_tol;
    ct.max_iter = cfg.coarse_max_iter;
    ct.min_iter = 0;
    auto pcg = std::make_unique<PCGT<T>>(c, A64, AT, true, ct);
    pcg->trace = c.trace_id(lv + ".CoarsePCG");
    return pcg;
  }
  Term ht;
  ht.mode = 2;
  ht.max_iter = std::max(1, cfg.h_cycle);
  auto omg = std::make_unique<OrthoMGT<T>>(c, AT, ht);
  omg->ortho.cap = std::max(2, t.cfg.ortho_max_krylov > 0 ? t.cfg.ortho_max_krylov : 96);
  omg->ortho.recalc_period = std::max(1, t.cfg.recalc_resi_period);
  omg->trace = c.trace_id(lv + ".OrthoMG");
  omg->sweeps = cfg.h_sweeps;
  omg->post = make_smoother<T>(c, A64, AT, cfg.h_smoother, cfg, lv);
  t.aggs.emplace_back(matrix_aggregate(*A64, c.st));
  const Aggregation* g = t.aggs.back().get();
  const Matrix* c64 = g->coarse.get();
  const Matrix* cT = level_matrix<T>(t, c64);
  auto ag = std::make_unique<AggregationT<T>>(c, g);
  ag->trace = c.trace_id(lv + ".Aggregation");
  ag->lower = build_hlevel<T>(t, c64, cT, hl + 1);
  omg->coarse = std::move(ag);
  return omg;
}

template <typename T>
std::unique_ptr<Solver<T>> make_smoother(Ctx& c, const Matrix* A64, const Matrix* AT, int kind,
                                         const bsgpu_solver_config& cfg, const std::string& name) {
  std::unique_ptr<Solver<T>> s;
  const char* tag = ".BlockJacobi";
  if (kind == BSGPU_SMOOTHER_BLOCKGS) {
    s = std::make_unique<BlockGST<T>>(c, A64, AT, cfg.bj_iters, cfg.bj_omega);
    tag = ".BlockGS";
  } else if (kind == BSGPU_SMOOTHER_SCHWARZ) {
    s = std::make_unique<SchwarzT<T>>(c, A64, AT, cfg.bj_iters);
    tag = ".Schwarz";
  } else if (kind == BSGPU_SMOOTHER_ILU) {
    s = std::make_unique<ILU0T<T>>(c, A64);
    tag = ".CellILU";
  } else if (kind == BSGPU_SMOOTHER_ILU_NATURAL) {
    s = std::make_unique<ILUNaturalT<T>>(c, A64);
    tag = ".CellILU";
  } else if (kind == BSGPU_SMOOTHER_SCHWARZ_BLOCKS) {
    s = std::make_unique<BlockSchwarzT<T>>(c, A64, AT, cfg.bj_iters, cfg.schwarz_parts, cfg.schwarz_overlap,
                                           cfg.schwarz_scaling != 0);
    tag = ".Schwarz";
  } else {
    s = std::make_unique<BlockJacobiT<T>>(c, A64, AT, cfg.bj_iters, cfg.bj_omega);
  }
  s->trace = c.trace_id(name + tag);
  return s;
}

// h-multigrid below the coarsest p-level: level k of the hierarchy is an OrthoMG with block-Jacobi smoothing and
// a TransferT coarse correction; level 0 (the p-level itself) iterates to the coarse tolerance, the others run
// h_cycle iterations; the last level is solved densely.
template <typename T>
std::unique_ptr<Solver<T>> build_hmg_level(Tree& t, const HmgHierarchy* H, const Matrix* AT, size_t k) {
  const bsgpu_solver_config& cfg = t.cfg;
  Ctx& c = *t.ctx;
  const std::string lv = "HMG" + std::to_string(k);
  const Matrix* A64 = H->levels[k].Aref;
  if (k + 1 == H->levels.size()) {
    if (H->n_dense) {
      auto d = std::make_unique<DenseDirectT<T>>(H->dense_inv, H->n_dense);
      d->trace = c.trace_id(lv + ".DenseDirect");
      return d;
    }
    Term ct;
    ct.mode = 1;
    ct.tol = cfg.coarse_tol;
    ct.max_iter = cfg.coarse_max_iter;
    ct.min_iter = 0;
    auto pcg = std::make_unique<PCGT<T>>(c, A64, AT, true, ct);
    pcg->trace = c.trace_id(lv + ".CoarsePCG");
    return pcg;
  }
  Term ht;
  if (k == 0) {
    ht.mode = 1;
    ht.tol = cfg.coarse_tol;
    ht.max_iter = cfg.coarse_max_iter;
    ht.min_iter = 1;
  } else {
    ht.mode = 2;
    ht.max_iter = std::max(1, cfg.h_cycle);
  }
  auto omg = std::make_unique<OrthoMGT<T>>(c, AT, ht);
  omg->ortho.cap = std::max(2, t.cfg.ortho_max_krylov > 0 ? t.cfg.ortho_max_krylov : 96);
  omg->ortho.recalc_period = std::max(1, t.cfg.recalc_resi_period);
  omg->trace = c.trace_id(lv + ".OrthoMG");
  omg->sweeps = std::max(1, cfg.h_sweeps);
  omg->post = make_smoother<T>(c, A64, AT, cfg.h_smoother, cfg, lv);
  const HmgLevel& L = H->levels[k];
  auto tr = std::make_unique<TransferT<T>>(c, L.P.get(), L.R.get());
  tr->trace = c.trace_id(lv + ".Transfer");
  const Matrix* next64 = H->levels[k + 1].Aref;
  tr->lower = build_hmg_level<T>(t, H, level_matrix<T>(t, next64), k + 1);
  omg->coarse = std::move(tr);
  return omg;
}

// A64: FP64 level operator (factorisations are computed from it); AT: the same operator in the precision T the
// level runs in (AT == A64 for T = double).
template <typename T>
std::unique_ptr<Solver<T>> build_level(Tree& t, const Matrix* A64, const Matrix* AT, int level, const Term& top) {
  const bsgpu_solver_config& cfg = t.cfg;
  Ctx& c = *t.ctx;
  if (level == cfg.n_levels - 1) {
    if (cfg.coarse_kind == BSGPU_COARSE_HMG) {
      require(t.info.hprol != nullptr && !t.info.hprol->empty() && t.info.top != nullptr,
              "the h-multigrid coarse solve needs h-level prolongations (bsgpu_mgop_add_h_level)");
      t.hmgs.emplace_back(hmg_setup(*A64, *t.info.top, t.info.L, cfg.level_keep[level], *t.info.hprol,
                                    cfg.dense_limit, c.st));
      return build_hmg_level<T>(t, t.hmgs.back().get(), AT, 0);
    }
    if (cfg.coarse_kind == BSGPU_COARSE_AMG) {
      t.amgs.emplace_back(amg_setup(*A64, std::max(1, cfg.h_levels), cfg.dense_limit, c.st));
      Term ct;
      ct.mode = 1;
      ct.tol = cfg.coarse_tol;
      ct.max_iter = cfg.coarse_max_iter;
      auto s = std::make_unique<AmgPcgT<T>>(t, t.amgs.back().get(), AT, std::max(1, cfg.h_sweeps), ct);
      s->trace = c.trace_id("L" + std::to_string(level) + ".AmgPCG");
      return s;
    }
    if (cfg.h_levels > 0 && A64->uniform && A64->Np == 1) return build_hlevel<T>(t, A64, AT, 0);
    if (cfg.coarse_kind == BSGPU_COARSE_DENSE) {
      require(A64->uniform && A64->Np == 1, "the dense coarse solve needs a p = 0 last level", BSGPU_ERR_UNSUPPORTED);
      require(A64->N <= 4096, "the dense coarse solve is limited to 4096 unknowns", BSGPU_ERR_UNSUPPORTED);
      auto d = std::make_unique<DenseDirectT<T>>(c, A64);
      d->trace = c.trace_id("L" + std::to_string(level) + ".DenseDirect");
      return d;
    }
    require(cfg.coarse_kind == BSGPU_COARSE_PCG, "unknown coarse solver", BSGPU_ERR_UNSUPPORTED);
    Term ct;
    ct.mode = 1;
    ct.tol = cfg.coarse_tol;
    ct.max_iter = cfg.coarse_max_iter;
    ct.min_iter = 0;
    auto pcg = std::make_unique<PCGT<T>>(c, A64, AT, true, ct);
    pcg->trace = c.trace_id("L" + std::to_string(level) + ".CoarsePCG");
    return pcg;
  }
  Term lt = top;
  if (level > 0) {
    lt.mode = 3;
    lt.reduction = cfg.sub_reduction;
    lt.max_iter = cfg.sub_max_iter;
  }
  const std::string lv = "L" + std::to_string(level);
  auto omg = std::make_unique<OrthoMGT<T>>(c, AT, lt);
  omg->ortho.cap = std::max(2, t.cfg.ortho_max_krylov > 0 ? t.cfg.ortho_max_krylov : 96);
  omg->ortho.recalc_period = std::max(1, t.cfg.recalc_resi_period);
  omg->trace = c.trace_id(lv + ".OrthoMG");
  if (level == 0 && t.net && (cfg.learned & BSGPU_LEARNED_PRESMOOTH)) {
    omg->pre = std::make_unique<LearnedPrecondT<T>>(c, t.net.get());
    omg->pre->trace = c.trace_id(lv + ".LearnedPreSmoother");
    omg->pre_on = &t.learned_on;
  }
  omg->sweeps = cfg.post_sweeps;
  omg->post = make_smoother<T>(c, A64, AT, cfg.smoother, cfg, lv);
  const int keep = cfg.level_keep[level + 1];
  t.owned.emplace_back(matrix_restrict(*A64, keep, c.st));
  const Matrix* sub64 = t.owned.back().get();
  const Matrix* subT = level_matrix<T>(t, sub64);
  auto gr = std::make_unique<GridAndDegT<T>>(c, AT, subT, keep);
  gr->trace = c.trace_id(lv + ".GridAndDegRestriction");
  gr->lower = build_level<T>(t, sub64, subT, level + 1, top);
  omg->coarse = std::move(gr);
  return omg;
}

}  // namespace

RecordedSolve* recorded_form(Tree& t) {
  auto* f = dynamic_cast<FlexGMRES*>(t.top.get());
  return (f && f->whole) ? static_cast<RecordedSolve*>(f) : nullptr;
}

Tree* build_tree(const Matrix* A, const bsgpu_solver_config& cfg, const OperatorInfo& info) {
  require(!A->single, "the solver operator must be FP64");
  require(cfg.n_levels >= 1 && cfg.n_levels <= 8, "n_levels must be in 1..8");
  auto t = std::make_unique<Tree>();
  t->ctx = std::make_unique<Ctx>();
  t->ctx->autotune = cfg.autotune != 0;
  if (cfg.solver == BSGPU_SOLVER_FGMRES_PMG || cfg.solver == BSGPU_SOLVER_SOFTGMRES) t->ctx->tune(*A, 0);
  const char* tr = std::getenv("BSGPU_TRACE");
  t->ctx->tracing = tr != nullptr && tr[0] != '\0' && tr[0] != '0';
  t->A = A;
  t->cfg = cfg;
  t->info = info;
  Term top;
  top.mode = cfg.termination == BSGPU_TERM_RELATIVE ? 1 : 0;
  top.tol = cfg.tol;
  top.max_iter = cfg.max_iter;
  top.min_iter = cfg.min_iter;
  if (cfg.solver != BSGPU_SOLVER_SOFTPCG && cfg.solver != BSGPU_SOLVER_BLOCKJACOBI &&
      !(cfg.solver == BSGPU_SOLVER_SOFTGMRES && cfg.n_levels <= 1)) {
    require(cfg.level_keep[0] == A->Np, "level_keep[0] must equal Np");
    for (int l = 1; l < cfg.n_levels; ++l)
      require(cfg.level_keep[l] >= 1 && cfg.level_keep[l] < cfg.level_keep[l - 1], "level_keep must decrease");
  }
  const bool mixed = cfg.precision == BSGPU_PRECISION_MIXED;
  require(cfg.graph >= 0 && cfg.graph <= 2, "graph must be 0, 1 or 2");
  if (cfg.learned != BSGPU_LEARNED_OFF) {
    require(cfg.solver == BSGPU_SOLVER_FGMRES_PMG, "the learned stage needs the FGMRES + p-multigrid solver");
    require(info.nbr != nullptr && info.nfaces > 0, "the learned stage needs the cell graph (bsgpu_mgop_set_cell_neighbours)");
    require(A->uniform, "the learned stage needs one species per cell", BSGPU_ERR_UNSUPPORTED);
    require((int64_t)info.nbr->size() == A->nb * info.nfaces, "cell neighbour table size mismatch");
    if (info.nfeat) require((int64_t)info.feats->size() == A->nb * info.nfeat, "cell feature table size mismatch");
    t->net = std::make_unique<LearnedNet>();
    if (cfg.learned_hidden > 0) {
      require(cfg.learned_hidden % 16 == 0 && cfg.learned_hidden <= 128, "learned_hidden must be a multiple of 16, <= 128");
      t->net->H = cfg.learned_hidden;
    }
    t->net->init(A->Np, A->nb, info.nfaces, info.nfeat, info.nbr->data(), info.nfeat ? info.feats->data() : nullptr,
                 0x5eed);
  }
  switch (cfg.solver) {
    case BSGPU_SOLVER_SOFTPCG: {
      require(!mixed, "mixed precision is available for the FGMRES preconditioner", BSGPU_ERR_UNSUPPORTED);
      t->top = std::make_unique<PCGT<double>>(*t->ctx, A, A, cfg.bj_iters >= 0, top);
      t->top->trace = t->ctx->trace_id("SoftPCG");
      break;
    }
    case BSGPU_SOLVER_BLOCKJACOBI:
      require(!mixed, "mixed precision is available for the FGMRES preconditioner", BSGPU_ERR_UNSUPPORTED);
      t->top = make_smoother<double>(*t->ctx, A, A, cfg.smoother, cfg, "");
      break;
    case BSGPU_SOLVER_ORTHOMG:
      require(!mixed, "mixed precision is available for the FGMRES preconditioner", BSGPU_ERR_UNSUPPORTED);
      t->top = build_level<double>(*t, A, A, 0, top);
      break;
    case BSGPU_SOLVER_FGMRES_PMG: {
      require(cfg.max_krylov >= 1 && cfg.max_krylov <= 256, "max_krylov must be in 1..256");
      Term one;
      one.mode = 2;
      one.max_iter = 1;
      auto f = std::make_unique<FlexGMRES>(*t->ctx, A, cfg.max_krylov, top);
      f->trace = t->ctx->trace_id("FlexGMRES");
      if (mixed) {
        auto ad = std::make_unique<MixedAdapter>(A->N);
        auto lvl = build_level<float>(*t, A, level_matrix<float>(*t, A), 0, one);
        if (cfg.graph) {
          require(lvl->graphable(), "the V-cycle cannot be recorded as a graph with this coarse solver",
                  BSGPU_ERR_UNSUPPORTED);
          auto g = std::make_unique<GraphedT<float>>(A->N, std::move(lvl));
          g->Xs = ad->x32.p;
          g->Bs = ad->b32.p;
          g->key_src = &t->learned_on;
          if (cfg.graph == 1) g->ensure(*t->ctx);  // recorded at set-up, not in the first solve
          ad->inner = std::move(g);
        } else {
          ad->inner = std::move(lvl);
        }
        f->pc = std::move(ad);
      } else {
        auto lvl = build_level<double>(*t, A, A, 0, one);
        if (cfg.graph) {
          require(lvl->graphable(), "the V-cycle cannot be recorded as a graph with this coarse solver",
                  BSGPU_ERR_UNSUPPORTED);
          auto g = std::make_unique<GraphedT<double>>(A->N, std::move(lvl));
          g->key_src = &t->learned_on;
          if (cfg.graph == 1) g->ensure(*t->ctx);  // recorded at set-up, not in the first solve
          f->pc = std::move(g);
        } else {
          f->pc = std::move(lvl);
        }
      }
      f->tree = t.get();
      if (t->net && (cfg.learned & BSGPU_LEARNED_FGMRES)) {
        f->pc2 = std::make_unique<LearnedPrecondT<double>>(*t->ctx, t->net.get());
        f->pc2->trace = t->ctx->trace_id("LearnedStage");
        f->stall = cfg.learned_stall > 0 ? cfg.learned_stall : 0.99;
      }
      // cfg.graph == 2: the handle records the whole solve (recorded_form) at set-up
      f->whole = cfg.graph == 2;
      t->top = std::move(f);
      break;
    }
    case BSGPU_SOLVER_SOFTGMRES: {
      require(cfg.max_krylov >= 1 && cfg.max_krylov <= 256, "max_krylov must be in 1..256");
      Term one;
      one.mode = 2;
      one.max_iter = 1;
      // left preconditioning needs the same operator M^{-1} in every application: a block smoother, not the
      // p-multigrid V-cycle (its ORTHOMIN minimisation and capped coarse solves vary between calls; FlexGMRES
      // is the Krylov method for it)
      require(cfg.n_levels <= 1, "SoftGMRES takes a block-smoother preconditioner (n_levels <= 1); use "
              "FlexGMRES for the p-multigrid V-cycle", BSGPU_ERR_UNSUPPORTED);
      require(!mixed, "mixed precision is available for the FlexGMRES p-multigrid preconditioner",
              BSGPU_ERR_UNSUPPORTED);
      (void)one;
      auto f = std::make_unique<SoftGMRES>(*t->ctx, A, cfg.max_krylov, top);
      f->trace = t->ctx->trace_id("SoftGMRES");
      if (cfg.bj_iters >= 0) f->pc = make_smoother<double>(*t->ctx, A, A, cfg.smoother, cfg, "");
      t->top = std::move(f);
      break;
    }
    default:
      throw Error(BSGPU_ERR_ARGUMENT, "unknown solver kind");
  }
  BSGPU_CUDA(cudaStreamSynchronize(t->ctx->st));
  return t.release();
}

}  // namespace bsgpu

namespace bsgpu {

double train_learned(Tree& t, int n_rhs, int steps, double lr, uint64_t seed) {
  require(t.net != nullptr, "the solver was created without the learned stage (cfg.learned = 0)");
  require(n_rhs >= 1 && steps >= 1 && lr > 0, "n_rhs, steps and lr must be positive");
  Ctx& c = *t.ctx;
  const int64_t N = t.A->N;
  // 1. training residuals generated by the solver itself: Arnoldi vectors of solves with random right-hand sides
  std::vector<DBuf<double>> pool;
  const bool was_on = t.learned_on;
  t.learned_on = false;
  t.collect = &pool;
  // cfg.learned_pairs residuals in total (default 12 per right-hand side), spread evenly over the solves
  const size_t pairs = t.cfg.learned_pairs > 0 ? (size_t)t.cfg.learned_pairs : (size_t)n_rhs * 12;
  const size_t per = (pairs + n_rhs - 1) / n_rhs;
  DBuf<double> b(std::max<int64_t>(N, 1)), x(std::max<int64_t>(N, 1));
  for (int k = 0; k < n_rhs && pool.size() < pairs; ++k) {
    fill_random(b.p, N, seed + 7919ull * k, c.st);
    fill(0.0, x.p, N, c.st);
    t.collect_cap = std::min(pairs, pool.size() + per);
    t.top->solve(c, x.p, b.p, true);
  }
  t.collect = nullptr;
  t.learned_pool = (int)pool.size();
  require(!pool.empty(), "no training residuals were generated");
  // 2. Adam on the energy-norm loss
  DBuf<double> z(N), Az(N), g(N);
  double* scal = c.scal(8);
  double loss_acc = 0.0;
  int loss_n = 0;
  for (int s = 0; s < steps; ++s) {
    learned_train_step(*t.net, *t.A, pool[s % pool.size()].p, z.p, Az.p, g.p, c.red, scal, lr, c.st);
    if (s >= steps - 8) {
      c.fetch(scal, 5);
      const double* h = c.hscal + (scal - c.dscal.p);
      loss_acc += (h[3] - 2.0 * h[4]) / h[2];
      ++loss_n;
    }
  }
  BSGPU_CUDA(cudaStreamSynchronize(c.st));
  learned_check(*t.net, c.st);
  t.net->trained = true;
  t.learned_on = true;
  (void)was_on;
  return loss_n ? loss_acc / loss_n : 0.0;
}

}  // namespace bsgpu
