// extern "C" boundary of the library (declarations and reference citations in include/bsgpu.h).
#include <algorithm>
#include <atomic>
#include <cstring>
#include <exception>
#include <memory>

#include "solvers.cuh"

struct bsgpu_matrix_s {
  std::unique_ptr<bsgpu::Matrix> m;
  bool borrowed = false;
  bsgpu::Matrix* get() { return m.get(); }
};

struct bsgpu_mgop_s {
  bsgpu::Matrix* A = nullptr;  // original operator (owned by the caller's handle)
  std::unique_ptr<bsgpu::Matrix> Aop;
  bsgpu::DBuf<double> L;       // per-block left change of basis, row-major
  int mode = 0;
  bsgpu_matrix_s op_handle;    // borrowed handle returned by bsgpu_mgop_get_operator
  std::vector<bsgpu::HostBsr> hprol;  // h-level prolongations below the coarsest p-level
  int nfaces = 0, nfeat = 0;          // cell graph and features for the learned stage
  std::vector<int32_t> nbr;
  std::vector<float> feats;
  const bsgpu::Matrix* op() const { return mode == BSGPU_COB_EYE ? A : Aop.get(); }
};

struct bsgpu_solver_s {
  bsgpu_mgop_s* op = nullptr;
  std::unique_ptr<bsgpu::Tree> tree;
  bsgpu::DBuf<double> X, B, Xt, Bt;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  std::vector<double> history;
  double* lscal = nullptr;  // device scalars of the learned-stage entry points
  // cfg.graph == 2: the whole solve (change of basis, FlexGMRES with its V-cycle, back-transform) recorded once on
  // the staging vectors X, B and replayed by one graph launch
  cudaGraphExec_t rec_exec = nullptr;
  long long rec_top = 0;  // kernels at the top level of the recording
  int rec_key = -1;
  int device = 0;         // the device the handle's memory lives on
  ~bsgpu_solver_s() {
    if (rec_exec) cudaGraphExecDestroy(rec_exec);
  }
};

// Many handles recorded as one CUDA graph: every handle's recorded solve is one branch of the graph, all branches
// run concurrently from one launch.
struct bsgpu_batch_s {
  std::vector<bsgpu_solver_s*> s;
  std::vector<int> keys;
  cudaStream_t st = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long top = 0;
  cudaEvent_t start = nullptr;
  std::vector<cudaEvent_t> done;  // recorded at the end of every branch (external event nodes)
  bsgpu::DBuf<const double*> src;
  bsgpu::DBuf<double*> dst;
  bsgpu::DBuf<int64_t> len;
  const double** h_src = nullptr;  // pinned staging of the copy tables
  double** h_dst = nullptr;
  ~bsgpu_batch_s() {
    if (exec) cudaGraphExecDestroy(exec);
    for (cudaEvent_t e : done) cudaEventDestroy(e);
    if (start) cudaEventDestroy(start);
    if (st) cudaStreamDestroy(st);
    if (h_src) cudaFreeHost(h_src);
    if (h_dst) cudaFreeHost(h_dst);
  }
};

namespace bsgpu {

thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }
static std::atomic<unsigned long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
void add_launches(long long n) { g_launches.fetch_add((unsigned long long)n, std::memory_order_relaxed); }
unsigned long long launches_now() { return g_launches.load(); }
const Matrix* matrix_from_handle(bsgpu_matrix_t A) { return A ? A->get() : nullptr; }

namespace {

template <typename F>
int guarded(F&& f) {
  try {
    f();
    return BSGPU_OK;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return BSGPU_ERR_NOMEM;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return BSGPU_ERR_ARGUMENT;
  }
}

// transformed RHS / initial guess and back-transform (MultigridOperator.TransformRhsInto / TransformSolFrom)
void to_transformed(bsgpu_mgop_s* op, const double* X, const double* B, double* Xt, double* Bt, cudaStream_t st) {
  const Matrix& A = *op->A;
  if (op->mode == BSGPU_COB_EYE) {
    BSGPU_CUDA(cudaMemcpyAsync(Bt, B, A.N * 8, cudaMemcpyDeviceToDevice, st));
    BSGPU_CUDA(cudaMemcpyAsync(Xt, X, A.N * 8, cudaMemcpyDeviceToDevice, st));
    return;
  }
  block_gemv(op->L.p, A.doff.p, A.len.p, A.i0.p, A.row2blk.p, A.uniform ? A.Np : 0, false, B, Bt, A.N, st);
  block_trsv_lt(A, op->L.p, X, Xt, st);
}

void from_transformed(bsgpu_mgop_s* op, const double* Xt, double* X, cudaStream_t st) {
  const Matrix& A = *op->A;
  if (op->mode == BSGPU_COB_EYE) {
    BSGPU_CUDA(cudaMemcpyAsync(X, Xt, A.N * 8, cudaMemcpyDeviceToDevice, st));
    return;
  }
  block_gemv(op->L.p, A.doff.p, A.len.p, A.i0.p, A.row2blk.p, A.uniform ? A.Np : 0, true, Xt, X, A.N, st);
}

// The recorded solve of a handle: staging vectors X, B -> transformed basis, FlexGMRES, back into X.
void record_branch(bsgpu_solver_s* s, RecordedSolve* r) {
  Ctx& c = *s->tree->ctx;
  to_transformed(s->op, s->X.p, s->B.p, s->Xt.p, s->Bt.p, c.st);
  r->record(c, s->Xt.p, s->Bt.p);
  from_transformed(s->op, s->Xt.p, s->X.p, c.st);
}

// (Re)records the handle's whole solve when there is none or the learned stage was switched since.
void ensure_recorded(bsgpu_solver_s* s) {
  RecordedSolve* r = recorded_form(*s->tree);
  if (!r || (s->rec_exec && r->key() == s->rec_key)) return;
  if (s->rec_exec) {
    cudaGraphExecDestroy(s->rec_exec);
    s->rec_exec = nullptr;
  }
  Ctx& c = *s->tree->ctx;
  r->prepare(c);
  c.capture_begin();
  cudaGraph_t g = nullptr;
  try {
    record_branch(s, r);
  } catch (...) {
    c.capture_abort();
    cudaStreamEndCapture(c.st, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  s->rec_top = c.capture_end(&g);
  const cudaError_t e = cudaGraphInstantiate(&s->rec_exec, g, 0);
  cudaGraphDestroy(g);
  BSGPU_CUDA(e);
  s->rec_key = r->key();
}

void fill_stats(bsgpu_solver_s* s, bsgpu_solve_stats* stats, double seconds) {
  Tree& t = *s->tree;
  s->history = t.top->history;
  if (!stats) return;
  stats->iterations = t.top->this_level_iterations;
  stats->nested = t.top->nested();
  stats->converged = t.top->converged ? 1 : 0;
  stats->n_history = (int32_t)s->history.size();
  stats->res0 = s->history.empty() ? 0.0 : s->history.front();
  stats->res = s->history.empty() ? 0.0 : s->history.back();
  stats->seconds = seconds;
}

void solve_device(bsgpu_solver_s* s, double* dX, const double* dB, bsgpu_solve_stats* stats) {
  Tree& t = *s->tree;
  Ctx& c = *t.ctx;
  const int64_t N = s->op->A->N;
  RecordedSolve* rec = recorded_form(t);
  if (rec && !c.tracing && !t.collect) {
    ensure_recorded(s);
    BSGPU_CUDA(cudaEventRecord(s->e0, c.st));
    if (N && dX != s->X.p) BSGPU_CUDA(cudaMemcpyAsync(s->X.p, dX, N * 8, cudaMemcpyDeviceToDevice, c.st));
    if (N && dB != s->B.p) BSGPU_CUDA(cudaMemcpyAsync(s->B.p, dB, N * 8, cudaMemcpyDeviceToDevice, c.st));
    BSGPU_CUDA(cudaGraphLaunch(s->rec_exec, c.st));
    add_launches(s->rec_top);
    c.graph_ran = true;
    if (N && dX != s->X.p) BSGPU_CUDA(cudaMemcpyAsync(dX, s->X.p, N * 8, cudaMemcpyDeviceToDevice, c.st));
    BSGPU_CUDA(cudaEventRecord(s->e1, c.st));
    rec->queue_result(c, c.st);
    BSGPU_CUDA(cudaStreamSynchronize(c.st));
    rec->take_result(c);
    c.flush_graph_counts();  // raises an error the device recorded
    if (t.net) learned_check(*t.net, c.st);
    float ms = 0;
    BSGPU_CUDA(cudaEventElapsedTime(&ms, s->e0, s->e1));
    fill_stats(s, stats, ms * 1e-3);
    return;
  }
  BSGPU_CUDA(cudaEventRecord(s->e0, c.st));
  to_transformed(s->op, dX, dB, s->Xt.p, s->Bt.p, c.st);
  t.top->this_level_iterations = 0;
  t.top->solve(c, s->Xt.p, s->Bt.p, false);
  from_transformed(s->op, s->Xt.p, dX, c.st);
  BSGPU_CUDA(cudaEventRecord(s->e1, c.st));
  BSGPU_CUDA(cudaEventSynchronize(s->e1));
  c.flush_graph_counts();
  if (t.net) learned_check(*t.net, c.st);
  float ms = 0;
  BSGPU_CUDA(cudaEventElapsedTime(&ms, s->e0, s->e1));
  fill_stats(s, stats, ms * 1e-3);
  (void)N;
}

}  // namespace
}  // namespace bsgpu

using namespace bsgpu;

extern "C" {

BSGPU_API int bsgpu_get_version(int* major, int* minor) {
  if (major) *major = 0;
  if (minor) *minor = 1;
  return BSGPU_OK;
}

BSGPU_API int bsgpu_get_launch_count(uint64_t* n) {
  if (!n) return BSGPU_ERR_ARGUMENT;
  *n = g_launches.load();
  return BSGPU_OK;
}

BSGPU_API int bsgpu_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return BSGPU_ERR_ARGUMENT;
  std::strncpy(buf, g_last_error.c_str(), len - 1);
  buf[len - 1] = '\0';
  return BSGPU_OK;
}

BSGPU_API int bsgpu_set_device(int device) {
  return guarded([&] { BSGPU_CUDA(cudaSetDevice(device)); });
}

BSGPU_API int bsgpu_matrix_autotune(bsgpu_matrix_t A) {
  return guarded([&] {
    require(A != nullptr && A->get() != nullptr, "null matrix");
    autotune(*A->get(), 0, nullptr, nullptr);
    BSGPU_CUDA(cudaStreamSynchronize(nullptr));
  });
}

BSGPU_API int bsgpu_autotune_report(char* buf, size_t len) {
  return guarded([&] {
    require(buf != nullptr && len > 0, "null argument");
    const std::string r = autotune_report();
    std::strncpy(buf, r.c_str(), len - 1);
    buf[len - 1] = '\0';
  });
}

BSGPU_API int bsgpu_matrix_create(bsgpu_matrix_t* A, int64_t nb, int32_t Np, const int32_t* nspc,
                                  const int64_t* row_ptr, const int32_t* col_idx, const double* values,
                                  int32_t flags) {
  return guarded([&] {
    require(A != nullptr, "null handle pointer");
    auto h = std::make_unique<bsgpu_matrix_s>();
    h->m.reset(matrix_create(nb, Np, nspc, row_ptr, col_idx, values, flags));
    *A = h.release();
  });
}

BSGPU_API int bsgpu_assemble_sip_cartesian(bsgpu_matrix_t* A, int32_t D, const int32_t* shape, double lo, double hi,
                                           int32_t p, double penalty, const double* nu, int32_t flags) {
  return guarded([&] {
    require(A != nullptr && shape != nullptr, "null argument");
    require(flags == BSGPU_HOST_POINTERS || flags == BSGPU_DEVICE_POINTERS, "bad pointer flag");
    auto h = std::make_unique<bsgpu_matrix_s>();
    h->m.reset(assemble_sip_cartesian(D, shape, lo, hi, p, penalty, nu, flags == BSGPU_DEVICE_POINTERS));
    *A = h.release();
  });
}

BSGPU_API int bsgpu_sip_templates(int32_t D, int32_t p, const double* h, double* out, int64_t cap, int64_t* n) {
  return guarded([&] {
    require(h != nullptr, "null argument");
    const std::vector<double> T = sip_templates(D, p, h);
    if (n) *n = (int64_t)T.size();
    if (out) {
      require(cap >= (int64_t)T.size(), "output buffer too small");
      std::copy(T.begin(), T.end(), out);
    }
  });
}

BSGPU_API int bsgpu_schwarz_blocks(int64_t nb, const int64_t* row_ptr, const int32_t* col_idx, int64_t parts,
                                   int32_t overlap, int64_t* ptr, int32_t* cells, int64_t* nblocks, int64_t* total) {
  return guarded([&] {
    require(nb >= 0 && row_ptr != nullptr && (col_idx != nullptr || nb == 0), "null argument");
    Matrix M;  // host structure only: no device memory is touched
    M.nb = nb;
    M.h_rp.assign(row_ptr, row_ptr + nb + 1);
    M.nnzb = M.h_rp[nb];
    M.h_ci.assign(col_idx, col_idx + M.nnzb);
    for (int64_t k = 0; k < M.nnzb; ++k)
      require(M.h_ci[k] >= 0 && M.h_ci[k] < nb, "column index out of range");
    auto blocks = schwarz_partition(M, parts > 0 ? parts : std::max<int64_t>(1, (nb + 7) / 8));
    schwarz_extend(M, blocks, overlap);
    int64_t n = 0;
    for (auto& bl : blocks) n += (int64_t)bl.size();
    if (nblocks) *nblocks = (int64_t)blocks.size();
    if (total) *total = n;
    if (ptr && cells) {
      int64_t o = 0;
      ptr[0] = 0;
      for (size_t b = 0; b < blocks.size(); ++b) {
        for (int32_t c : blocks[b]) cells[o++] = c;
        ptr[b + 1] = o;
      }
    }
  });
}

BSGPU_API int bsgpu_ilu_wavefronts(int64_t nb, const int64_t* row_ptr, const int32_t* col_idx, int64_t* level_ptr,
                                   int32_t* rows, int64_t* nlevels) {
  return guarded([&] {
    require(nb >= 0 && row_ptr != nullptr && (col_idx != nullptr || nb == 0), "null argument");
    Matrix M;  // host structure only: no device memory is touched
    M.nb = nb;
    M.h_rp.assign(row_ptr, row_ptr + nb + 1);
    M.nnzb = M.h_rp[nb];
    M.h_ci.assign(col_idx, col_idx + M.nnzb);
    for (int64_t k = 0; k < M.nnzb; ++k)
      require(M.h_ci[k] >= 0 && M.h_ci[k] < nb, "column index out of range");
    std::vector<int64_t> lptr;
    std::vector<int32_t> order;
    ilu_wavefronts(M, lptr, order);
    if (nlevels) *nlevels = (int64_t)lptr.size() - 1;
    if (level_ptr) std::copy(lptr.begin(), lptr.end(), level_ptr);
    if (rows) std::copy(order.begin(), order.end(), rows);
  });
}

BSGPU_API int bsgpu_project_separable(int32_t D, const int32_t* shape, int32_t p, int32_t M, const double* coef,
                                      const double* tables, double* out, int32_t flags) {
  return guarded([&] {
    require(shape && out && (M == 0 || (coef && tables)), "null argument");
    require(flags == BSGPU_HOST_POINTERS || flags == BSGPU_DEVICE_POINTERS, "bad pointer flag");
    int64_t nc = 1;
    for (int d = 0; d < D && d < 3; ++d) nc *= std::max(shape[d], 1);
    const int64_t N = nc * (int64_t)modes_count(D, p);
    if (flags == BSGPU_DEVICE_POINTERS) {
      project_separable(D, shape, p, M, coef, tables, out, nullptr);
    } else {
      DBuf<double> d(std::max<int64_t>(N, 1));
      project_separable(D, shape, p, M, coef, tables, d.p, nullptr);
      BSGPU_CUDA(cudaMemcpy(out, d.p, N * 8, cudaMemcpyDeviceToHost));
    }
  });
}

BSGPU_API int bsgpu_matrix_destroy(bsgpu_matrix_t A) {
  return guarded([&] {
    if (A && !A->borrowed) delete A;
  });
}

BSGPU_API int bsgpu_matrix_get_info(bsgpu_matrix_t A, int64_t* nrows, int64_t* nb, int64_t* nnzb, int32_t* Np) {
  return guarded([&] {
    require(A && A->get(), "null matrix");
    const Matrix& M = *A->get();
    if (nrows) *nrows = M.N;
    if (nb) *nb = M.nb;
    if (nnzb) *nnzb = M.nnzb;
    if (Np) *Np = M.Np;
  });
}

BSGPU_API int bsgpu_matrix_read_values(bsgpu_matrix_t A, double* values, int32_t flags) {
  return guarded([&] {
    require(A && A->get() && values, "null argument");
    matrix_read_values(*A->get(), values, flags == BSGPU_DEVICE_POINTERS, nullptr);
  });
}

BSGPU_API int bsgpu_matrix_spmv(bsgpu_matrix_t A, double alpha, const double* x, double beta, double* y) {
  return guarded([&] {
    require(A && A->get() && x && y, "null argument");
    require(x != y, "In-Place computation is not supported.");
    const Matrix& M = *A->get();
    DBuf<double> dx(std::max<int64_t>(M.N, 1)), dy(std::max<int64_t>(M.N, 1));
    if (M.N) {
      BSGPU_CUDA(cudaMemcpy(dx.p, x, M.N * 8, cudaMemcpyHostToDevice));
      if (beta != 0.0) BSGPU_CUDA(cudaMemcpy(dy.p, y, M.N * 8, cudaMemcpyHostToDevice));
    }
    spmv(M, alpha, dx.p, beta, beta != 0.0 ? dy.p : nullptr, dy.p, nullptr);
    if (M.N) BSGPU_CUDA(cudaMemcpy(y, dy.p, M.N * 8, cudaMemcpyDeviceToHost));
  });
}

BSGPU_API int bsgpu_matrix_spmv_device(bsgpu_matrix_t A, double alpha, const double* x, double beta, double* y,
                                       void* stream) {
  return guarded([&] {
    require(A && A->get() && x && y, "null argument");
    require(x != y, "In-Place computation is not supported.");
    spmv(*A->get(), alpha, x, beta, beta != 0.0 ? y : nullptr, y, (cudaStream_t)stream);
  });
}

BSGPU_API int bsgpu_matrix_create_single(bsgpu_matrix_t A, bsgpu_matrix_t* A32) {
  return guarded([&] {
    require(A && A->get() && A32, "null argument");
    auto h = std::make_unique<bsgpu_matrix_s>();
    h->m.reset(matrix_to_single(*A->get(), nullptr));
    *A32 = h.release();
  });
}

BSGPU_API int bsgpu_matrix_spmv_device_f32(bsgpu_matrix_t A32, float alpha, const float* x, float beta, float* y,
                                           void* stream) {
  return guarded([&] {
    require(A32 && A32->get() && x && y, "null argument");
    require(x != y, "In-Place computation is not supported.");
    spmv(*A32->get(), alpha, x, beta, beta != 0.0f ? y : nullptr, y, (cudaStream_t)stream);
  });
}

BSGPU_API int bsgpu_matrix_restrict(bsgpu_matrix_t A, int32_t keep, bsgpu_matrix_t* Asub) {
  return guarded([&] {
    require(A && A->get() && Asub, "null argument");
    auto h = std::make_unique<bsgpu_matrix_s>();
    h->m.reset(matrix_restrict(*A->get(), keep, nullptr));
    *Asub = h.release();
  });
}

BSGPU_API int bsgpu_mgop_create(bsgpu_mgop_t* op, bsgpu_matrix_t A, int32_t mode) {
  return guarded([&] {
    require(op && A && A->get(), "null argument");
    require(mode == BSGPU_COB_EYE || mode == BSGPU_COB_DIAG_BLOCK_EQUILIB, "unknown change-of-basis mode");
    require(!A->get()->single, "the operator must be FP64");
    auto h = std::make_unique<bsgpu_mgop_s>();
    h->A = A->get();
    h->mode = mode;
    if (mode == BSGPU_COB_DIAG_BLOCK_EQUILIB) {
      const Matrix& M = *h->A;
      std::vector<int64_t> o = diag_offsets(M);
      h->L.alloc(std::max<int64_t>(o.back(), 1));
      DBuf<int> err(1);
      BSGPU_CUDA(cudaMemset(err.p, 0, sizeof(int)));
      symminv_batched(M, h->L.p, err.p, nullptr);
      int herr = 0;
      BSGPU_CUDA(cudaMemcpy(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost));
      if (herr)
        throw Error(BSGPU_ERR_ARITHMETIC, "SymmInv: zero or indefinite pivot in diagonal block " + std::to_string(herr - 1));
      h->Aop.reset(matrix_like(M, false));
      change_of_basis_apply(M, h->L.p, *h->Aop, nullptr);
    }
    h->op_handle.m.reset(const_cast<Matrix*>(h->op()));
    h->op_handle.borrowed = true;
    *op = h.release();
  });
}

BSGPU_API int bsgpu_mgop_destroy(bsgpu_mgop_t op) {
  return guarded([&] {
    if (!op) return;
    op->op_handle.m.release();  // borrowed
    delete op;
  });
}

BSGPU_API int bsgpu_mgop_get_operator(bsgpu_mgop_t op, bsgpu_matrix_t* Aop) {
  return guarded([&] {
    require(op && Aop, "null argument");
    *Aop = &op->op_handle;
  });
}

BSGPU_API int bsgpu_mgop_add_h_level(bsgpu_mgop_t op, int32_t Np, int64_t nb_fine, int64_t nb_coarse,
                                     const int64_t* row_ptr, const int32_t* col_idx, const double* values) {
  return guarded([&] {
    require(op && row_ptr && (col_idx || nb_fine == 0) && (values || nb_fine == 0), "null argument");
    require(Np > 0 && nb_fine > 0 && nb_coarse > 0 && nb_coarse <= nb_fine, "bad h-level sizes");
    if (!op->hprol.empty())
      require(op->hprol.back().nb_cols == nb_fine, "h-level rows must equal the previous level's coarse blocks");
    HostBsr P;
    P.Np = Np;
    P.nb_rows = nb_fine;
    P.nb_cols = nb_coarse;
    P.rp.assign(row_ptr, row_ptr + nb_fine + 1);
    require(P.rp[0] == 0, "row_ptr[0] must be 0");
    for (int64_t i = 0; i < nb_fine; ++i) require(P.rp[i + 1] >= P.rp[i], "row_ptr must be non-decreasing");
    const int64_t nnzb = P.rp[nb_fine];
    P.ci.assign(col_idx, col_idx + nnzb);
    for (int32_t c : P.ci) require(c >= 0 && c < nb_coarse, "col_idx out of range");
    P.v.assign(values, values + nnzb * (int64_t)Np * Np);
    op->hprol.push_back(std::move(P));
  });
}

BSGPU_API int bsgpu_mgop_set_cell_neighbours(bsgpu_mgop_t op, int32_t nfaces, const int32_t* nbr) {
  return guarded([&] {
    require(op && nbr && nfaces > 0 && nfaces <= 16, "bad cell neighbour table");
    const int64_t nb = op->A->nb;
    for (int64_t i = 0; i < nb * nfaces; ++i) require(nbr[i] >= -1 && nbr[i] < nb, "neighbour index out of range");
    op->nfaces = nfaces;
    op->nbr.assign(nbr, nbr + nb * nfaces);
  });
}

BSGPU_API int bsgpu_mgop_set_cell_features(bsgpu_mgop_t op, int32_t nfeat, const float* feats) {
  return guarded([&] {
    require(op && (feats || nfeat == 0) && nfeat >= 0 && nfeat <= 64, "bad cell feature table");
    op->nfeat = nfeat;
    op->feats.assign(feats, feats + op->A->nb * (int64_t)nfeat);
  });
}

BSGPU_API int bsgpu_mgop_read_left_cob(bsgpu_mgop_t op, double* L) {
  return guarded([&] {
    require(op && L, "null argument");
    require(op->mode == BSGPU_COB_DIAG_BLOCK_EQUILIB, "no change of basis (mode Eye)");
    std::vector<int64_t> o = diag_offsets(*op->A);
    BSGPU_CUDA(cudaMemcpy(L, op->L.p, o.back() * 8, cudaMemcpyDeviceToHost));
  });
}

BSGPU_API int bsgpu_solver_config_default(bsgpu_solver_config* cfg) {
  return guarded([&] {
    require(cfg != nullptr, "null config");
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->solver = BSGPU_SOLVER_FGMRES_PMG;
    cfg->termination = BSGPU_TERM_DEFAULT;
    cfg->tol = 1e-10;
    cfg->max_iter = 300;
    cfg->min_iter = 1;
    cfg->max_krylov = 30;
    cfg->n_levels = 1;
    cfg->post_sweeps = 10;
    cfg->bj_iters = 1;
    cfg->bj_omega = 1.0;
    cfg->coarse_kind = BSGPU_COARSE_PCG;
    cfg->coarse_tol = 1e-3;
    cfg->coarse_max_iter = 2000;
    cfg->sub_max_iter = 100;
    cfg->sub_reduction = 0.1;
    cfg->precision = BSGPU_PRECISION_FP64;
    cfg->h_levels = 0;
    cfg->h_sweeps = 3;
    cfg->h_cycle = 1;
    cfg->dense_limit = 1024;
    cfg->learned = BSGPU_LEARNED_OFF;
    cfg->learned_hidden = 64;
    cfg->learned_stall = 0.99;
    cfg->ortho_max_krylov = 96;
    cfg->recalc_resi_period = 1;
    cfg->learned_pairs = 0;
    cfg->graph = 0;
    cfg->autotune = 0;
    cfg->fp16_storage = 0;
    cfg->schwarz_parts = 0;
    cfg->schwarz_overlap = 1;
    cfg->schwarz_scaling = 0;
  });
}

BSGPU_API int bsgpu_solver_create(bsgpu_solver_t* s, bsgpu_mgop_t op, const bsgpu_solver_config* cfg) {
  return guarded([&] {
    require(s && op && cfg, "null argument");
    auto h = std::make_unique<bsgpu_solver_s>();
    h->op = op;
    OperatorInfo info;
    info.top = op->A;
    info.L = op->mode == BSGPU_COB_DIAG_BLOCK_EQUILIB ? op->L.p : nullptr;
    info.hprol = &op->hprol;
    info.nfaces = op->nfaces;
    info.nbr = op->nfaces ? &op->nbr : nullptr;
    info.nfeat = op->nfeat;
    info.feats = op->nfeat ? &op->feats : nullptr;
    h->tree.reset(build_tree(op->op(), *cfg, info));
    const int64_t N = std::max<int64_t>(op->A->N, 1);
    h->X.alloc(N); h->B.alloc(N); h->Xt.alloc(N); h->Bt.alloc(N);
    BSGPU_CUDA(cudaEventCreate(&h->e0));
    BSGPU_CUDA(cudaEventCreate(&h->e1));
    BSGPU_CUDA(cudaGetDevice(&h->device));
    ensure_recorded(h.get());  // cfg.graph == 2: the whole solve is recorded at set-up
    *s = h.release();
  });
}

BSGPU_API int bsgpu_batch_create(bsgpu_batch_t* b, const bsgpu_solver_t* solvers, int32_t n) {
  return guarded([&] {
    require(b && solvers && n >= 1, "null argument or empty batch");
    require(solvers[0] != nullptr, "null solver handle in the batch");
    int cur = 0;
    BSGPU_CUDA(cudaGetDevice(&cur));
    require(cur == solvers[0]->device, "the current device must be the batch members' device (bsgpu_set_device)");
    auto h = std::make_unique<bsgpu_batch_s>();
    for (int32_t i = 0; i < n; ++i) {
      bsgpu_solver_s* s = solvers[i];
      require(s != nullptr, "null solver handle in the batch");
      for (int32_t q = 0; q < i; ++q) require(solvers[q] != s, "a solver handle appears twice in the batch");
      require(s->device == solvers[0]->device, "batch members must live on one device");
      RecordedSolve* r = recorded_form(*s->tree);
      require(r != nullptr, "batch members must be FlexGMRES solvers created with graph = 2", BSGPU_ERR_UNSUPPORTED);
      r->prepare(*s->tree->ctx);
      BSGPU_CUDA(cudaStreamSynchronize(s->tree->ctx->st));
      h->s.push_back(s);
      h->keys.push_back(r->key());
    }
    BSGPU_CUDA(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
    BSGPU_CUDA(cudaEventCreate(&h->start));
    h->done.assign(n, nullptr);
    for (auto& e : h->done) BSGPU_CUDA(cudaEventCreate(&e));
    h->src.alloc(3 * n);  // copy tables: right-hand sides in, initial guesses in, solutions out
    h->dst.alloc(3 * n);
    h->len.alloc(n);
    BSGPU_CUDA(cudaMallocHost(&h->h_src, 3 * n * sizeof(double*)));
    BSGPU_CUDA(cudaMallocHost(&h->h_dst, 3 * n * sizeof(double*)));
    std::vector<int64_t> lens(n);
    for (int32_t i = 0; i < n; ++i) lens[i] = h->s[i]->op->A->N;
    BSGPU_CUDA(cudaMemcpy(h->len.p, lens.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice));
    cudaEvent_t fork = nullptr, join = nullptr;
    BSGPU_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    BSGPU_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
    cudaGraph_t g = nullptr;
    BSGPU_CUDA(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeRelaxed));
    int32_t i = 0;
    try {
      BSGPU_CUDA(cudaEventRecord(fork, h->st));
      for (; i < n; ++i) {
        Ctx& c = *h->s[i]->tree->ctx;
        BSGPU_CUDA(cudaStreamWaitEvent(c.st, fork, 0));
        c.capture_join();
        record_branch(h->s[i], recorded_form(*h->s[i]->tree));
        h->top += c.capture_leave();
        BSGPU_CUDA(cudaEventRecordWithFlags(h->done[i], c.st, cudaEventRecordExternal));
        BSGPU_CUDA(cudaEventRecord(join, c.st));
        BSGPU_CUDA(cudaStreamWaitEvent(h->st, join, 0));
      }
    } catch (...) {
      if (i < n) {
        Ctx& c = *h->s[i]->tree->ctx;
        c.capture_abort();
        cudaEventRecord(join, c.st);
        cudaStreamWaitEvent(h->st, join, 0);
      }
      cudaStreamEndCapture(h->st, &g);
      if (g) cudaGraphDestroy(g);
      cudaEventDestroy(fork);
      cudaEventDestroy(join);
      throw;
    }
    BSGPU_CUDA(cudaStreamEndCapture(h->st, &g));
    cudaEventDestroy(fork);
    cudaEventDestroy(join);
    const cudaError_t e = cudaGraphInstantiate(&h->exec, g, 0);
    cudaGraphDestroy(g);
    BSGPU_CUDA(e);
    *b = h.release();
  });
}

BSGPU_API int bsgpu_batch_solve_device(bsgpu_batch_t b, double* const* X, const double* const* B,
                                       bsgpu_solve_stats* stats) {
  return guarded([&] {
    require(b && X && B, "null argument");
    const int n = (int)b->s.size();
    int cur = 0;
    BSGPU_CUDA(cudaGetDevice(&cur));
    require(cur == b->s[0]->device, "the current device must be the batch members' device (bsgpu_set_device)");
    for (int i = 0; i < n; ++i) {
      require(X[i] && B[i], "null vector in the batch");
      require((const double*)X[i] != B[i], "a batch member's X and B must be different vectors");
      require(recorded_form(*b->s[i]->tree)->key() == b->keys[i],
              "a batch member's learned stage was switched after the batch was recorded; create the batch again");
    }
    cudaStream_t st = b->st;
    // staging: B_i -> handle i's B, X_i -> handle i's X (initial guess) before the graph, handle i's X -> X_i after
    for (int i = 0; i < n; ++i) {
      b->h_src[i] = B[i];
      b->h_dst[i] = b->s[i]->B.p;
      b->h_src[n + i] = X[i];
      b->h_dst[n + i] = b->s[i]->X.p;
      b->h_src[2 * n + i] = b->s[i]->X.p;
      b->h_dst[2 * n + i] = X[i];
    }
    // ordered after the caller's work on the legacy default stream, as bsgpu_solver_solve_device
    BSGPU_CUDA(cudaEventRecord(b->start, cudaStreamLegacy));
    BSGPU_CUDA(cudaStreamWaitEvent(st, b->start, 0));
    BSGPU_CUDA(cudaMemcpyAsync(b->src.p, b->h_src, 3 * n * sizeof(double*), cudaMemcpyHostToDevice, st));
    BSGPU_CUDA(cudaMemcpyAsync(b->dst.p, b->h_dst, 3 * n * sizeof(double*), cudaMemcpyHostToDevice, st));
    batch_copy(b->src.p, b->dst.p, b->len.p, n, st);
    batch_copy(b->src.p + n, b->dst.p + n, b->len.p, n, st);
    BSGPU_CUDA(cudaEventRecord(b->start, st));
    BSGPU_CUDA(cudaGraphLaunch(b->exec, st));
    add_launches(b->top);
    batch_copy(b->src.p + 2 * n, b->dst.p + 2 * n, b->len.p, n, st);
    for (int i = 0; i < n; ++i) recorded_form(*b->s[i]->tree)->queue_result(*b->s[i]->tree->ctx, st);
    BSGPU_CUDA(cudaStreamSynchronize(st));
    // results of every member first, then the first error any of them recorded
    std::exception_ptr first;
    for (int i = 0; i < n; ++i) {
      bsgpu_solver_s* s = b->s[i];
      Ctx& c = *s->tree->ctx;
      recorded_form(*s->tree)->take_result(c);
      c.graph_ran = true;
      float ms = 0;
      BSGPU_CUDA(cudaEventElapsedTime(&ms, b->start, b->done[i]));
      fill_stats(s, stats ? stats + i : nullptr, ms * 1e-3);
      try {
        c.flush_graph_counts();
      } catch (...) {
        if (!first) first = std::current_exception();
      }
    }
    if (first) std::rethrow_exception(first);
  });
}

BSGPU_API int bsgpu_batch_destroy(bsgpu_batch_t b) {
  return guarded([&] { delete b; });
}

BSGPU_API int bsgpu_solver_destroy(bsgpu_solver_t s) {
  return guarded([&] {
    if (!s) return;
    if (s->e0) cudaEventDestroy(s->e0);
    if (s->e1) cudaEventDestroy(s->e1);
    delete s;
  });
}

BSGPU_API int bsgpu_solver_solve(bsgpu_solver_t s, double* X, const double* B, bsgpu_solve_stats* stats) {
  return guarded([&] {
    require(s && X && B, "null argument");
    const int64_t N = s->op->A->N;
    cudaStream_t st = s->tree->ctx->st;
    if (N) {
      BSGPU_CUDA(cudaMemcpyAsync(s->B.p, B, N * 8, cudaMemcpyHostToDevice, st));
      BSGPU_CUDA(cudaMemcpyAsync(s->X.p, X, N * 8, cudaMemcpyHostToDevice, st));
    }
    solve_device(s, s->X.p, s->B.p, stats);
    if (N) {
      BSGPU_CUDA(cudaMemcpyAsync(X, s->X.p, N * 8, cudaMemcpyDeviceToHost, st));
      BSGPU_CUDA(cudaStreamSynchronize(st));
    }
  });
}

BSGPU_API int bsgpu_solver_solve_device(bsgpu_solver_t s, double* X, const double* B, bsgpu_solve_stats* stats) {
  return guarded([&] {
    require(s && X && B, "null argument");
    // order after the caller's work on the legacy default stream only, so that solves driven from several host
    // threads (one handle each) overlap on the device
    BSGPU_CUDA(cudaEventRecord(s->e0, cudaStreamLegacy));
    BSGPU_CUDA(cudaStreamWaitEvent(s->tree->ctx->st, s->e0, 0));
    solve_device(s, X, B, stats);
  });
}

BSGPU_API int bsgpu_solver_train_learned(bsgpu_solver_t s, int32_t n_rhs, int32_t steps, double lr, uint64_t seed,
                                         double* loss) {
  return guarded([&] {
    require(s != nullptr, "null solver");
    const double l = train_learned(*s->tree, n_rhs, steps, lr, seed);
    if (loss) *loss = l;
  });
}

BSGPU_API int bsgpu_solver_set_tracing(bsgpu_solver_t s, int32_t on) {
  return guarded([&] {
    require(s != nullptr, "null solver");
    s->tree->ctx->tracing = on != 0;
    s->tree->ctx->graph_counts.clear();
    for (auto& e : s->tree->ctx->trace) {
      e.calls = 0;
      e.seconds = 0;
      e.iterations = 0;
    }
  });
}

BSGPU_API int bsgpu_solver_get_trace(bsgpu_solver_t s, char* buf, size_t len) {
  return guarded([&] {
    require(s != nullptr && buf != nullptr && len > 0, "null argument");
    std::string out = "[";
    char tmp[512];
    bool first = true;
    for (auto& e : s->tree->ctx->trace) {
      std::snprintf(tmp, sizeof(tmp), "%s{\"name\": \"%s\", \"calls\": %ld, \"seconds\": %.6f, \"iterations\": %ld}",
                    first ? "" : ", ", e.name.c_str(), e.calls, e.seconds, e.iterations);
      out += tmp;
      first = false;
    }
    // executions of the conditional bodies of the recorded V-cycle (graph mode)
    for (auto& g : s->tree->ctx->graph_counts) {
      std::snprintf(tmp, sizeof(tmp), "%s{\"name\": \"graph: %s\", \"calls\": %llu, \"seconds\": 0, \"iterations\": 0}",
                    first ? "" : ", ", g.first.c_str(), g.second);
      out += tmp;
      first = false;
    }
    out += "]";
    std::strncpy(buf, out.c_str(), len - 1);
    buf[len - 1] = '\0';
  });
}

static LearnedNet& learned_of(bsgpu_solver_t s) {
  require(s != nullptr, "null solver");
  require(s->tree->net != nullptr, "the solver was created without the learned stage (cfg.learned = 0)");
  return *s->tree->net;
}

BSGPU_API int bsgpu_solver_learned_info(bsgpu_solver_t s, int32_t* dims) {
  return guarded([&] {
    LearnedNet& n = learned_of(s);
    require(dims != nullptr, "null argument");
    const int32_t d[8] = {n.Np, n.nfaces, n.nextra, n.F, n.Fp, n.H, n.Op, s->tree->learned_pool};
    std::memcpy(dims, d, sizeof(d));
  });
}

BSGPU_API int bsgpu_solver_learned_get_weights(bsgpu_solver_t s, float* w1, float* w2, float* w3) {
  return guarded([&] {
    LearnedNet& n = learned_of(s);
    require(w1 && w2 && w3, "null argument");
    BSGPU_CUDA(cudaStreamSynchronize(s->tree->ctx->st));
    learned_get_weights(n, w1, w2, w3);
  });
}

BSGPU_API int bsgpu_solver_learned_set_weights(bsgpu_solver_t s, const float* w1, const float* w2, const float* w3) {
  return guarded([&] {
    LearnedNet& n = learned_of(s);
    require(w1 && w2 && w3, "null argument");
    BSGPU_CUDA(cudaStreamSynchronize(s->tree->ctx->st));
    learned_set_weights(n, w1, w2, w3);
  });
}

BSGPU_API int bsgpu_solver_learned_apply(bsgpu_solver_t s, const double* r, double* z) {
  return guarded([&] {
    LearnedNet& n = learned_of(s);
    require(r && z, "null argument");
    Ctx& c = *s->tree->ctx;
    const int64_t N = n.ncells * n.Np;
    BSGPU_CUDA(cudaMemcpyAsync(s->B.p, r, N * 8, cudaMemcpyHostToDevice, c.st));
    if (!s->lscal) s->lscal = c.scal(8);
    double* d = s->lscal;
    const double* a[1] = {s->B.p};
    dots(c.red, 1, a, a, N, d, 1, c.st);
    learned_scale(d, d + 1, N, c.st);
    learned_apply(n, s->B.p, s->X.p, d + 1, c.st);
    BSGPU_CUDA(cudaMemcpyAsync(z, s->X.p, N * 8, cudaMemcpyDeviceToHost, c.st));
    BSGPU_CUDA(cudaStreamSynchronize(c.st));
    learned_check(n, c.st);
  });
}

BSGPU_API int bsgpu_solver_learned_gradient(bsgpu_solver_t s, const double* r, float* g1, float* g2, float* g3,
                                            double* loss) {
  return guarded([&] {
    LearnedNet& n = learned_of(s);
    require(r && g1 && g2 && g3, "null argument");
    Ctx& c = *s->tree->ctx;
    const int64_t N = n.ncells * n.Np;
    DBuf<double> Az(std::max<int64_t>(N, 1)), g(std::max<int64_t>(N, 1));
    BSGPU_CUDA(cudaMemcpyAsync(s->B.p, r, N * 8, cudaMemcpyHostToDevice, c.st));
    if (!s->lscal) s->lscal = c.scal(8);
    double* scal = s->lscal;
    learned_gradient(n, *s->tree->A, s->B.p, s->X.p, Az.p, g.p, c.red, scal, c.st);
    learned_take_gradient(n, g1, g2, g3, c.st);
    c.fetch(scal, 5);
    const double* h = c.hscal + (scal - c.dscal.p);
    if (loss) *loss = (h[3] - 2.0 * h[4]) / h[2];
  });
}

BSGPU_API int bsgpu_solver_get_history(bsgpu_solver_t s, double* hist, int32_t cap, int32_t* n) {
  return guarded([&] {
    require(s != nullptr, "null solver");
    const int32_t k = (int32_t)s->history.size();
    if (n) *n = k;
    if (hist)
      for (int32_t i = 0; i < k && i < cap; ++i) hist[i] = s->history[i];
  });
}

}  // extern "C"
