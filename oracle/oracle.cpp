// ORACLE -- test infrastructure only.  CPU restatement of the BoSSS linear-solver hot path, used by tests/ as the
// parity checker and by bench.py as the timed CPU baseline.  Nothing in the product library links or calls it.
//
// Every routine cites the reference file:line (paths relative to the BoSSS source tree) whose algorithm it
// restates.  Block storage is the BlockMsrMatrix view (BlockMsrMatrix.cs:315,1133,2453-2560): one dense,
// row-major block per occupied (block row, block column) pair, block columns ascending inside a block row.
//
// Parity status: no golden vectors exist in the reference (its solver tests pin tolerances, not values); the
// restatement is pinned by the reference's own known-answer tests restated in tests/ (TestCartesian1 exactness,
// convergence slopes, SpMV against an independent CSR product, multigrid transfer exactness, Schwarz 1e-14).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {
#include "oracle.h"
}

namespace {

thread_local std::string g_err;

using Vec = std::vector<double>;

// ---------------------------------------------------------------------------------------------------------------
// Block-sparse matrix
// ---------------------------------------------------------------------------------------------------------------
struct Mat {
  int64_t nb = 0, N = 0;
  std::vector<int64_t> i0;   // nb+1 first DOF of each block row
  std::vector<int32_t> len;  // nb   block length
  std::vector<int64_t> rp;   // nb+1 block row pointer
  std::vector<int32_t> ci;   // nnzb block column index
  std::vector<int64_t> vp;   // nnzb+1 offset of each block in v
  std::vector<double> v;     // values (owned copy)
  const double* val = nullptr;  // values actually used (v.data() or external)
  std::vector<int32_t> nspc;  // species per block (XDG); block length = nspc * Np
  int Np = 0;

  int64_t nnzb() const { return (int64_t)ci.size(); }
  const double* blk(int64_t k) const { return val + vp[k]; }
};

void build_offsets(Mat& A) {
  A.i0.assign(A.nb + 1, 0);
  for (int64_t i = 0; i < A.nb; ++i) A.i0[i + 1] = A.i0[i] + A.len[i];
  A.N = A.i0[A.nb];
  A.vp.assign(A.nnzb() + 1, 0);
  for (int64_t i = 0; i < A.nb; ++i)
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
      A.vp[k + 1] = A.vp[k] + (int64_t)A.len[i] * A.len[A.ci[k]];
}

// BlockMsrMatrix.SpMV(alpha, x, beta, y): y = beta*y + alpha*A*x, per block row an accumulator over the row's
// blocks, scalar loop per block (BlockMsrMatrix.cs:2970-3410; row loop :3089-3239, accumulate :3211-3216).
// With beta == 0 the old y is not read (BLAS convention).
void spmv(const Mat& A, double alpha, const double* x, double beta, double* y) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < A.nb; ++i) {
    const int I = A.len[i];
    double acc[512];
    for (int r = 0; r < I; ++r) acc[r] = 0.0;
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      const int j = A.ci[k];
      const int J = A.len[j];
      const double* b = A.blk(k);
      const double* xj = x + A.i0[j];
      for (int r = 0; r < I; ++r) {
        double s = 0.0;
        for (int c = 0; c < J; ++c) s += b[r * J + c] * xj[c];
        acc[r] += s;
      }
    }
    double* yi = y + A.i0[i];
    if (beta == 0.0)
      for (int r = 0; r < I; ++r) yi[r] = alpha * acc[r];
    else
      for (int r = 0; r < I; ++r) yi[r] = yi[r] * beta + alpha * acc[r];
  }
}

// ---------------------------------------------------------------------------------------------------------------
// BLAS-1 (MPI-free restatement of ilPSP GenericBlas / BLAS.ddot, daxpy, dscal)
// ---------------------------------------------------------------------------------------------------------------
double dot(const Vec& a, const Vec& b) {
  double s = 0.0;
  const int64_t n = (int64_t)a.size();
#pragma omp parallel for reduction(+ : s) schedule(static)
  for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}
double nrm2(const Vec& a) { return std::sqrt(dot(a, a)); }
void axpy(double alpha, const Vec& x, Vec& y) {
  const int64_t n = (int64_t)x.size();
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) y[i] += alpha * x[i];
}
void scal(double alpha, Vec& x) {
  const int64_t n = (int64_t)x.size();
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) x[i] *= alpha;
}
void copyv(const Vec& src, Vec& dst) { dst = src; }
bool has_nan(const Vec& a) {
  for (double v : a)
    if (!std::isfinite(v)) return true;
  return false;
}

// ---------------------------------------------------------------------------------------------------------------
// Dense block kernels
// ---------------------------------------------------------------------------------------------------------------

// SymmInv (MultigridOperator_ChangeOfBasis.cs:624-760): symmetric elimination that reduces M to diag(+-1) by
// row/column scaling and row/column additions, applying the same row operations to L (starting from I).  On exit
// L*M_in*L^T = diag(+-1) and L is lower triangular.  M is destroyed.  Returns 0 or an error code.
int symminv(int n, double* M, double* L) {
  for (int i = 0; i < n * n; ++i) L[i] = 0.0;
  for (int i = 0; i < n; ++i) L[i * n + i] = 1.0;
  for (int i = 0; i < n; ++i) {
    double Mii = M[i * n + i];
    if (Mii == 0.0) return OR_ERR_ARITHMETIC;
    double scl = 1.0 / std::sqrt(std::fabs(Mii));
    for (int c = 0; c < n; ++c) M[i * n + c] *= scl;   // RowScale(M)
    for (int c = 0; c < n; ++c) L[i * n + c] *= scl;   // RowScale(L)
    for (int r = 0; r < n; ++r) M[r * n + i] *= scl;   // ColScale(M)
    double diagsign = (M[i * n + i] > 0) ? 1.0 : ((M[i * n + i] < 0) ? -1.0 : 0.0);
    if (diagsign == 0.0) return OR_ERR_ARITHMETIC;
    if (std::fabs(std::fabs(M[i * n + i]) - 1.0) > 1.0e-8) return OR_ERR_ARITHMETIC;
    for (int k = i + 1; k < n; ++k) {
      double Mki = M[k * n + i];
      double a = -Mki * diagsign;
      for (int c = 0; c < n; ++c) M[k * n + c] += M[i * n + c] * a;  // RowAdd(M, i -> k)
      for (int c = 0; c < n; ++c) L[k * n + c] += L[i * n + c] * a;  // RowAdd(L, i -> k)
      for (int r = 0; r < n; ++r) M[r * n + k] += M[r * n + i] * a;  // ColAdd(M, i -> k)
    }
  }
  return 0;
}

// InvertInPlace (IMatrixExtensions.cs:2221-2330): LU with partial pivoting (LAPACK dgetrf/dgetri semantics),
// closed forms for n <= 1.  A is row-major and replaced by its inverse.
int invert(int n, double* A) {
  if (n == 0) return 0;
  if (n == 1) {
    if (A[0] == 0.0) return OR_ERR_ARITHMETIC;
    A[0] = 1.0 / A[0];
    return 0;
  }
  std::vector<double> LU(A, A + n * n), inv((size_t)n * n, 0.0);
  std::vector<int> piv(n);
  for (int k = 0; k < n; ++k) {
    int p = k;
    double mx = std::fabs(LU[k * n + k]);
    for (int r = k + 1; r < n; ++r)
      if (std::fabs(LU[r * n + k]) > mx) { mx = std::fabs(LU[r * n + k]); p = r; }
    piv[k] = p;
    if (mx == 0.0) return OR_ERR_ARITHMETIC;
    if (p != k)
      for (int c = 0; c < n; ++c) std::swap(LU[k * n + c], LU[p * n + c]);
    for (int r = k + 1; r < n; ++r) {
      double f = LU[r * n + k] / LU[k * n + k];
      LU[r * n + k] = f;
      for (int c = k + 1; c < n; ++c) LU[r * n + c] -= f * LU[k * n + c];
    }
  }
  for (int col = 0; col < n; ++col) {
    std::vector<double> e(n, 0.0);
    e[col] = 1.0;
    for (int k = 0; k < n; ++k)
      if (piv[k] != k) std::swap(e[k], e[piv[k]]);
    for (int r = 0; r < n; ++r) {
      double s = e[r];
      for (int c = 0; c < r; ++c) s -= LU[r * n + c] * e[c];
      e[r] = s;
    }
    for (int r = n - 1; r >= 0; --r) {
      double s = e[r];
      for (int c = r + 1; c < n; ++c) s -= LU[r * n + c] * e[c];
      e[r] = s / LU[r * n + r];
    }
    for (int r = 0; r < n; ++r) inv[r * n + col] = e[r];
  }
  std::copy(inv.begin(), inv.end(), A);
  return 0;
}

// ---------------------------------------------------------------------------------------------------------------
// Termination (IterativeSolverConfig.cs:48-62)
// ---------------------------------------------------------------------------------------------------------------
struct Term {
  int mode = 0;  // 0: default (R < R0*tol + tol), 1: relative (R < R0*tol), 2: fixed count, 3: sub-level
  double tol = 1e-10;
  int max_iter = 300, min_iter = 1;
  double reduction = 0.1;  // mode 3
  // returns {notTerminate, success}
  std::pair<bool, bool> operator()(int iter, double R0, double R) const {
    const double eps = 2.2204460492503131e-16 * 1000;
    if (mode == 2) return {iter <= max_iter, true};
    if (mode == 3) {  // PmgConfig.cs:202-215 SubLevelTermination
      if (iter <= 1) return {true, false};
      if (R < R0 * reduction) return {false, true};
      if (iter > max_iter) return {false, false};
      return {true, false};
    }
    if (iter <= min_iter) return {true, false};
    bool ok = (mode == 0) ? (R < R0 * tol + tol) : (R < R0 * tol);
    if (ok) return {false, true};
    if (iter > max_iter) return {false, false};
    if (R0 < eps || R < eps) return {false, true};
    return {true, false};
  }
};

// ---------------------------------------------------------------------------------------------------------------
// Solver interface (ISmootherTemplate.cs:29-83)
// ---------------------------------------------------------------------------------------------------------------
struct Solver {
  int this_level_iterations = 0;
  bool converged = false;
  virtual ~Solver() {}
  virtual void solve(Vec& X, const Vec& B) = 0;  // X: initial guess in, solution out
  virtual int nested() const { return 0; }
};

// BlockJacobi (BlockJacobi.cs:68-266).
struct BlockJacobi : Solver {
  const Mat* A;
  Mat Dg, Dinv;  // block-diagonal matrices (same row partition)
  int iters = 1;
  double omega = 1.0;
  BlockJacobi(const Mat* A_, int it, double om) : A(A_), iters(it), omega(om) {
    for (Mat* M : {&Dg, &Dinv}) {
      M->nb = A->nb; M->len = A->len; M->Np = A->Np; M->nspc = A->nspc;
      M->rp.resize(A->nb + 1);
      M->ci.resize(A->nb);
      for (int64_t i = 0; i <= A->nb; ++i) M->rp[i] = i;
      for (int64_t i = 0; i < A->nb; ++i) M->ci[i] = (int32_t)i;
      build_offsets(*M);
      M->v.assign(M->vp.back(), 0.0);
      M->val = M->v.data();
    }
    int err = 0;
#pragma omp parallel for schedule(static) reduction(| : err)
    for (int64_t i = 0; i < A->nb; ++i) {
      const int n = A->len[i];
      int64_t kd = -1;
      for (int64_t k = A->rp[i]; k < A->rp[i + 1]; ++k)
        if (A->ci[k] == i) kd = k;
      double* d = Dg.v.data() + Dg.vp[i];
      double* di = Dinv.v.data() + Dinv.vp[i];
      if (kd >= 0) std::copy(A->blk(kd), A->blk(kd) + n * n, d);
      std::copy(d, d + n * n, di);
      err |= invert(n, di);
    }
    if (err) throw std::runtime_error("BlockJacobi: singular diagonal block");
  }
  void solve(Vec& x, const Vec& b) override {
    Vec q(b.size());
    for (int it = 0;; ++it) {
      q = b;
      spmv(*A, -1.0, x.data(), 1.0, q.data());
      // ResNorm only feeds the termination check, which is iteration-count based (BlockJacobi.cs:171-173).
      if (!(it <= iters)) { converged = true; return; }
      spmv(Dg, 1.0, x.data(), 1.0, q.data());
      spmv(Dinv, omega, q.data(), 1.0 - omega, x.data());
    }
  }
};

// Restriction of an operator to the leading `keep` modes of every species in every block
// (GridAndDegRestriction.cs:47-99 MgOperatorRestriction, BlockMask.GetSubBlockMatrix).
struct Restriction {
  const Mat* A;
  Mat sub;
  std::vector<int64_t> map;  // sub index -> full index
  Restriction(const Mat* A_, int keep) : A(A_) {
    sub.nb = A->nb; sub.Np = keep; sub.nspc = A->nspc;
    sub.len.resize(A->nb);
    std::vector<std::vector<int>> loc(A->nb);
    for (int64_t i = 0; i < A->nb; ++i) {
      int ns = A->nspc.empty() ? 1 : A->nspc[i];
      for (int s = 0; s < ns; ++s)
        for (int m = 0; m < keep; ++m) loc[i].push_back(s * A->Np + m);
      sub.len[i] = (int32_t)loc[i].size();
    }
    sub.rp = A->rp;
    sub.ci = A->ci;
    build_offsets(sub);
    sub.v.assign(sub.vp.back(), 0.0);
    sub.val = sub.v.data();
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < A->nb; ++i)
      for (int64_t k = A->rp[i]; k < A->rp[i + 1]; ++k) {
        int j = A->ci[k];
        int Jf = A->len[j];
        const double* b = A->blk(k);
        double* o = sub.v.data() + sub.vp[k];
        int Js = sub.len[j];
        for (size_t r = 0; r < loc[i].size(); ++r)
          for (size_t c = 0; c < loc[j].size(); ++c) o[r * Js + c] = b[loc[i][r] * Jf + loc[j][c]];
      }
    map.resize(sub.N);
    for (int64_t i = 0; i < A->nb; ++i)
      for (size_t r = 0; r < loc[i].size(); ++r) map[sub.i0[i] + r] = A->i0[i] + loc[i][r];
  }
  void get(const Vec& full, Vec& s) const {  // BlockMask.GetSubVec
    s.resize(map.size());
    for (size_t i = 0; i < map.size(); ++i) s[i] = full[map[i]];
  }
  void acc(const Vec& s, Vec& full) const {  // BlockMask.AccSubVec
    for (size_t i = 0; i < map.size(); ++i) full[map[i]] += s[i];
  }
};

// GridAndDegRestriction.Solve (GridAndDegRestriction.cs:379-439).
struct GridAndDegRestriction : Solver {
  Restriction R;
  Solver* lower = nullptr;
  GridAndDegRestriction(const Mat* A, int keep) : R(A, keep) {}
  ~GridAndDegRestriction() { delete lower; }
  void solve(Vec& X, const Vec& B) override {
    Vec xLo, bLo;
    R.get(X, xLo);
    R.get(B, bLo);
    if (lower) {
      if (nrm2(bLo) <= 0) { converged = true; return; }
      lower->solve(xLo, bLo);
      converged = lower->converged;
    }
    R.acc(xLo, X);
  }
  int nested() const override { return lower ? lower->this_level_iterations + lower->nested() : 0; }
};

// Dense direct solve of the coarsest level (stand-in for DirectSolver's LAPACK/PARDISO path,
// DirectSolver.cs:308-345): the assembled level matrix is inverted once.
struct DenseDirect : Solver {
  const Mat* A;
  std::vector<double> inv;
  int64_t n;
  explicit DenseDirect(const Mat* A_) : A(A_), n(A_->N) {
    if (n > 12000) throw std::runtime_error("DenseDirect: level too large for a dense factorisation");
    inv.assign((size_t)n * n, 0.0);
    for (int64_t i = 0; i < A->nb; ++i)
      for (int64_t k = A->rp[i]; k < A->rp[i + 1]; ++k) {
        int j = A->ci[k];
        const double* b = A->blk(k);
        for (int r = 0; r < A->len[i]; ++r)
          for (int c = 0; c < A->len[j]; ++c) inv[(A->i0[i] + r) * n + A->i0[j] + c] = b[r * A->len[j] + c];
      }
    if (invert((int)n, inv.data())) throw std::runtime_error("DenseDirect: singular");
  }
  void solve(Vec& X, const Vec& B) override {
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n; ++r) {
      double s = 0.0;
      for (int64_t c = 0; c < n; ++c) s += inv[r * n + c] * B[c];
      X[r] = s;
    }
    converged = true;
    this_level_iterations = 1;
  }
};

// SoftPCG (SoftPCG.cs:113-194) with an optional preconditioner.
struct SoftPCG : Solver {
  const Mat* A;
  Solver* precond = nullptr;  // owned
  Term term;
  std::vector<double>* hist = nullptr;
  SoftPCG(const Mat* A_, Solver* pc, Term t) : A(A_), precond(pc), term(t) {}
  ~SoftPCG() { delete precond; }
  void apply_pc(Vec& z, const Vec& r) {
    if (precond) {
      std::fill(z.begin(), z.end(), 0.0);
      precond->solve(z, r);
    } else {
      z = r;
    }
  }
  void solve(Vec& x, const Vec& B) override {
    const size_t L = x.size();
    Vec P(L), V(L), Z(L), Res = B;
    spmv(*A, -1.0, x.data(), 1.0, Res.data());
    apply_pc(Z, Res);
    P = Z;
    double alpha = dot(Res, Z);
    double R = nrm2(Res), R0 = R;
    if (hist) hist->push_back(R);
    auto st = term(0, R0, R);
    bool cont = st.first;
    int n = 1;
    for (; cont; ++n) {
      spmv(*A, 1.0, P.data(), 0.0, V.data());
      double VxP = dot(V, P);
      double lambda = alpha / VxP;
      if (!std::isfinite(lambda)) throw std::runtime_error("SoftPCG: breakdown");
      axpy(lambda, P, x);
      axpy(-lambda, V, Res);
      apply_pc(Z, Res);
      double alpha_neu = dot(Res, Z);
      scal(alpha_neu / alpha, P);
      axpy(1.0, Z, P);
      R = nrm2(Res);
      alpha = alpha_neu;
      if (hist) hist->push_back(R);
      st = term(n, R0, R);
      cont = st.first;
    }
    converged = st.second;
    this_level_iterations = n - 1;
  }
};

// CoreOrthonormalizationProcedure (OrthonormalizationMultigrid.cs:58-445).
struct Ortho {
  const Mat* A;
  std::vector<Vec> Sol, Mxx;
  std::mt19937_64 rng{12345};
  bool more_than_one = false;
  bool cancellation = false;
  explicit Ortho(const Mat* A_) : A(A_) {}
  void clear() { Sol.clear(); Mxx.clear(); }
  double fill_random(Vec& X, Vec& M) {
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    for (auto& v : X) v = U(rng);
    spmv(*A, 1.0, X.data(), 0.0, M.data());
    double nm = nrm2(M);
    if (nm == 0 || !std::isfinite(nm)) throw std::runtime_error("Ortho: breakdown with random vector");
    return nm;
  }
  // AddSol (:219-345): A-orthonormalisation of X against the history (modified Gram-Schmidt, up to 10 sweeps).
  void add_sol(Vec X) {
    more_than_one = false;
    const size_t L = X.size();
    Vec M(L);
    spmv(*A, 1.0, X.data(), 0.0, M.data());
    double nM = nrm2(M);
    if (!std::isfinite(nM)) throw std::runtime_error("Ortho: NaN/Inf");
    if (nM == 0) nM = fill_random(X, M);
    scal(1.0 / nM, M);
    scal(1.0 / nM, X);
    const int MaxOrtho = 10;
    bool canc = false;
    for (int jj = 0; jj <= MaxOrtho; ++jj) {
      more_than_one = jj > 0;
      for (size_t i = 0; i < Sol.size(); ++i) {
        double beta = dot(M, Mxx[i]);
        axpy(-beta, Sol[i], X);
        axpy(-beta, Mxx[i], M);
      }
      double nn = nrm2(M);
      if (nn <= 1e-5) {
        canc = true;
        if (jj < MaxOrtho) {
          double Xn = nrm2(X);
          if (Xn < 1e-200 || jj == MaxOrtho - 1) {
            fill_random(X, M);
          } else {
            scal(1.0 / Xn, X);
            spmv(*A, 1.0, X.data(), 0.0, M.data());
            if (nrm2(M) == 0) fill_random(X, M);
          }
          double gamma = 1.0 / nn;
          scal(gamma, M);
          scal(gamma, X);
        } else {
          throw std::runtime_error("Ortho: numerical breakdown");
        }
      } else {
        double gamma = 1.0 / nn;
        scal(gamma, M);
        scal(gamma, X);
        break;
      }
    }
    cancellation = canc;
    Sol.push_back(std::move(X));
    Mxx.push_back(std::move(M));
  }
  // MinimizeResidual (:149-209): the residual is updated, and recomputed from scratch when the history length is
  // a multiple of RecalcResiPeriod or the last AddSol needed more than one sweep (:179-190).
  int recalc_period = 1;
  double minimize(Vec& X, Vec& Sol0, const Vec& Res0, Vec& Res) {
    double oldN = nrm2(Res);
    size_t i = Sol.size() - 1;
    double alpha = dot(Mxx[i], Res0);
    axpy(alpha, Sol[i], X);
    axpy(-alpha, Mxx[i], Res);
    if (recalc_period <= 1 || more_than_one || Sol.size() % (size_t)recalc_period == 0) {
      Res = Res0;
      axpy(-1.0, X, Sol0);
      spmv(*A, 1.0, Sol0.data(), 1.0, Res.data());
      axpy(1.0, X, Sol0);
    }
    double N = nrm2(Res);
    double tol = std::max(std::max(N, oldN) * 0.2, 1.0e-7);
    if (N > oldN + tol) throw std::runtime_error("Ortho: residual increase");
    return N;
  }
};

// OrthonormalizationMultigrid.Solve (OrthonormalizationMultigrid.cs:797-1104), CoarseOnLowerLevel = false,
// m_omega = 1, no pre-smoother (the PmgConfig setup, PmgConfig.cs:80-245).
struct OrthoMG : Solver {
  const Mat* A;
  Solver* coarse = nullptr;  // owned
  Solver* post = nullptr;    // owned
  int sweeps = 10;
  Term term;
  Ortho ortho;
  std::vector<double>* hist = nullptr;
  OrthoMG(const Mat* A_, Term t) : A(A_), term(t), ortho(A_) {}
  ~OrthoMG() { delete coarse; delete post; }
  int nested() const override {
    int s = 0;
    if (coarse) s += coarse->this_level_iterations + coarse->nested();
    if (post) s += post->this_level_iterations + post->nested();
    return s;
  }
  void solve(Vec& X, const Vec& B) override {
    const size_t L = X.size();
    Vec Sol0 = X, Res0 = B;
    spmv(*A, -1.0, Sol0.data(), 1.0, Res0.data());
    Vec Res = Res0;
    double r0 = nrm2(Res0), rn = r0;
    if (hist) hist->push_back(rn);
    ortho.clear();
    int iIter;
    for (iIter = 1;; ++iIter) {
      auto st = term(iIter, r0, rn);
      if (!st.first) { converged = st.second; break; }
      if (coarse) {
        Vec vl(L, 0.0);
        coarse->solve(vl, Res);
        if (has_nan(vl)) throw std::runtime_error("OrthoMG: coarse solver produced NaN/Inf");
        ortho.add_sol(std::move(vl));
        rn = ortho.minimize(X, Sol0, Res0, Res);
        st = term(iIter, r0, rn);
        if (!st.first) { converged = st.second; break; }
      }
      bool termPost = false;
      if (post) {
        for (int g = 0; g < sweeps; ++g) {
          Vec pc(L, 0.0);
          post->solve(pc, Res);
          if (has_nan(pc)) throw std::runtime_error("OrthoMG: smoother produced NaN/Inf");
          ortho.add_sol(std::move(pc));
          rn = ortho.minimize(X, Sol0, Res0, Res);
          st = term(iIter, r0, rn);
          if (!st.first) { converged = st.second; termPost = true; break; }
          if (ortho.cancellation) break;
        }
      }
      if (termPost) break;
      this_level_iterations++;
      if (hist) hist->push_back(rn);
    }
  }
};

// FlexGMRES (FlexGMRES.cs:144-277).  Saad-1993 FGMRES(m) with modified Gram-Schmidt Arnoldi; the
// least-squares problem is solved by Givens rotations (mathematically the dgelsy solution for full-rank H).
// `reference_defect` reproduces FlexGMRES.cs:259-260, where the least-squares result is overwritten by
// alpha = (beta, 0, ..., 0), i.e. X += beta*Z_0; it also checks termination only once per restart, as the
// reference does (:168-183).  Without it the implicit residual is checked after every Arnoldi step.
// SoftGMRES.Solve (SoftGMRES.cs:227-460): restarted GMRES(m), left preconditioned (r = M^{-1}(b - A x), Arnoldi
// on M^{-1} A with modified Gram-Schmidt), Givens rotations (rotmat, :196-210), x += V y at convergence and at
// each restart; the termination test compares |s_i| (preconditioned residual estimate) with the initial
// unpreconditioned residual |b - A x0| (:260-268, :372).  At the iteration limit the cycle's update is applied.
struct SoftGMRES : Solver {
  const Mat* A;
  Solver* precond = nullptr;  // owned; nullptr = identity
  int m = 80;
  Term term;
  std::vector<double>* hist = nullptr;
  SoftGMRES(const Mat* A_, Solver* pc, int m_, Term t) : A(A_), precond(pc), m(m_), term(t) {}
  ~SoftGMRES() { delete precond; }
  void apply_pc(const Vec& in, Vec& out) {
    if (!precond) { out = in; return; }
    std::fill(out.begin(), out.end(), 0.0);
    precond->solve(out, in);
  }
  static void rotmat(double& c, double& s, double a, double b) {
    if (b == 0.0) { c = 1.0; s = 0.0; }
    else if (std::fabs(b) > std::fabs(a)) { double t = a / b; s = 1.0 / std::sqrt(1.0 + t * t); c = t * s; }
    else { double t = b / a; c = 1.0 / std::sqrt(1.0 + t * t); s = t * c; }
  }
  void solve(Vec& X, const Vec& B) override {
    const size_t L = B.size();
    Vec z(L), r(L), w(L);
    z = B;
    spmv(*A, -1.0, X.data(), 1.0, z.data());
    const double r0 = nrm2(z);
    if (hist) hist->push_back(r0);
    auto t0 = term(0, r0, r0);
    if (!t0.first) { converged = t0.second; return; }
    std::vector<Vec> V(m + 1, Vec(L));
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), s(m + 2), y(m);
    int tot = 0;
    bool first = true;
    while (true) {
      if (!first) { z = B; spmv(*A, -1.0, X.data(), 1.0, z.data()); }
      first = false;
      apply_pc(z, r);
      const double beta = nrm2(r);
      if (!std::isfinite(beta)) throw std::runtime_error("SoftGMRES: NaN/Inf");
      if (beta == 0.0) { converged = true; break; }
      V[0] = r;
      scal(1.0 / beta, V[0]);
      std::fill(s.begin(), s.end(), 0.0);
      s[0] = beta;
      int i;
      bool stop = false;
      double err = beta;
      for (i = 1; i <= m; ++i) {
        spmv(*A, 1.0, V[i - 1].data(), 0.0, z.data());
        apply_pc(z, w);
        for (int k = 0; k < i; ++k) {
          H[k * m + (i - 1)] = dot(w, V[k]);
          axpy(-H[k * m + (i - 1)], V[k], w);
        }
        const double nw = nrm2(w);
        H[i * m + (i - 1)] = nw;
        V[i] = w;
        if (nw > 0) scal(1.0 / nw, V[i]);
        for (int k = 1; k <= i - 1; ++k) {
          const double tmp = cs[k - 1] * H[(k - 1) * m + i - 1] + sn[k - 1] * H[k * m + i - 1];
          H[k * m + i - 1] = -sn[k - 1] * H[(k - 1) * m + i - 1] + cs[k - 1] * H[k * m + i - 1];
          H[(k - 1) * m + i - 1] = tmp;
        }
        rotmat(cs[i - 1], sn[i - 1], H[(i - 1) * m + i - 1], H[i * m + i - 1]);
        const double tmp = cs[i - 1] * s[i - 1];
        H[(i - 1) * m + i - 1] = cs[i - 1] * H[(i - 1) * m + i - 1] + sn[i - 1] * H[i * m + i - 1];
        H[i * m + i - 1] = 0.0;
        s[i] = -sn[i - 1] * s[i - 1];
        s[i - 1] = tmp;
        err = std::fabs(s[i]);
        if (hist) hist->push_back(err);
        auto t1 = term(tot, r0, err);
        ++tot;
        if (!t1.first || nw == 0.0) { stop = true; converged = t1.second || nw == 0.0; break; }
      }
      const int kk = stop ? i : m;
      for (int a = kk - 1; a >= 0; --a) {
        double acc = s[a];
        for (int q = a + 1; q < kk; ++q) acc -= H[a * m + q] * y[q];
        y[a] = acc / H[a * m + a];
      }
      for (int a = 0; a < kk; ++a) axpy(y[a], V[a], X);
      if (stop) break;
      auto t2 = term(tot, r0, err);
      if (!t2.first) { converged = t2.second; break; }
    }
    this_level_iterations = tot;
  }
};

struct FlexGMRES : Solver {
  const Mat* A;
  Solver* precond = nullptr;  // owned
  int m = 30;
  Term term;
  bool reference_defect = false;
  std::vector<double>* hist = nullptr;
  FlexGMRES(const Mat* A_, Solver* pc, int m_, Term t) : A(A_), precond(pc), m(m_), term(t) {}
  ~FlexGMRES() { delete precond; }
  int nested() const override { return precond ? precond->this_level_iterations + precond->nested() : 0; }
  void solve(Vec& X, const Vec& B) override {
    const size_t L = B.size();
    Vec R0(L);
    int iIter = 0;
    double r0 = 0;
    std::vector<Vec> V, Z;
    std::vector<double> H((size_t)(m + 1) * m), cs(m), sn(m), g(m + 1);
    while (true) {
      R0 = B;
      spmv(*A, -1.0, X.data(), 1.0, R0.data());
      double r = nrm2(R0);
      if (iIter == 0) r0 = r;
      if (hist) hist->push_back(r);
      auto st = term(iIter, r0, r);
      if (!st.first || st.second) { converged = st.second; this_level_iterations = iIter; return; }
      double beta = r;
      V.clear(); Z.clear();
      V.push_back(R0);
      scal(1.0 / beta, V[0]);
      std::fill(g.begin(), g.end(), 0.0);
      g[0] = beta;
      int j;
      for (j = 0; j < m; ++j) {
        Vec Zj(L, 0.0);
        precond->solve(Zj, V[j]);
        iIter++;
        Vec W(L);
        spmv(*A, 1.0, Zj.data(), 0.0, W.data());
        Z.push_back(std::move(Zj));
        for (int i = 0; i <= j; ++i) {
          double h = dot(W, V[i]);
          H[i * m + j] = h;
          axpy(-h, V[i], W);
        }
        double wn = nrm2(W);
        H[(j + 1) * m + j] = wn;
        scal(1.0 / wn, W);
        V.push_back(std::move(W));
        // Givens update of column j
        for (int i = 0; i < j; ++i) {
          double a = H[i * m + j], b = H[(i + 1) * m + j];
          H[i * m + j] = cs[i] * a + sn[i] * b;
          H[(i + 1) * m + j] = -sn[i] * a + cs[i] * b;
        }
        double a = H[j * m + j], b = H[(j + 1) * m + j];
        double den = std::hypot(a, b);
        cs[j] = a / den;
        sn[j] = b / den;
        H[j * m + j] = den;
        H[(j + 1) * m + j] = 0.0;
        g[j + 1] = -sn[j] * g[j];
        g[j] = cs[j] * g[j];
        if (!reference_defect) {
          double est = std::fabs(g[j + 1]);
          if (hist) hist->push_back(est);
          auto st2 = term(iIter, r0, est);
          if (!st2.first || st2.second || wn == 0.0) { ++j; break; }
        }
      }
      int k = j;  // number of Krylov vectors used
      std::vector<double> y(k, 0.0);
      if (reference_defect) {
        y[0] = beta;
      } else {
        for (int i = k - 1; i >= 0; --i) {
          double s = g[i];
          for (int c = i + 1; c < k; ++c) s -= H[i * m + c] * y[c];
          y[i] = s / H[i * m + i];
        }
      }
      for (int i = 0; i < k; ++i) axpy(y[i], Z[i], X);
    }
  }
};

// ChangeOfBasis with Mode.DiagBlockEquilib (MultigridOperator_ChangeOfBasis.cs:260,819-828 and
// MultigridOperator.cs:650-700): per block row L_i from SymmInv(A_ii); operator A'_ij = L_i A_ij L_j^T.
int change_of_basis(const Mat& A, Mat& Ap, std::vector<double>& Lblk) {
  Ap = Mat();
  Ap.nb = A.nb; Ap.len = A.len; Ap.rp = A.rp; Ap.ci = A.ci; Ap.nspc = A.nspc; Ap.Np = A.Np;
  build_offsets(Ap);
  Ap.v.assign(Ap.vp.back(), 0.0);
  Ap.val = Ap.v.data();
  std::vector<int64_t> lp(A.nb + 1, 0);
  for (int64_t i = 0; i < A.nb; ++i) lp[i + 1] = lp[i] + (int64_t)A.len[i] * A.len[i];
  Lblk.assign(lp.back(), 0.0);
  int err = 0;
#pragma omp parallel for schedule(static) reduction(| : err)
  for (int64_t i = 0; i < A.nb; ++i) {
    int n = A.len[i];
    int64_t kd = -1;
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k)
      if (A.ci[k] == i) kd = k;
    if (kd < 0) { err |= OR_ERR_ARITHMETIC; continue; }
    std::vector<double> M(A.blk(kd), A.blk(kd) + n * n);
    err |= symminv(n, M.data(), Lblk.data() + lp[i]);
  }
  if (err) return err;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < A.nb; ++i) {
    int I = A.len[i];
    const double* Li = Lblk.data() + lp[i];
    std::vector<double> T;
    for (int64_t k = A.rp[i]; k < A.rp[i + 1]; ++k) {
      int j = A.ci[k];
      int J = A.len[j];
      const double* Lj = Lblk.data() + lp[j];
      const double* b = A.blk(k);
      T.assign((size_t)I * J, 0.0);
      for (int r = 0; r < I; ++r)       // T = L_i * A_ij
        for (int q = 0; q <= r; ++q) {
          double l = Li[r * I + q];
          for (int c = 0; c < J; ++c) T[r * J + c] += l * b[q * J + c];
        }
      double* o = Ap.v.data() + Ap.vp[k];
      for (int r = 0; r < I; ++r)       // A' = T * L_j^T
        for (int c = 0; c < J; ++c) {
          double s = 0.0;
          for (int q = 0; q <= c; ++q) s += T[r * J + q] * Lj[c * J + q];
          o[r * J + c] = s;
        }
    }
  }
  return 0;
}

void load_mat(Mat& A, const or_bsr* m) {
  A.nb = m->nb;
  A.Np = m->Np;
  A.len.resize(A.nb);
  A.nspc.assign(A.nb, 1);
  for (int64_t i = 0; i < A.nb; ++i) {
    A.nspc[i] = m->nspc ? m->nspc[i] : 1;
    A.len[i] = A.nspc[i] * m->Np;
  }
  A.rp.assign(m->row_ptr, m->row_ptr + A.nb + 1);
  A.ci.assign(m->col_idx, m->col_idx + A.rp[A.nb]);
  build_offsets(A);
  A.val = m->values;  // external storage, not copied
}

// Schwarz patch inverses restated for patches = one cell plus the cells of its block row (Schwarz.cs:623-840):
// the rows of the centre cell of each patch inverse, in A's layout.
int schwarz_rows_mat(const Mat& A, double* values_out) {
  {
    int err = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(| : err)
    for (int64_t K = 0; K < A.nb; ++K) {
      std::vector<int32_t> cells(A.ci.begin() + A.rp[K], A.ci.begin() + A.rp[K + 1]);
      std::vector<int> off(cells.size() + 1, 0);
      for (size_t a = 0; a < cells.size(); ++a) off[a + 1] = off[a] + A.len[cells[a]];
      const int n = off.back();
      std::vector<double> P((size_t)n * n, 0.0);
      for (size_t a = 0; a < cells.size(); ++a) {
        const int32_t ca = cells[a];
        for (int64_t q = A.rp[ca]; q < A.rp[ca + 1]; ++q) {
          auto it = std::find(cells.begin(), cells.end(), A.ci[q]);
          if (it == cells.end()) continue;
          const size_t b = it - cells.begin();
          const int I = A.len[ca], J = A.len[A.ci[q]];
          const double* blk = A.blk(q);
          for (int r = 0; r < I; ++r)
            for (int c = 0; c < J; ++c) P[(size_t)(off[a] + r) * n + off[b] + c] = blk[r * J + c];
        }
      }
      err |= invert(n, P.data());
      const size_t aK = std::find(cells.begin(), cells.end(), (int32_t)K) - cells.begin();
      const int I = A.len[K];
      for (size_t b = 0; b < cells.size(); ++b) {
        const int J = A.len[cells[b]];
        double* o = values_out + A.vp[A.rp[K] + b];
        for (int r = 0; r < I; ++r)
          for (int c = 0; c < J; ++c) o[r * J + c] = P[(size_t)(off[aK] + r) * n + off[b] + c];
      }
    }
    if (err) { g_err = "Schwarz: singular block"; return OR_ERR_ARITHMETIC; }
    return 0;
  }
}


// helpers of the block ILU(0) restatement
void gemm_sub(int I, int K, int J, const double* A, const double* B, double* C) {  // C -= A B, row-major
  for (int r = 0; r < I; ++r)
    for (int k = 0; k < K; ++k) {
      const double a = A[r * K + k];
      for (int c = 0; c < J; ++c) C[r * J + c] -= a * B[k * J + c];
    }
}
int64_t find_block(const Mat& A, int64_t i, int32_t j) {
  const int32_t* b = A.ci.data() + A.rp[i];
  const int32_t* e = A.ci.data() + A.rp[i + 1];
  const int32_t* p = std::lower_bound(b, e, j);
  return (p != e && *p == j) ? A.rp[i] + (p - b) : -1;
}
std::vector<int64_t> positions(const Mat& A, const int32_t* order) {
  std::vector<int64_t> pos(A.nb);
  for (int64_t q = 0; q < A.nb; ++q) pos[order ? order[q] : q] = q;
  return pos;
}

int ilu0_factor_mat(const Mat& A, const int32_t* order, double* factor_out) {
  {
    std::vector<int64_t> pos = positions(A, order);
    std::copy(A.val, A.val + A.vp[A.nnzb()], factor_out);
    auto W = [&](int64_t k) { return factor_out + A.vp[k]; };
    for (int64_t kk = 0; kk + 1 < A.nb; ++kk) {
      const int64_t k = order ? order[kk] : kk;
      const int Sk = A.len[k];
      if (Sk == 0) continue;
      const int64_t dkk = find_block(A, k, (int32_t)k);
      if (dkk < 0) continue;
      std::vector<double> inv(W(dkk), W(dkk) + (size_t)Sk * Sk);
      if (invert(Sk, inv.data()) != 0) continue;
      // rows i > k (in the ordering) with an occupied block (i, k); the pattern is structurally symmetric
      for (int64_t q = A.rp[k]; q < A.rp[k + 1]; ++q) {
        const int64_t i = A.ci[q];
        if (pos[i] <= pos[k]) continue;
        const int64_t qik = find_block(A, i, (int32_t)k);
        if (qik < 0) continue;
        const int Si = A.len[i];
        std::vector<double> L((size_t)Si * Sk, 0.0);
        gemm_sub(Si, Sk, Sk, W(qik), inv.data(), L.data());          // L = -A_ik inv(A_kk)
        for (auto& v : L) v = -v;
        std::copy(L.begin(), L.end(), W(qik));
        for (int64_t p = A.rp[i]; p < A.rp[i + 1]; ++p) {
          const int32_t j = A.ci[p];
          if (pos[j] <= pos[k]) continue;
          const int64_t qkj = find_block(A, k, j);
          if (qkj < 0) continue;                                      // (k, j) outside the ILU(0) pattern
          gemm_sub(Si, Sk, A.len[j], L.data(), W(qkj), W(p));
        }
      }
    }
    return 0;
  }
}


int ilu0_solve_mat(const Mat& A, const int32_t* order, const double* factor, const double* b, double* x) {
  {
    std::vector<int64_t> pos = positions(A, order);
    std::vector<double> y(b, b + A.N);
    for (int64_t q = 0; q < A.nb; ++q) {
      const int64_t i = order ? order[q] : q;
      const int I = A.len[i];
      for (int64_t p = A.rp[i]; p < A.rp[i + 1]; ++p) {
        const int32_t k = A.ci[p];
        if (pos[k] >= pos[i]) continue;
        const int K = A.len[k];
        const double* L = factor + A.vp[p];
        for (int r = 0; r < I; ++r)
          for (int c = 0; c < K; ++c) y[A.i0[i] + r] -= L[r * K + c] * y[A.i0[k] + c];
      }
    }
    for (int64_t q = A.nb - 1; q >= 0; --q) {
      const int64_t i = order ? order[q] : q;
      const int I = A.len[i];
      std::vector<double> s(y.begin() + A.i0[i], y.begin() + A.i0[i] + I);
      for (int64_t p = A.rp[i]; p < A.rp[i + 1]; ++p) {
        const int32_t j = A.ci[p];
        if (pos[j] <= pos[i]) continue;
        const int J = A.len[j];
        const double* U = factor + A.vp[p];
        for (int r = 0; r < I; ++r)
          for (int c = 0; c < J; ++c) s[r] -= U[r * J + c] * x[A.i0[j] + c];
      }
      const int64_t d = find_block(A, i, (int32_t)i);
      if (d < 0) { g_err = "ILU: missing diagonal block"; return OR_ERR_ARGUMENT; }
      std::vector<double> inv(factor + A.vp[d], factor + A.vp[d] + (size_t)I * I);
      if (invert(I, inv.data()) != 0) { g_err = "ILU: singular diagonal block"; return OR_ERR_ARITHMETIC; }
      for (int r = 0; r < I; ++r) {
        double acc = 0.0;
        for (int c = 0; c < I; ++c) acc += inv[r * I + c] * s[c];
        x[A.i0[i] + r] = acc;
      }
    }
    return 0;
  }
}


// Restricted additive Schwarz smoother (Schwarz.cs:996-1147 with the patches of schwarz_rows_mat):
// x <- x + M (b - A x), FixedNoOfIterations = iters + 1 updates.
struct SchwarzSmoother : Solver {
  const Mat* A;
  Mat M;
  int updates;
  SchwarzSmoother(const Mat* A_, int iters) : A(A_), M(*A_), updates(iters + 1) {
    M.v.assign(A->vp.back(), 0.0);
    M.val = M.v.data();
    if (schwarz_rows_mat(*A, M.v.data()) != 0) throw std::runtime_error("Schwarz: singular block");
  }
  void solve(Vec& x, const Vec& b) override {
    Vec r(b.size());
    for (int s = 0; s < updates; ++s) {
      r = b;
      spmv(*A, -1.0, x.data(), 1.0, r.data());
      spmv(M, 1.0, r.data(), 1.0, x.data());
    }
    converged = true;
  }
};

// Additive Schwarz with multi-cell blocks (Schwarz.cs:56).  Blocks: METISBlockingStrategy (Schwarz.cs:190-320)
// partitions the cell graph into NoOfPartsOnCurrentProcess parts with METIS; the restatement partitions it with a
// greedy breadth-first aggregation (seeds in ascending cell order, neighbours in ascending order, ceil(nb/parts)
// cells per block), then grows every block by `overlap` layers as Schwarz.cs:690-735 (each sweep visits the members
// present at its start) and sorts it.  Solve (:996-1147): per iteration Res = B - A X (the product skipped while X
// is zero), every block's dense system solved and its solution added to X, then X scaled by one over the number of
// blocks covering each DOF with overlap and EnableOverlapScaling (:790-815, :1093-1104).
std::vector<std::vector<int32_t>> schwarz_partition_mat(const Mat& A, int64_t parts) {
  const int64_t target = std::max<int64_t>(1, (A.nb + parts - 1) / parts);
  std::vector<int32_t> part(A.nb, -1);
  std::vector<std::vector<int32_t>> blocks;
  for (int64_t seed = 0; seed < A.nb; ++seed) {
    if (part[seed] >= 0) continue;
    const int32_t id = (int32_t)blocks.size();
    std::vector<int32_t> q(1, (int32_t)seed);
    part[seed] = id;
    size_t head = 0;
    while (head < q.size() && (int64_t)q.size() < target) {
      const int32_t c = q[head++];
      for (int64_t k = A.rp[c]; k < A.rp[c + 1] && (int64_t)q.size() < target; ++k) {
        const int32_t j = A.ci[k];
        if (j != c && part[j] < 0) {
          part[j] = id;
          q.push_back(j);
        }
      }
    }
    std::sort(q.begin(), q.end());
    blocks.push_back(q);
  }
  return blocks;
}

void schwarz_extend_mat(const Mat& A, std::vector<std::vector<int32_t>>& blocks, int overlap) {
  std::vector<char> marker(A.nb, 0);
  for (auto& bl : blocks) {
    for (int32_t c : bl) marker[c] = 1;
    for (int s = 0; s < overlap; ++s) {
      const size_t members = bl.size();
      for (size_t m = 0; m < members; ++m)
        for (int64_t k = A.rp[bl[m]]; k < A.rp[bl[m] + 1]; ++k)
          if (!marker[A.ci[k]]) {
            marker[A.ci[k]] = 1;
            bl.push_back(A.ci[k]);
          }
    }
    std::sort(bl.begin(), bl.end());
    for (int32_t c : bl) marker[c] = 0;
  }
}

struct BlockSchwarz : Solver {
  const Mat* A;
  std::vector<std::vector<int64_t>> dofs;   // DOFs of every block
  std::vector<std::vector<double>> inv;     // dense inverses, row-major
  std::vector<double> scale;                // 1 / multiplicity, or empty
  int iters;
  BlockSchwarz(const Mat* A_, int64_t parts, int overlap, bool scaling, int iters_) : A(A_), iters(iters_) {
    auto blocks = schwarz_partition_mat(*A, parts > 0 ? parts : std::max<int64_t>(1, (A->nb + 7) / 8));
    schwarz_extend_mat(*A, blocks, overlap);
    std::vector<int> count(A->N, 0);
    for (auto& bl : blocks) {
      std::vector<int64_t> d;
      std::vector<int64_t> first;  // local offset of each cell
      for (int32_t c : bl) {
        first.push_back((int64_t)d.size());
        for (int64_t g = A->i0[c]; g < A->i0[c + 1]; ++g) {
          d.push_back(g);
          count[g]++;
        }
      }
      const int64_t n = (int64_t)d.size();
      std::vector<double> M((size_t)(n * n), 0.0);
      for (size_t p = 0; p < bl.size(); ++p)
        for (size_t q = 0; q < bl.size(); ++q) {
          const int64_t k = find_block(*A, bl[p], bl[q]);
          if (k < 0) continue;
          const int I = A->len[bl[p]], J = A->len[bl[q]];
          for (int r = 0; r < I; ++r)
            for (int cc = 0; cc < J; ++cc) M[(first[p] + r) * n + first[q] + cc] = A->blk(k)[r * J + cc];
        }
      if (invert((int)n, M.data()) != 0) throw std::runtime_error("Schwarz: singular block");
      dofs.push_back(d);
      inv.push_back(M);
    }
    if (scaling && overlap > 0) {
      scale.resize(A->N);
      for (int64_t g = 0; g < A->N; ++g) scale[g] = 1.0 / count[g];
    }
  }
  void solve(Vec& x, const Vec& b) override {
    Vec r(b.size());
    for (int it = 0; it < iters; ++it) {
      r = b;
      if (dot(x, x) != 0.0) spmv(*A, -1.0, x.data(), 1.0, r.data());
#pragma omp parallel for schedule(dynamic, 4)
      for (int64_t bi = 0; bi < (int64_t)dofs.size(); ++bi) {
        const auto& d = dofs[bi];
        const int64_t n = (int64_t)d.size();
        std::vector<double> y(n, 0.0);
        for (int64_t p = 0; p < n; ++p) {
          double acc = 0.0;
          for (int64_t q = 0; q < n; ++q) acc += inv[bi][p * n + q] * r[d[q]];
          y[p] = acc;
        }
        for (int64_t p = 0; p < n; ++p) {
#pragma omp atomic
          x[d[p]] += y[p];
        }
      }
      if (!scale.empty())
        for (int64_t g = 0; g < A->N; ++g) x[g] *= scale[g];
    }
    converged = true;
  }
};

// Block ILU(0) smoother (CellILU.Solve, CellILU.cs:182-250): x = U^{-1} L^{-1} b with the factors computed in the
// natural cell order (the reference's) or with the cells ordered by a greedy colouring of the block graph (colour
// 0 first; the order the GPU smoother uses).
struct ILUSmoother : Solver {
  const Mat* A;
  std::vector<double> F;
  std::vector<int32_t> order;
  ILUSmoother(const Mat* A_, bool coloured) : A(A_) {
    if (coloured) {
      std::vector<int32_t> col(A->nb, -1);
      int ncol = 0;
      for (int64_t i = 0; i < A->nb; ++i) {
        std::vector<char> used(ncol + 1, 0);
        for (int64_t k = A->rp[i]; k < A->rp[i + 1]; ++k)
          if (A->ci[k] != i && col[A->ci[k]] >= 0) used[col[A->ci[k]]] = 1;
        int cc = 0;
        while (cc < ncol && used[cc]) ++cc;
        col[i] = cc;
        if (cc == ncol) ++ncol;
      }
      for (int cc = 0; cc < ncol; ++cc)
        for (int64_t i = 0; i < A->nb; ++i)
          if (col[i] == cc) order.push_back((int32_t)i);
    }
    F.assign(A->vp.back(), 0.0);
    ilu0_factor_mat(*A, order.empty() ? nullptr : order.data(), F.data());
  }
  void solve(Vec& x, const Vec& b) override {
    if (ilu0_solve_mat(*A, order.empty() ? nullptr : order.data(), F.data(), b.data(), x.data()) != 0)
      throw std::runtime_error("ILU: singular pivot block");
    converged = true;
  }
};

Solver* build_level(const Mat* A, const or_solver_cfg* c, int level, std::vector<Restriction*>& keep);

Solver* make_coarsest(const Mat* A, const or_solver_cfg* c) {
  if (c->coarse_kind == OR_COARSE_DENSE) return new DenseDirect(A);
  Term t;
  t.mode = 1;
  t.tol = c->coarse_tol;
  t.max_iter = c->coarse_max_iter;
  t.min_iter = 0;
  return new SoftPCG(A, new BlockJacobi(A, 0, 1.0), t);
}

// PmgConfig.CreateInstanceImpl__Kummer (PmgConfig.cs:80-245), UseILU = false: every OrthoMG level uses a
// BlockJacobi post-smoother with NoOfPostSmootherSweeps = 10; coarse correction through GridAndDegRestriction.
Solver* build_level(const Mat* A, const or_solver_cfg* c, int level, std::vector<Restriction*>& keep) {
  if (level == c->n_levels - 1) return make_coarsest(A, c);
  Term t;
  if (level == 0) {
    t.mode = c->top_mode;
    t.tol = c->tol;
    t.max_iter = c->max_iter;
    t.min_iter = c->min_iter;
  } else {
    t.mode = 3;
    t.reduction = c->sub_reduction;
    t.max_iter = c->sub_max_iter;
  }
  auto* omg = new OrthoMG(A, t);
  omg->ortho.recalc_period = c->recalc_resi_period;
  omg->sweeps = c->post_sweeps;
  if (c->smoother == OR_SMOOTHER_SCHWARZ)
    omg->post = new SchwarzSmoother(A, c->bj_iters);
  else if (c->smoother == OR_SMOOTHER_SCHWARZ_BLOCKS)
    omg->post = new BlockSchwarz(A, c->schwarz_parts, c->schwarz_overlap, c->schwarz_scaling != 0, c->bj_iters + 1);
  else if (c->smoother == OR_SMOOTHER_ILU_COLOURED || c->smoother == OR_SMOOTHER_ILU_NATURAL)
    omg->post = new ILUSmoother(A, c->smoother == OR_SMOOTHER_ILU_COLOURED);
  else
    omg->post = new BlockJacobi(A, c->bj_iters, c->bj_omega);
  auto* gr = new GridAndDegRestriction(A, c->level_keep[level + 1]);
  gr->lower = build_level(&gr->R.sub, c, level + 1, keep);
  omg->coarse = gr;
  return omg;
}

}  // namespace

extern "C" {

const char* or_last_error(void) { return g_err.c_str(); }

int or_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

int or_spmv(const or_bsr* m, double alpha, const double* x, double beta, double* y) {
  try {
    Mat A;
    load_mat(A, m);
    spmv(A, alpha, x, beta, y);
    return 0;
  } catch (std::exception& e) {
    g_err = e.what();
    return OR_ERR_ARGUMENT;
  }
}

int or_symminv(int n, double* M, double* L) { return symminv(n, M, L); }
int or_invert(int n, double* A) { return invert(n, A); }

int or_change_of_basis(const or_bsr* m, double* values_out, double* L_out) {
  try {
    Mat A, Ap;
    load_mat(A, m);
    std::vector<double> L;
    int e = change_of_basis(A, Ap, L);
    if (e) { g_err = "SymmInv failed (zero or non-unit diagonal)"; return e; }
    std::copy(Ap.v.begin(), Ap.v.end(), values_out);
    if (L_out) std::copy(L.begin(), L.end(), L_out);
    return 0;
  } catch (std::exception& e) {
    g_err = e.what();
    return OR_ERR_ARGUMENT;
  }
}

int or_restrict(const or_bsr* m, int keep, double* values_out, int64_t* map_out) {
  try {
    Mat A;
    load_mat(A, m);
    Restriction R(&A, keep);
    std::copy(R.sub.v.begin(), R.sub.v.end(), values_out);
    if (map_out) std::copy(R.map.begin(), R.map.end(), map_out);
    return 0;
  } catch (std::exception& e) {
    g_err = e.what();
    return OR_ERR_ARGUMENT;
  }
}

// Schwarz block set-up restated for blocks = one cell plus the cells of its block row (overlap 1), restricted
// form: the rows of the centre cell of each block inverse (Schwarz.cs:623-840 extracts each block's sub-matrix
// and factors it with LAPACK; here the sub-matrix is inverted with InvertInPlace).  values_out has A's layout.
int or_schwarz_rows(const or_bsr* m, double* values_out) {
  try {
    Mat A;
    load_mat(A, m);
    return schwarz_rows_mat(A, values_out);
  } catch (std::exception& e) {
    g_err = e.what();
    return OR_ERR_ARGUMENT;
  }
}

// Block ILU(0) (CellILU.ComputeILU, CellILU.cs:1229-1330, ILU_level = 0 as PmgConfig.cs:131 sets it): Saad's
// in-place KIJ form over the block rows taken in the order `order` (NULL: natural order, the reference's).
// factor_out receives the factors in A's layout: strictly lower blocks L_ik (unit lower factor), upper blocks and
// the diagonal U_ij.  A diagonal block whose factorisation fails is skipped, as the reference does.
int or_ilu0_factor(const or_bsr* m, const int32_t* order, double* factor_out) {
  try {
    Mat A;
    load_mat(A, m);
    return ilu0_factor_mat(A, order, factor_out);
  } catch (std::exception& e) {
    g_err = e.what();
    return OR_ERR_ARGUMENT;
  }
}

// x = U^{-1} L^{-1} b with the factors of or_ilu0_factor (CellILU.Solve, CellILU.cs:182-250: LoTriDiagonalSolve
// with the unit lower factor, then UpTriDiagonalSolve with the upper factor and its diagonal blocks).
int or_ilu0_solve(const or_bsr* m, const int32_t* order, const double* factor, const double* b, double* x) {
  try {
    Mat A;
    load_mat(A, m);
    return ilu0_solve_mat(A, order, factor, b, x);
  } catch (std::exception& e) {
    g_err = e.what();
    return OR_ERR_ARGUMENT;
  }
}

int or_schwarz_blocks(const or_bsr* m, int64_t parts, int overlap, int64_t* ptr, int32_t* cells, int64_t* nblocks,
                      int64_t* total) {
  try {
    Mat A;
    load_mat(A, m);
    auto blocks = schwarz_partition_mat(A, parts > 0 ? parts : std::max<int64_t>(1, (A.nb + 7) / 8));
    schwarz_extend_mat(A, blocks, overlap);
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
    return 0;
  } catch (std::exception& e) {
    g_err = e.what();
    return OR_ERR_ARITHMETIC;
  }
}

int or_block_schwarz(const or_bsr* m, int64_t parts, int overlap, int scaling, int iters, double* x, const double* b) {
  try {
    Mat A;
    load_mat(A, m);
    BlockSchwarz s(&A, parts, overlap, scaling != 0, iters);
    Vec X(x, x + A.N), B(b, b + A.N);
    s.solve(X, B);
    std::copy(X.begin(), X.end(), x);
    return 0;
  } catch (std::exception& e) {
    g_err = e.what();
    return OR_ERR_ARITHMETIC;
  }
}

int or_blockjacobi(const or_bsr* m, int iters, double omega, double* x, const double* b) {
  try {
    Mat A;
    load_mat(A, m);
    BlockJacobi bj(&A, iters, omega);
    Vec X(x, x + A.N), B(b, b + A.N);
    bj.solve(X, B);
    std::copy(X.begin(), X.end(), x);
    return 0;
  } catch (std::exception& e) {
    g_err = e.what();
    return OR_ERR_ARITHMETIC;
  }
}

// Persistent solver: set-up once (level matrices, block inverses), solve many times.
struct or_solver_s {
  Mat A;
  Solver* s = nullptr;
  std::vector<Restriction*> keep;
  std::vector<double> hist;
  ~or_solver_s() { delete s; }
};

or_solver_t or_solver_create(const or_bsr* m, const or_solver_cfg* c) {
  try {
    auto* h = new or_solver_s();
    load_mat(h->A, m);
    Term top;
    top.mode = c->top_mode;
    top.tol = c->tol;
    top.max_iter = c->max_iter;
    top.min_iter = c->min_iter;
    if (c->solver == OR_SOLVER_FGMRES_PMG) {
      or_solver_cfg pc = *c;
      pc.top_mode = 2;
      pc.max_iter = 1;
      Solver* prec = build_level(&h->A, &pc, 0, h->keep);
      auto* f = new FlexGMRES(&h->A, prec, c->max_krylov, top);
      f->reference_defect = c->reference_fgmres_defect != 0;
      f->hist = &h->hist;
      h->s = f;
    } else if (c->solver == OR_SOLVER_ORTHOMG) {
      h->s = build_level(&h->A, c, 0, h->keep);
    } else {
      h->s = new SoftPCG(&h->A, c->bj_iters >= 0 ? new BlockJacobi(&h->A, c->bj_iters, c->bj_omega) : nullptr, top);
    }
    return h;
  } catch (std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}

int or_solver_solve(or_solver_t h, const double* b, double* x, or_stats* stats) {
  try {
    Vec X(x, x + h->A.N), B(b, b + h->A.N);
    h->hist.clear();
    h->s->this_level_iterations = 0;
    h->s->solve(X, B);
    std::copy(X.begin(), X.end(), x);
    if (stats) {
      stats->iterations = h->s->this_level_iterations;
      stats->nested = h->s->nested();
      stats->converged = h->s->converged ? 1 : 0;
      stats->n_hist = (int)h->hist.size();
      stats->res0 = h->hist.empty() ? 0 : h->hist.front();
      stats->res = h->hist.empty() ? 0 : h->hist.back();
    }
    return 0;
  } catch (std::exception& e) {
    g_err = e.what();
    return OR_ERR_ARITHMETIC;
  }
}

void or_solver_destroy(or_solver_t h) { delete h; }

int or_solve(const or_bsr* m, const or_solver_cfg* c, const double* b, double* x, or_stats* stats,
             double* hist, int hist_cap) {
  try {
    Mat A;
    load_mat(A, m);
    Vec X(x, x + A.N), B(b, b + A.N);
    std::vector<double> h;
    std::vector<Restriction*> keep;
    Solver* s = nullptr;
    Term top;
    top.mode = c->top_mode;
    top.tol = c->tol;
    top.max_iter = c->max_iter;
    top.min_iter = c->min_iter;
    if (c->solver == OR_SOLVER_PCG) {
      auto* p = new SoftPCG(&A, c->bj_iters >= 0 ? new BlockJacobi(&A, c->bj_iters, c->bj_omega) : nullptr, top);
      p->hist = &h;
      s = p;
    } else if (c->solver == OR_SOLVER_ORTHOMG) {
      s = build_level(&A, c, 0, keep);
      static_cast<OrthoMG*>(s)->hist = &h;
    } else if (c->solver == OR_SOLVER_FGMRES_PMG) {
      or_solver_cfg pc = *c;
      pc.top_mode = 2;  // one V-cycle per preconditioner call
      pc.max_iter = 1;
      Solver* prec = build_level(&A, &pc, 0, keep);
      auto* f = new FlexGMRES(&A, prec, c->max_krylov, top);
      f->reference_defect = c->reference_fgmres_defect != 0;
      f->hist = &h;
      s = f;
    } else if (c->solver == OR_SOLVER_SOFTGMRES) {
      auto* g = new SoftGMRES(&A, c->bj_iters >= 0 ? new BlockJacobi(&A, c->bj_iters, c->bj_omega) : nullptr,
                              c->max_krylov, top);
      g->hist = &h;
      s = g;
    } else {
      g_err = "unknown solver kind";
      return OR_ERR_ARGUMENT;
    }
    s->solve(X, B);
    std::copy(X.begin(), X.end(), x);
    if (stats) {
      stats->iterations = s->this_level_iterations;
      stats->nested = s->nested();
      stats->converged = s->converged ? 1 : 0;
      stats->n_hist = (int)h.size();
      Vec R = B;
      spmv(A, -1.0, X.data(), 1.0, R.data());
      stats->res = nrm2(R);
      stats->res0 = h.empty() ? 0 : h[0];
    }
    if (hist)
      for (int i = 0; i < hist_cap && i < (int)h.size(); ++i) hist[i] = h[i];
    delete s;
    return 0;
  } catch (std::exception& e) {
    g_err = e.what();
    return OR_ERR_ARITHMETIC;
  }
}

}  // extern "C"
