// Smoothed-aggregation AMG below the coarsest p-level.
//
// BoSSS solves its coarsest p-level with a sparse direct solver (PARDISO in single precision, PmgConfig.cs:167-177;
// DirectSolver.cs:308-345).  No sparse direct factorisation is written here; instead the coarsest level is solved
// by CG preconditioned with a smoothed-aggregation V-cycle (Vanek, Mandel, Brezina 1996), set up once on the host
// from the level matrix:
//   * aggregates: greedy, on the block graph for the block level (cells) and on the strong-connection graph
//     (|a_ij| >= theta*sqrt(|a_ii a_jj|)) for the scalar levels;
//   * near-null space: the constant function, which in the orthonormal, lower-triangularly transformed DG basis
//     lives in mode 0 of every block only; tentative prolongator = that vector, normalised per aggregate;
//   * P = (I - omega D^-1 A) P_tent with omega = 4 / (3 rho(D^-1 A)) (power iteration), A_c = P^T A P;
//   * last level (<= dense_limit unknowns): dense inverse.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>

#include "aggregation.cuh"
#include "amg.cuh"

namespace bsgpu {

namespace {

struct HCsr {
  int64_t rows = 0, cols = 0;
  std::vector<int64_t> rp;
  std::vector<int32_t> ci;
  std::vector<double> v;
};

HCsr block_to_csr(const Matrix& A, cudaStream_t st) {
  std::vector<double> vals(A.nvals);
  if (A.nvals) matrix_read_values(A, vals.data(), false, st);
  HCsr M;
  M.rows = M.cols = A.N;
  M.rp.assign(A.N + 1, 0);
  for (int64_t i = 0; i < A.nb; ++i) {
    int64_t w = 0;
    for (int64_t k = A.h_rp[i]; k < A.h_rp[i + 1]; ++k) w += A.h_len[A.h_ci[k]];
    for (int r = 0; r < A.h_len[i]; ++r) M.rp[A.h_i0[i] + r + 1] = w;
  }
  for (int64_t r = 0; r < A.N; ++r) M.rp[r + 1] += M.rp[r];
  M.ci.resize(M.rp.back());
  M.v.resize(M.rp.back());
  int64_t off = 0;
  for (int64_t i = 0; i < A.nb; ++i) {
    const int I = A.h_len[i];
    std::vector<int64_t> pos(I);
    for (int r = 0; r < I; ++r) pos[r] = M.rp[A.h_i0[i] + r];
    for (int64_t k = A.h_rp[i]; k < A.h_rp[i + 1]; ++k) {
      const int32_t j = A.h_ci[k];
      const int J = A.h_len[j];
      for (int r = 0; r < I; ++r)
        for (int c = 0; c < J; ++c) {
          M.ci[pos[r]] = (int32_t)(A.h_i0[j] + c);
          M.v[pos[r]] = vals[off + (int64_t)r * J + c];
          ++pos[r];
        }
      off += (int64_t)I * J;
    }
  }
  return M;
}

std::vector<double> diagonal(const HCsr& A) {
  std::vector<double> d(A.rows, 0.0);
  for (int64_t r = 0; r < A.rows; ++r)
    for (int64_t k = A.rp[r]; k < A.rp[r + 1]; ++k)
      if (A.ci[k] == r) d[r] = A.v[k];
  return d;
}

void csr_mv(const HCsr& A, const std::vector<double>& x, std::vector<double>& y) {
  y.assign(A.rows, 0.0);
  for (int64_t r = 0; r < A.rows; ++r) {
    double s = 0;
    for (int64_t k = A.rp[r]; k < A.rp[r + 1]; ++k) s += A.v[k] * x[A.ci[k]];
    y[r] = s;
  }
}

// largest eigenvalue of D^-1 A by power iteration
double rho_dinv_a(const HCsr& A, const std::vector<double>& d) {
  std::mt19937_64 g(7);
  std::uniform_real_distribution<double> U(-1, 1);
  std::vector<double> x(A.rows), y;
  for (auto& t : x) t = U(g);
  double lam = 1.0;
  for (int it = 0; it < 20; ++it) {
    csr_mv(A, x, y);
    double n2 = 0;
    for (int64_t r = 0; r < A.rows; ++r) {
      y[r] /= (d[r] != 0 ? d[r] : 1.0);
      n2 += y[r] * y[r];
    }
    double nx = 0;
    for (double t : x) nx += t * t;
    lam = std::sqrt(n2 / std::max(nx, 1e-300));
    const double s = 1.0 / std::sqrt(std::max(n2, 1e-300));
    for (int64_t r = 0; r < A.rows; ++r) x[r] = y[r] * s;
  }
  return lam;
}

// greedy aggregation of a graph (rp, ci); `strong(row, k)` tells whether entry k of row is a strong connection
template <typename Strong>
std::vector<int32_t> aggregate(int64_t n, const std::vector<int64_t>& rp, const std::vector<int32_t>& ci,
                               Strong strong, int32_t& nagg) {
  std::vector<int32_t> agg(n, -1);
  nagg = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (agg[i] >= 0) continue;
    bool free = true;
    for (int64_t k = rp[i]; k < rp[i + 1] && free; ++k)
      if (strong(i, k) && agg[ci[k]] >= 0) free = false;
    if (!free) continue;
    agg[i] = nagg;
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k)
      if (strong(i, k)) agg[ci[k]] = nagg;
    ++nagg;
  }
  std::vector<int32_t> a2 = agg;
  for (int64_t i = 0; i < n; ++i) {
    if (agg[i] >= 0) continue;
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k)
      if (strong(i, k) && agg[ci[k]] >= 0) { a2[i] = agg[ci[k]]; break; }
  }
  for (int64_t i = 0; i < n; ++i)
    if (a2[i] < 0) a2[i] = nagg++;
  return a2;
}

// C = A * B (sparse x sparse, row by row with a dense marker); columns sorted
HCsr spgemm(const HCsr& A, const HCsr& B) {
  HCsr C;
  C.rows = A.rows;
  C.cols = B.cols;
  C.rp.assign(A.rows + 1, 0);
  std::vector<int64_t> mark(B.cols, -1);
  std::vector<double> acc(B.cols, 0.0);
  std::vector<int32_t> cols;
  for (int64_t r = 0; r < A.rows; ++r) {
    cols.clear();
    for (int64_t k = A.rp[r]; k < A.rp[r + 1]; ++k) {
      const int32_t j = A.ci[k];
      const double a = A.v[k];
      for (int64_t q = B.rp[j]; q < B.rp[j + 1]; ++q) {
        const int32_t c = B.ci[q];
        if (mark[c] != r) {
          mark[c] = r;
          acc[c] = 0.0;
          cols.push_back(c);
        }
        acc[c] += a * B.v[q];
      }
    }
    std::sort(cols.begin(), cols.end());
    for (int32_t c : cols) {
      C.ci.push_back(c);
      C.v.push_back(acc[c]);
    }
    C.rp[r + 1] = (int64_t)C.ci.size();
  }
  return C;
}

HCsr transpose(const HCsr& A) {
  HCsr T;
  T.rows = A.cols;
  T.cols = A.rows;
  T.rp.assign(A.cols + 1, 0);
  for (int32_t c : A.ci) T.rp[c + 1]++;
  for (int64_t r = 0; r < A.cols; ++r) T.rp[r + 1] += T.rp[r];
  T.ci.resize(A.ci.size());
  T.v.resize(A.v.size());
  std::vector<int64_t> pos(T.rp.begin(), T.rp.end() - 1);
  for (int64_t r = 0; r < A.rows; ++r)
    for (int64_t k = A.rp[r]; k < A.rp[r + 1]; ++k) {
      const int64_t p = pos[A.ci[k]]++;
      T.ci[p] = (int32_t)r;
      T.v[p] = A.v[k];
    }
  return T;
}

std::unique_ptr<Csr> upload(const HCsr& M) {
  auto d = std::make_unique<Csr>();
  d->rows = M.rows;
  d->cols = M.cols;
  d->nnz = (int64_t)M.ci.size();
  require(d->nnz < (int64_t)1 << 31, "AMG transfer operator too large", BSGPU_ERR_UNSUPPORTED);
  std::vector<int32_t> rp(M.rp.begin(), M.rp.end());
  d->rp.alloc(M.rows + 1);
  d->ci.alloc(std::max<int64_t>(d->nnz, 1));
  d->v64.alloc(std::max<int64_t>(d->nnz, 1));
  d->v32.alloc(std::max<int64_t>(d->nnz, 1));
  BSGPU_CUDA(cudaMemcpy(d->rp.p, rp.data(), (M.rows + 1) * 4, cudaMemcpyHostToDevice));
  if (d->nnz) {
    std::vector<float> v32(M.v.begin(), M.v.end());
    BSGPU_CUDA(cudaMemcpy(d->ci.p, M.ci.data(), d->nnz * 4, cudaMemcpyHostToDevice));
    BSGPU_CUDA(cudaMemcpy(d->v64.p, M.v.data(), d->nnz * 8, cudaMemcpyHostToDevice));
    BSGPU_CUDA(cudaMemcpy(d->v32.p, v32.data(), d->nnz * 4, cudaMemcpyHostToDevice));
  }
  return d;
}

void set_diag(AmgLevel& L, const std::vector<double>& d) {
  std::vector<double> inv(d.size());
  std::vector<float> inv32(d.size());
  for (size_t i = 0; i < d.size(); ++i) {
    inv[i] = d[i] != 0 ? 1.0 / d[i] : 0.0;
    inv32[i] = (float)inv[i];
  }
  L.dinv64.alloc(std::max<size_t>(d.size(), 1));
  L.dinv32.alloc(std::max<size_t>(d.size(), 1));
  if (!d.empty()) {
    BSGPU_CUDA(cudaMemcpy(L.dinv64.p, inv.data(), d.size() * 8, cudaMemcpyHostToDevice));
    BSGPU_CUDA(cudaMemcpy(L.dinv32.p, inv32.data(), d.size() * 4, cudaMemcpyHostToDevice));
  }
}

template <typename T>
__global__ void csr_spmv_kernel(int64_t rows, const int32_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                const T* __restrict__ v, T alpha, const T* __restrict__ x, T beta,
                                T* __restrict__ y) {
  // 8 threads per row
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t row = t >> 3;
  const int lane = threadIdx.x & 7;
  double s = 0.0;
  if (row < rows)
    for (int32_t k = rp[row] + lane; k < rp[row + 1]; k += 8) s = fma((double)v[k], (double)x[ci[k]], s);
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o, 8);
  if (row < rows && lane == 0) y[row] = (T)(alpha * s + (beta != T(0) ? (double)beta * (double)y[row] : 0.0));
}

// Ax == nullptr: x is taken as zero (first sweep from a zero guess), x = omega * Dinv b
template <typename T>
__global__ void jacobi_kernel(const T* __restrict__ dinv, T omega, const T* __restrict__ b, const T* __restrict__ Ax,
                              T* __restrict__ x, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (Ax)
      x[i] += omega * dinv[i] * (b[i] - Ax[i]);
    else
      x[i] = omega * dinv[i] * b[i];
  }
}

int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 8)); }

}  // namespace

AmgHierarchy* amg_setup(const Matrix& A0, int max_levels, int dense_limit, cudaStream_t st) {
  require(!A0.single, "AMG set-up needs the FP64 level matrix");
  auto H = std::make_unique<AmgHierarchy>();
  HCsr A = block_to_csr(A0, st);
  // near-null vector: mode 0 of every block
  std::vector<double> B(A.rows, 0.0);
  for (int64_t i = 0; i < A0.nb; ++i) B[A0.h_i0[i]] = 1.0;
  const double theta = 0.08;
  for (int lev = 0;; ++lev) {
    H->levels.emplace_back();
    AmgLevel& L = H->levels.back();
    L.n = A.rows;
    std::vector<double> d = diagonal(A);
    set_diag(L, d);
    const double rho = rho_dinv_a(A, d);
    L.omega = 4.0 / (3.0 * rho);
    if (lev == 0) {
      L.Aref = &A0;
    } else {
      L.A.reset(matrix_create(A.rows, 1, nullptr, A.rp.data(), A.ci.data(), A.v.data(), BSGPU_HOST_POINTERS));
      L.Aref = L.A.get();
    }
    if (A.rows <= dense_limit || lev >= max_levels) break;
    // aggregates
    int32_t nagg = 0;
    std::vector<int32_t> agg;
    std::vector<int32_t> dof2agg(A.rows, -1);
    if (lev == 0) {
      auto all = [](int64_t, int64_t) { return true; };
      agg = aggregate(A0.nb, A0.h_rp, A0.h_ci, all, nagg);
      for (int64_t i = 0; i < A0.nb; ++i) dof2agg[A0.h_i0[i]] = agg[i];  // only mode-0 rows carry B
    } else {
      auto strong = [&](int64_t r, int64_t k) {
        const int32_t c = A.ci[k];
        return c == r || std::fabs(A.v[k]) >= theta * std::sqrt(std::fabs(d[r] * d[c]));
      };
      agg = aggregate(A.rows, A.rp, A.ci, strong, nagg);
      dof2agg = agg;
    }
    if (nagg >= A.rows) break;  // no coarsening possible
    // tentative prolongator: B normalised per aggregate
    std::vector<double> norm(nagg, 0.0);
    for (int64_t r = 0; r < A.rows; ++r)
      if (dof2agg[r] >= 0) norm[dof2agg[r]] += B[r] * B[r];
    for (auto& t : norm) t = std::sqrt(t);
    HCsr Pt;
    Pt.rows = A.rows;
    Pt.cols = nagg;
    Pt.rp.assign(A.rows + 1, 0);
    for (int64_t r = 0; r < A.rows; ++r) {
      if (dof2agg[r] >= 0 && norm[dof2agg[r]] > 0) {
        Pt.ci.push_back(dof2agg[r]);
        Pt.v.push_back(B[r] / norm[dof2agg[r]]);
      }
      Pt.rp[r + 1] = (int64_t)Pt.ci.size();
    }
    if (lev > 0) {
      // below the first level the tentative prolongator is used unsmoothed: smoothing it again would widen the
      // Galerkin stencils level by level until the small levels are dense
      HCsr R = transpose(Pt);
      HCsr Ac = spgemm(R, spgemm(A, Pt));
      L.P = upload(Pt);
      L.R = upload(R);
      B = norm;
      A = std::move(Ac);
      continue;
    }
    // smoothed prolongator P = Pt - omega D^-1 A Pt
    HCsr AP = spgemm(A, Pt);
    HCsr P;
    P.rows = A.rows;
    P.cols = nagg;
    P.rp.assign(A.rows + 1, 0);
    const double w = L.omega;
    for (int64_t r = 0; r < A.rows; ++r) {
      const double s = d[r] != 0 ? w / d[r] : 0.0;
      int64_t q = Pt.rp[r];
      for (int64_t k = AP.rp[r]; k < AP.rp[r + 1]; ++k) {
        double val = -s * AP.v[k];
        if (q < Pt.rp[r + 1] && Pt.ci[q] == AP.ci[k]) val += Pt.v[q++];
        P.ci.push_back(AP.ci[k]);
        P.v.push_back(val);
      }
      for (; q < Pt.rp[r + 1]; ++q) {  // tentative entries without an A*Pt counterpart
        P.ci.push_back(Pt.ci[q]);
        P.v.push_back(Pt.v[q]);
      }
      P.rp[r + 1] = (int64_t)P.ci.size();
    }
    HCsr R = transpose(P);
    HCsr Ac = spgemm(R, spgemm(A, P));
    L.P = upload(P);
    L.R = upload(R);
    B = norm;
    A = std::move(Ac);
  }
  // dense inverse of the last level
  AmgLevel& last = H->levels.back();
  if (last.n <= 4096 && H->levels.size() > 1) {
    dense_inverse(*last.Aref, H->dense_inv, st);
    H->n_dense = last.n;
  }
  return H.release();
}

namespace {

// scalar CSR with uniform Np x Np block structure -> block-CSR Matrix (row-major blocks)
Matrix* csr_to_matrix(const HCsr& A, int Np) {
  require(A.rows % Np == 0, "internal: level size not a multiple of the block size");
  const int64_t nb = A.rows / Np;
  std::vector<int64_t> rp(nb + 1, 0);
  std::vector<int32_t> ci;
  std::vector<double> v;
  std::vector<int32_t> cols;
  for (int64_t b = 0; b < nb; ++b) {
    cols.clear();
    for (int r = 0; r < Np; ++r)
      for (int64_t k = A.rp[b * Np + r]; k < A.rp[b * Np + r + 1]; ++k) cols.push_back(A.ci[k] / Np);
    std::sort(cols.begin(), cols.end());
    cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
    const size_t base = v.size();
    v.resize(base + cols.size() * Np * Np, 0.0);
    for (int r = 0; r < Np; ++r)
      for (int64_t k = A.rp[b * Np + r]; k < A.rp[b * Np + r + 1]; ++k) {
        const int32_t cb = A.ci[k] / Np, cc = A.ci[k] % Np;
        const size_t q = std::lower_bound(cols.begin(), cols.end(), cb) - cols.begin();
        v[base + q * Np * Np + (size_t)r * Np + cc] += A.v[k];
      }
    ci.insert(ci.end(), cols.begin(), cols.end());
    rp[b + 1] = (int64_t)ci.size();
  }
  return matrix_create(nb, Np, nullptr, rp.data(), ci.data(), v.data(), BSGPU_HOST_POINTERS);
}

void dense_inverse_csr(const HCsr& A, std::vector<double>& inv) {
  const int64_t n = A.rows;
  require(n <= 4096, "dense direct solve limited to 4096 unknowns", BSGPU_ERR_UNSUPPORTED);
  std::vector<double> M((size_t)n * n, 0.0);
  for (int64_t r = 0; r < n; ++r)
    for (int64_t k = A.rp[r]; k < A.rp[r + 1]; ++k) M[r * n + A.ci[k]] += A.v[k];
  inv.assign((size_t)n * n, 0.0);
  for (int64_t i = 0; i < n; ++i) inv[i * n + i] = 1.0;
  for (int64_t p = 0; p < n; ++p) {
    int64_t best = p;
    for (int64_t r = p + 1; r < n; ++r)
      if (std::fabs(M[r * n + p]) > std::fabs(M[best * n + p])) best = r;
    if (!(std::fabs(M[best * n + p]) > 0.0)) throw Error(BSGPU_ERR_ARITHMETIC, "dense direct solve: singular matrix");
    if (best != p) {
      std::swap_ranges(M.begin() + p * n, M.begin() + (p + 1) * n, M.begin() + best * n);
      std::swap_ranges(inv.begin() + p * n, inv.begin() + (p + 1) * n, inv.begin() + best * n);
    }
    const double d = 1.0 / M[p * n + p];
    for (int64_t c = 0; c < n; ++c) {
      M[p * n + c] *= d;
      inv[p * n + c] *= d;
    }
    for (int64_t r = 0; r < n; ++r) {
      if (r == p) continue;
      const double f = M[r * n + p];
      if (f == 0.0) continue;
      for (int64_t c = 0; c < n; ++c) {
        M[r * n + c] -= f * M[p * n + c];
        inv[r * n + c] -= f * inv[p * n + c];
      }
    }
  }
}

}  // namespace

HmgHierarchy* hmg_setup(const Matrix& Ap, const Matrix& top, const double* Ltop, int keep,
                        const std::vector<HostBsr>& prol, int dense_limit, cudaStream_t st) {
  require(!Ap.single && Ap.uniform && top.uniform, "h-levels need an FP64 operator with one species per block");
  require(!prol.empty(), "no h-level prolongations were given to the MultigridOperator");
  require(Ap.Np == keep, "internal: coarsest p-level block size");
  auto H = std::make_unique<HmgHierarchy>();
  HCsr A = block_to_csr(Ap, st);
  // U_i = (L_p,i)^{-T} for the first prolongation
  std::vector<double> U;
  const int Nt = top.Np;
  if (Ltop) {
    std::vector<double> Lh((size_t)top.nb * Nt * Nt);
    BSGPU_CUDA(cudaMemcpy(Lh.data(), Ltop, Lh.size() * 8, cudaMemcpyDeviceToHost));
    U.assign((size_t)top.nb * keep * keep, 0.0);
    std::vector<double> Li(keep * keep), Inv(keep * keep);
    for (int64_t i = 0; i < top.nb; ++i) {
      for (int r = 0; r < keep; ++r)
        for (int c = 0; c < keep; ++c) Li[r * keep + c] = Lh[(size_t)i * Nt * Nt + r * Nt + c];
      // inverse of the lower-triangular Li by forward substitution, column by column
      for (int c = 0; c < keep; ++c)
        for (int r = 0; r < keep; ++r) {
          double s = (r == c) ? 1.0 : 0.0;
          for (int q = 0; q < r; ++q) s -= Li[r * keep + q] * Inv[q * keep + c];
          Inv[r * keep + c] = s / Li[r * keep + r];
        }
      for (int r = 0; r < keep; ++r)
        for (int c = 0; c < keep; ++c) U[(size_t)i * keep * keep + r * keep + c] = Inv[c * keep + r];
    }
  }
  H->levels.emplace_back();
  H->levels[0].Aref = &Ap;
  for (size_t k = 0; k < prol.size(); ++k) {
    const HostBsr& Pb = prol[k];
    const int64_t nbf = A.rows / keep;
    require(Pb.Np == keep, "h-level prolongation block size differs from the coarsest p-level block size");
    require(Pb.nb_rows == nbf, "h-level prolongation rows do not match the level");
    HCsr P;
    P.rows = A.rows;
    P.cols = Pb.nb_cols * keep;
    P.rp.assign(P.rows + 1, 0);
    std::vector<double> blk(keep * keep);
    for (int64_t i = 0; i < nbf; ++i) {
      for (int r = 0; r < keep; ++r) {
        for (int64_t kb = Pb.rp[i]; kb < Pb.rp[i + 1]; ++kb) {
          const double* b = Pb.v.data() + (size_t)kb * keep * keep;
          for (int c = 0; c < keep; ++c) {
            double s;
            if (k == 0 && Ltop) {
              s = 0.0;
              for (int q = 0; q < keep; ++q) s += U[(size_t)i * keep * keep + r * keep + q] * b[q * keep + c];
            } else {
              s = b[r * keep + c];
            }
            if (s != 0.0) {
              P.ci.push_back((int32_t)(Pb.ci[kb] * keep + c));
              P.v.push_back(s);
            }
          }
        }
        P.rp[i * keep + r + 1] = (int64_t)P.ci.size();
      }
    }
    HCsr R = transpose(P);
    HCsr Ac = spgemm(R, spgemm(A, P));
    H->levels.back().P = upload(P);
    H->levels.back().R = upload(R);
    H->levels.emplace_back();
    HmgLevel& L = H->levels.back();
    L.A.reset(csr_to_matrix(Ac, keep));
    L.Aref = L.A.get();
    A = std::move(Ac);
    if (A.rows <= dense_limit) break;
  }
  if (A.rows <= 4096) {
    dense_inverse_csr(A, H->dense_inv);
    H->n_dense = A.rows;
  }
  return H.release();
}

void csr_spmv(const Csr& M, double alpha, const double* x, double beta, double* y, cudaStream_t st) {
  if (!M.rows) return;
  const int64_t threads = M.rows * 8;
  csr_spmv_kernel<double><<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(M.rows, M.rp.p, M.ci.p, M.v64.p, alpha,
                                                                             x, beta, y);
  BSGPU_CHECK_LAUNCH();
}
void csr_spmv(const Csr& M, float alpha, const float* x, float beta, float* y, cudaStream_t st) {
  if (!M.rows) return;
  const int64_t threads = M.rows * 8;
  csr_spmv_kernel<float><<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(M.rows, M.rp.p, M.ci.p, M.v32.p, alpha,
                                                                           x, beta, y);
  BSGPU_CHECK_LAUNCH();
}
void jacobi_update(const double* dinv, double omega, const double* b, const double* Ax, double* x, int64_t n,
                   cudaStream_t st) {
  if (!n) return;
  jacobi_kernel<double><<<grid_for(n), 256, 0, st>>>(dinv, omega, b, Ax, x, n);
  BSGPU_CHECK_LAUNCH();
}
void jacobi_update(const float* dinv, float omega, const float* b, const float* Ax, float* x, int64_t n,
                   cudaStream_t st) {
  if (!n) return;
  jacobi_kernel<float><<<grid_for(n), 256, 0, st>>>(dinv, omega, b, Ax, x, n);
  BSGPU_CHECK_LAUNCH();
}

}  // namespace bsgpu
