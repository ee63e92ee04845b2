// Smoothed-aggregation algebraic multigrid for the coarsest p-level (see amg.cu).
#pragma once
#include "matrix.cuh"

namespace bsgpu {

// Rectangular CSR matrix on the device (prolongation P and its transpose).
struct Csr {
  int64_t rows = 0, cols = 0, nnz = 0;
  DBuf<int32_t> rp, ci;
  DBuf<double> v64;
  DBuf<float> v32;
};

struct AmgLevel {
  std::unique_ptr<Matrix> A;   // level operator (FP64); level 0 borrows the p-level matrix instead
  const Matrix* Aref = nullptr;
  std::unique_ptr<Csr> P, R;   // prolongation (rows = this level, cols = next) and restriction R = P^T
  double omega = 0.0;          // damping of the point-Jacobi smoother, 4 / (3 rho(D^-1 A))
  DBuf<double> dinv64;         // point-diagonal inverse
  DBuf<float> dinv32;
  int64_t n = 0;
};

struct AmgHierarchy {
  std::vector<AmgLevel> levels;      // levels[0] is the p-level operator
  std::vector<double> dense_inv;     // inverse of the last level (row-major)
  int64_t n_dense = 0;
};

// Builds the hierarchy below the block matrix A0 (its DOF 0 of every block carries the near-null space, the
// constant function), with at most max_levels coarse levels, stopping at dense_limit unknowns.
AmgHierarchy* amg_setup(const Matrix& A0, int max_levels, int dense_limit, cudaStream_t st);

// Block-sparse prolongation supplied by the caller (host copy): row block = fine cell, column block = coarse
// cell, blocks Np x Np row-major, in the untransformed orthonormal DG basis.
struct HostBsr {
  int Np = 0;
  int64_t nb_rows = 0, nb_cols = 0;
  std::vector<int64_t> rp;
  std::vector<int32_t> ci;
  std::vector<double> v;
};

// Geometric h-levels below the coarsest p-level (agglomerated cells, caller-supplied prolongations).
struct HmgLevel {
  std::unique_ptr<Matrix> A;  // Galerkin operator of this level (levels >= 1)
  const Matrix* Aref = nullptr;
  std::unique_ptr<Csr> P, R;  // to the next coarser level
};
struct HmgHierarchy {
  std::vector<HmgLevel> levels;
  std::vector<double> dense_inv;
  int64_t n_dense = 0;
};

// Ap: coarsest p-level operator (transformed basis, FP64, uniform blocks of `keep` modes); top / Ltop: the
// finest level's matrix and its left change of basis (device, per block row I x I row-major; nullptr = Eye).
// The first prolongation is mapped into the transformed basis with L_p^{-T} (L_p = leading keep x keep block of
// L, lower triangular); coarse operators are P^T A P.  The last level is inverted densely.
HmgHierarchy* hmg_setup(const Matrix& Ap, const Matrix& top, const double* Ltop, int keep,
                        const std::vector<HostBsr>& prol, int dense_limit, cudaStream_t st);

// y = alpha * M x + beta * y
void csr_spmv(const Csr& M, double alpha, const double* x, double beta, double* y, cudaStream_t st);
void csr_spmv(const Csr& M, float alpha, const float* x, float beta, float* y, cudaStream_t st);
// x += omega * Dinv .* (b - r) where r = A x was computed before (point Jacobi update), element-wise
void jacobi_update(const double* dinv, double omega, const double* b, const double* Ax, double* x, int64_t n,
                   cudaStream_t st);
void jacobi_update(const float* dinv, float omega, const float* b, const float* Ax, float* x, int64_t n,
                   cudaStream_t st);

}  // namespace bsgpu
