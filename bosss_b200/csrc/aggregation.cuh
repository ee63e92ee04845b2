// h-coarsening by aggregation and the dense coarsest-level solve (see aggregation.cu).
#pragma once
#include "matrix.cuh"

namespace bsgpu {

struct Aggregation {
  std::unique_ptr<Matrix> coarse;  // P^T A P (FP64, 1x1 blocks)
  DBuf<int32_t> agg;               // fine node -> aggregate
  DBuf<int32_t> mptr, mem;         // aggregate -> members (CSR)
  int64_t nf = 0, nc = 0;
};

Aggregation* matrix_aggregate(const Matrix& A, cudaStream_t st);
// inverse of a small matrix with 1x1 blocks, row-major, computed on the host in FP64 at set-up
void dense_inverse(const Matrix& A, std::vector<double>& inv, cudaStream_t st);

void agg_restrict(const Aggregation& g, const double* fine, double* coarse, cudaStream_t st);
void agg_restrict(const Aggregation& g, const float* fine, float* coarse, cudaStream_t st);
void agg_prolong_add(const Aggregation& g, const double* coarse, double* fine, cudaStream_t st);
void agg_prolong_add(const Aggregation& g, const float* coarse, float* fine, cudaStream_t st);
void dense_gemv(const double* M, const double* x, double* y, int n, cudaStream_t st);
void dense_gemv(const float* M, const float* x, float* y, int n, cudaStream_t st);

}  // namespace bsgpu
