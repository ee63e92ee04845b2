// Vector kernels of the solver path (dot products, multi-axpy, scaling, precision conversion).
//
// Dot products are single-launch grid reductions: every CTA writes its partial sums to a scratch array, the last
// CTA to finish (threadfence + atomic ticket) adds the partials in a fixed order and writes the result, so a
// result never depends on CTA scheduling and no second launch or host round trip is needed.  Results stay in
// device memory; later kernels read their coefficients from there.
#pragma once
#include "common.cuh"

namespace bsgpu {

constexpr int kMaxDots = 16;  // dot products per launch

// Scratch of the grid reductions: partial sums [kMaxDots][grid] and a ticket counter (zero between launches).
struct ReduceScratch {
  DBuf<double> partial;
  DBuf<unsigned int> ticket;
  int grid = 0;
  void init();
};

// out[k] = sum_i a[k][i] * b[k][i], k < K (K <= kMaxDots).  `post`: 0 = plain sum, 1 = sqrt(sum).
// `active`: optional device predicate (no-op when *active == 0).
void dots(ReduceScratch& s, int K, const double* const* a, const double* const* b, int64_t n, double* out, int post,
          cudaStream_t st, const int* active = nullptr);
void dots(ReduceScratch& s, int K, const float* const* a, const float* const* b, int64_t n, double* out, int post,
          cudaStream_t st, const int* active = nullptr);

// y[i] += sign * sum_k coef[k] * x[k][i]; coefficients either from device memory (dcoef) or from the host list.
void axpys(int K, const double* dcoef, const double* hcoef, double sign, const double* const* x, double* y, int64_t n,
           cudaStream_t st, const int* active = nullptr);
void axpys(int K, const double* dcoef, const double* hcoef, double sign, const float* const* x, float* y, int64_t n,
           cudaStream_t st, const int* active = nullptr);

// y1 += sign * sum_k dcoef[k] * x1[k][i] and y2 += sign * sum_k dcoef[k] * x2[k][i] in one pass.
void axpys2(int K, const double* dcoef, double sign, const double* const* x1, double* y1, const double* const* x2,
            double* y2, int64_t n, cudaStream_t st);
void axpys2(int K, const double* dcoef, double sign, const float* const* x1, float* y1, const float* const* x2,
            float* y2, int64_t n, cudaStream_t st);

// x *= 1/dscal[0] and (if y) y *= 1/dscal[0]; sets *err = 1 when dscal[0] is 0 or not finite.
void scale_inv2(const double* dscal, double* x, double* y, int64_t n, int* err, cudaStream_t st,
                const int* active = nullptr);
void scale_inv2(const double* dscal, float* x, float* y, int64_t n, int* err, cudaStream_t st,
                const int* active = nullptr);

// y = alpha * x + beta * y  (host scalars)
void axpby(double alpha, const double* x, double beta, double* y, int64_t n, cudaStream_t st);
void axpby(float alpha, const float* x, float beta, float* y, int64_t n, cudaStream_t st);
void fill(double v, double* x, int64_t n, cudaStream_t st);
void fill(float v, float* x, int64_t n, cudaStream_t st);
void convert(const double* x, float* y, int64_t n, cudaStream_t st);
void convert(const float* x, double* y, int64_t n, cudaStream_t st);
// reproducible pseudo-random fill in [-1, 1) (counter-based hash)
void fill_random(double* x, int64_t n, uint64_t seed, cudaStream_t st);
void fill_random(float* x, int64_t n, uint64_t seed, cudaStream_t st);

// sub-vector gather/scatter of p-restriction (BlockMask.GetSubVec / AccSubVec, SubBlockSelectorExt.cs:573-700):
// the sub vector holds, per block, nspc species of `keep` leading modes out of Np.
void restrict_gather(const double* full, double* sub, int64_t nsub, int Np, int keep, const int64_t* map,
                     cudaStream_t st);
void restrict_gather(const float* full, float* sub, int64_t nsub, int Np, int keep, const int64_t* map, cudaStream_t st);
void restrict_scatter_add(const double* sub, double* full, int64_t nsub, int Np, int keep, const int64_t* map,
                          cudaStream_t st);
void restrict_scatter_add(const float* sub, float* full, int64_t nsub, int Np, int keep, const int64_t* map,
                          cudaStream_t st);

// y_b = M_b x_b for per-block dense I x I matrices (row-major), optionally transposed; used by the change of basis.
void block_gemv(const double* M, const int64_t* moff, const int32_t* len, const int64_t* i0, const int32_t* row2blk,
                int uniformNp, bool transpose, const double* x, double* y, int64_t N, cudaStream_t st);

}  // namespace bsgpu
