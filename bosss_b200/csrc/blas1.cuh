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

// SoftPCG's scalar step after r.z and r.r are known (SoftPCG.cs:113-194 with IterativeSolverConfig's termination):
// s[0] = r.z (old), s[2] = r.z (new), s[3] = r.r, s[4] = r0.r0, s[5] = iteration count; writes beta to s[6],
// advances the count and clears *active when the iteration terminates.  Device side, one thread.
__device__ __forceinline__ void pcg_beta_step(double* s, int* active, int mode, double tol, int max_iter,
                                              int min_iter) {
  const double rz_new = s[2], rr = s[3];
  s[6] = rz_new / s[0];
  s[0] = rz_new;
  const double it = s[5] + 1.0;
  s[5] = it;
  const double R = sqrt(rr), R0 = sqrt(s[4]);
  const double eps = 2.2204460492503131e-16 * 1000;
  bool stop = false;
  if (it > min_iter) {
    const bool ok = (mode == 0) ? (R < R0 * tol + tol) : (R < R0 * tol);
    if (ok || it > max_iter || R < eps || R0 < eps) stop = true;
  }
  if (!isfinite(rz_new) || !isfinite(rr)) stop = true;
  if (stop) *active = 0;
}

// One fused PCG update for uniform blocks of NP in {4, 6, 10, 20} with a block-Jacobi preconditioner (Dinv
// column-major per block): alpha = s[0]/s[1]; x += alpha p; r -= alpha q; z = Dinv r; s[2] = r.z, s[3] = r.r;
// then pcg_beta_step.  No-op when *active == 0.  Returns false (nothing launched) for other block sizes.
bool pcg_update(ReduceScratch& red, int NP, double* s, int* active, double* x, const double* p, const double* q,
                double* r, double* z, const double* dinv, int64_t nb, int mode, double tol, int max_iter,
                int min_iter, cudaStream_t st);
bool pcg_update(ReduceScratch& red, int NP, double* s, int* active, float* x, const float* p, const float* q,
                float* r, float* z, const float* dinv, int64_t nb, int mode, double tol, int max_iter, int min_iter,
                cudaStream_t st);

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
