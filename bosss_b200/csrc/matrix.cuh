// Device-resident block-sparse matrix (the BlockMsrMatrix of the solver path) and its kernels' launchers.
//
// Device layout ("row-interleaved slab").  Block row i, with block length I and occupied blocks k = rp[i] ..
// rp[i+1]-1 of widths J_k, is one slab of I rows and sum_k J_k columns.  The slab is cut into column chunks of
// V consecutive entries (V = 2 for FP64 and V = 4 for FP32 when the block widths allow it, else smaller); the
// chunks are stored chunk-major, row-minor:   value(k, r, c) = boff[k] + (c / V) * I * V + r * V + c % V.
// A thread that owns DOF row r of block row i therefore streams its row with V-wide vector loads while the
// I threads of the block row read one contiguous run of I*V values per step: every HBM sector that is fetched
// is fully used and no shuffle or shared-memory reduction is needed.  Blocks never straddle a chunk because V
// divides every block width.
#pragma once
#include <cuda_fp16.h>

#include "common.cuh"

namespace bsgpu {

struct Matrix {
  int64_t nb = 0, N = 0, nnzb = 0;
  int Np = 0;            // modes per species
  bool uniform = true;   // every block has Np rows (one species)
  bool single = false;   // values stored as float (FP32 arithmetic)
  bool half = false;     // with single: values stored as FP16 (v16), FP32 arithmetic
  int V = 1;             // chunk width (elements)
  // host copies of the structure
  std::vector<int64_t> h_rp, h_i0;
  std::vector<int32_t> h_ci, h_len, h_nspc;
  // device structure
  DBuf<int64_t> rp, i0, boff;
  DBuf<int32_t> ci, len, row2blk;
  DBuf<int64_t> doff;      // offsets of the per-block-row diagonal factors (I*I each)
  DBuf<int64_t> cta_row0;  // CTA packing for the variable-size kernels (whole block rows per CTA)
  int64_t ncta = 0;
  // Blocks of one or two species (XDG): the block rows with one species, then those with two, each list in
  // ascending order; the typed kernels specialise on the species count of the row (typed == false: the general
  // kernel with per-row lookups serves the matrix).
  bool typed = false;
  DBuf<int32_t> grp_rows;
  int64_t grp_n1 = 0, grp_n2 = 0;
  // Launch shape of the uniform and species-count kernels: threads per CTA (whole block rows each) for the plain
  // product (cta[0]) and the fused block-Jacobi update (cta[1]); 256 unless the autotuner picked otherwise.
  mutable int cta[2] = {256, 256};
  mutable bool tuned[2] = {false, false};
  int cta_threads = 256;
  DBuf<double> v64;
  DBuf<float> v32;
  DBuf<__half> v16;
  int64_t nvals = 0;

  size_t value_bytes() const { return (size_t)nvals * (half ? 2 : single ? 4 : 8); }
  int64_t max_len() const;
};

// Creation from block-CSR arrays with row-major blocks (host or device pointers).
Matrix* matrix_create(int64_t nb, int32_t Np, const int32_t* nspc, const int64_t* row_ptr, const int32_t* col_idx,
                      const double* values, int32_t flags);
// A matrix with the same structure as `A` and values given in the device layout of `A` (used for transforms).
Matrix* matrix_like(const Matrix& A, bool single);
void matrix_read_values(const Matrix& A, double* dst, bool dst_device, cudaStream_t st);
Matrix* matrix_to_single(const Matrix& A, cudaStream_t st);
// FP16 copy of an FP64 matrix (uniform blocks of 4, 10 or 20) for the preconditioner: products in FP32 arithmetic on
// half the value traffic.  Marked single (it serves the FP32 kernels' entry points).
Matrix* matrix_to_half(const Matrix& A, cudaStream_t st);
Matrix* matrix_restrict(const Matrix& A, int keep, cudaStream_t st);
// SIP operator of -div(nu grad u) on a uniform Cartesian grid of shape[0..D) cells over [lo, hi]^D, degree p,
// homogeneous Dirichlet boundaries, assembled on the GPU (assembly.cu).  nu: per-cell diffusivity or null (1).
Matrix* assemble_sip_cartesian(int D, const int32_t* shape, double lo, double hi, int p, double penalty,
                               const double* nu, bool nu_device);
// the assembly's block templates for cell sizes h[0..D) (host computation, no device work): sip_template_count()
// matrices of Np x Np, row-major (0 volume; 1 + 4d .. 4 + 4d the face terms of direction d on the +d and -d sides;
// 13 + 6d .. 15 + 6d the off-diagonal terms of direction d)
std::vector<double> sip_templates(int D, int p, const double* h);
int sip_template_count();
int modes_count(int D, int p);  // modes of total degree <= p in D dimensions
// load vector of a separable right-hand side sum_m coef[m] prod_d f_{m,d}(x_d) on a Cartesian grid: tables holds the
// 1-D projections [M][D][shape[d]][p + 1] (integral of f_{m,d} times the 1-D basis over each cell interval, with
// the 1-D scaling); out_device[c * Np + a] = sum_m coef[m] prod_d tables[m][d][i_d(c)][mode_a[d]]
void project_separable(int D, const int32_t* shape, int p, int M, const double* coef, const double* tables,
                       double* out_device, cudaStream_t st);

// y = alpha*A*x + beta*z (z may be y; z == nullptr: beta ignored).  `active`: optional device flag, the launch
// is a no-op when *active == 0.
void spmv(const Matrix& A, double alpha, const double* x, double beta, const double* z, double* y, cudaStream_t st,
          const int* active = nullptr);
void spmv(const Matrix& A, float alpha, const float* x, float beta, const float* z, float* y, cudaStream_t st,
          const int* active = nullptr);
// Block-Jacobi update fused into the SpMV: xo = x + omega * Dinv * (b - A*x).  Dinv: per block row, column-major.
void bj_update(const Matrix& A, const double* dinv, double omega, const double* x, const double* b, double* xo,
               cudaStream_t st, const int* active = nullptr);
void bj_update(const Matrix& A, const float* dinv, float omega, const float* x, const float* b, float* xo,
               cudaStream_t st, const int* active = nullptr);
// In-place block Gauss-Seidel half-sweep over one colour: x_i += omega * Dinv_i * (b - A*x)_i for the listed
// block rows (no two of which are neighbours).  Uniform blocks of 4, 6, 10 or 20 only.
void gs_update_rows(const Matrix& A, const double* dinv, double omega, const int32_t* rows, int64_t nrows,
                    const double* b, double* x, cudaStream_t st);
void gs_update_rows(const Matrix& A, const float* dinv, float omega, const int32_t* rows, int64_t nrows,
                    const float* b, float* x, cudaStream_t st);
// In-place unit-diagonal update over listed block rows: x_i += (b - A*x)_i (no two listed rows neighbours).  With
// x zero on the rows not yet visited this is the forward substitution of a unit lower factor stored in A.
void unit_update_rows(const Matrix& A, const int32_t* rows, int64_t nrows, const double* b, double* x,
                      cudaStream_t st);
void unit_update_rows(const Matrix& A, const int32_t* rows, int64_t nrows, const float* b, float* x, cudaStream_t st);
// Greedy colouring of the block graph (lists of block rows per colour).
std::vector<std::vector<int32_t>> greedy_colouring(const Matrix& A);
// y = omega * Dinv * b (first block-Jacobi sweep from a zero guess).
void blockdiag_apply(const Matrix& A, const double* dinv, double omega, const double* b, double* y, cudaStream_t st,
                     const int* active = nullptr);
void blockdiag_apply(const Matrix& A, const float* dinv, float omega, const float* b, float* y, cudaStream_t st,
                     const int* active = nullptr);

// Offsets of the per-block-row dense diagonal factors (column-major I x I each) and their total size.
std::vector<int64_t> diag_offsets(const Matrix& A);

// Autotuner of the launch shape (threads per CTA: 256, 128 or 64, whole block rows per CTA) of the product
// (mode 0) or of the fused block-Jacobi update (mode 1, with the factors dinv of the matrix's precision) on the
// matrix itself: every candidate is timed with CUDA events and the fastest is kept in A.cta.  Results are cached
// per device and matrix shape and recorded for autotune_report.  Not during a graph capture.
void autotune(const Matrix& A, int mode, const void* dinv, cudaStream_t st);
std::string autotune_report();

}  // namespace bsgpu
