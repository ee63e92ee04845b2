// h-coarsening of the lowest p-level: greedy aggregation of the block graph with piecewise-constant prolongation
// and Galerkin coarse operators, plus the dense direct solve of the last level.
//
// In BoSSS the levels below the p-hierarchy are geometric h-levels on aggregation grids (AggregationGridBasis,
// used by OrthoMGSchwarzConfig.cs:177-860) and the coarsest system goes to a direct solver (DirectSolver.cs:43,
// PmgConfig.cs:167-177).  Here the aggregates are formed from the matrix graph alone (no grid needed): phase 1
// makes an aggregate of every node whose neighbours are all free, phase 2 attaches the remaining nodes to an
// aggregate of a neighbour, phase 3 keeps isolated nodes on their own.  Restriction sums the members of an
// aggregate, prolongation injects the aggregate value; A_c = P^T A P.
#include <algorithm>
#include <cmath>
#include <numeric>

#include "aggregation.cuh"
#include "blas1.cuh"

namespace bsgpu {

namespace {

template <typename T>
__global__ void agg_restrict_kernel(const T* __restrict__ fine, T* __restrict__ coarse, const int32_t* __restrict__ mptr,
                                    const int32_t* __restrict__ mem, int64_t nc) {
  for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < nc; a += (int64_t)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int32_t k = mptr[a]; k < mptr[a + 1]; ++k) s += (double)fine[mem[k]];
    coarse[a] = (T)s;
  }
}

template <typename T>
__global__ void agg_prolong_kernel(const T* __restrict__ coarse, T* __restrict__ fine, const int32_t* __restrict__ agg,
                                   int64_t nf) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nf; i += (int64_t)gridDim.x * blockDim.x)
    fine[i] += coarse[agg[i]];
}

// one warp per row: y = M x for a dense row-major n x n matrix
template <typename T>
__global__ void dense_gemv_kernel(const T* __restrict__ M, const T* __restrict__ x, T* __restrict__ y, int n) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const T* row = M + (int64_t)warp * n;
  double s = 0.0;
  for (int c = lane; c < n; c += 32) s = fma((double)row[c], (double)x[c], s);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if (lane == 0) y[warp] = (T)s;
}

int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 8)); }

}  // namespace

Aggregation* matrix_aggregate(const Matrix& A, cudaStream_t st) {
  require(A.uniform && A.Np == 1 && !A.single, "aggregation needs an FP64 matrix with 1x1 blocks");
  const int64_t n = A.nb;
  std::vector<double> v(A.nnzb);
  if (A.nnzb) matrix_read_values(A, v.data(), false, st);
  std::vector<int32_t> agg(n, -1);
  int32_t nc = 0;
  // phase 1: seeds whose neighbourhood is entirely free
  for (int64_t i = 0; i < n; ++i) {
    if (agg[i] >= 0) continue;
    bool free = true;
    for (int64_t k = A.h_rp[i]; k < A.h_rp[i + 1] && free; ++k)
      if (agg[A.h_ci[k]] >= 0) free = false;
    if (!free) continue;
    bool has_nb = false;
    for (int64_t k = A.h_rp[i]; k < A.h_rp[i + 1]; ++k) {
      agg[A.h_ci[k]] = nc;
      if (A.h_ci[k] != i) has_nb = true;
    }
    agg[i] = nc;
    (void)has_nb;
    ++nc;
  }
  // phase 2: attach leftovers to the neighbouring aggregate with the strongest coupling
  std::vector<int32_t> agg2 = agg;
  for (int64_t i = 0; i < n; ++i) {
    if (agg[i] >= 0) continue;
    double best = -1.0;
    int32_t ba = -1;
    for (int64_t k = A.h_rp[i]; k < A.h_rp[i + 1]; ++k) {
      const int32_t j = A.h_ci[k];
      if (j == i || agg[j] < 0) continue;
      const double w = std::fabs(v[k]);
      if (w > best) { best = w; ba = agg[j]; }
    }
    agg2[i] = ba;
  }
  // phase 3: isolated nodes
  for (int64_t i = 0; i < n; ++i)
    if (agg2[i] < 0) agg2[i] = nc++;
  agg.swap(agg2);
  // members CSR
  std::vector<int32_t> mptr(nc + 1, 0), mem(n);
  for (int64_t i = 0; i < n; ++i) mptr[agg[i] + 1]++;
  for (int32_t a = 0; a < nc; ++a) mptr[a + 1] += mptr[a];
  {
    std::vector<int32_t> fillp(mptr.begin(), mptr.end() - 1);
    for (int64_t i = 0; i < n; ++i) mem[fillp[agg[i]]++] = (int32_t)i;
  }
  // Galerkin product P^T A P, row by row with a dense marker
  std::vector<int64_t> crp(nc + 1, 0);
  std::vector<int32_t> cci;
  std::vector<double> cv;
  cci.reserve(A.nnzb / 2);
  cv.reserve(A.nnzb / 2);
  std::vector<int64_t> pos(nc, -1);
  for (int32_t a = 0; a < nc; ++a) {
    const int64_t start = (int64_t)cci.size();
    for (int32_t m = mptr[a]; m < mptr[a + 1]; ++m) {
      const int32_t i = mem[m];
      for (int64_t k = A.h_rp[i]; k < A.h_rp[i + 1]; ++k) {
        const int32_t b = agg[A.h_ci[k]];
        if (pos[b] < start) {
          pos[b] = (int64_t)cci.size();
          cci.push_back(b);
          cv.push_back(v[k]);
        } else {
          cv[pos[b]] += v[k];
        }
      }
    }
    // sort the row's columns ascending (BlockMsrMatrix order)
    std::vector<std::pair<int32_t, double>> row;
    for (int64_t q = start; q < (int64_t)cci.size(); ++q) row.emplace_back(cci[q], cv[q]);
    std::sort(row.begin(), row.end());
    for (size_t q = 0; q < row.size(); ++q) {
      cci[start + q] = row[q].first;
      cv[start + q] = row[q].second;
    }
    crp[a + 1] = (int64_t)cci.size();
  }
  auto out = std::make_unique<Aggregation>();
  out->nf = n;
  out->nc = nc;
  out->coarse.reset(matrix_create(nc, 1, nullptr, crp.data(), cci.data(), cv.data(), BSGPU_HOST_POINTERS));
  out->agg.alloc(std::max<int64_t>(n, 1));
  out->mptr.alloc(nc + 1);
  out->mem.alloc(std::max<int64_t>(n, 1));
  if (n) BSGPU_CUDA(cudaMemcpy(out->agg.p, agg.data(), n * 4, cudaMemcpyHostToDevice));
  BSGPU_CUDA(cudaMemcpy(out->mptr.p, mptr.data(), (nc + 1) * 4, cudaMemcpyHostToDevice));
  if (n) BSGPU_CUDA(cudaMemcpy(out->mem.p, mem.data(), n * 4, cudaMemcpyHostToDevice));
  return out.release();
}

void dense_inverse(const Matrix& A, std::vector<double>& inv, cudaStream_t st) {
  require(A.uniform && A.Np == 1 && !A.single, "dense inverse needs an FP64 matrix with 1x1 blocks");
  const int64_t n = A.nb;
  require(n <= 4096, "dense direct solve limited to 4096 unknowns", BSGPU_ERR_UNSUPPORTED);
  std::vector<double> v(A.nnzb);
  if (A.nnzb) matrix_read_values(A, v.data(), false, st);
  std::vector<double> M((size_t)n * n, 0.0);
  for (int64_t i = 0; i < n; ++i)
    for (int64_t k = A.h_rp[i]; k < A.h_rp[i + 1]; ++k) M[i * n + A.h_ci[k]] = v[k];
  inv.assign((size_t)n * n, 0.0);
  for (int64_t i = 0; i < n; ++i) inv[i * n + i] = 1.0;
  // Gauss-Jordan with partial pivoting
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

void agg_restrict(const Aggregation& g, const double* fine, double* coarse, cudaStream_t st) {
  if (!g.nc) return;
  agg_restrict_kernel<double><<<grid_for(g.nc), 256, 0, st>>>(fine, coarse, g.mptr.p, g.mem.p, g.nc);
  BSGPU_CHECK_LAUNCH();
}
void agg_restrict(const Aggregation& g, const float* fine, float* coarse, cudaStream_t st) {
  if (!g.nc) return;
  agg_restrict_kernel<float><<<grid_for(g.nc), 256, 0, st>>>(fine, coarse, g.mptr.p, g.mem.p, g.nc);
  BSGPU_CHECK_LAUNCH();
}
void agg_prolong_add(const Aggregation& g, const double* coarse, double* fine, cudaStream_t st) {
  if (!g.nf) return;
  agg_prolong_kernel<double><<<grid_for(g.nf), 256, 0, st>>>(coarse, fine, g.agg.p, g.nf);
  BSGPU_CHECK_LAUNCH();
}
void agg_prolong_add(const Aggregation& g, const float* coarse, float* fine, cudaStream_t st) {
  if (!g.nf) return;
  agg_prolong_kernel<float><<<grid_for(g.nf), 256, 0, st>>>(coarse, fine, g.agg.p, g.nf);
  BSGPU_CHECK_LAUNCH();
}
void dense_gemv(const double* M, const double* x, double* y, int n, cudaStream_t st) {
  if (!n) return;
  dense_gemv_kernel<double><<<(n * 32 + 255) / 256, 256, 0, st>>>(M, x, y, n);
  BSGPU_CHECK_LAUNCH();
}
void dense_gemv(const float* M, const float* x, float* y, int n, cudaStream_t st) {
  if (!n) return;
  dense_gemv_kernel<float><<<(n * 32 + 255) / 256, 256, 0, st>>>(M, x, y, n);
  BSGPU_CHECK_LAUNCH();
}

}  // namespace bsgpu
