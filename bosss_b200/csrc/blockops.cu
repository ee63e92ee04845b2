// Batched dense block operations on the diagonal / all blocks of a block-sparse matrix.
#include <algorithm>

#include "blockops.cuh"

namespace bsgpu {

namespace {

__device__ __forceinline__ int64_t diag_block(const int64_t* rp, const int32_t* ci, int64_t i) {
  for (int64_t k = rp[i]; k < rp[i + 1]; ++k)
    if (ci[k] == i) return k;
  return -1;
}

__device__ __forceinline__ double packed_at(const double* v, int64_t boff, int I, int V, int r, int c) {
  return v[boff + (int64_t)(c / V) * I * V + r * V + (c % V)];
}

// One CTA per block row: symmetric elimination of the diagonal block in shared memory.
// Row/column scalings and additions are those of SymmInv; the additions of one elimination step are applied
// together as M <- E M E^T, L <- E L with E = I + sum_k a_k e_k e_i^T (the elementary operations of one step
// commute, so this equals the reference's sequential order up to rounding).
__global__ void symminv_kernel(const int64_t* __restrict__ rp, const int32_t* __restrict__ ci,
                               const int32_t* __restrict__ len, const int64_t* __restrict__ boff,
                               const double* __restrict__ vals, int V, const int64_t* __restrict__ doff,
                               double* __restrict__ Lout, int* __restrict__ err, int64_t nb) {
  extern __shared__ double sm[];
  for (int64_t i = blockIdx.x; i < nb; i += gridDim.x) {
    const int n = len[i];
    double* M = sm;
    double* L = sm + n * n;
    double* rowi = L + n * n;
    double* coli = rowi + n;
    double* a = coli + n;
    __shared__ int bad;
    const int64_t kd = diag_block(rp, ci, i);
    if (threadIdx.x == 0) bad = (kd < 0);
    __syncthreads();
    if (bad) {
      if (threadIdx.x == 0) atomicCAS(err, 0, (int)(i + 1 < 0x7fffffff ? i + 1 : 0x7fffffff));
      __syncthreads();
      continue;
    }
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int r = e / n, c = e - r * n;
      M[e] = packed_at(vals, boff[kd], n, V, r, c);
      L[e] = (r == c) ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int p = 0; p < n; ++p) {
      const double Mpp = M[p * n + p];
      if (Mpp == 0.0 || !isfinite(Mpp)) {
        if (threadIdx.x == 0) { bad = 1; atomicCAS(err, 0, (int)(i + 1 < 0x7fffffff ? i + 1 : 0x7fffffff)); }
        __syncthreads();
        break;
      }
      const double scl = 1.0 / sqrt(fabs(Mpp));
      for (int c = threadIdx.x; c < n; c += blockDim.x) {
        M[p * n + c] *= scl;
        L[p * n + c] *= scl;
      }
      __syncthreads();
      for (int r = threadIdx.x; r < n; r += blockDim.x) M[r * n + p] *= scl;
      __syncthreads();
      const double d = M[p * n + p];
      const double sgn = d > 0 ? 1.0 : -1.0;
      if (fabs(fabs(d) - 1.0) > 1.0e-8) {
        if (threadIdx.x == 0) { bad = 1; atomicCAS(err, 0, (int)(i + 1 < 0x7fffffff ? i + 1 : 0x7fffffff)); }
        __syncthreads();
        break;
      }
      for (int q = threadIdx.x; q < n; q += blockDim.x) {
        rowi[q] = M[p * n + q];
        coli[q] = M[q * n + p];
        a[q] = (q > p) ? -M[q * n + p] * sgn : 0.0;
      }
      __syncthreads();
      const double mpp = M[p * n + p];
      for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - r * n;
        M[e] += a[r] * rowi[c] + a[c] * coli[r] + a[r] * a[c] * mpp;
        if (r > p) L[e] += a[r] * L[p * n + c];
      }
      __syncthreads();
    }
    double* out = Lout + doff[i];
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) out[e] = L[e];
    __syncthreads();
  }
}

// Aout(k) = L_i A(k) L_j^T, one CTA per block, L lower triangular.
__global__ void cob_kernel(const int64_t* __restrict__ rp, const int32_t* __restrict__ ci,
                           const int32_t* __restrict__ len, const int32_t* __restrict__ blk_row,
                           const int64_t* __restrict__ boff_in, int Vin, const double* __restrict__ vin,
                           const int64_t* __restrict__ boff_out, int Vout, double* __restrict__ vout,
                           const double* __restrict__ L, const int64_t* __restrict__ doff, int64_t nnzb) {
  extern __shared__ double sm[];
  for (int64_t k = blockIdx.x; k < nnzb; k += gridDim.x) {
    const int i = blk_row[k], j = ci[k];
    const int I = len[i], J = len[j];
    double* A = sm;
    double* T = A + I * J;
    double* Li = T + I * J;
    double* Lj = Li + I * I;
    for (int e = threadIdx.x; e < I * J; e += blockDim.x) {
      const int r = e / J, c = e - r * J;
      A[e] = packed_at(vin, boff_in[k], I, Vin, r, c);
    }
    for (int e = threadIdx.x; e < I * I; e += blockDim.x) Li[e] = L[doff[i] + e];
    for (int e = threadIdx.x; e < J * J; e += blockDim.x) Lj[e] = L[doff[j] + e];
    __syncthreads();
    for (int e = threadIdx.x; e < I * J; e += blockDim.x) {
      const int r = e / J, c = e - r * J;
      double s = 0.0;
      for (int q = 0; q <= r; ++q) s = fma(Li[r * I + q], A[q * J + c], s);
      T[e] = s;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < I * J; e += blockDim.x) {
      const int r = e / J, c = e - r * J;
      double s = 0.0;
      for (int q = 0; q <= c; ++q) s = fma(T[r * J + q], Lj[c * J + q], s);
      vout[boff_out[k] + (int64_t)(c / Vout) * I * Vout + r * Vout + (c % Vout)] = s;
    }
    __syncthreads();
  }
}

// Gauss-Jordan inversion with partial pivoting of the diagonal block, one CTA per block row.
__global__ void invert_kernel(const int64_t* __restrict__ rp, const int32_t* __restrict__ ci,
                              const int32_t* __restrict__ len, const int64_t* __restrict__ boff,
                              const double* __restrict__ vals, int V, const int64_t* __restrict__ doff,
                              double* __restrict__ D64, float* __restrict__ D32, int* __restrict__ err, int64_t nb) {
  extern __shared__ double sm[];
  for (int64_t i = blockIdx.x; i < nb; i += gridDim.x) {
    const int n = len[i];
    double* M = sm;
    double* prow = sm + n * n;
    double* pcol = prow + n;
    int* perm = reinterpret_cast<int*>(pcol + n);
    __shared__ int piv;
    __shared__ int bad;
    const int64_t kd = diag_block(rp, ci, i);
    if (threadIdx.x == 0) bad = (kd < 0);
    __syncthreads();
    if (bad) {
      if (threadIdx.x == 0) atomicCAS(err, 0, (int)(i + 1 < 0x7fffffff ? i + 1 : 0x7fffffff));
      __syncthreads();
      continue;
    }
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
      const int r = e / n, c = e - r * n;
      M[e] = packed_at(vals, boff[kd], n, V, r, c);
    }
    __syncthreads();
    for (int p = 0; p < n; ++p) {
      if (threadIdx.x == 0) {
        int best = p;
        double mx = fabs(M[p * n + p]);
        for (int r = p + 1; r < n; ++r)
          if (fabs(M[r * n + p]) > mx) { mx = fabs(M[r * n + p]); best = r; }
        piv = best;
        perm[p] = best;
        if (!(mx > 0.0) || !isfinite(mx)) { bad = 1; atomicCAS(err, 0, (int)(i + 1 < 0x7fffffff ? i + 1 : 0x7fffffff)); }
      }
      __syncthreads();
      if (bad) break;
      if (piv != p)
        for (int c = threadIdx.x; c < n; c += blockDim.x) {
          const double t = M[p * n + c];
          M[p * n + c] = M[piv * n + c];
          M[piv * n + c] = t;
        }
      __syncthreads();
      const double inv = 1.0 / M[p * n + p];
      for (int q = threadIdx.x; q < n; q += blockDim.x) {
        prow[q] = (q == p) ? inv : M[p * n + q] * inv;
        pcol[q] = M[q * n + p];
      }
      __syncthreads();
      for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - r * n;
        if (r == p)
          M[e] = prow[c];
        else if (c == p)
          M[e] = -pcol[r] * prow[p];
        else
          M[e] -= pcol[r] * prow[c];
      }
      __syncthreads();
    }
    if (!bad) {
      // undo the row interchanges as column interchanges, in reverse order
      for (int p = n - 1; p >= 0; --p) {
        const int q = perm[p];
        if (q != p)
          for (int r = threadIdx.x; r < n; r += blockDim.x) {
            const double t = M[r * n + p];
            M[r * n + p] = M[r * n + q];
            M[r * n + q] = t;
          }
        __syncthreads();
      }
      for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - r * n;
        const double v = M[r * n + c];
        if (D64) D64[doff[i] + (int64_t)c * n + r] = v;
        if (D32) D32[doff[i] + (int64_t)c * n + r] = (float)v;
      }
    }
    __syncthreads();
  }
}

// y_i = L_i^{-T} x_i, one thread per block row (back substitution with the upper-triangular L^T)
__global__ void trsv_lt_kernel(const int32_t* __restrict__ len, const int64_t* __restrict__ i0,
                               const int64_t* __restrict__ doff, const double* __restrict__ L,
                               const double* __restrict__ x, double* __restrict__ y, int64_t nb) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += (int64_t)gridDim.x * blockDim.x) {
    const int n = len[i];
    const double* Li = L + doff[i];
    const int64_t s0 = i0[i];
    for (int r = n - 1; r >= 0; --r) {
      double s = x[s0 + r];
      for (int c = r + 1; c < n; ++c) s -= Li[c * n + r] * y[s0 + c];
      y[s0 + r] = s / Li[r * n + r];
    }
  }
}

// Restricted additive Schwarz factors with one block per cell: the block of cell K is K plus the cells its block
// row couples to (face neighbours, i.e. overlap 1).  The dense block matrix is assembled in shared memory,
// inverted by Gauss-Jordan with partial pivoting in FP64, and the rows of cell K are written into M, which has
// A's block structure: M_{K,L} = [P_K^-1]_{K,L}.  One CTA per cell; block sizes may differ between cells.
template <typename TO>
__global__ void schwarz_factor_kernel(const int64_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                      const int32_t* __restrict__ len, const int64_t* __restrict__ boff,
                                      const double* __restrict__ vals, int V, const int64_t* __restrict__ boffM,
                                      int VM, TO* __restrict__ M, int maxp, int* __restrict__ err, int64_t nb) {
  extern __shared__ double sm[];
  __shared__ int offs[33];
  __shared__ int piv;
  __shared__ int bad;
  for (int64_t K = blockIdx.x; K < nb; K += gridDim.x) {
    const int64_t k0 = rp[K], k1 = rp[K + 1];
    const int nc = (int)(k1 - k0);
    if (threadIdx.x == 0) {
      bad = nc > 32;
      int o = 0;
      for (int a = 0; a < nc && a < 32; ++a) {
        offs[a] = o;
        o += len[ci[k0 + a]];
      }
      offs[nc < 32 ? nc : 32] = o;
      if (o > maxp) bad = 1;
    }
    __syncthreads();
    if (bad) {
      if (threadIdx.x == 0) atomicCAS(err, 0, (int)(K + 1 < 0x7fffffff ? K + 1 : 0x7fffffff));
      __syncthreads();
      continue;
    }
    const int n = offs[nc];
    double* P = sm;                 // n x n
    double* prow = sm + n * n;
    double* pcol = prow + n;
    int* perm = reinterpret_cast<int*>(pcol + n);
    for (int e = threadIdx.x; e < n * n; e += blockDim.x) P[e] = 0.0;
    __syncthreads();
    // assemble: for every patch cell a, the blocks of its row whose column is a patch cell
    for (int a = 0; a < nc; ++a) {
      const int32_t ca = ci[k0 + a];
      const int I = len[ca];
      for (int64_t q = rp[ca]; q < rp[ca + 1]; ++q) {
        const int32_t cb = ci[q];
        int b = -1;
        for (int t = 0; t < nc; ++t)
          if (ci[k0 + t] == cb) b = t;
        if (b < 0) continue;
        const int J = len[cb];
        for (int e = threadIdx.x; e < I * J; e += blockDim.x) {
          const int r = e / J, c = e - r * J;
          P[(offs[a] + r) * n + offs[b] + c] = vals[boff[q] + (int64_t)(c / V) * I * V + r * V + (c % V)];
        }
      }
    }
    __syncthreads();
    // Gauss-Jordan inversion with partial pivoting
    for (int p = 0; p < n; ++p) {
      if (threadIdx.x == 0) {
        int best = p;
        double mx = fabs(P[p * n + p]);
        for (int r = p + 1; r < n; ++r)
          if (fabs(P[r * n + p]) > mx) { mx = fabs(P[r * n + p]); best = r; }
        piv = best;
        perm[p] = best;
        if (!(mx > 0.0) || !isfinite(mx)) { bad = 1; atomicCAS(err, 0, (int)(K + 1 < 0x7fffffff ? K + 1 : 0x7fffffff)); }
      }
      __syncthreads();
      if (bad) break;
      if (piv != p)
        for (int c = threadIdx.x; c < n; c += blockDim.x) {
          const double t = P[p * n + c];
          P[p * n + c] = P[piv * n + c];
          P[piv * n + c] = t;
        }
      __syncthreads();
      const double inv = 1.0 / P[p * n + p];
      for (int q = threadIdx.x; q < n; q += blockDim.x) {
        prow[q] = (q == p) ? inv : P[p * n + q] * inv;
        pcol[q] = P[q * n + p];
      }
      __syncthreads();
      for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
        const int r = e / n, c = e - r * n;
        if (r == p)
          P[e] = prow[c];
        else if (c == p)
          P[e] = -pcol[r] * prow[p];
        else
          P[e] -= pcol[r] * prow[c];
      }
      __syncthreads();
    }
    if (!bad) {
      for (int p = n - 1; p >= 0; --p) {
        const int q = perm[p];
        if (q != p)
          for (int r = threadIdx.x; r < n; r += blockDim.x) {
            const double t = P[r * n + p];
            P[r * n + p] = P[r * n + q];
            P[r * n + q] = t;
          }
        __syncthreads();
      }
      // rows of the centre cell K -> block row K of M
      int aK = 0;
      for (int t = 0; t < nc; ++t)
        if (ci[k0 + t] == K) aK = t;
      const int I = len[K];
      for (int b = 0; b < nc; ++b) {
        const int J = len[ci[k0 + b]];
        for (int e = threadIdx.x; e < I * J; e += blockDim.x) {
          const int r = e / J, c = e - r * J;
          M[boffM[k0 + b] + (int64_t)(c / VM) * I * VM + r * VM + (c % VM)] =
              (TO)P[(offs[aK] + r) * n + offs[b] + c];
        }
      }
    }
    __syncthreads();
  }
}

// Block ILU(0) of a two-colour block graph with the rows ordered colour 0 first (CellILU.ComputeILU,
// CellILU.cs:1229-1330, applied to the reordered matrix).  Colour-0 rows have no lower neighbours, so their
// factors are A's blocks (copied beforehand); every colour-1 row b only has colour-0 neighbours r, hence
//   L_br = A_br A_rr^{-1},   U_bb = A_bb - sum_r L_br A_rb,
// and no other block of the pattern changes.  One CTA per colour-1 row; dinv: A_rr^{-1}, column-major per block
// row at doff.  M (FP64, A's structure and layout) receives L_br and U_bb.
__global__ void ilu0_two_colour_kernel(const int64_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                       const int32_t* __restrict__ len, const int64_t* __restrict__ boff,
                                       const double* __restrict__ vals, int V, const int64_t* __restrict__ doff,
                                       const double* __restrict__ dinv, const int32_t* __restrict__ rows,
                                       int64_t nrows, double* __restrict__ M, int* __restrict__ err) {
  extern __shared__ double sm[];
  for (int64_t q = blockIdx.x; q < nrows; q += gridDim.x) {
    const int64_t b = rows[q];
    const int I = len[b];
    double* U = sm;            // I x I row-major
    double* L = sm + I * I;    // I x J row-major (J <= max block length)
    int64_t kd = -1;
    for (int64_t k = rp[b]; k < rp[b + 1]; ++k)
      if (ci[k] == b) kd = k;
    if (kd < 0) {
      if (threadIdx.x == 0) atomicCAS(err, 0, (int)(b + 1 < 0x7fffffff ? b + 1 : 0x7fffffff));
      continue;
    }
    for (int e = threadIdx.x; e < I * I; e += blockDim.x) {
      const int r = e / I, c = e - r * I;
      U[e] = vals[boff[kd] + (int64_t)(c / V) * I * V + r * V + (c % V)];
    }
    __syncthreads();
    for (int64_t k = rp[b]; k < rp[b + 1]; ++k) {
      const int64_t r = ci[k];
      if (r == b) continue;
      const int J = len[r];
      // block (r, b) in row r (structurally symmetric pattern)
      int64_t krb = -1;
      for (int64_t t = rp[r]; t < rp[r + 1]; ++t)
        if (ci[t] == b) krb = t;
      if (krb < 0) {
        if (threadIdx.x == 0) atomicCAS(err, 0, (int)(b + 1 < 0x7fffffff ? b + 1 : 0x7fffffff));
        break;
      }
      const double* D = dinv + doff[r];
      for (int e = threadIdx.x; e < I * J; e += blockDim.x) {
        const int i = e / J, c = e - i * J;
        double acc = 0.0;
        for (int p = 0; p < J; ++p)
          acc = fma(vals[boff[k] + (int64_t)(p / V) * I * V + i * V + (p % V)], D[c * J + p], acc);
        L[e] = acc;
        M[boff[k] + (int64_t)(c / V) * I * V + i * V + (c % V)] = acc;
      }
      __syncthreads();
      for (int e = threadIdx.x; e < I * I; e += blockDim.x) {
        const int i = e / I, c = e - i * I;
        double acc = 0.0;
        for (int p = 0; p < J; ++p)
          acc = fma(L[i * J + p], vals[boff[krb] + (int64_t)(c / V) * J * V + p * V + (c % V)], acc);
        U[e] -= acc;
      }
      __syncthreads();
    }
    for (int e = threadIdx.x; e < I * I; e += blockDim.x) {
      const int r = e / I, c = e - r * I;
      M[boff[kd] + (int64_t)(c / V) * I * V + r * V + (c % V)] = U[e];
    }
    __syncthreads();
  }
}

// Block ILU(0) in the natural block-row order (CellILU.ComputeILU, CellILU.cs:1229-1330), one wavefront of block
// rows per launch: the rows of a wavefront have all their lower neighbours in earlier wavefronts, so each CTA
// factors one row completely (row-wise "IKJ" order, which performs the same updates of every block in the same
// order as the reference's column-wise loop):
//   for every lower neighbour k of i, ascending:  L_ik = A_ik U_kk^{-1};  A_ij -= L_ik U_kj  (j > k, (k,j) in the
//   pattern), and finally U_ii^{-1} for the rows after it.
// M holds the factors in place (a copy of A's values beforehand); uinv receives U_ii^{-1} column-major at doff
// (FP64, and FP32 when u32 != null).
__global__ void ilu0_level_kernel(const int64_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                  const int32_t* __restrict__ len, const int64_t* __restrict__ boff, int V,
                                  const int64_t* __restrict__ doff, const int32_t* __restrict__ rows, int64_t nrows,
                                  double* __restrict__ M, double* __restrict__ uinv, float* __restrict__ u32,
                                  int* __restrict__ err) {
  extern __shared__ double sm[];
  __shared__ int piv, bad;
  for (int64_t q = blockIdx.x; q < nrows; q += gridDim.x) {
    const int64_t i = rows[q];
    const int I = len[i];
    double* L = sm;  // I x K row-major (K <= max block length)
    int64_t kd = -1;
    for (int64_t t = rp[i]; t < rp[i + 1]; ++t)
      if (ci[t] == i) kd = t;
    if (threadIdx.x == 0) bad = (kd < 0);
    __syncthreads();
    if (bad) {
      if (threadIdx.x == 0) atomicCAS(err, 0, (int)(i + 1 < 0x7fffffff ? i + 1 : 0x7fffffff));
      __syncthreads();
      continue;
    }
    for (int64_t pk = rp[i]; pk < rp[i + 1]; ++pk) {
      const int64_t k = ci[pk];
      if (k >= i) break;  // block columns ascend: the lower neighbours come first
      const int K = len[k];
      const double* D = uinv + doff[k];
      for (int e = threadIdx.x; e < I * K; e += blockDim.x) {
        const int r = e / K, c = e - r * K;
        double acc = 0.0;
        for (int t = 0; t < K; ++t)
          acc = fma(M[boff[pk] + (int64_t)(t / V) * I * V + r * V + (t % V)], D[(int64_t)c * K + t], acc);
        L[e] = acc;
      }
      __syncthreads();
      for (int e = threadIdx.x; e < I * K; e += blockDim.x) {
        const int r = e / K, c = e - r * K;
        M[boff[pk] + (int64_t)(c / V) * I * V + r * V + (c % V)] = L[e];
      }
      for (int64_t pj = pk + 1; pj < rp[i + 1]; ++pj) {
        const int64_t j = ci[pj];
        int64_t kj = -1;
        {
          int64_t lo = rp[k], hi = rp[k + 1];  // binary search of column j in row k
          while (lo < hi) {
            const int64_t mid = (lo + hi) / 2;
            if (ci[mid] < j)
              lo = mid + 1;
            else
              hi = mid;
          }
          if (lo < rp[k + 1] && ci[lo] == j) kj = lo;
        }
        if (kj < 0) continue;  // (k, j) outside the ILU(0) pattern
        const int J = len[j];
        for (int e = threadIdx.x; e < I * J; e += blockDim.x) {
          const int r = e / J, c = e - r * J;
          double acc = 0.0;
          for (int t = 0; t < K; ++t) acc = fma(L[r * K + t], M[boff[kj] + (int64_t)(c / V) * K * V + t * V + (c % V)], acc);
          M[boff[pj] + (int64_t)(c / V) * I * V + r * V + (c % V)] -= acc;
        }
      }
      __syncthreads();
    }
    // U_ii^{-1}: Gauss-Jordan with partial pivoting in shared memory
    double* U = sm;
    double* prow = sm + I * I;
    double* pcol = prow + I;
    int* perm = reinterpret_cast<int*>(pcol + I);
    for (int e = threadIdx.x; e < I * I; e += blockDim.x) {
      const int r = e / I, c = e - r * I;
      U[e] = M[boff[kd] + (int64_t)(c / V) * I * V + r * V + (c % V)];
    }
    __syncthreads();
    for (int p = 0; p < I; ++p) {
      if (threadIdx.x == 0) {
        int best = p;
        double mx = fabs(U[p * I + p]);
        for (int r = p + 1; r < I; ++r)
          if (fabs(U[r * I + p]) > mx) {
            mx = fabs(U[r * I + p]);
            best = r;
          }
        piv = best;
        perm[p] = best;
        if (!(mx > 0.0) || !isfinite(mx)) {
          bad = 1;
          atomicCAS(err, 0, (int)(i + 1 < 0x7fffffff ? i + 1 : 0x7fffffff));
        }
      }
      __syncthreads();
      if (bad) break;
      if (piv != p)
        for (int c = threadIdx.x; c < I; c += blockDim.x) {
          const double t = U[p * I + c];
          U[p * I + c] = U[piv * I + c];
          U[piv * I + c] = t;
        }
      __syncthreads();
      const double inv = 1.0 / U[p * I + p];
      for (int t = threadIdx.x; t < I; t += blockDim.x) {
        prow[t] = (t == p) ? inv : U[p * I + t] * inv;
        pcol[t] = U[t * I + p];
      }
      __syncthreads();
      for (int e = threadIdx.x; e < I * I; e += blockDim.x) {
        const int r = e / I, c = e - r * I;
        if (r == p)
          U[e] = prow[c];
        else if (c == p)
          U[e] = -pcol[r] * prow[p];
        else
          U[e] -= pcol[r] * prow[c];
      }
      __syncthreads();
    }
    if (!bad) {
      for (int p = I - 1; p >= 0; --p) {
        const int t = perm[p];
        if (t != p)
          for (int r = threadIdx.x; r < I; r += blockDim.x) {
            const double w = U[r * I + p];
            U[r * I + p] = U[r * I + t];
            U[r * I + t] = w;
          }
        __syncthreads();
      }
      for (int e = threadIdx.x; e < I * I; e += blockDim.x) {
        const int r = e / I, c = e - r * I;
        uinv[doff[i] + (int64_t)c * I + r] = U[e];
        if (u32) u32[doff[i] + (int64_t)c * I + r] = (float)U[e];
      }
    }
    __syncthreads();
  }
}

DBuf<int32_t> blk_rows(const Matrix& A) {
  std::vector<int32_t> br(A.nnzb);
  for (int64_t i = 0; i < A.nb; ++i)
    for (int64_t k = A.h_rp[i]; k < A.h_rp[i + 1]; ++k) br[k] = (int32_t)i;
  DBuf<int32_t> d(std::max<int64_t>(A.nnzb, 1));
  if (A.nnzb) BSGPU_CUDA(cudaMemcpy(d.p, br.data(), A.nnzb * 4, cudaMemcpyHostToDevice));
  return d;
}

int grid_for(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>(n, (int64_t)num_sms() * 16)); }

}  // namespace

void symminv_batched(const Matrix& A, double* L, int* err, cudaStream_t st) {
  require(!A.single, "SymmInv needs the FP64 matrix");
  if (A.nb == 0) return;
  const int64_t n = A.max_len();
  const size_t smem = (size_t)(2 * n * n + 3 * n) * sizeof(double);
  require(smem <= 200 * 1024, "block too large for SymmInv", BSGPU_ERR_UNSUPPORTED);
  if (smem > 48 * 1024) BSGPU_CUDA(cudaFuncSetAttribute(symminv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  symminv_kernel<<<grid_for(A.nb), 128, smem, st>>>(A.rp.p, A.ci.p, A.len.p, A.boff.p, A.v64.p, A.V, A.doff.p, L, err,
                                                   A.nb);
  BSGPU_CHECK_LAUNCH();
}

void change_of_basis_apply(const Matrix& A, const double* L, Matrix& Aout, cudaStream_t st) {
  require(!A.single && !Aout.single, "change of basis needs FP64 matrices");
  if (A.nnzb == 0) return;
  const int64_t n = A.max_len();
  const size_t smem = (size_t)(4 * n * n) * sizeof(double);
  require(smem <= 200 * 1024, "block too large for the change of basis", BSGPU_ERR_UNSUPPORTED);
  if (smem > 48 * 1024) BSGPU_CUDA(cudaFuncSetAttribute(cob_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  DBuf<int32_t> br = blk_rows(A);
  cob_kernel<<<grid_for(A.nnzb), 128, smem, st>>>(A.rp.p, A.ci.p, A.len.p, br.p, A.boff.p, A.V, A.v64.p, Aout.boff.p,
                                                 Aout.V, Aout.v64.p, L, A.doff.p, A.nnzb);
  BSGPU_CHECK_LAUNCH();
  BSGPU_CUDA(cudaStreamSynchronize(st));
}

void invert_diag_blocks(const Matrix& A, double* D64, float* D32, int* err, cudaStream_t st) {
  require(!A.single, "inversion needs the FP64 matrix");
  if (A.nb == 0) return;
  const int64_t n = A.max_len();
  const size_t smem = (size_t)(n * n + 2 * n) * sizeof(double) + (size_t)n * sizeof(int);
  require(smem <= 200 * 1024, "block too large for the inversion", BSGPU_ERR_UNSUPPORTED);
  if (smem > 48 * 1024) BSGPU_CUDA(cudaFuncSetAttribute(invert_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  invert_kernel<<<grid_for(A.nb), 128, smem, st>>>(A.rp.p, A.ci.p, A.len.p, A.boff.p, A.v64.p, A.V, A.doff.p, D64, D32,
                                                  err, A.nb);
  BSGPU_CHECK_LAUNCH();
}

void ilu0_levels(const Matrix& A, const int32_t* rows, const std::vector<int64_t>& level_ptr, Matrix& M,
                 double* uinv, float* u32, int* err, cudaStream_t st) {
  require(!A.single && !M.single && M.V == A.V && M.nvals == A.nvals, "ILU(0) factors need FP64 matrices");
  BSGPU_CUDA(cudaMemcpyAsync(M.v64.p, A.v64.p, (size_t)A.nvals * 8, cudaMemcpyDeviceToDevice, st));
  const int64_t n = A.max_len();
  const size_t smem = (size_t)(n * n + 2 * n) * sizeof(double) + (size_t)n * sizeof(int);
  require(smem <= 200 * 1024, "block too large for ILU(0)", BSGPU_ERR_UNSUPPORTED);
  if (smem > 48 * 1024)
    BSGPU_CUDA(cudaFuncSetAttribute(ilu0_level_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (size_t l = 0; l + 1 < level_ptr.size(); ++l) {
    const int64_t nr = level_ptr[l + 1] - level_ptr[l];
    if (nr == 0) continue;
    ilu0_level_kernel<<<grid_for(nr), 128, smem, st>>>(A.rp.p, A.ci.p, A.len.p, A.boff.p, A.V, A.doff.p,
                                                       rows + level_ptr[l], nr, M.v64.p, uinv, u32, err);
    BSGPU_CHECK_LAUNCH();
  }
}

void ilu0_two_colour(const Matrix& A, const double* dinv, const int32_t* rows1, int64_t n1, Matrix& M, int* err,
                     cudaStream_t st) {
  require(!A.single && !M.single && M.V == A.V && M.nvals == A.nvals, "ILU(0) factors need FP64 matrices");
  BSGPU_CUDA(cudaMemcpyAsync(M.v64.p, A.v64.p, (size_t)A.nvals * 8, cudaMemcpyDeviceToDevice, st));
  if (n1 == 0) return;
  const int64_t n = A.max_len();
  const size_t smem = (size_t)(2 * n * n) * sizeof(double);
  require(smem <= 200 * 1024, "block too large for ILU(0)", BSGPU_ERR_UNSUPPORTED);
  if (smem > 48 * 1024)
    BSGPU_CUDA(cudaFuncSetAttribute(ilu0_two_colour_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  ilu0_two_colour_kernel<<<grid_for(n1), 128, smem, st>>>(A.rp.p, A.ci.p, A.len.p, A.boff.p, A.v64.p, A.V, A.doff.p,
                                                          dinv, rows1, n1, M.v64.p, err);
  BSGPU_CHECK_LAUNCH();
}

void schwarz_factor(const Matrix& A, Matrix& M, int* err, cudaStream_t st) {
  require(!A.single, "Schwarz factorisation needs the FP64 matrix");
  if (A.nb == 0) return;
  // largest patch: the block row with the most DOFs
  int64_t maxp = 0;
  for (int64_t i = 0; i < A.nb; ++i) {
    int64_t s = 0;
    for (int64_t k = A.h_rp[i]; k < A.h_rp[i + 1]; ++k) s += A.h_len[A.h_ci[k]];
    maxp = std::max(maxp, s);
    require(A.h_rp[i + 1] - A.h_rp[i] <= 32, "Schwarz: more than 32 coupled cells in a block row",
            BSGPU_ERR_UNSUPPORTED);
  }
  const size_t smem = (size_t)(maxp * maxp + 2 * maxp) * 8 + (size_t)maxp * 4;
  require(smem <= 220 * 1024, "Schwarz: patch of " + std::to_string(maxp) + " unknowns exceeds shared memory",
          BSGPU_ERR_UNSUPPORTED);
  const int grid = (int)std::min<int64_t>(A.nb, (int64_t)num_sms() * 8);
  if (M.single) {
    BSGPU_CUDA(cudaFuncSetAttribute(schwarz_factor_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    schwarz_factor_kernel<float><<<grid, 256, smem, st>>>(A.rp.p, A.ci.p, A.len.p, A.boff.p, A.v64.p, A.V, M.boff.p,
                                                          M.V, M.v32.p, (int)maxp, err, A.nb);
  } else {
    BSGPU_CUDA(cudaFuncSetAttribute(schwarz_factor_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    schwarz_factor_kernel<double><<<grid, 256, smem, st>>>(A.rp.p, A.ci.p, A.len.p, A.boff.p, A.v64.p, A.V, M.boff.p,
                                                           M.V, M.v64.p, (int)maxp, err, A.nb);
  }
  BSGPU_CHECK_LAUNCH();
}

void block_trsv_lt(const Matrix& A, const double* L, const double* x, double* y, cudaStream_t st) {
  if (A.nb == 0) return;
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((A.nb + 127) / 128, (int64_t)num_sms() * 8));
  trsv_lt_kernel<<<grid, 128, 0, st>>>(A.len.p, A.i0.p, A.doff.p, L, x, y, A.nb);
  BSGPU_CHECK_LAUNCH();
}

}  // namespace bsgpu
