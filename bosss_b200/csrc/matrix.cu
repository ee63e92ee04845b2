// Block-sparse matrix storage and the SpMV family (BlockMsrMatrix.SpMV, BlockMsrMatrix.cs:2970-3410).
#include <algorithm>
#include <map>
#include <mutex>
#include <numeric>
#include <sstream>

#include "ldst.cuh"
#include "matrix.cuh"

namespace bsgpu {

int64_t Matrix::max_len() const {
  int64_t m = 0;
  for (int32_t l : h_len) m = std::max<int64_t>(m, l);
  return m;
}

namespace {

// ---------------------------------------------------------------------------------------------------------------
// layout conversion
// ---------------------------------------------------------------------------------------------------------------
template <typename TI, typename TO>
__global__ void repack_kernel(const TI* __restrict__ in, const int64_t* __restrict__ in_off, TO* __restrict__ out,
                              const int64_t* __restrict__ boff, const int32_t* __restrict__ blk_row,
                              const int32_t* __restrict__ ci, const int32_t* __restrict__ len, int V,
                              int64_t nnzb) {
  for (int64_t k = blockIdx.x; k < nnzb; k += gridDim.x) {
    const int I = len[blk_row[k]], J = len[ci[k]];
    const int64_t src = in_off[k], dst = boff[k];
    for (int e = threadIdx.x; e < I * J; e += blockDim.x) {
      const int r = e / J, c = e - r * J;
      out[dst + (int64_t)(c / V) * I * V + r * V + (c % V)] = (TO)in[src + e];
    }
  }
}

template <typename TI, typename TO>
__global__ void unpack_kernel(const TI* __restrict__ in, const int64_t* __restrict__ boff, TO* __restrict__ out,
                              const int64_t* __restrict__ out_off, const int32_t* __restrict__ blk_row,
                              const int32_t* __restrict__ ci, const int32_t* __restrict__ len, int V,
                              int64_t nnzb) {
  for (int64_t k = blockIdx.x; k < nnzb; k += gridDim.x) {
    const int I = len[blk_row[k]], J = len[ci[k]];
    const int64_t src = boff[k], dst = out_off[k];
    for (int e = threadIdx.x; e < I * J; e += blockDim.x) {
      const int r = e / J, c = e - r * J;
      out[dst + e] = (TO)in[src + (int64_t)(c / V) * I * V + r * V + (c % V)];
    }
  }
}

// element-wise conversion between layouts of two matrices with identical structure
template <typename TI, typename TO>
__global__ void relayout_kernel(const TI* __restrict__ in, const int64_t* __restrict__ boff_in, int Vin,
                                TO* __restrict__ out, const int64_t* __restrict__ boff_out, int Vout,
                                const int32_t* __restrict__ blk_row, const int32_t* __restrict__ ci,
                                const int32_t* __restrict__ len, int64_t nnzb) {
  for (int64_t k = blockIdx.x; k < nnzb; k += gridDim.x) {
    const int I = len[blk_row[k]], J = len[ci[k]];
    for (int e = threadIdx.x; e < I * J; e += blockDim.x) {
      const int r = e / J, c = e - r * J;
      out[boff_out[k] + (int64_t)(c / Vout) * I * Vout + r * Vout + (c % Vout)] =
          (TO)in[boff_in[k] + (int64_t)(c / Vin) * I * Vin + r * Vin + (c % Vin)];
    }
  }
}

// sub-matrix of the leading `keep` modes of every species (full block = nspc species x Np modes)
template <typename T>
__global__ void restrict_kernel(const T* __restrict__ in, const int64_t* __restrict__ boff_in, int Vin,
                                T* __restrict__ out, const int64_t* __restrict__ boff_out, int Vout,
                                const int32_t* __restrict__ blk_row, const int32_t* __restrict__ ci,
                                const int32_t* __restrict__ len_in, const int32_t* __restrict__ len_out, int Np,
                                int keep, int64_t nnzb) {
  for (int64_t k = blockIdx.x; k < nnzb; k += gridDim.x) {
    const int i = blk_row[k], j = ci[k];
    const int Ii = len_in[i], Ji = len_in[j], Io = len_out[i], Jo = len_out[j];
    (void)Ji;
    for (int e = threadIdx.x; e < Io * Jo; e += blockDim.x) {
      const int r = e / Jo, c = e - r * Jo;
      const int rf = (r / keep) * Np + (r % keep), cf = (c / keep) * Np + (c % keep);
      out[boff_out[k] + (int64_t)(c / Vout) * Io * Vout + r * Vout + (c % Vout)] =
          in[boff_in[k] + (int64_t)(cf / Vin) * Ii * Vin + rf * Vin + (cf % Vin)];
    }
  }
}

// ---------------------------------------------------------------------------------------------------------------
// SpMV kernels
// ---------------------------------------------------------------------------------------------------------------
template <typename T>
struct Acc { using type = T; };

// Uniform Np x Np blocks, Np known at compile time.  A CTA owns BPC = blockDim/NP whole block rows; thread t is DOF
// row r = t % NP of block row t / NP.  MODE 0: y = alpha*A*x + beta*z.  MODE 1: fused block-Jacobi update
// y = x + alpha * Dinv * (z - A*x) (z = b), the block row's residual exchanged through shared memory.
template <typename T, int NP, int V, int MODE, typename S = T>
__global__ void __launch_bounds__(256) spmv_uniform_kernel(
    const int64_t* __restrict__ rp, const int32_t* __restrict__ ci, const S* __restrict__ vals,
    const T* x, const T* __restrict__ z, T* y, T alpha, T beta, int64_t nb,
    const T* __restrict__ dinv, const int* __restrict__ active, const int32_t* __restrict__ row_list = nullptr) {
  static_assert(NP % V == 0, "chunk width must divide the block size");
  if (active != nullptr && *active == 0) return;
  const int BPC = blockDim.x / NP;  // block rows per CTA (the launch shape the autotuner picks)
  const int t = threadIdx.x;
  const int lb = t / NP;
  const int r = t - lb * NP;
  // MODE 2 (block Gauss-Seidel half-sweep): the block rows come from `row_list` (one colour; nb is the list
  // length) and the update is in place (x == y): all reads of x precede the barrier, the write follows it, and
  // no block row of the list reads another row of the list.
  int64_t i = (int64_t)blockIdx.x * BPC + lb;
  bool valid = (lb < BPC) && (i < nb);
  if constexpr (MODE == 2 || MODE == 3) {
    if (valid) i = row_list[i];
  }
  const uint64_t pol = policy_evict_first();
  T acc0 = 0, acc1 = 0;
  if (valid) {
    const int64_t k0 = rp[i], k1 = rp[i + 1];
    for (int64_t k = k0; k < k1; ++k) {
      const int64_t j = ci[k];
      const S* vb = vals + k * (NP * NP) + r * V;
      const T* xb = x + j * NP;
#pragma unroll
      for (int c = 0; c < NP / V; ++c) {
        Vec<S, V> a = ldv_stream<S, V>(vb + c * (NP * V), pol);
        Vec<T, V> xv = ldv_cached<T, V>(xb + c * V);
#pragma unroll
        for (int q = 0; q < V; ++q) {
          if ((c * V + q) & 1)
            acc1 = fma(widen<T>(a.a[q]), xv.a[q], acc1);
          else
            acc0 = fma(widen<T>(a.a[q]), xv.a[q], acc0);
        }
      }
    }
  }
  const T acc = acc0 + acc1;
  const int64_t g = i * NP + r;
  if constexpr (MODE == 0) {
    if (valid) {
      T out = alpha * acc;
      if (z != nullptr) out = fma(beta, z[g], out);
      y[g] = out;
    }
  } else if constexpr (MODE == 3) {
    // unit-diagonal in-place update over a row list (forward substitution with a unit lower factor): every read of
    // x in the CTA precedes the barrier, the writes follow it
    const T val = valid ? fma(alpha, z[g] - acc, x[g]) : T(0);
    __syncthreads();
    if (valid) y[g] = val;
  } else {
    __shared__ T q[256];
    q[t] = valid ? (z[g] - acc) : T(0);
    __syncthreads();
    if (valid) {
      const T* D = dinv + i * (NP * NP) + r;
      const T* qb = q + lb * NP;
      T s0 = 0, s1 = 0;
#pragma unroll
      for (int c = 0; c < NP; c += 2) {
        s0 = fma(D[c * NP], qb[c], s0);
        if (c + 1 < NP) s1 = fma(D[(c + 1) * NP], qb[c + 1], s1);
      }
      y[g] = fma(alpha, s0 + s1, x[g]);
    }
  }
}

// General block sizes (XDG: 1..n species per block).  CTA b owns DOF rows cta_row0[b] .. cta_row0[b+1]-1,
// which are whole block rows (packed on the host).
template <typename T, int V, int MODE>
__global__ void __launch_bounds__(256) spmv_general_kernel(
    const int64_t* __restrict__ rp, const int32_t* __restrict__ ci, const int32_t* __restrict__ len,
    const int64_t* __restrict__ i0, const int64_t* __restrict__ boff, const int32_t* __restrict__ row2blk,
    const int64_t* __restrict__ cta_row0, const T* __restrict__ vals, const T* __restrict__ x,
    const T* __restrict__ z, T* __restrict__ y, T alpha, T beta, const T* __restrict__ dinv,
    const int64_t* __restrict__ doff, const int* __restrict__ active) {
  if (active != nullptr && *active == 0) return;
  const int64_t row0 = cta_row0[blockIdx.x], row1 = cta_row0[blockIdx.x + 1];
  const int64_t g = row0 + threadIdx.x;
  const bool valid = g < row1;
  const uint64_t pol = policy_evict_first();
  T acc0 = 0, acc1 = 0;
  int64_t i = 0;
  int r = 0, I = 0;
  if (valid) {
    i = row2blk[g];
    r = (int)(g - i0[i]);
    I = len[i];
    for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
      const int64_t j = ci[k];
      const int J = len[j];
      const T* vb = vals + boff[k] + r * V;
      const T* xb = x + i0[j];
      int c = 0;
      for (; c + 2 * V <= J; c += 2 * V) {
        Vec<T, V> a = ldv_stream<T, V>(vb + (int64_t)(c / V) * I * V, pol);
        Vec<T, V> b = ldv_stream<T, V>(vb + (int64_t)(c / V + 1) * I * V, pol);
        Vec<T, V> xa = ldv_cached<T, V>(xb + c);
        Vec<T, V> xc = ldv_cached<T, V>(xb + c + V);
#pragma unroll
        for (int q = 0; q < V; ++q) {
          acc0 = fma(a.a[q], xa.a[q], acc0);
          acc1 = fma(b.a[q], xc.a[q], acc1);
        }
      }
      for (; c < J; c += V) {
        Vec<T, V> a = ldv_stream<T, V>(vb + (int64_t)(c / V) * I * V, pol);
        Vec<T, V> xa = ldv_cached<T, V>(xb + c);
#pragma unroll
        for (int q = 0; q < V; ++q) acc0 = fma(a.a[q], xa.a[q], acc0);
      }
    }
  }
  const T acc = acc0 + acc1;
  if constexpr (MODE == 0) {
    if (valid) {
      T out = alpha * acc;
      if (z != nullptr) out = fma(beta, z[g], out);
      y[g] = out;
    }
  } else {
    __shared__ T q[256];
    q[threadIdx.x] = valid ? (z[g] - acc) : T(0);
    __syncthreads();
    if (valid) {
      const T* D = dinv + doff[i] + r;
      const int base = (int)(i0[i] - row0);
      T s = 0;
      for (int c = 0; c < I; ++c) s = fma(D[(int64_t)c * I], q[base + c], s);
      y[g] = fma(alpha, s, x[g]);
    }
  }
}

// Blocks of one or two species of NP modes each (XDG cut cells carry two).  The block rows of one species count are
// listed in `rows`; a CTA owns blockDim / (NS*NP) of them, thread t being DOF row r of list entry t / (NS*NP), as in
// the uniform kernel, so the row length is a compile-time constant.  A block in column j has len[j] / NP species
// sub-blocks of NP columns, each streamed with the fully unrolled chunk loop of the uniform kernel (V divides NP,
// so no chunk straddles a species boundary and there is no scalar tail).
template <typename T, int NP, int NS, int V, int MODE>
__device__ __forceinline__ void typed_rows(int BPC, int64_t b0, int64_t nrows, const int32_t* __restrict__ rows,
                                           const int64_t* __restrict__ rp, const int32_t* __restrict__ ci,
                                           const int32_t* __restrict__ len, const int64_t* __restrict__ i0,
                                           const int64_t* __restrict__ boff, const T* __restrict__ vals,
                                           const T* __restrict__ x, const T* __restrict__ z, T* __restrict__ y,
                                           T alpha, T beta, const T* __restrict__ dinv,
                                           const int64_t* __restrict__ doff) {
  constexpr int I = NP * NS;
  static_assert(NP % V == 0, "chunk width must divide the species block");
  const int t = threadIdx.x;
  const int lb = t / I;
  const int r = t - lb * I;
  const int64_t b = b0 + lb;
  const bool valid = (lb < BPC) && (b < nrows);
  const int64_t i = valid ? rows[b] : 0;
  const uint64_t pol = policy_evict_first();
  T acc0 = 0, acc1 = 0;
  if (valid) {
    const int64_t k0 = rp[i], k1 = rp[i + 1];
    for (int64_t k = k0; k < k1; ++k) {
      const int64_t j = ci[k];
      const int sj = len[j] / NP;
      const T* vb = vals + boff[k] + r * V;
      const T* xb = x + i0[j];
      for (int sp = 0; sp < sj; ++sp) {
#pragma unroll
        for (int c = 0; c < NP / V; ++c) {
          const int col = sp * NP + c * V;
          Vec<T, V> a = ldv_stream<T, V>(vb + (int64_t)(col / V) * (I * V), pol);
          Vec<T, V> xv = ldv_cached<T, V>(xb + col);
#pragma unroll
          for (int q = 0; q < V; ++q) {
            if ((c * V + q) & 1)
              acc1 = fma(a.a[q], xv.a[q], acc1);
            else
              acc0 = fma(a.a[q], xv.a[q], acc0);
          }
        }
      }
    }
  }
  const T acc = acc0 + acc1;
  const int64_t g = valid ? i0[i] + r : 0;
  if constexpr (MODE == 0) {
    if (valid) {
      T out = alpha * acc;
      if (z != nullptr) out = fma(beta, z[g], out);
      y[g] = out;
    }
  } else {
    __shared__ T q[256];
    q[t] = valid ? (z[g] - acc) : T(0);
    __syncthreads();
    if (valid) {
      const T* D = dinv + doff[i] + r;
      const T* qb = q + lb * I;
      T s0 = 0, s1 = 0;
#pragma unroll
      for (int c = 0; c < I; c += 2) {
        s0 = fma(D[c * I], qb[c], s0);
        if (c + 1 < I) s1 = fma(D[(c + 1) * I], qb[c + 1], s1);
      }
      y[g] = fma(alpha, s0 + s1, x[g]);
    }
  }
}

// One launch for both species counts: CTAs [0, cta1) take the one-species rows, the rest the two-species rows.
template <typename T, int NP, int V, int MODE>
__global__ void __launch_bounds__(256) spmv_typed_kernel(
    const int64_t* __restrict__ rp, const int32_t* __restrict__ ci, const int32_t* __restrict__ len,
    const int64_t* __restrict__ i0, const int64_t* __restrict__ boff, const int32_t* __restrict__ rows,
    int64_t n1, int64_t n2, int64_t cta1, const T* __restrict__ vals, const T* __restrict__ x,
    const T* __restrict__ z, T* __restrict__ y, T alpha, T beta, const T* __restrict__ dinv,
    const int64_t* __restrict__ doff, const int* __restrict__ active) {
  if (active != nullptr && *active == 0) return;
  const int bpc1 = blockDim.x / NP, bpc2 = blockDim.x / (2 * NP);
  if ((int64_t)blockIdx.x < cta1)
    typed_rows<T, NP, 1, V, MODE>(bpc1, (int64_t)blockIdx.x * bpc1, n1, rows, rp, ci, len, i0, boff, vals, x, z, y,
                                  alpha, beta, dinv, doff);
  else
    typed_rows<T, NP, 2, V, MODE>(bpc2, ((int64_t)blockIdx.x - cta1) * bpc2, n2, rows + n1, rp, ci, len, i0, boff,
                                  vals, x, z, y, alpha, beta, dinv, doff);
}

// y = alpha * Dinv * b (block diagonal, column-major blocks)
template <typename T>
__global__ void blockdiag_kernel(const int32_t* __restrict__ len, const int64_t* __restrict__ i0,
                                 const int32_t* __restrict__ row2blk, const int64_t* __restrict__ doff,
                                 const T* __restrict__ dinv, T alpha, const T* __restrict__ b, T* __restrict__ y,
                                 int64_t N, int uniformNp, const int* __restrict__ active) {
  if (active != nullptr && *active == 0) return;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < N; g += (int64_t)gridDim.x * blockDim.x) {
    int64_t i;
    int I;
    int64_t o;
    if (uniformNp > 0) {
      i = g / uniformNp;
      I = uniformNp;
      o = i * I * I;
    } else {
      i = row2blk[g];
      I = len[i];
      o = doff[i];
    }
    const int64_t s0 = uniformNp > 0 ? i * I : i0[i];
    const int r = (int)(g - s0);
    const T* D = dinv + o + r;
    T s = 0;
    for (int c = 0; c < I; ++c) s = fma(D[(int64_t)c * I], b[s0 + c], s);
    y[g] = alpha * s;
  }
}

int pick_V(const std::vector<int32_t>& len, bool single) {
  const int cand = single ? 4 : 2;
  for (int V = cand; V > 1; V /= 2) {
    bool ok = true;
    for (int32_t l : len)
      if (l % V) { ok = false; break; }
    if (ok) return V;
  }
  return 1;
}

// host-side derived structure (offsets, packing), uploaded to the device
void finish_structure(Matrix& M) {
  M.nb = (int64_t)M.h_len.size();
  M.nnzb = (int64_t)M.h_ci.size();
  M.h_i0.assign(M.nb + 1, 0);
  for (int64_t i = 0; i < M.nb; ++i) M.h_i0[i + 1] = M.h_i0[i] + M.h_len[i];
  M.N = M.h_i0[M.nb];
  M.V = pick_V(M.h_len, M.single);
  std::vector<int64_t> boff(M.nnzb);
  int64_t off = 0;
  for (int64_t i = 0; i < M.nb; ++i)
    for (int64_t k = M.h_rp[i]; k < M.h_rp[i + 1]; ++k) {
      boff[k] = off;
      off += (int64_t)M.h_len[i] * M.h_len[M.h_ci[k]];
    }
  M.nvals = off;
  M.rp.alloc(M.nb + 1);
  M.ci.alloc(std::max<int64_t>(M.nnzb, 1));
  M.len.alloc(std::max<int64_t>(M.nb, 1));
  M.i0.alloc(M.nb + 1);
  M.boff.alloc(std::max<int64_t>(M.nnzb, 1));
  BSGPU_CUDA(cudaMemcpy(M.rp.p, M.h_rp.data(), (M.nb + 1) * 8, cudaMemcpyHostToDevice));
  if (M.nnzb) BSGPU_CUDA(cudaMemcpy(M.ci.p, M.h_ci.data(), M.nnzb * 4, cudaMemcpyHostToDevice));
  if (M.nb) BSGPU_CUDA(cudaMemcpy(M.len.p, M.h_len.data(), M.nb * 4, cudaMemcpyHostToDevice));
  BSGPU_CUDA(cudaMemcpy(M.i0.p, M.h_i0.data(), (M.nb + 1) * 8, cudaMemcpyHostToDevice));
  if (M.nnzb) BSGPU_CUDA(cudaMemcpy(M.boff.p, boff.data(), M.nnzb * 8, cudaMemcpyHostToDevice));
  // row -> block map and CTA packing (whole block rows, at most 256 DOF rows per CTA)
  std::vector<int32_t> r2b(M.N);
  for (int64_t i = 0; i < M.nb; ++i)
    for (int64_t g = M.h_i0[i]; g < M.h_i0[i + 1]; ++g) r2b[g] = (int32_t)i;
  std::vector<int64_t> packs{0};
  int64_t cur = 0;
  for (int64_t i = 0; i < M.nb; ++i) {
    if (cur + M.h_len[i] > M.cta_threads) {
      packs.push_back(M.h_i0[i]);
      cur = 0;
    }
    cur += M.h_len[i];
  }
  packs.push_back(M.N);
  if (packs.size() >= 2 && packs[packs.size() - 2] == M.N) packs.pop_back();
  M.ncta = (int64_t)packs.size() - 1;
  std::vector<int64_t> dof(M.nb + 1, 0);
  for (int64_t i = 0; i < M.nb; ++i) dof[i + 1] = dof[i] + (int64_t)M.h_len[i] * M.h_len[i];
  M.doff.alloc(M.nb + 1);
  BSGPU_CUDA(cudaMemcpy(M.doff.p, dof.data(), (M.nb + 1) * 8, cudaMemcpyHostToDevice));
  // species-count groups for the typed kernels (one or two species of Np modes, Np in {1, 4, 10, 20})
  M.typed = false;
  M.grp_n1 = M.grp_n2 = 0;
  bool two_at_most = M.nb > 0;
  for (int64_t i = 0; i < M.nb && two_at_most; ++i) two_at_most = M.h_len[i] == M.Np || M.h_len[i] == 2 * M.Np;
  const bool np_ok = M.Np == 1 || M.Np == 4 || M.Np == 10 || M.Np == 20;
  if (!M.uniform && two_at_most && np_ok && M.Np % M.V == 0) {
    std::vector<int32_t> g;
    g.reserve(M.nb);
    for (int64_t i = 0; i < M.nb; ++i)
      if (M.h_len[i] == M.Np) g.push_back((int32_t)i);
    M.grp_n1 = (int64_t)g.size();
    for (int64_t i = 0; i < M.nb; ++i)
      if (M.h_len[i] == 2 * M.Np) g.push_back((int32_t)i);
    M.grp_n2 = (int64_t)g.size() - M.grp_n1;
    M.grp_rows.alloc(g.size());
    BSGPU_CUDA(cudaMemcpy(M.grp_rows.p, g.data(), g.size() * 4, cudaMemcpyHostToDevice));
    M.typed = true;
  }
  M.row2blk.alloc(std::max<int64_t>(M.N, 1));
  M.cta_row0.alloc(packs.size());
  if (M.N) BSGPU_CUDA(cudaMemcpy(M.row2blk.p, r2b.data(), M.N * 4, cudaMemcpyHostToDevice));
  BSGPU_CUDA(cudaMemcpy(M.cta_row0.p, packs.data(), packs.size() * 8, cudaMemcpyHostToDevice));
}

DBuf<int32_t> block_rows(const Matrix& M) {
  std::vector<int32_t> br(M.nnzb);
  for (int64_t i = 0; i < M.nb; ++i)
    for (int64_t k = M.h_rp[i]; k < M.h_rp[i + 1]; ++k) br[k] = (int32_t)i;
  DBuf<int32_t> d(std::max<int64_t>(M.nnzb, 1));
  if (M.nnzb) BSGPU_CUDA(cudaMemcpy(d.p, br.data(), M.nnzb * 4, cudaMemcpyHostToDevice));
  return d;
}

std::vector<int64_t> rowmajor_offsets(const Matrix& M) {
  std::vector<int64_t> o(M.nnzb + 1, 0);
  for (int64_t i = 0; i < M.nb; ++i)
    for (int64_t k = M.h_rp[i]; k < M.h_rp[i + 1]; ++k) o[k + 1] = o[k] + (int64_t)M.h_len[i] * M.h_len[M.h_ci[k]];
  return o;
}

int conv_grid(int64_t nnzb) { return (int)std::min<int64_t>(std::max<int64_t>(nnzb, 1), 1 << 20); }

bool specialised(const Matrix& A) {
  if (!A.uniform) return false;
  switch (A.Np) {
    case 4: case 6: case 10: case 20: return A.V == (A.single ? (A.Np % 4 == 0 ? 4 : 2) : 2);
    default: return false;
  }
}

template <typename T, int NP, int V, int MODE, typename S = T>
void launch_uniform(const Matrix& A, const S* vals, const T* x, const T* z, T* y, T alpha, T beta, const T* dinv,
                    cudaStream_t st, const int* active) {
  const int BPC = std::max(1, A.cta[MODE == 1 ? 1 : 0] / NP);
  const int64_t grid = (A.nb + BPC - 1) / BPC;
  if (grid == 0) return;
  spmv_uniform_kernel<T, NP, V, MODE, S><<<(unsigned)grid, BPC * NP, 0, st>>>(A.rp.p, A.ci.p, vals, x, z, y, alpha,
                                                                             beta, A.nb, dinv, active);
  BSGPU_CHECK_LAUNCH();
}

// FP16 values, FP32 vectors and arithmetic (the preconditioner's level matrices stored in half precision); uniform
// blocks of 4, 10 or 20 with the chunk width of the half layout
template <int MODE>
void dispatch_half(const Matrix& A, const float* x, const float* z, float* y, float alpha, float beta,
                   const float* dinv, cudaStream_t st, const int* active) {
  const __half* v = A.v16.p;
  if (A.uniform && A.Np == 20 && A.V == 4)
    return launch_uniform<float, 20, 4, MODE, __half>(A, v, x, z, y, alpha, beta, dinv, st, active);
  if (A.uniform && A.Np == 10 && A.V == 2)
    return launch_uniform<float, 10, 2, MODE, __half>(A, v, x, z, y, alpha, beta, dinv, st, active);
  if (A.uniform && A.Np == 4 && A.V == 4)
    return launch_uniform<float, 4, 4, MODE, __half>(A, v, x, z, y, alpha, beta, dinv, st, active);
  throw Error(BSGPU_ERR_UNSUPPORTED, "FP16 matrices: uniform blocks of 4, 10 or 20 only");
}

template <typename T, int V, int MODE>
void launch_general(const Matrix& A, const T* vals, const T* x, const T* z, T* y, T alpha, T beta, const T* dinv,
                    const int64_t* doff, cudaStream_t st, const int* active) {
  if (A.ncta == 0) return;
  spmv_general_kernel<T, V, MODE><<<(unsigned)A.ncta, A.cta_threads, 0, st>>>(
      A.rp.p, A.ci.p, A.len.p, A.i0.p, A.boff.p, A.row2blk.p, A.cta_row0.p, vals, x, z, y, alpha, beta, dinv, doff,
      active);
  BSGPU_CHECK_LAUNCH();
}

template <typename T, int NP, int V, int MODE>
void launch_typed(const Matrix& A, const T* vals, const T* x, const T* z, T* y, T alpha, T beta, const T* dinv,
                  const int64_t* doff, cudaStream_t st, const int* active) {
  const int threads = std::max(A.cta[MODE == 1 ? 1 : 0], 2 * NP);
  const int64_t bpc1 = threads / NP, bpc2 = threads / (2 * NP);
  const int64_t cta1 = (A.grp_n1 + bpc1 - 1) / bpc1, cta2 = (A.grp_n2 + bpc2 - 1) / bpc2;
  if (cta1 + cta2 == 0) return;
  spmv_typed_kernel<T, NP, V, MODE><<<(unsigned)(cta1 + cta2), threads, 0, st>>>(
      A.rp.p, A.ci.p, A.len.p, A.i0.p, A.boff.p, A.grp_rows.p, A.grp_n1, A.grp_n2, cta1, vals, x, z, y, alpha, beta,
      dinv, doff, active);
  BSGPU_CHECK_LAUNCH();
}

// the (Np, V) pairs of the typed kernels; false: not covered (the general kernel serves the matrix)
template <typename T, int MODE>
bool dispatch_typed(const Matrix& A, const T* vals, const T* x, const T* z, T* y, T alpha, T beta, const T* dinv,
                    const int64_t* doff, cudaStream_t st, const int* active) {
  if (!A.typed) return false;
#define BSGPU_TYPED(NP, VV)                                                                       \
  if (A.Np == NP && A.V == VV) {                                                                  \
    launch_typed<T, NP, VV, MODE>(A, vals, x, z, y, alpha, beta, dinv, doff, st, active);         \
    return true;                                                                                  \
  }
  BSGPU_TYPED(1, 1)
  BSGPU_TYPED(4, 2)
  BSGPU_TYPED(10, 2)
  BSGPU_TYPED(20, 2)
  if constexpr (sizeof(T) == 4) {
    BSGPU_TYPED(4, 4)
    BSGPU_TYPED(20, 4)
  }
#undef BSGPU_TYPED
  return false;
}

template <typename T, int MODE>
void dispatch(const Matrix& A, const T* vals, const T* x, const T* z, T* y, T alpha, T beta, const T* dinv,
              const int64_t* doff, cudaStream_t st, const int* active) {
  if (dispatch_typed<T, MODE>(A, vals, x, z, y, alpha, beta, dinv, doff, st, active)) return;
  if (specialised(A)) {
    constexpr int VW = sizeof(T) == 8 ? 2 : 4;
    switch (A.Np) {
      case 20: return launch_uniform<T, 20, VW, MODE>(A, vals, x, z, y, alpha, beta, dinv, st, active);
      case 4: return launch_uniform<T, 4, VW, MODE>(A, vals, x, z, y, alpha, beta, dinv, st, active);
      case 10: return launch_uniform<T, 10, 2, MODE>(A, vals, x, z, y, alpha, beta, dinv, st, active);
      case 6: return launch_uniform<T, 6, 2, MODE>(A, vals, x, z, y, alpha, beta, dinv, st, active);
    }
  }
  switch (A.V) {
    case 1: return launch_general<T, 1, MODE>(A, vals, x, z, y, alpha, beta, dinv, doff, st, active);
    case 2: return launch_general<T, 2, MODE>(A, vals, x, z, y, alpha, beta, dinv, doff, st, active);
    default:
      if constexpr (sizeof(T) == 4) return launch_general<T, 4, MODE>(A, vals, x, z, y, alpha, beta, dinv, doff, st, active);
      throw Error(BSGPU_ERR_UNSUPPORTED, "unsupported chunk width");
  }
}

void check_aligned(const void* p, size_t a, const char* what) {
  require(((uintptr_t)p % a) == 0, std::string(what) + " must be aligned to " + std::to_string(a) + " bytes");
}

}  // namespace

std::vector<int64_t> diag_offsets(const Matrix& A) {
  std::vector<int64_t> o(A.nb + 1, 0);
  for (int64_t i = 0; i < A.nb; ++i) o[i + 1] = o[i] + (int64_t)A.h_len[i] * A.h_len[i];
  return o;
}

Matrix* matrix_create(int64_t nb, int32_t Np, const int32_t* nspc, const int64_t* row_ptr, const int32_t* col_idx,
                      const double* values, int32_t flags) {
  require(nb >= 0 && Np > 0, "nb must be >= 0 and Np > 0");
  require(row_ptr && (col_idx || nb == 0) && (values || nb == 0), "null array");
  require(flags == BSGPU_HOST_POINTERS || flags == BSGPU_DEVICE_POINTERS, "bad pointer flag");
  auto M = std::make_unique<Matrix>();
  M->Np = Np;
  M->h_rp.resize(nb + 1);
  const bool dev = flags == BSGPU_DEVICE_POINTERS;
  if (dev)
    BSGPU_CUDA(cudaMemcpy(M->h_rp.data(), row_ptr, (nb + 1) * 8, cudaMemcpyDeviceToHost));
  else
    std::copy(row_ptr, row_ptr + nb + 1, M->h_rp.begin());
  require(M->h_rp[0] == 0, "row_ptr[0] must be 0");
  for (int64_t i = 0; i < nb; ++i) require(M->h_rp[i + 1] >= M->h_rp[i], "row_ptr must be non-decreasing");
  const int64_t nnzb = M->h_rp[nb];
  M->h_ci.resize(nnzb);
  M->h_nspc.assign(nb, 1);
  if (dev) {
    if (nnzb) BSGPU_CUDA(cudaMemcpy(M->h_ci.data(), col_idx, nnzb * 4, cudaMemcpyDeviceToHost));
    if (nspc && nb) BSGPU_CUDA(cudaMemcpy(M->h_nspc.data(), nspc, nb * 4, cudaMemcpyDeviceToHost));
  } else {
    std::copy(col_idx, col_idx + nnzb, M->h_ci.begin());
    if (nspc) std::copy(nspc, nspc + nb, M->h_nspc.begin());
  }
  for (int64_t i = 0; i < nb; ++i) {
    require(M->h_nspc[i] >= 1, "nspc must be >= 1");
    for (int64_t k = M->h_rp[i]; k < M->h_rp[i + 1]; ++k) {
      require(M->h_ci[k] >= 0 && M->h_ci[k] < nb, "col_idx out of range");
      if (k > M->h_rp[i]) require(M->h_ci[k] > M->h_ci[k - 1], "block columns must be strictly ascending");
    }
  }
  M->h_len.resize(nb);
  M->uniform = true;
  for (int64_t i = 0; i < nb; ++i) {
    M->h_len[i] = M->h_nspc[i] * Np;
    if (M->h_nspc[i] != 1) M->uniform = false;
  }
  require((int64_t)Np * (M->uniform ? 1 : *std::max_element(M->h_nspc.begin(), M->h_nspc.end())) <= 256,
          "block length above 256 is not supported", BSGPU_ERR_UNSUPPORTED);
  finish_structure(*M);
  // values: row-major blocks in input order -> device layout
  std::vector<int64_t> in_off = rowmajor_offsets(*M);
  M->v64.alloc(std::max<int64_t>(M->nvals, 1));
  if (M->nvals) {
    DBuf<double> tmp;
    const double* src = values;
    if (!dev) {
      tmp.alloc(M->nvals);
      BSGPU_CUDA(cudaMemcpy(tmp.p, values, M->nvals * 8, cudaMemcpyHostToDevice));
      src = tmp.p;
    }
    DBuf<int64_t> d_in_off(M->nnzb);
    BSGPU_CUDA(cudaMemcpy(d_in_off.p, in_off.data(), M->nnzb * 8, cudaMemcpyHostToDevice));
    DBuf<int32_t> br = block_rows(*M);
    repack_kernel<double, double><<<conv_grid(M->nnzb), 128>>>(src, d_in_off.p, M->v64.p, M->boff.p, br.p, M->ci.p,
                                                              M->len.p, M->V, M->nnzb);
    BSGPU_CHECK_LAUNCH();
    BSGPU_CUDA(cudaDeviceSynchronize());
  }
  return M.release();
}

Matrix* matrix_like(const Matrix& A, bool single) {
  auto M = std::make_unique<Matrix>();
  M->Np = A.Np;
  M->uniform = A.uniform;
  M->single = single;
  M->h_rp = A.h_rp;
  M->h_ci = A.h_ci;
  M->h_len = A.h_len;
  M->h_nspc = A.h_nspc;
  finish_structure(*M);
  if (single)
    M->v32.alloc(std::max<int64_t>(M->nvals, 1));
  else
    M->v64.alloc(std::max<int64_t>(M->nvals, 1));
  return M.release();
}

void matrix_read_values(const Matrix& A, double* dst, bool dst_device, cudaStream_t st) {
  require(!A.single, "read_values: FP64 matrices only");
  if (!A.nvals) return;
  std::vector<int64_t> out_off = rowmajor_offsets(A);
  DBuf<int64_t> d_off(A.nnzb);
  BSGPU_CUDA(cudaMemcpy(d_off.p, out_off.data(), A.nnzb * 8, cudaMemcpyHostToDevice));
  DBuf<int32_t> br = block_rows(A);
  DBuf<double> tmp;
  double* out = dst;
  if (!dst_device) {
    tmp.alloc(A.nvals);
    out = tmp.p;
  }
  unpack_kernel<double, double><<<conv_grid(A.nnzb), 128, 0, st>>>(A.v64.p, A.boff.p, out, d_off.p, br.p, A.ci.p,
                                                                   A.len.p, A.V, A.nnzb);
  BSGPU_CHECK_LAUNCH();
  if (!dst_device) BSGPU_CUDA(cudaMemcpyAsync(dst, tmp.p, A.nvals * 8, cudaMemcpyDeviceToHost, st));
  BSGPU_CUDA(cudaStreamSynchronize(st));
}

Matrix* matrix_to_single(const Matrix& A, cudaStream_t st) {
  require(!A.single, "matrix is already single precision");
  std::unique_ptr<Matrix> M(matrix_like(A, true));
  DBuf<int32_t> br = block_rows(A);
  if (A.nvals) {
    relayout_kernel<double, float><<<conv_grid(A.nnzb), 128, 0, st>>>(A.v64.p, A.boff.p, A.V, M->v32.p, M->boff.p,
                                                                      M->V, br.p, A.ci.p, A.len.p, A.nnzb);
    BSGPU_CHECK_LAUNCH();
  }
  BSGPU_CUDA(cudaStreamSynchronize(st));
  return M.release();
}

Matrix* matrix_to_half(const Matrix& A, cudaStream_t st) {
  require(!A.single, "the FP16 copy is made from the FP64 matrix");
  require(A.uniform && (A.Np == 4 || A.Np == 10 || A.Np == 20), "FP16 matrices: uniform blocks of 4, 10 or 20 only",
          BSGPU_ERR_UNSUPPORTED);
  auto M = std::make_unique<Matrix>();
  M->Np = A.Np;
  M->uniform = true;
  M->single = true;
  M->half = true;
  M->h_rp = A.h_rp;
  M->h_ci = A.h_ci;
  M->h_len = A.h_len;
  M->h_nspc = A.h_nspc;
  finish_structure(*M);
  M->V = A.Np == 10 ? 2 : 4;  // the widest chunk (up to 8 bytes of halves) dividing the block width
  M->typed = false;
  M->v16.alloc(std::max<int64_t>(M->nvals, 1));
  DBuf<int32_t> br = block_rows(A);
  if (A.nvals) {
    relayout_kernel<double, __half><<<conv_grid(A.nnzb), 128, 0, st>>>(A.v64.p, A.boff.p, A.V, M->v16.p, M->boff.p,
                                                                       M->V, br.p, A.ci.p, A.len.p, A.nnzb);
    BSGPU_CHECK_LAUNCH();
  }
  BSGPU_CUDA(cudaStreamSynchronize(st));
  return M.release();
}

Matrix* matrix_restrict(const Matrix& A, int keep, cudaStream_t st) {
  require(keep >= 1 && keep <= A.Np, "restriction: keep must be in 1..Np");
  auto M = std::make_unique<Matrix>();
  M->Np = keep;
  M->uniform = A.uniform;
  M->single = A.single;
  M->h_rp = A.h_rp;
  M->h_ci = A.h_ci;
  M->h_nspc = A.h_nspc;
  M->h_len.resize(A.nb);
  for (int64_t i = 0; i < A.nb; ++i) M->h_len[i] = A.h_nspc[i] * keep;
  finish_structure(*M);
  DBuf<int32_t> br = block_rows(A);
  if (M->single) {
    M->v32.alloc(std::max<int64_t>(M->nvals, 1));
    if (M->nvals)
      restrict_kernel<float><<<conv_grid(A.nnzb), 128, 0, st>>>(A.v32.p, A.boff.p, A.V, M->v32.p, M->boff.p, M->V,
                                                                br.p, A.ci.p, A.len.p, M->len.p, A.Np, keep, A.nnzb);
  } else {
    M->v64.alloc(std::max<int64_t>(M->nvals, 1));
    if (M->nvals)
      restrict_kernel<double><<<conv_grid(A.nnzb), 128, 0, st>>>(A.v64.p, A.boff.p, A.V, M->v64.p, M->boff.p, M->V,
                                                                 br.p, A.ci.p, A.len.p, M->len.p, A.Np, keep, A.nnzb);
  }
  BSGPU_CHECK_LAUNCH();
  BSGPU_CUDA(cudaStreamSynchronize(st));
  return M.release();
}

// ---------------------------------------------------------------------------------------------------------------
// SpMV entry points
// ---------------------------------------------------------------------------------------------------------------
void spmv(const Matrix& A, double alpha, const double* x, double beta, const double* z, double* y, cudaStream_t st,
          const int* active) {
  require(!A.single, "FP64 SpMV on an FP32 matrix");
  check_aligned(x, 16, "x");
  dispatch<double, 0>(A, A.v64.p, x, z, y, alpha, beta, nullptr, nullptr, st, active);
}

void spmv(const Matrix& A, float alpha, const float* x, float beta, const float* z, float* y, cudaStream_t st,
          const int* active) {
  require(A.single, "FP32 SpMV on an FP64 matrix");
  check_aligned(x, 16, "x");
  if (A.half) return dispatch_half<0>(A, x, z, y, alpha, beta, nullptr, st, active);
  dispatch<float, 0>(A, A.v32.p, x, z, y, alpha, beta, nullptr, nullptr, st, active);
}

namespace {
template <typename T>
void bj_update_impl(const Matrix& A, const T* vals, const T* dinv, T omega, const T* x, const T* b, T* xo,
                    cudaStream_t st, const int* active) {
  check_aligned(x, 16, "x");
  dispatch<T, 1>(A, vals, x, b, xo, omega, T(0), dinv, A.doff.p, st, active);
}
}  // namespace

namespace {
template <typename T>
void gs_rows_impl(const Matrix& A, const T* vals, const T* dinv, T omega, const int32_t* rows, int64_t nrows,
                  const T* b, T* x, cudaStream_t st) {
  require(specialised(A) && !A.half, "block Gauss-Seidel needs uniform blocks of 4, 6, 10 or 20 (FP32/FP64 values)",
          BSGPU_ERR_UNSUPPORTED);
  if (nrows == 0) return;
  constexpr int VW = sizeof(T) == 8 ? 2 : 4;
#define BSGPU_GS(NP, VV)                                                                                     \
  spmv_uniform_kernel<T, NP, VV, 2><<<(unsigned)((nrows + 256 / NP - 1) / (256 / NP)), (256 / NP) * NP, 0, st>>>( \
      A.rp.p, A.ci.p, vals, x, b, x, omega, T(0), nrows, dinv, nullptr, rows)
  switch (A.Np) {
    case 20: BSGPU_GS(20, VW); break;
    case 4: BSGPU_GS(4, VW); break;
    case 10: BSGPU_GS(10, 2); break;
    case 6: BSGPU_GS(6, 2); break;
  }
#undef BSGPU_GS
  BSGPU_CHECK_LAUNCH();
}
}  // namespace

void gs_update_rows(const Matrix& A, const double* dinv, double omega, const int32_t* rows, int64_t nrows,
                    const double* b, double* x, cudaStream_t st) {
  require(!A.single, "precision mismatch");
  gs_rows_impl<double>(A, A.v64.p, dinv, omega, rows, nrows, b, x, st);
}

namespace {
template <typename T>
void unit_rows_impl(const Matrix& A, const T* vals, const int32_t* rows, int64_t nrows, const T* b, T* x,
                    cudaStream_t st) {
  require(specialised(A) && !A.half, "unit-diagonal row update needs uniform blocks of 4, 6, 10 or 20 (FP32/FP64 values)",
          BSGPU_ERR_UNSUPPORTED);
  if (nrows == 0) return;
  constexpr int VW = sizeof(T) == 8 ? 2 : 4;
#define BSGPU_UNIT(NP, VV)                                                                                   \
  spmv_uniform_kernel<T, NP, VV, 3><<<(unsigned)((nrows + 256 / NP - 1) / (256 / NP)), (256 / NP) * NP, 0, st>>>( \
      A.rp.p, A.ci.p, vals, x, b, x, T(1), T(0), nrows, nullptr, nullptr, rows)
  switch (A.Np) {
    case 20: BSGPU_UNIT(20, VW); break;
    case 4: BSGPU_UNIT(4, VW); break;
    case 10: BSGPU_UNIT(10, 2); break;
    case 6: BSGPU_UNIT(6, 2); break;
  }
#undef BSGPU_UNIT
  BSGPU_CHECK_LAUNCH();
}
}  // namespace

void unit_update_rows(const Matrix& A, const int32_t* rows, int64_t nrows, const double* b, double* x,
                      cudaStream_t st) {
  require(!A.single, "precision mismatch");
  unit_rows_impl<double>(A, A.v64.p, rows, nrows, b, x, st);
}
void unit_update_rows(const Matrix& A, const int32_t* rows, int64_t nrows, const float* b, float* x,
                      cudaStream_t st) {
  require(A.single, "precision mismatch");
  unit_rows_impl<float>(A, A.v32.p, rows, nrows, b, x, st);
}
void gs_update_rows(const Matrix& A, const float* dinv, float omega, const int32_t* rows, int64_t nrows,
                    const float* b, float* x, cudaStream_t st) {
  require(A.single, "precision mismatch");
  gs_rows_impl<float>(A, A.v32.p, dinv, omega, rows, nrows, b, x, st);
}

std::vector<std::vector<int32_t>> greedy_colouring(const Matrix& A) {
  std::vector<int32_t> col(A.nb, -1);
  int ncol = 0;
  std::vector<char> used;
  for (int64_t i = 0; i < A.nb; ++i) {
    used.assign(ncol + 1, 0);
    for (int64_t k = A.h_rp[i]; k < A.h_rp[i + 1]; ++k) {
      const int32_t j = A.h_ci[k];
      if (j != i && col[j] >= 0) used[col[j]] = 1;
    }
    int c = 0;
    while (c < ncol && used[c]) ++c;
    col[i] = c;
    if (c == ncol) ++ncol;
  }
  std::vector<std::vector<int32_t>> lists(ncol);
  for (int64_t i = 0; i < A.nb; ++i) lists[col[i]].push_back((int32_t)i);
  return lists;
}

void bj_update(const Matrix& A, const double* dinv, double omega, const double* x, const double* b, double* xo,
               cudaStream_t st, const int* active) {
  require(!A.single, "precision mismatch");
  bj_update_impl<double>(A, A.v64.p, dinv, omega, x, b, xo, st, active);
}
void bj_update(const Matrix& A, const float* dinv, float omega, const float* x, const float* b, float* xo,
               cudaStream_t st, const int* active) {
  require(A.single, "precision mismatch");
  if (A.half) {
    check_aligned(x, 16, "x");
    return dispatch_half<1>(A, x, b, xo, omega, 0.0f, dinv, st, active);
  }
  bj_update_impl<float>(A, A.v32.p, dinv, omega, x, b, xo, st, active);
}

namespace {
template <typename T>
void blockdiag_impl(const Matrix& A, const T* dinv, T alpha, const T* b, T* y, cudaStream_t st, const int* active) {
  if (A.N == 0) return;
  const int grid = (int)std::min<int64_t>((A.N + 255) / 256, (int64_t)num_sms() * 16);
  blockdiag_kernel<T><<<grid, 256, 0, st>>>(A.len.p, A.i0.p, A.row2blk.p, A.doff.p, dinv, alpha, b, y, A.N,
                                            A.uniform ? A.Np : 0, active);
  BSGPU_CHECK_LAUNCH();
}
}  // namespace

void blockdiag_apply(const Matrix& A, const double* dinv, double omega, const double* b, double* y, cudaStream_t st,
                     const int* active) {
  blockdiag_impl<double>(A, dinv, omega, b, y, st, active);
}
void blockdiag_apply(const Matrix& A, const float* dinv, float omega, const float* b, float* y, cudaStream_t st,
                     const int* active) {
  blockdiag_impl<float>(A, dinv, omega, b, y, st, active);
}

// ---------------------------------------------------------------------------------------------------------------
// autotuner of the launch shape
// ---------------------------------------------------------------------------------------------------------------
namespace {

std::mutex g_tune_mutex;
std::map<std::string, int> g_tune_cache;
std::vector<std::string> g_tune_log;

template <typename T>
float time_launches(const Matrix& A, int mode, const T* dinv, const T* x, const T* b, T* y, cudaStream_t st, int reps) {
  cudaEvent_t e0, e1;
  BSGPU_CUDA(cudaEventCreate(&e0));
  BSGPU_CUDA(cudaEventCreate(&e1));
  const T* vals = A.single ? (const T*)(const void*)A.v32.p : (const T*)(const void*)A.v64.p;
  auto one = [&]() {
    if constexpr (sizeof(T) == 4) {
      if (A.half) {
        if (mode == 0)
          dispatch_half<0>(A, x, nullptr, y, 1.0f, 0.0f, nullptr, st, nullptr);
        else
          dispatch_half<1>(A, x, b, y, 1.0f, 0.0f, dinv, st, nullptr);
        return;
      }
    }
    if (mode == 0)
      dispatch<T, 0>(A, vals, x, nullptr, y, T(1), T(0), nullptr, nullptr, st, nullptr);
    else
      dispatch<T, 1>(A, vals, x, b, y, T(1), T(0), dinv, A.doff.p, st, nullptr);
  };
  for (int i = 0; i < 2; ++i) one();
  BSGPU_CUDA(cudaEventRecord(e0, st));
  for (int i = 0; i < reps; ++i) one();
  BSGPU_CUDA(cudaEventRecord(e1, st));
  BSGPU_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  BSGPU_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return ms / reps;
}

template <typename T>
void autotune_impl(const Matrix& A, int mode, const T* dinv, cudaStream_t st) {
  const bool tunable = A.typed || specialised(A) || A.half;
  if (!tunable || A.tuned[mode] || A.N == 0) return;
  int dev = 0;
  BSGPU_CUDA(cudaGetDevice(&dev));
  std::ostringstream key;
  key << dev << (A.typed ? ":typed:" : ":uniform:") << (A.half ? "f16" : A.single ? "f32" : "f64") << ":Np" << A.Np
      << ":V" << A.V
      << ":mode" << mode << ":nb" << A.nb << ":nnzb" << A.nnzb << ":N" << A.N;
  {
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune_cache.find(key.str());
    if (it != g_tune_cache.end()) {
      A.cta[mode] = it->second;
      A.tuned[mode] = true;
      return;
    }
  }
  // launches costing about 2 ms in total per candidate, at least 5
  const double bytes = (double)A.value_bytes() + 3.0 * (double)A.N * sizeof(T);
  const int reps = (int)std::max(5.0, std::min(200.0, 2e-3 / (bytes / 5e12)));
  DBuf<T> x(A.N), b(A.N), y(A.N);
  BSGPU_CUDA(cudaMemsetAsync(x.p, 0, A.N * sizeof(T), st));
  BSGPU_CUDA(cudaMemsetAsync(b.p, 0, A.N * sizeof(T), st));
  const int cands[3] = {256, 128, 64};
  const int saved = A.cta[mode];
  std::ostringstream rec;
  rec << "{\"matrix\": \"" << key.str() << "\", \"times_ms\": {";
  int best = 256;
  float tbest = 1e30f;
  for (int ci = 0; ci < 3; ++ci) {
    const int c = cands[ci];
    if (!A.typed && c < A.Np) continue;
    if (A.typed && c < 2 * A.Np) continue;
    A.cta[mode] = c;
    const float t = time_launches<T>(A, mode, dinv, x.p, b.p, y.p, st, reps);
    rec << (ci ? ", " : "") << "\"" << c << "\": " << t;
    if (t < tbest) {
      tbest = t;
      best = c;
    }
  }
  (void)saved;
  A.cta[mode] = best;
  A.tuned[mode] = true;
  rec << "}, \"threads_per_cta\": " << best << ", \"reps\": " << reps << "}";
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  g_tune_cache[key.str()] = best;
  g_tune_log.push_back(rec.str());
}

}  // namespace

void autotune(const Matrix& A, int mode, const void* dinv, cudaStream_t st) {
  require(mode == 0 || mode == 1, "autotune: mode 0 (product) or 1 (block-Jacobi update)");
  require(mode == 0 || dinv != nullptr, "autotune: the block-Jacobi update needs the factors");
  cudaStreamCaptureStatus cs;
  BSGPU_CUDA(cudaStreamIsCapturing(st, &cs));
  require(cs == cudaStreamCaptureStatusNone, "autotune inside a graph capture");
  if (A.single)
    autotune_impl<float>(A, mode, (const float*)dinv, st);
  else
    autotune_impl<double>(A, mode, (const double*)dinv, st);
}

std::string autotune_report() {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  std::string out = "[";
  for (size_t i = 0; i < g_tune_log.size(); ++i) out += (i ? ", " : "") + g_tune_log[i];
  return out + "]";
}

}  // namespace bsgpu
