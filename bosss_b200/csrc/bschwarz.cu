// Additive Schwarz with multi-cell blocks (see bschwarz.cuh).
#include <algorithm>
#include <numeric>

#include "bschwarz.cuh"

namespace bsgpu {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ int64_t find_col(const int64_t* rp, const int32_t* ci, int64_t row, int32_t col) {
  int64_t lo = rp[row], hi = rp[row + 1];
  while (lo < hi) {
    const int64_t mid = (lo + hi) / 2;
    if (ci[mid] < col)
      lo = mid + 1;
    else
      hi = mid;
  }
  return (lo < rp[row + 1] && ci[lo] == col) ? lo : -1;
}

// One CTA per block: the dense block (rows and columns = the block's DOFs, cells in ascending order) is gathered
// from the block-sparse matrix into its slot of W and inverted in place by Gauss-Jordan with partial pivoting
// (FP64); the FP32 copy is written to w32 when given.
__global__ void __launch_bounds__(kThreads) factor_kernel(
    const int64_t* __restrict__ rp, const int32_t* __restrict__ ci, const int32_t* __restrict__ len,
    const int64_t* __restrict__ boff, const double* __restrict__ vals, int V, const int64_t* __restrict__ cell_ptr,
    const int32_t* __restrict__ cells, const int64_t* __restrict__ dof_ptr, const int64_t* __restrict__ inv_off,
    double* __restrict__ W, float* __restrict__ w32, int* __restrict__ err, int64_t nblk) {
  __shared__ int loff[kMaxSchwarzDofs + 1];
  __shared__ int perm[kMaxSchwarzDofs];
  __shared__ double prow[kMaxSchwarzDofs];
  __shared__ double pcol[kMaxSchwarzDofs];
  __shared__ double wmax[kThreads / 32];
  __shared__ int wrow[kThreads / 32];
  __shared__ int piv, bad;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t b = blockIdx.x; b < nblk; b += gridDim.x) {
    const int64_t c0 = cell_ptr[b];
    const int nc = (int)(cell_ptr[b + 1] - c0);
    const int n = (int)(dof_ptr[b + 1] - dof_ptr[b]);
    double* M = W + inv_off[b];
    if (threadIdx.x == 0) {
      int acc = 0;
      for (int p = 0; p < nc; ++p) {
        loff[p] = acc;
        acc += len[cells[c0 + p]];
      }
      loff[nc] = acc;
      bad = 0;
    }
    for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += blockDim.x) M[e] = 0.0;
    __syncthreads();
    for (int pair = threadIdx.x; pair < nc * nc; pair += blockDim.x) {
      const int p = pair / nc, q = pair - p * nc;
      const int32_t cp = cells[c0 + p], cq = cells[c0 + q];
      const int64_t k = find_col(rp, ci, cp, cq);
      if (k < 0) continue;
      const int I = len[cp], J = len[cq];
      for (int r = 0; r < I; ++r)
        for (int c = 0; c < J; ++c)
          M[(int64_t)(loff[p] + r) * n + loff[q] + c] = vals[boff[k] + (int64_t)(c / V) * I * V + r * V + (c % V)];
    }
    __syncthreads();
    for (int p = 0; p < n; ++p) {
      // pivot: largest |M[r][p]|, r >= p
      double best = -1.0;
      int brow = p;
      for (int r = p + threadIdx.x; r < n; r += blockDim.x) {
        const double v = fabs(M[(int64_t)r * n + p]);
        if (v > best) {
          best = v;
          brow = r;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_down_sync(0xffffffffu, best, o);
        const int orow = __shfl_down_sync(0xffffffffu, brow, o);
        if (ov > best || (ov == best && orow < brow)) {
          best = ov;
          brow = orow;
        }
      }
      if (lane == 0) {
        wmax[warp] = best;
        wrow[warp] = brow;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        double bv = wmax[0];
        int br = wrow[0];
        for (int w = 1; w < kThreads / 32; ++w)
          if (wmax[w] > bv || (wmax[w] == bv && wrow[w] < br)) {
            bv = wmax[w];
            br = wrow[w];
          }
        piv = br;
        perm[p] = br;
        if (!(bv > 0.0) || !isfinite(bv)) {
          bad = 1;
          atomicCAS(err, 0, (int)(b + 1 < 0x7fffffff ? b + 1 : 0x7fffffff));
        }
      }
      __syncthreads();
      if (bad) break;
      if (piv != p)
        for (int c = threadIdx.x; c < n; c += blockDim.x) {
          const double t = M[(int64_t)p * n + c];
          M[(int64_t)p * n + c] = M[(int64_t)piv * n + c];
          M[(int64_t)piv * n + c] = t;
        }
      __syncthreads();
      const double inv = 1.0 / M[(int64_t)p * n + p];
      for (int t = threadIdx.x; t < n; t += blockDim.x) {
        prow[t] = (t == p) ? inv : M[(int64_t)p * n + t] * inv;
        pcol[t] = M[(int64_t)t * n + p];
      }
      __syncthreads();
      for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += blockDim.x) {
        const int r = (int)(e / n), c = (int)(e - (int64_t)r * n);
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
      for (int p = n - 1; p >= 0; --p) {
        const int q = perm[p];
        if (q != p)
          for (int r = threadIdx.x; r < n; r += blockDim.x) {
            const double t = M[(int64_t)r * n + p];
            M[(int64_t)r * n + p] = M[(int64_t)r * n + q];
            M[(int64_t)r * n + q] = t;
          }
        __syncthreads();
      }
      if (w32)
        for (int64_t e = threadIdx.x; e < (int64_t)n * n; e += blockDim.x) w32[inv_off[b] + e] = (float)M[e];
    }
    __syncthreads();
  }
}

// One CTA per block: the residual's block entries into shared memory, one warp per row of the inverse (lanes along
// the row, coalesced), the row's value added to x atomically (blocks overlap).
template <typename T, typename TI>
__global__ void __launch_bounds__(kThreads) apply_kernel(const int64_t* __restrict__ dof_ptr,
                                                         const int32_t* __restrict__ dofs,
                                                         const int64_t* __restrict__ inv_off,
                                                         const TI* __restrict__ inv, const T* __restrict__ r,
                                                         T* __restrict__ x, int64_t nblk) {
  __shared__ T rb[kMaxSchwarzDofs];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t b = blockIdx.x; b < nblk; b += gridDim.x) {
    const int64_t d0 = dof_ptr[b];
    const int n = (int)(dof_ptr[b + 1] - d0);
    __syncthreads();
    for (int q = threadIdx.x; q < n; q += blockDim.x) rb[q] = r[dofs[d0 + q]];
    __syncthreads();
    const TI* Mi = inv + inv_off[b];
    for (int p = warp; p < n; p += kThreads / 32) {
      double acc = 0.0;
      for (int q = lane; q < n; q += 32) acc = fma((double)Mi[(int64_t)p * n + q], (double)rb[q], acc);
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
      if (lane == 0) atomicAdd(x + dofs[d0 + p], (T)acc);
    }
  }
}

template <typename T>
__global__ void scale_kernel(const T* __restrict__ s, T* __restrict__ x, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] *= s[i];
}

int blocks_grid(int64_t nblk) { return (int)std::max<int64_t>(1, std::min<int64_t>(nblk, (int64_t)num_sms() * 8)); }

template <typename T>
void add_impl(const SchwarzBlocks& S, const T* r, T* x, cudaStream_t st) {
  if (S.nblk == 0) return;
  if constexpr (sizeof(T) == 4) {
    if (S.inv32.p) {
      apply_kernel<T, float><<<blocks_grid(S.nblk), kThreads, 0, st>>>(S.dof_ptr.p, S.dofs.p, S.inv_off.p,
                                                                        S.inv32.p, r, x, S.nblk);
      BSGPU_CHECK_LAUNCH();
      return;
    }
  }
  require(S.inv64.p != nullptr, "Schwarz blocks: FP64 inverses missing");
  apply_kernel<T, double><<<blocks_grid(S.nblk), kThreads, 0, st>>>(S.dof_ptr.p, S.dofs.p, S.inv_off.p, S.inv64.p, r,
                                                                     x, S.nblk);
  BSGPU_CHECK_LAUNCH();
}

}  // namespace

std::vector<std::vector<int32_t>> schwarz_partition(const Matrix& A, int64_t parts) {
  require(parts >= 1, "Schwarz: the number of blocks must be at least 1");
  const int64_t nb = A.nb;
  const int64_t target = std::max<int64_t>(1, (nb + parts - 1) / parts);
  std::vector<int32_t> part(nb, -1);
  std::vector<std::vector<int32_t>> blocks;
  std::vector<int32_t> queue;
  for (int64_t seed = 0; seed < nb; ++seed) {
    if (part[seed] >= 0) continue;
    const int32_t id = (int32_t)blocks.size();
    queue.assign(1, (int32_t)seed);
    part[seed] = id;
    size_t head = 0;
    while (head < queue.size() && (int64_t)queue.size() < target) {
      const int32_t c = queue[head++];
      for (int64_t k = A.h_rp[c]; k < A.h_rp[c + 1] && (int64_t)queue.size() < target; ++k) {
        const int32_t j = A.h_ci[k];
        if (j == c || part[j] >= 0) continue;
        part[j] = id;
        queue.push_back(j);
      }
    }
    std::sort(queue.begin(), queue.end());
    blocks.push_back(queue);
  }
  return blocks;
}

void schwarz_extend(const Matrix& A, std::vector<std::vector<int32_t>>& blocks, int overlap) {
  require(overlap >= 0 && overlap <= 2, "Schwarz: overlap must be 0, 1 or 2 (Schwarz.cs:501-516)");
  std::vector<char> marker(A.nb, 0);
  for (auto& bl : blocks) {
    for (int32_t c : bl) marker[c] = 1;
    for (int s = 0; s < overlap; ++s) {
      const size_t members = bl.size();
      for (size_t m = 0; m < members; ++m) {
        const int32_t c = bl[m];
        for (int64_t k = A.h_rp[c]; k < A.h_rp[c + 1]; ++k) {
          const int32_t j = A.h_ci[k];
          if (!marker[j]) {
            marker[j] = 1;
            bl.push_back(j);
          }
        }
      }
    }
    std::sort(bl.begin(), bl.end());
    for (int32_t c : bl) marker[c] = 0;
  }
}

SchwarzBlocks* schwarz_blocks_setup(const Matrix& A64, const std::vector<std::vector<int32_t>>& blocks, bool scaling,
                                    bool single, int* err, cudaStream_t st) {
  require(!A64.single, "Schwarz blocks are factored from the FP64 matrix");
  require(A64.N < (int64_t(1) << 31), "Schwarz blocks: too many unknowns for 32-bit DOF lists", BSGPU_ERR_UNSUPPORTED);
  auto S = std::make_unique<SchwarzBlocks>();
  S->nblk = (int64_t)blocks.size();
  S->N = A64.N;
  std::vector<int64_t> cell_ptr(1, 0), dof_ptr(1, 0), inv_off(1, 0);
  std::vector<int32_t> cells, dofs;
  std::vector<int32_t> count(A64.N, 0);
  for (const auto& bl : blocks) {
    int64_t n = 0;
    for (int32_t c : bl) {
      cells.push_back(c);
      for (int64_t g = A64.h_i0[c]; g < A64.h_i0[c + 1]; ++g) {
        dofs.push_back((int32_t)g);
        count[g]++;
      }
      n += A64.h_len[c];
    }
    require(n <= kMaxSchwarzDofs, "Schwarz: a block has " + std::to_string(n) + " unknowns, more than " +
                                      std::to_string(kMaxSchwarzDofs) + " (use more blocks or less overlap)",
            BSGPU_ERR_UNSUPPORTED);
    S->max_n = std::max<int>(S->max_n, (int)n);
    cell_ptr.push_back((int64_t)cells.size());
    dof_ptr.push_back((int64_t)dofs.size());
    inv_off.push_back(inv_off.back() + n * n);
  }
  S->total = inv_off.back();
  DBuf<int64_t> d_cell_ptr(cell_ptr.size());
  DBuf<int32_t> d_cells(std::max<size_t>(cells.size(), 1));
  S->dof_ptr.alloc(dof_ptr.size());
  S->dofs.alloc(std::max<size_t>(dofs.size(), 1));
  S->inv_off.alloc(inv_off.size());
  BSGPU_CUDA(cudaMemcpy(d_cell_ptr.p, cell_ptr.data(), cell_ptr.size() * 8, cudaMemcpyHostToDevice));
  if (!cells.empty()) BSGPU_CUDA(cudaMemcpy(d_cells.p, cells.data(), cells.size() * 4, cudaMemcpyHostToDevice));
  BSGPU_CUDA(cudaMemcpy(S->dof_ptr.p, dof_ptr.data(), dof_ptr.size() * 8, cudaMemcpyHostToDevice));
  if (!dofs.empty()) BSGPU_CUDA(cudaMemcpy(S->dofs.p, dofs.data(), dofs.size() * 4, cudaMemcpyHostToDevice));
  BSGPU_CUDA(cudaMemcpy(S->inv_off.p, inv_off.data(), inv_off.size() * 8, cudaMemcpyHostToDevice));
  S->inv64.alloc(std::max<int64_t>(S->total, 1));
  if (single) S->inv32.alloc(std::max<int64_t>(S->total, 1));
  if (S->nblk)
    factor_kernel<<<blocks_grid(S->nblk), kThreads, 0, st>>>(A64.rp.p, A64.ci.p, A64.len.p, A64.boff.p, A64.v64.p,
                                                             A64.V, d_cell_ptr.p, d_cells.p, S->dof_ptr.p,
                                                             S->inv_off.p, S->inv64.p, single ? S->inv32.p : nullptr,
                                                             err, S->nblk);
  BSGPU_CHECK_LAUNCH();
  BSGPU_CUDA(cudaStreamSynchronize(st));
  if (single) S->inv64.release();
  if (scaling) {
    std::vector<double> sc(A64.N);
    for (int64_t g = 0; g < A64.N; ++g) sc[g] = count[g] > 0 ? 1.0 / count[g] : 1.0;
    if (single) {
      std::vector<float> s32(sc.begin(), sc.end());
      S->scale32.alloc(std::max<int64_t>(A64.N, 1));
      if (A64.N) BSGPU_CUDA(cudaMemcpy(S->scale32.p, s32.data(), A64.N * 4, cudaMemcpyHostToDevice));
    } else {
      S->scale64.alloc(std::max<int64_t>(A64.N, 1));
      if (A64.N) BSGPU_CUDA(cudaMemcpy(S->scale64.p, sc.data(), A64.N * 8, cudaMemcpyHostToDevice));
    }
  }
  return S.release();
}

void schwarz_blocks_add(const SchwarzBlocks& S, const double* r, double* x, cudaStream_t st) {
  add_impl<double>(S, r, x, st);
}
void schwarz_blocks_add(const SchwarzBlocks& S, const float* r, float* x, cudaStream_t st) {
  add_impl<float>(S, r, x, st);
}
void schwarz_blocks_scale(const SchwarzBlocks& S, double* x, cudaStream_t st) {
  require(S.scale64.p != nullptr, "Schwarz blocks: no FP64 scaling");
  scale_kernel<double><<<blocks_grid((S.N + kThreads - 1) / kThreads), kThreads, 0, st>>>(S.scale64.p, x, S.N);
  BSGPU_CHECK_LAUNCH();
}
void schwarz_blocks_scale(const SchwarzBlocks& S, float* x, cudaStream_t st) {
  require(S.scale32.p != nullptr, "Schwarz blocks: no FP32 scaling");
  scale_kernel<float><<<blocks_grid((S.N + kThreads - 1) / kThreads), kThreads, 0, st>>>(S.scale32.p, x, S.N);
  BSGPU_CHECK_LAUNCH();
}

}  // namespace bsgpu
