// Additive Schwarz with multi-cell blocks (Schwarz.cs:56): the reference partitions the cells into
// NoOfPartsOnCurrentProcess blocks with METIS (METISBlockingStrategy, Schwarz.cs:190-320), grows each block by
// `Overlap` layers of face neighbours (:690-735), solves every block directly and adds the block solutions
// (:996-1147), optionally scaled by one over the number of blocks that cover a DOF (EnableOverlapScaling,
// :790-815, :1093-1104).
//
// Here the partition is a deterministic greedy breadth-first aggregation of the cell graph to blocks of
// ceil(nb / parts) cells (a stand-in for METIS's k-way partition: connected, balanced blocks), the blocks are dense
// (at most kMaxSchwarzDofs unknowns after the overlap growth), their inverses are computed in FP64 on the GPU (one
// CTA per block, Gauss-Jordan with partial pivoting in global memory) and stored in FP64 or FP32, and one Schwarz
// application is   x <- x + sum_b R_b^T A_b^{-1} R_b (b - A x),   x <- x * s  (scaling),   one CTA per block
// (gather, dense product by warps, atomic scatter-add).
#pragma once
#include "matrix.cuh"

namespace bsgpu {

constexpr int kMaxSchwarzDofs = 1024;

// cell lists of the blocks (ascending cell numbers within a block)
std::vector<std::vector<int32_t>> schwarz_partition(const Matrix& A, int64_t parts);
// grows every block by `overlap` layers of neighbours in the block graph, as Schwarz.cs:690-735 (each sweep visits
// the members present at its start), then sorts it
void schwarz_extend(const Matrix& A, std::vector<std::vector<int32_t>>& blocks, int overlap);

struct SchwarzBlocks {
  int64_t nblk = 0, N = 0, total = 0;
  int max_n = 0;
  DBuf<int64_t> dof_ptr;   // [nblk + 1] offsets into dofs
  DBuf<int32_t> dofs;      // DOFs of every block (the cells' DOFs in ascending cell order)
  DBuf<int64_t> inv_off;   // [nblk + 1] offsets of the row-major n_b x n_b inverses
  DBuf<double> inv64;
  DBuf<float> inv32;
  DBuf<double> scale64;    // 1 / multiplicity per DOF (overlap scaling), or empty
  DBuf<float> scale32;
};

// dense inverses of the blocks of A64 (FP64 arithmetic; kept as FP32 when single); err <- first failing block + 1
SchwarzBlocks* schwarz_blocks_setup(const Matrix& A64, const std::vector<std::vector<int32_t>>& blocks, bool scaling,
                                    bool single, int* err, cudaStream_t st);
// x += sum_b R_b^T A_b^{-1} R_b r
void schwarz_blocks_add(const SchwarzBlocks& S, const double* r, double* x, cudaStream_t st);
void schwarz_blocks_add(const SchwarzBlocks& S, const float* r, float* x, cudaStream_t st);
// x *= scale (overlap scaling)
void schwarz_blocks_scale(const SchwarzBlocks& S, double* x, cudaStream_t st);
void schwarz_blocks_scale(const SchwarzBlocks& S, float* x, cudaStream_t st);

}  // namespace bsgpu
