// Batched dense block operations: SymmInv change of basis, diagonal-block inversion, block triangular solves.
#pragma once
#include "matrix.cuh"

namespace bsgpu {

// L_i for every block row from SymmInv of the diagonal block (MultigridOperator_ChangeOfBasis.cs:624-760).
// L: per block row I x I row-major at offsets diag_offsets(A).  Returns 0 or the first failing block + 1.
void symminv_batched(const Matrix& A, double* L, int* err, cudaStream_t st);
// Aout_ij = L_i * A_ij * L_j^T for every block (Aout has A's structure, FP64).
void change_of_basis_apply(const Matrix& A, const double* L, Matrix& Aout, cudaStream_t st);
// Inverses of the diagonal blocks (BlockJacobi.cs:125-146 InvertInPlace), stored column-major per block at
// diag_offsets(A); computed in FP64 and written as FP64 (D64) and/or FP32 (D32).
void invert_diag_blocks(const Matrix& A, double* D64, float* D32, int* err, cudaStream_t st);
// Restricted additive Schwarz factors, one overlapping block per cell (the cell and the cells of its block
// row): M (A's structure, FP64 or FP32 values) gets the centre-cell rows of each block inverse
// (Schwarz.cs:623-840 block set-up; blocks here are cell patches with overlap 1).  One launch for all blocks,
// whatever their sizes.
void schwarz_factor(const Matrix& A, Matrix& M, int* err, cudaStream_t st);
// Block ILU(0) of a two-colour block graph, rows ordered colour 0 first (CellILU.cs:1229-1330 on the reordered
// matrix): M (FP64, A's structure) <- A with L_br = A_br A_rr^{-1} and U_bb = A_bb - sum_r L_br A_rb on the
// colour-1 rows `rows1`.  dinv: inverses of A's diagonal blocks (invert_diag_blocks layout).
void ilu0_two_colour(const Matrix& A, const double* dinv, const int32_t* rows1, int64_t n1, Matrix& M, int* err,
                     cudaStream_t st);
// Block ILU(0) in the natural block-row order (CellILU.cs:1229-1330), wavefront by wavefront: rows[level_ptr[l] ..
// level_ptr[l+1]) are the block rows whose lower neighbours all lie in earlier wavefronts.  M (FP64, A's
// structure) <- the factors (unit-lower L below the diagonal, U on and above it); uinv (and u32 if not null) <-
// U_ii^{-1} per block row, column-major at diag_offsets(A).
void ilu0_levels(const Matrix& A, const int32_t* rows, const std::vector<int64_t>& level_ptr, Matrix& M,
                 double* uinv, float* u32, int* err, cudaStream_t st);
// y_i = L_i^{-T} x_i per block (initial-guess transform with a lower-triangular L, row-major).
void block_trsv_lt(const Matrix& A, const double* L, const double* x, double* y, cudaStream_t st);

}  // namespace bsgpu
