// Learned preconditioner stage: a one-hop message-passing MLP over the cell graph (see learned.cu).
#pragma once
#include "blas1.cuh"
#include "matrix.cuh"

namespace bsgpu {

struct LearnedNet {
  int Np = 0;        // modes per cell (input and output block)
  int nfaces = 6;    // neighbours per cell in the table
  int nextra = 0;    // extra per-cell features (e.g. log k of the cell and its neighbours)
  int F = 0, Fp = 0; // input width and its padding to 16
  int H = 64;        // hidden width
  int Op = 0;        // output width padded to 16
  int64_t ncells = 0;
  DBuf<int32_t> nbr;      // [ncells x nfaces], -1 = none
  DBuf<float> extra;      // [ncells x nextra]
  // weights: bf16 copies used by the kernels, FP32 master copies and Adam moments for training
  DBuf<uint16_t> w1, w2, w3;                 // [Fp x H], [H x H], [H x Op], row-major (k, n)
  DBuf<float> m1, m2, m3, g1, g2, g3, a1, a2, a3, v1, v2, v3;
  DBuf<float> act;                           // training activations [ncells x 2H]
  DBuf<int> err;                             // set when a bounded wait of the forward kernel gave up
  int adam_t = 0;
  bool trained = false;
  void init(int Np_, int64_t ncells_, int nfaces_, int nextra_, const int32_t* nbr_host, const float* extra_host,
            uint64_t seed);
  size_t nweights() const { return (size_t)Fp * H + (size_t)H * H + (size_t)H * Op; }
};

// z = NN(r) for every cell (r, z: length ncells*Np, FP64 or FP32).  `scale`: device scalar; inputs are divided
// by it and outputs multiplied (bf16 range safety; the network is positively homogeneous).
void learned_apply(const LearnedNet& net, const double* r, double* z, const double* scale, cudaStream_t st);
void learned_apply(const LearnedNet& net, const float* r, float* z, const double* scale, cudaStream_t st);

// Raises BSGPU_ERR_TIMEOUT (and clears the flag) when a forward launch reported a wait that gave up.
void learned_check(const LearnedNet& net, cudaStream_t st);
// scale = |r| / sqrt(n) from a device norm (input normalisation of the stage)
void learned_scale(const double* nrm, double* scale, int64_t n, cudaStream_t st);

// One training step on the energy-norm loss (z^T A z - 2 z^T r) / |r|^2, z = NN(r): forward over all cells
// (activations kept), gradient g = 2 (A z - r)/|r|^2 through one SpMV, backward over the cells and an Adam step.
// Returns the loss through a device scalar (loss_out).
void learned_train_step(LearnedNet& net, const Matrix& A, const double* r, double* z, double* Az, double* g,
                        ReduceScratch& red, double* scal, double lr, cudaStream_t st);
// The same loss and its gradient without the update: the gradient is accumulated into net.g1..g3 (which must be
// zero), the loss terms into scal[0..4] as above.
void learned_gradient(LearnedNet& net, const Matrix& A, const double* r, double* z, double* Az, double* g,
                      ReduceScratch& red, double* scal, cudaStream_t st);
// Host copies of the weights the kernels use (BF16, widened exactly to float; padded shapes Fp x H, H x H, H x Op,
// row-major), and replacement of the weights (FP32 master copies = the given values, BF16 copies rounded to
// nearest even; Adam state reset).
void learned_get_weights(const LearnedNet& net, float* w1, float* w2, float* w3);
void learned_set_weights(LearnedNet& net, const float* w1, const float* w2, const float* w3);
// Copies the accumulated gradient to the host and zeroes it.
void learned_take_gradient(LearnedNet& net, float* g1, float* g2, float* g3, cudaStream_t st);

}  // namespace bsgpu
