// Learned preconditioner stage (no counterpart in the reference; it plugs into FlexGMRES's list of
// preconditioners, FlexGMRES.cs:50-56,196-199).
//
// Per cell c the network sees its own residual block, the blocks of its face neighbours (zero where a face has
// none) and optional per-cell features, and returns a correction block:
//     z_c = W3^T relu(W2^T relu(W1^T f_c)),   f_c = [r_c, r_n1, ..., r_n6, extra_c]
// No biases: with ReLU the map is positively homogeneous, z(a r) = a z(r) for a > 0, so it commutes with the
// arbitrary scaling of Krylov vectors.  Weights are BF16 (FP32 master copies for training), products accumulate in
// FP32 on the tensor cores (wmma bf16 16x16x16 tiles), one CTA per tile of 64 cells with all weights in shared
// memory.  Training minimises the energy norm of the error left after the correction,
//     |e - z|_A^2 = z^T A z - 2 z^T r + e^T A e,   A e = r,
// i.e. it fits a local approximate inverse of the operator, with one SpMV per step for A z.
#include <cuda_bf16.h>
#include <mma.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>

#include "learned.cuh"

namespace bsgpu {

namespace {

using namespace nvcuda;
constexpr int kTile = 64;    // cells per CTA tile (forward)
constexpr int kBTile = 32;   // cells per CTA tile (backward)

__device__ __forceinline__ __nv_bfloat16 bf(float x) { return __float2bfloat16(x); }

template <typename TV>
__device__ __forceinline__ float feature(const TV* __restrict__ r, const int32_t* __restrict__ nbr,
                                         const float* __restrict__ extra, int64_t c, int f, int Np, int nfaces,
                                         int nextra, float inv_scale) {
  const int block = f / Np;
  if (block <= nfaces) {
    const int m = f - block * Np;
    int64_t cell = c;
    if (block > 0) {
      const int32_t n = nbr[c * nfaces + block - 1];
      if (n < 0) return 0.0f;
      cell = n;
    }
    return (float)r[cell * Np + m] * inv_scale;
  }
  const int e = f - (nfaces + 1) * Np;
  return e < nextra ? extra[c * nextra + e] : 0.0f;
}

struct FwdArgs {
  const int32_t* nbr;
  const float* extra;
  const __nv_bfloat16* w1;
  const __nv_bfloat16* w2;
  const __nv_bfloat16* w3;
  float* act;  // training: [ncells x 2H] post-ReLU activations, or nullptr
  const double* scale;
  int64_t ncells;
  int Np, nfaces, nextra, F, Fp, H, Op;
};

// C[64 x N] = A[64 x K] * B[K x N], all in shared memory (A, B bf16 row-major, C float row-major); 8 warps
template <int NW>
__device__ __forceinline__ void tile_gemm(const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb,
                                          float* C, int ldc, int K, int N) {
  const int warp = threadIdx.x >> 5;
  const int mt = kTile / 16, nt = N / 16;
  for (int t = warp; t < mt * nt; t += NW) {
    const int i = t / nt, j = t % nt;
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc;
    wmma::fill_fragment(acc, 0.0f);
    for (int k = 0; k < K; k += 16) {
      wmma::fragment<wmma::matrix_a, 16, 16, 16, __nv_bfloat16, wmma::row_major> a;
      wmma::fragment<wmma::matrix_b, 16, 16, 16, __nv_bfloat16, wmma::row_major> b;
      wmma::load_matrix_sync(a, A + (size_t)i * 16 * lda + k, lda);
      wmma::load_matrix_sync(b, B + (size_t)k * ldb + j * 16, ldb);
      wmma::mma_sync(acc, a, b, acc);
    }
    wmma::store_matrix_sync(C + (size_t)i * 16 * ldc + j * 16, acc, ldc, wmma::mem_row_major);
  }
}

template <typename TV>
__global__ void __launch_bounds__(256) mlp_fwd_kernel(FwdArgs a, const TV* __restrict__ r, TV* __restrict__ z) {
  extern __shared__ __align__(128) unsigned char smem[];
  __nv_bfloat16* W1 = reinterpret_cast<__nv_bfloat16*>(smem);
  __nv_bfloat16* W2 = W1 + a.Fp * a.H;
  __nv_bfloat16* W3 = W2 + a.H * a.H;
  __nv_bfloat16* X = W3 + a.H * a.Op;
  __nv_bfloat16* Hb = X + kTile * a.Fp;
  float* Cf = reinterpret_cast<float*>(Hb + kTile * a.H);
  const int nthr = blockDim.x;
  for (int e = threadIdx.x; e < a.Fp * a.H; e += nthr) W1[e] = a.w1[e];
  for (int e = threadIdx.x; e < a.H * a.H; e += nthr) W2[e] = a.w2[e];
  for (int e = threadIdx.x; e < a.H * a.Op; e += nthr) W3[e] = a.w3[e];
  const double sc = a.scale ? *a.scale : 1.0;
  const float inv = sc > 0 ? (float)(1.0 / sc) : 1.0f;
  const int ldc = a.H > a.Op ? a.H : a.Op;
  for (int64_t t0 = (int64_t)blockIdx.x * kTile; t0 < a.ncells; t0 += (int64_t)gridDim.x * kTile) {
    __syncthreads();
    for (int e = threadIdx.x; e < kTile * a.Fp; e += nthr) {
      const int cl = e / a.Fp, f = e - cl * a.Fp;
      const int64_t c = t0 + cl;
      float v = 0.0f;
      if (c < a.ncells && f < a.F) v = feature<TV>(r, a.nbr, a.extra, c, f, a.Np, a.nfaces, a.nextra, inv);
      X[e] = bf(v);
    }
    __syncthreads();
    tile_gemm<8>(X, a.Fp, W1, a.H, Cf, ldc, a.Fp, a.H);
    __syncthreads();
    for (int e = threadIdx.x; e < kTile * a.H; e += nthr) {
      const int cl = e / a.H, j = e - cl * a.H;
      const float h = fmaxf(Cf[cl * ldc + j], 0.0f);
      Hb[e] = bf(h);
      if (a.act && t0 + cl < a.ncells) a.act[(t0 + cl) * 2 * a.H + j] = h;
    }
    __syncthreads();
    tile_gemm<8>(Hb, a.H, W2, a.H, Cf, ldc, a.H, a.H);
    __syncthreads();
    for (int e = threadIdx.x; e < kTile * a.H; e += nthr) {
      const int cl = e / a.H, j = e - cl * a.H;
      const float h = fmaxf(Cf[cl * ldc + j], 0.0f);
      Hb[e] = bf(h);
      if (a.act && t0 + cl < a.ncells) a.act[(t0 + cl) * 2 * a.H + a.H + j] = h;
    }
    __syncthreads();
    tile_gemm<8>(Hb, a.H, W3, a.Op, Cf, ldc, a.H, a.Op);
    __syncthreads();
    for (int e = threadIdx.x; e < kTile * a.Np; e += nthr) {
      const int cl = e / a.Np, o = e - cl * a.Np;
      const int64_t c = t0 + cl;
      if (c < a.ncells) z[c * a.Np + o] = (TV)((double)Cf[cl * ldc + o] * sc);
    }
  }
}

struct BwdArgs {
  const int32_t* nbr;
  const float* extra;
  const float* m2;   // FP32 master W2 [H x H]
  const float* m3;   // FP32 master W3 [H x Op]
  const float* act;  // [ncells x 2H]
  const double* g;   // dL/dz (per DOF)
  const double* scale;
  float* g1;
  float* g2;
  float* g3;
  int64_t ncells;
  int Np, nfaces, nextra, F, Fp, H, Op;
};

// Backward pass on the CUDA cores (FP32): per tile of 32 cells the activation gradients, then the weight
// gradients accumulated per CTA in shared memory and added to the global gradient once at the end.
__global__ void __launch_bounds__(256) mlp_bwd_kernel(BwdArgs a, const double* __restrict__ r) {
  extern __shared__ __align__(16) float sm[];
  const int Fp = a.Fp, H = a.H, Op = a.Op;
  float* dW1 = sm;                 // Fp x H
  float* dW2 = dW1 + Fp * H;       // H x H
  float* dW3 = dW2 + H * H;        // H x Op
  float* W2 = dW3 + H * Op;        // H x H
  float* W3 = W2 + H * H;          // H x Op
  float* X = W3 + H * Op;          // kBTile x Fp
  float* H1 = X + kBTile * Fp;     // kBTile x H
  float* H2 = H1 + kBTile * H;
  float* D1 = H2 + kBTile * H;
  float* D2 = D1 + kBTile * H;
  float* G = D2 + kBTile * H;      // kBTile x Op
  const int nthr = blockDim.x;
  for (int e = threadIdx.x; e < Fp * H + H * H + H * Op; e += nthr) dW1[e] = 0.0f;
  for (int e = threadIdx.x; e < H * H; e += nthr) W2[e] = a.m2[e];
  for (int e = threadIdx.x; e < H * Op; e += nthr) W3[e] = a.m3[e];
  const double sc = a.scale ? *a.scale : 1.0;
  const float inv = sc > 0 ? (float)(1.0 / sc) : 1.0f;
  for (int64_t t0 = (int64_t)blockIdx.x * kBTile; t0 < a.ncells; t0 += (int64_t)gridDim.x * kBTile) {
    __syncthreads();
    for (int e = threadIdx.x; e < kBTile * Fp; e += nthr) {
      const int cl = e / Fp, f = e - cl * Fp;
      const int64_t c = t0 + cl;
      X[e] = (c < a.ncells && f < a.F) ? feature<double>(r, a.nbr, a.extra, c, f, a.Np, a.nfaces, a.nextra, inv) : 0.0f;
    }
    for (int e = threadIdx.x; e < kBTile * H; e += nthr) {
      const int cl = e / H, j = e - cl * H;
      const int64_t c = t0 + cl;
      H1[e] = c < a.ncells ? a.act[c * 2 * H + j] : 0.0f;
      H2[e] = c < a.ncells ? a.act[c * 2 * H + H + j] : 0.0f;
    }
    for (int e = threadIdx.x; e < kBTile * Op; e += nthr) {
      const int cl = e / Op, o = e - cl * Op;
      const int64_t c = t0 + cl;
      // z = sc * y  ->  dL/dy = sc * dL/dz
      G[e] = (c < a.ncells && o < a.Np) ? (float)(a.g[c * a.Np + o] * sc) : 0.0f;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kBTile * H; e += nthr) {
      const int cl = e / H, k = e - cl * H;
      float s = 0.0f;
      for (int o = 0; o < Op; ++o) s = fmaf(G[cl * Op + o], W3[k * Op + o], s);
      D2[e] = H2[e] > 0.0f ? s : 0.0f;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kBTile * H; e += nthr) {
      const int cl = e / H, j = e - cl * H;
      float s = 0.0f;
      for (int k = 0; k < H; ++k) s = fmaf(D2[cl * H + k], W2[j * H + k], s);
      D1[e] = H1[e] > 0.0f ? s : 0.0f;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < H * Op; e += nthr) {
      const int k = e / Op, o = e - k * Op;
      float s = 0.0f;
      for (int cl = 0; cl < kBTile; ++cl) s = fmaf(H2[cl * H + k], G[cl * Op + o], s);
      dW3[e] += s;
    }
    for (int e = threadIdx.x; e < H * H; e += nthr) {
      const int j = e / H, k = e - j * H;
      float s = 0.0f;
      for (int cl = 0; cl < kBTile; ++cl) s = fmaf(H1[cl * H + j], D2[cl * H + k], s);
      dW2[e] += s;
    }
    for (int e = threadIdx.x; e < Fp * H; e += nthr) {
      const int f = e / H, j = e - f * H;
      float s = 0.0f;
      for (int cl = 0; cl < kBTile; ++cl) s = fmaf(X[cl * Fp + f], D1[cl * H + j], s);
      dW1[e] += s;
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < Fp * H; e += nthr) atomicAdd(a.g1 + e, dW1[e]);
  for (int e = threadIdx.x; e < H * H; e += nthr) atomicAdd(a.g2 + e, dW2[e]);
  for (int e = threadIdx.x; e < H * Op; e += nthr) atomicAdd(a.g3 + e, dW3[e]);
}

__global__ void adam_kernel(float* __restrict__ w, uint16_t* __restrict__ wb, float* __restrict__ grad,
                            float* __restrict__ m, float* __restrict__ v, int64_t n, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float g = grad[i];
    const float mi = b1 * m[i] + (1.0f - b1) * g;
    const float vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    w[i] = wi;
    const __nv_bfloat16 h = __float2bfloat16(wi);
    wb[i] = *reinterpret_cast<const uint16_t*>(&h);
    grad[i] = 0.0f;
  }
}

__global__ void rms_scale_kernel(const double* nrm, double* scale, double inv_sqrt_n) {
  const double s = nrm[0] * inv_sqrt_n;
  scale[0] = s > 0 ? s : 1.0;
}

// g = 2 (Az - r) / |r|^2
__global__ void energy_grad_kernel(const double* __restrict__ Az, const double* __restrict__ r,
                                   const double* __restrict__ rr, double* __restrict__ g, int64_t n) {
  const double f = 2.0 / rr[0];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    g[i] = f * (Az[i] - r[i]);
}

uint16_t to_bf16_bits(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  const uint32_t rounding = 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)((u + rounding) >> 16);
}

size_t fwd_smem(const LearnedNet& n) {
  const int ldc = std::max(n.H, n.Op);
  return (size_t)(n.Fp * n.H + n.H * n.H + n.H * n.Op + kTile * n.Fp + kTile * n.H) * 2 + (size_t)kTile * ldc * 4;
}

template <typename TV>
void apply_impl(const LearnedNet& net, const TV* r, TV* z, const double* scale, float* act, cudaStream_t st) {
  require(net.ncells > 0, "learned stage is not initialised");
  FwdArgs a{net.nbr.p, net.extra.p, reinterpret_cast<const __nv_bfloat16*>(net.w1.p),
            reinterpret_cast<const __nv_bfloat16*>(net.w2.p), reinterpret_cast<const __nv_bfloat16*>(net.w3.p), act,
            scale, net.ncells, net.Np, net.nfaces, net.nextra, net.F, net.Fp, net.H, net.Op};
  const size_t sm = fwd_smem(net);
  BSGPU_CUDA(cudaFuncSetAttribute(mlp_fwd_kernel<TV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  const int64_t tiles = (net.ncells + kTile - 1) / kTile;
  const int grid = (int)std::min<int64_t>(tiles, (int64_t)num_sms() * 2);
  mlp_fwd_kernel<TV><<<grid, 256, sm, st>>>(a, r, z);
  BSGPU_CHECK_LAUNCH();
}

}  // namespace

void LearnedNet::init(int Np_, int64_t ncells_, int nfaces_, int nextra_, const int32_t* nbr_host,
                      const float* extra_host, uint64_t seed) {
  Np = Np_;
  ncells = ncells_;
  nfaces = nfaces_;
  nextra = nextra_;
  F = (nfaces + 1) * Np + nextra;
  Fp = (F + 15) / 16 * 16;
  Op = (Np + 15) / 16 * 16;
  require(fwd_smem(*this) <= 200 * 1024, "learned stage: input too wide for one CTA", BSGPU_ERR_UNSUPPORTED);
  nbr.alloc(std::max<int64_t>(ncells * nfaces, 1));
  BSGPU_CUDA(cudaMemcpy(nbr.p, nbr_host, ncells * nfaces * 4, cudaMemcpyHostToDevice));
  extra.alloc(std::max<int64_t>(ncells * nextra, 1));
  if (nextra) BSGPU_CUDA(cudaMemcpy(extra.p, extra_host, ncells * nextra * 4, cudaMemcpyHostToDevice));
  // He initialisation; the last layer starts small so that the untrained stage is a mild scaled identity-free map
  std::mt19937_64 g(seed);
  auto fill_master = [&](std::vector<float>& w, int K, int N, int Kreal, int Nreal, float sd) {
    std::normal_distribution<float> nd(0.0f, sd);
    w.assign((size_t)K * N, 0.0f);
    for (int k = 0; k < Kreal; ++k)
      for (int n = 0; n < Nreal; ++n) w[(size_t)k * N + n] = nd(g);
  };
  std::vector<float> h1, h2, h3;
  fill_master(h1, Fp, H, F, H, std::sqrt(2.0f / F));
  fill_master(h2, H, H, H, H, std::sqrt(2.0f / H));
  fill_master(h3, H, Op, H, Np, 0.1f * std::sqrt(1.0f / H));
  auto upload = [&](const std::vector<float>& h, DBuf<float>& master, DBuf<uint16_t>& b, DBuf<float>& grad,
                    DBuf<float>& m, DBuf<float>& v) {
    master.alloc(h.size());
    b.alloc(h.size());
    grad.alloc(h.size());
    m.alloc(h.size());
    v.alloc(h.size());
    std::vector<uint16_t> hb(h.size());
    for (size_t i = 0; i < h.size(); ++i) hb[i] = to_bf16_bits(h[i]);
    BSGPU_CUDA(cudaMemcpy(master.p, h.data(), h.size() * 4, cudaMemcpyHostToDevice));
    BSGPU_CUDA(cudaMemcpy(b.p, hb.data(), h.size() * 2, cudaMemcpyHostToDevice));
    BSGPU_CUDA(cudaMemset(grad.p, 0, h.size() * 4));
    BSGPU_CUDA(cudaMemset(m.p, 0, h.size() * 4));
    BSGPU_CUDA(cudaMemset(v.p, 0, h.size() * 4));
  };
  upload(h1, m1, w1, g1, a1, v1);
  upload(h2, m2, w2, g2, a2, v2);
  upload(h3, m3, w3, g3, a3, v3);
  adam_t = 0;
  trained = false;
}

void learned_scale(const double* nrm, double* scale, int64_t n, cudaStream_t st) {
  rms_scale_kernel<<<1, 1, 0, st>>>(nrm, scale, 1.0 / std::sqrt((double)std::max<int64_t>(n, 1)));
  BSGPU_CHECK_LAUNCH();
}

void learned_apply(const LearnedNet& net, const double* r, double* z, const double* scale, cudaStream_t st) {
  apply_impl<double>(net, r, z, scale, nullptr, st);
}
void learned_apply(const LearnedNet& net, const float* r, float* z, const double* scale, cudaStream_t st) {
  apply_impl<float>(net, r, z, scale, nullptr, st);
}

void learned_get_weights(const LearnedNet& net, float* w1, float* w2, float* w3) {
  auto get = [](const DBuf<uint16_t>& b, float* out) {
    std::vector<uint16_t> h(b.n);
    BSGPU_CUDA(cudaMemcpy(h.data(), b.p, b.n * 2, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < h.size(); ++i) {
      const uint32_t u = (uint32_t)h[i] << 16;
      std::memcpy(out + i, &u, 4);
    }
  };
  get(net.w1, w1);
  get(net.w2, w2);
  get(net.w3, w3);
}

void learned_set_weights(LearnedNet& net, const float* w1, const float* w2, const float* w3) {
  auto set = [](const float* in, DBuf<float>& master, DBuf<uint16_t>& b, DBuf<float>& grad, DBuf<float>& m,
                DBuf<float>& v) {
    std::vector<uint16_t> hb(master.n);
    for (size_t i = 0; i < hb.size(); ++i) hb[i] = to_bf16_bits(in[i]);
    BSGPU_CUDA(cudaMemcpy(master.p, in, master.n * 4, cudaMemcpyHostToDevice));
    BSGPU_CUDA(cudaMemcpy(b.p, hb.data(), hb.size() * 2, cudaMemcpyHostToDevice));
    BSGPU_CUDA(cudaMemset(grad.p, 0, grad.n * 4));
    BSGPU_CUDA(cudaMemset(m.p, 0, m.n * 4));
    BSGPU_CUDA(cudaMemset(v.p, 0, v.n * 4));
  };
  set(w1, net.m1, net.w1, net.g1, net.a1, net.v1);
  set(w2, net.m2, net.w2, net.g2, net.a2, net.v2);
  set(w3, net.m3, net.w3, net.g3, net.a3, net.v3);
  net.adam_t = 0;
}

void learned_take_gradient(LearnedNet& net, float* g1, float* g2, float* g3, cudaStream_t st) {
  auto take = [&](DBuf<float>& g, float* out) {
    BSGPU_CUDA(cudaMemcpyAsync(out, g.p, g.n * 4, cudaMemcpyDeviceToHost, st));
    BSGPU_CUDA(cudaMemsetAsync(g.p, 0, g.n * 4, st));
  };
  take(net.g1, g1);
  take(net.g2, g2);
  take(net.g3, g3);
  BSGPU_CUDA(cudaStreamSynchronize(st));
}

void learned_gradient(LearnedNet& net, const Matrix& A, const double* r, double* z, double* Az, double* g,
                      ReduceScratch& red, double* scal, cudaStream_t st) {
  // scal: [0] |r|, [1] scale, [2] |r|^2, [3] z.Az, [4] z.r
  const int64_t N = net.ncells * net.Np;
  if (!net.act.p) net.act.alloc((size_t)net.ncells * 2 * net.H);
  const double* a1[1] = {r};
  dots(red, 1, a1, a1, N, scal, 1, st);
  rms_scale_kernel<<<1, 1, 0, st>>>(scal, scal + 1, 1.0 / std::sqrt((double)N));
  BSGPU_CHECK_LAUNCH();
  apply_impl<double>(net, r, z, scal + 1, net.act.p, st);
  spmv(A, 1.0, z, 0.0, (const double*)nullptr, Az, st);
  const double* da[3] = {r, z, z};
  const double* db[3] = {r, Az, r};
  dots(red, 3, da, db, N, scal + 2, 0, st);
  const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((N + 255) / 256, (int64_t)num_sms() * 8));
  energy_grad_kernel<<<grid, 256, 0, st>>>(Az, r, scal + 2, g, N);
  BSGPU_CHECK_LAUNCH();
  BwdArgs b{net.nbr.p, net.extra.p, net.m2.p, net.m3.p, net.act.p, g, scal + 1, net.g1.p, net.g2.p, net.g3.p,
            net.ncells, net.Np, net.nfaces, net.nextra, net.F, net.Fp, net.H, net.Op};
  const size_t sm = (size_t)(net.Fp * net.H + 2 * net.H * net.H + 2 * net.H * net.Op + kBTile * net.Fp +
                             4 * kBTile * net.H + kBTile * net.Op) * 4;
  require(sm <= 220 * 1024, "learned stage: backward tile does not fit shared memory", BSGPU_ERR_UNSUPPORTED);
  BSGPU_CUDA(cudaFuncSetAttribute(mlp_bwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  const int bgrid = (int)std::min<int64_t>((net.ncells + kBTile - 1) / kBTile, (int64_t)num_sms());
  mlp_bwd_kernel<<<bgrid, 256, sm, st>>>(b, r);
  BSGPU_CHECK_LAUNCH();
}

void learned_train_step(LearnedNet& net, const Matrix& A, const double* r, double* z, double* Az, double* g,
                        ReduceScratch& red, double* scal, double lr, cudaStream_t st) {
  learned_gradient(net, A, r, z, Az, g, red, scal, st);
  net.adam_t++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - std::pow(b1, (float)net.adam_t), c2 = 1.0f - std::pow(b2, (float)net.adam_t);
  auto step = [&](DBuf<float>& w, DBuf<uint16_t>& wb, DBuf<float>& gr, DBuf<float>& m, DBuf<float>& v) {
    const int64_t n = (int64_t)w.n;
    adam_kernel<<<(int)std::min<int64_t>((n + 255) / 256, 1024), 256, 0, st>>>(w.p, wb.p, gr.p, m.p, v.p, n, (float)lr,
                                                                               b1, b2, 1e-8f, c1, c2);
    BSGPU_CHECK_LAUNCH();
  };
  step(net.m1, net.w1, net.g1, net.a1, net.v1);
  step(net.m2, net.w2, net.g2, net.a2, net.v2);
  step(net.m3, net.w3, net.g3, net.a3, net.v3);
}

}  // namespace bsgpu
