// Learned preconditioner stage (no counterpart in the reference; it plugs into FlexGMRES's list of
// preconditioners, FlexGMRES.cs:50-56,196-199).
//
// Per cell c the network sees its own residual block, the blocks of its face neighbours (zero where a face has
// none) and optional per-cell features, and returns a correction block:
//     z_c = W3^T relu(W2^T relu(W1^T f_c)),   f_c = [r_c, r_n1, ..., r_n6, extra_c]
// No biases: with ReLU the map is positively homogeneous, z(a r) = a z(r) for a > 0, so it commutes with the
// arbitrary scaling of Krylov vectors.  Weights are BF16 (FP32 master copies for training), products accumulate in
// FP32 on the 5th-generation tensor cores (tcgen05.mma with tensor-memory accumulators), one CTA per tile of 128
// cells with all weights in shared memory.  Training minimises the energy norm of the error left after the correction,
//     |e - z|_A^2 = z^T A z - 2 z^T r + e^T A e,   A e = r,
// i.e. it fits a local approximate inverse of the operator, with one SpMV per step for A z.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>

#include "learned.cuh"

namespace bsgpu {

namespace {

constexpr int kBTile = 32;   // cells per CTA tile (backward)

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

// ---- tcgen05 forward pass -------------------------------------------------------------------------------------
// One CTA of 128 threads per tile of 128 cells, thread t owning cell row t.  Each layer is one M = 128 block of
// tcgen05.mma (kind::f16: BF16 operands, FP32 accumulation in tensor memory), K in steps of 16, issued by one
// thread; the operands sit in shared memory in the canonical K-major layout without swizzle (8-row x 16-byte core
// matrices, K-adjacent core matrices 128 bytes apart, 8-row groups K/8 x 128 bytes apart).  The accumulators are
// read back with tcgen05.ld (32x32b: warp w sees tensor-memory lanes 32w .. 32w+31, i.e. its own cells), passed
// through ReLU, rounded to BF16 and written as the next layer's A operand.  Tensor memory: layer 1 at columns
// [0, H), layer 2 at [H, 2H), the output layer at [0, Op).
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (r, k) of an R x K BF16 operand in the canonical K-major layout
__device__ __forceinline__ uint32_t kmajor_off(int r, int k, int K) {
  return (uint32_t)(((r >> 3) * (K >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor: start address, leading (K) and stride (M/N) byte offsets, descriptor version 1,
// no swizzle
__device__ __forceinline__ uint64_t desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor, kind::f16: FP32 accumulator (bits 4-5 = 1), BF16 A and B (bits 7-9, 10-12 = 1), both
// K-major (bits 15, 16 = 0), N >> 3 in bits 17-22, M >> 4 in bits 24-28
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}
__device__ __forceinline__ void commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// bounded wait on an mbarrier phase
__device__ __forceinline__ bool wait_phase(uint32_t mbar, uint32_t parity) {
  for (long long it = 0; it < (1ll << 22); ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 16 FP32 columns of this thread's tensor-memory lane
__device__ __forceinline__ void ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 8 consecutive K entries of one row as one 16-byte store
__device__ __forceinline__ void st8(unsigned char* base, uint32_t off, const float* v) {
  __nv_bfloat162 h[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) h[i] = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
  *reinterpret_cast<uint4*>(base + off) = *reinterpret_cast<const uint4*>(h);
}

constexpr int kRows = 128;  // cells per tile = MMA M = threads per CTA

}  // namespace tc

// shared memory of the tcgen05 forward kernel: W1^T [H x Fp], W2^T [H x H], W3^T [Op x H], A1 [128 x Fp],
// A2 [128 x H] (BF16, canonical layout), each at a 1024-byte boundary
struct TcSmem {
  uint32_t w1, w2, w3, a1, a2, total;
  __host__ __device__ TcSmem(int Fp, int H, int Op) {
    auto up = [](uint32_t x) { return (x + 1023u) & ~1023u; };
    w1 = 0;
    w2 = up(w1 + (uint32_t)(H * Fp * 2));
    w3 = up(w2 + (uint32_t)(H * H * 2));
    a1 = up(w3 + (uint32_t)(Op * H * 2));
    a2 = up(a1 + (uint32_t)(tc::kRows * Fp * 2));
    total = up(a2 + (uint32_t)(tc::kRows * H * 2));
  }
};

template <typename TV>
__global__ void __launch_bounds__(128) mlp_fwd_tc_kernel(FwdArgs a, const TV* __restrict__ r, TV* __restrict__ z,
                                                         int tmem_cols, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  const int t = threadIdx.x, warp = t >> 5;
  const int Fp = a.Fp, H = a.H, Op = a.Op;
  const TcSmem L(Fp, H, Op);
  unsigned char* W1 = smem + L.w1;
  unsigned char* W2 = smem + L.w2;
  unsigned char* W3 = smem + L.w3;
  unsigned char* A1 = smem + L.a1;
  unsigned char* A2 = smem + L.a2;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(&tmem_slot)),
                 "r"(tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc::smem_u32(&mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // weights as the B operands: B = W^T (N rows x K), element (n, k) = W[k][n]
  const uint16_t* w1 = reinterpret_cast<const uint16_t*>(a.w1);
  const uint16_t* w2 = reinterpret_cast<const uint16_t*>(a.w2);
  const uint16_t* w3 = reinterpret_cast<const uint16_t*>(a.w3);
  for (int e = t; e < Fp * H; e += blockDim.x) {
    const int k = e / H, n = e - k * H;
    *reinterpret_cast<uint16_t*>(W1 + tc::kmajor_off(n, k, Fp)) = w1[e];
  }
  for (int e = t; e < H * H; e += blockDim.x) {
    const int k = e / H, n = e - k * H;
    *reinterpret_cast<uint16_t*>(W2 + tc::kmajor_off(n, k, H)) = w2[e];
  }
  for (int e = t; e < H * Op; e += blockDim.x) {
    const int k = e / Op, n = e - k * Op;
    *reinterpret_cast<uint16_t*>(W3 + tc::kmajor_off(n, k, H)) = w3[e];
  }
  tc::fence_proxy();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tmem_slot;
  const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
  const uint32_t mb = tc::smem_u32(&mbar);
  const uint32_t sA1 = tc::smem_u32(A1), sA2 = tc::smem_u32(A2);
  const uint32_t sW1 = tc::smem_u32(W1), sW2 = tc::smem_u32(W2), sW3 = tc::smem_u32(W3);
  const double sc = a.scale ? *a.scale : 1.0;
  const float inv = sc > 0 ? (float)(1.0 / sc) : 1.0f;
  uint32_t parity = 0;
  bool bad = false;  // a wait gave up (uniform across the CTA)
  // one layer: D[128 x N] (tensor memory column dcol) = A[128 x K] * B^T, then wait for it
  auto layer = [&](uint32_t sA, uint32_t sB, int K, int N, uint32_t dcol) -> bool {
    tc::fence_proxy();
    tc::fence_before();
    __syncthreads();
    if (t == 0) {
      tc::fence_after();
      const uint32_t sbo = (uint32_t)(K / 8) * 128u;
      for (int s = 0; s < K / 16; ++s)
        tc::mma(tmem + dcol, tc::desc(sA + (uint32_t)s * 256u, 128u, sbo), tc::desc(sB + (uint32_t)s * 256u, 128u, sbo),
                tc::idesc_bf16(tc::kRows, N), s > 0 ? 1u : 0u);
      tc::commit(mb);
    }
    const bool ok = tc::wait_phase(mb, parity);
    tc::fence_after();
    if (__syncthreads_and(ok ? 1 : 0) == 0) return false;
    parity ^= 1u;
    return true;
  };
  for (int64_t t0 = (int64_t)blockIdx.x * tc::kRows; t0 < a.ncells; t0 += (int64_t)gridDim.x * tc::kRows) {
    const int64_t c = t0 + t;
    const bool valid = c < a.ncells;
    // layer-1 operand: this cell's features, 8 at a time
    for (int k0 = 0; k0 < Fp; k0 += 8) {
      float v[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int f = k0 + q;
        v[q] = (valid && f < a.F) ? feature<TV>(r, a.nbr, a.extra, c, f, a.Np, a.nfaces, a.nextra, inv) : 0.0f;
      }
      tc::st8(A1, tc::kmajor_off(t, k0, Fp), v);
    }
    if (!layer(sA1, sW1, Fp, H, 0)) {
      bad = true;
      break;
    }
    for (int cb = 0; cb < H; cb += 16) {
      float v[16];
      tc::ld16(tmem + lane_base + (uint32_t)cb, v);
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = fmaxf(v[q], 0.0f);
      if (a.act && valid)
        for (int q = 0; q < 16; ++q) a.act[c * 2 * H + cb + q] = v[q];
      tc::st8(A2, tc::kmajor_off(t, cb, H), v);
      tc::st8(A2, tc::kmajor_off(t, cb + 8, H), v + 8);
    }
    if (!layer(sA2, sW2, H, H, (uint32_t)H)) {
      bad = true;
      break;
    }
    for (int cb = 0; cb < H; cb += 16) {
      float v[16];
      tc::ld16(tmem + lane_base + (uint32_t)(H + cb), v);
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = fmaxf(v[q], 0.0f);
      if (a.act && valid)
        for (int q = 0; q < 16; ++q) a.act[c * 2 * H + H + cb + q] = v[q];
      tc::st8(A2, tc::kmajor_off(t, cb, H), v);
      tc::st8(A2, tc::kmajor_off(t, cb + 8, H), v + 8);
    }
    if (!layer(sA2, sW3, H, Op, 0)) {
      bad = true;
      break;
    }
    for (int cb = 0; cb < Op; cb += 16) {
      float y[16];
      tc::ld16(tmem + lane_base + (uint32_t)cb, y);
      if (valid)
        for (int o = 0; o < 16 && cb + o < a.Np; ++o) z[c * a.Np + cb + o] = (TV)((double)y[o] * sc);
    }
    tc::fence_before();
    __syncthreads();
  }
  if (bad) {
    // a wait gave up: flag it, and give the committed MMAs a bounded second chance to finish before the tensor
    // memory is freed
    if (t == 0) atomicExch(err, 1);
    tc::wait_phase(mb, parity);
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tmem_cols) : "memory");
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

int tmem_columns(int H) {
  int c = 32;
  while (c < 2 * H) c *= 2;
  return c;
}

template <typename TV>
void apply_impl(const LearnedNet& net, const TV* r, TV* z, const double* scale, float* act, cudaStream_t st) {
  require(net.ncells > 0, "learned stage is not initialised");
  FwdArgs a{net.nbr.p, net.extra.p, reinterpret_cast<const __nv_bfloat16*>(net.w1.p),
            reinterpret_cast<const __nv_bfloat16*>(net.w2.p), reinterpret_cast<const __nv_bfloat16*>(net.w3.p), act,
            scale, net.ncells, net.Np, net.nfaces, net.nextra, net.F, net.Fp, net.H, net.Op};
  const TcSmem L(net.Fp, net.H, net.Op);
  BSGPU_CUDA(cudaFuncSetAttribute(mlp_fwd_tc_kernel<TV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.total));
  const int64_t tiles = (net.ncells + tc::kRows - 1) / tc::kRows;
  const int grid = (int)std::min<int64_t>(tiles, (int64_t)num_sms() * 2);
  mlp_fwd_tc_kernel<TV><<<grid, tc::kRows, L.total, st>>>(a, r, z, tmem_columns(net.H), net.err.p);
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
  require(H % 16 == 0 && H >= 16 && H <= 128, "learned stage: hidden width must be a multiple of 16 in 16..128",
          BSGPU_ERR_UNSUPPORTED);
  require(Op <= H, "learned stage: the hidden width must be at least the modes per cell (padded to 16)",
          BSGPU_ERR_UNSUPPORTED);
  require(TcSmem(Fp, H, Op).total <= 200 * 1024, "learned stage: input too wide for one CTA", BSGPU_ERR_UNSUPPORTED);
  err.alloc(1);
  BSGPU_CUDA(cudaMemset(err.p, 0, sizeof(int)));
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

void learned_check(const LearnedNet& net, cudaStream_t st) {
  int h = 0;
  BSGPU_CUDA(cudaMemcpyAsync(&h, net.err.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  BSGPU_CUDA(cudaStreamSynchronize(st));
  if (h) {
    BSGPU_CUDA(cudaMemset(net.err.p, 0, sizeof(int)));
    throw Error(BSGPU_ERR_TIMEOUT, "learned stage: a tensor-core wait gave up");
  }
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
