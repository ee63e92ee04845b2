// Vector kernels: grid-reduction dot products, multi-term axpy, scaling, conversion, p-restriction transfer.
// MPI-free counterparts of the BLAS-1 calls of the solvers (ddot/daxpy/dscal in OrthonormalizationMultigrid.cs,
// FlexGMRES.cs, SoftPCG.cs) and of BlockMask.GetSubVec/AccSubVec (SubBlockSelectorExt.cs:573-700).
#include <algorithm>

#include "blas1.cuh"
#include "reduce.cuh"

namespace bsgpu {

namespace {

constexpr int kThreads = 256;

template <typename T>
struct DotArgs {
  const T* a[kMaxDots];
  const T* b[kMaxDots];
};

using gridred::finish_dots;
using gridred::warp_sum;

template <typename T, int KC>
__global__ void __launch_bounds__(kThreads) dots_kernel(DotArgs<T> args, int K, int64_t n, double* __restrict__ partial,
                                                        unsigned int* __restrict__ ticket, double* __restrict__ out,
                                                        int post, const int* __restrict__ active) {
  if (active != nullptr && *active == 0) return;
  double acc[KC];
#pragma unroll
  for (int k = 0; k < KC; ++k) acc[k] = 0.0;
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  for (; i + stride < n; i += 2 * stride) {
#pragma unroll
    for (int k = 0; k < KC; ++k) {
      if (k < K) {
        const T* a = args.a[k];
        const T* b = args.b[k];
        double a0 = (double)a[i], a1 = (double)a[i + stride];
        double b0 = (a == b) ? a0 : (double)b[i];
        double b1 = (a == b) ? a1 : (double)b[i + stride];
        acc[k] = fma(a0, b0, acc[k]);
        acc[k] = fma(a1, b1, acc[k]);
      }
    }
  }
  if (i < n) {
#pragma unroll
    for (int k = 0; k < KC; ++k)
      if (k < K) acc[k] = fma((double)args.a[k][i], (double)args.b[k][i], acc[k]);
  }
  finish_dots<KC>(acc, K, partial, ticket, out, post);
}

// K products against one shared vector b (Gram-Schmidt projections, Arnoldi): b is read once per element and
// every vector moves in 16-byte loads (all pointers 16-byte aligned; the host checks), so the launch streams
// (K+1) vectors at HBM rate.
template <typename T> struct Vec16;
template <> struct Vec16<float> { using type = float4; static constexpr int W = 4; };
template <> struct Vec16<double> { using type = double2; static constexpr int W = 2; };

__device__ __forceinline__ double dot16(const float4& a, const float4& b) {
  return (double)a.x * b.x + (double)a.y * b.y + (double)a.z * b.z + (double)a.w * b.w;
}
__device__ __forceinline__ double dot16(const double2& a, const double2& b) { return fma(a.x, b.x, a.y * b.y); }

template <typename T, int KC>
__global__ void __launch_bounds__(kThreads) dots_sharedb_kernel(DotArgs<T> args, int K, int64_t n,
                                                                double* __restrict__ partial,
                                                                unsigned int* __restrict__ ticket,
                                                                double* __restrict__ out, int post,
                                                                const int* __restrict__ active) {
  if (active != nullptr && *active == 0) return;
  using V = typename Vec16<T>::type;
  constexpr int W = Vec16<T>::W;
  double acc[KC];
#pragma unroll
  for (int k = 0; k < KC; ++k) acc[k] = 0.0;
  const int64_t nv = n / W;
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  const V* bv = reinterpret_cast<const V*>(args.b[0]);
  for (int64_t j = (int64_t)blockIdx.x * kThreads + threadIdx.x; j < nv; j += stride) {
    const V bb = __ldg(bv + j);
    V aa[KC];
#pragma unroll
    for (int k = 0; k < KC; ++k)
      if (k < K) aa[k] = __ldcs(reinterpret_cast<const V*>(args.a[k]) + j);
#pragma unroll
    for (int k = 0; k < KC; ++k)
      if (k < K) acc[k] += dot16(aa[k], bb);
  }
  for (int64_t i = nv * W + (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += stride) {
    const double b = (double)args.b[0][i];
#pragma unroll
    for (int k = 0; k < KC; ++k)
      if (k < K) acc[k] = fma((double)args.a[k][i], b, acc[k]);
  }
  finish_dots<KC>(acc, K, partial, ticket, out, post);
}

template <typename T, int NP>
__global__ void __launch_bounds__(256) pcg_update_kernel(double* __restrict__ s, int* __restrict__ active,
                                                         T* __restrict__ x, const T* __restrict__ p,
                                                         const T* __restrict__ q, T* __restrict__ r, T* __restrict__ z,
                                                         const T* __restrict__ dinv, int64_t nb,
                                                         double* __restrict__ partial,
                                                         unsigned int* __restrict__ ticket, int mode, double tol,
                                                         int max_iter, int min_iter) {
  if (*active == 0) return;
  constexpr int BPC = 256 / NP;  // block rows per tile; thread t owns DOF row t % NP of block row t / NP
  const double alpha = s[0] / s[1];
  __shared__ T rs[256];
  double acc[2] = {0.0, 0.0};
  const int t = threadIdx.x;
  const int lb = t / NP;
  const int rr = t - lb * NP;
  for (int64_t tile = blockIdx.x; tile * BPC < nb; tile += gridDim.x) {
    const int64_t i = tile * BPC + lb;
    const bool valid = (lb < BPC) && (i < nb);
    const int64_t g = i * NP + rr;
    T rn = T(0);
    if (valid) {
      x[g] = (T)((double)x[g] + alpha * (double)p[g]);
      rn = (T)((double)r[g] - alpha * (double)q[g]);
      r[g] = rn;
    }
    rs[t] = rn;
    __syncthreads();
    if (valid) {
      const T* D = dinv + i * (NP * NP) + rr;
      const T* rb = rs + lb * NP;
      T zz = T(0);
#pragma unroll
      for (int c = 0; c < NP; ++c) zz = fma(D[c * NP], rb[c], zz);
      z[g] = zz;
      acc[0] = fma((double)rn, (double)zz, acc[0]);
      acc[1] = fma((double)rn, (double)rn, acc[1]);
    }
    __syncthreads();
  }
  if (finish_dots<2>(acc, 2, partial, ticket, s + 2, 0)) {
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      pcg_beta_step(s, active, mode, tol, max_iter, min_iter);
    }
  }
}

template <typename T>
bool pcg_update_impl(ReduceScratch& red, int NP, double* s, int* active, T* x, const T* p, const T* q, T* r, T* z,
                     const T* dinv, int64_t nb, int mode, double tol, int max_iter, int min_iter, cudaStream_t st) {
  if (NP != 4 && NP != 6 && NP != 10 && NP != 20) return false;
  if (nb == 0) return false;
  if (!red.grid) red.init();
  const int64_t tiles = (nb + 256 / NP - 1) / (256 / NP);
  // one full wave (8 CTAs of 256 threads per SM at 32 registers); more CTAs serialise on the reduction's ticket
  const int grid = (int)std::min<int64_t>(tiles, 2 * (int64_t)red.grid);
#define BSGPU_PCGU(N_)                                                                                          \
  pcg_update_kernel<T, N_><<<grid, 256, 0, st>>>(s, active, x, p, q, r, z, dinv, nb, red.partial.p, red.ticket.p, \
                                                 mode, tol, max_iter, min_iter)
  switch (NP) {
    case 4: BSGPU_PCGU(4); break;
    case 6: BSGPU_PCGU(6); break;
    case 10: BSGPU_PCGU(10); break;
    default: BSGPU_PCGU(20); break;
  }
#undef BSGPU_PCGU
  BSGPU_CHECK_LAUNCH();
  return true;
}

template <typename T>
void dots_impl(ReduceScratch& s, int K, const T* const* a, const T* const* b, int64_t n, double* out, int post,
               cudaStream_t st, const int* active) {
  require(K >= 1 && K <= kMaxDots, "dots: 1 <= K <= 16");
  if (!s.grid) s.init();
  DotArgs<T> args{};
  for (int k = 0; k < K; ++k) {
    args.a[k] = a[k];
    args.b[k] = b[k];
  }
  const int grid = s.grid;
  bool shared = true;
  for (int k = 0; k < K; ++k)
    shared = shared && b[k] == b[0] && (reinterpret_cast<uintptr_t>(a[k]) % 16 == 0);
  shared = shared && (reinterpret_cast<uintptr_t>(b[0]) % 16 == 0);
#define BSGPU_DOTS(KC)                                                                                        \
  do {                                                                                                        \
    if (shared)                                                                                               \
      dots_sharedb_kernel<T, KC><<<grid, kThreads, 0, st>>>(args, K, n, s.partial.p, s.ticket.p, out, post,   \
                                                            active);                                          \
    else                                                                                                      \
      dots_kernel<T, KC><<<grid, kThreads, 0, st>>>(args, K, n, s.partial.p, s.ticket.p, out, post, active);  \
  } while (0)
  if (K == 1)
    BSGPU_DOTS(1);
  else if (K == 2)
    BSGPU_DOTS(2);
  else if (K <= 4)
    BSGPU_DOTS(4);
  else if (K <= 8)
    BSGPU_DOTS(8);
  else
    BSGPU_DOTS(16);
#undef BSGPU_DOTS
  BSGPU_CHECK_LAUNCH();
}

constexpr int kMaxAxpy = 32;
template <typename T>
struct AxpyArgs {
  const T* x[kMaxAxpy];
  double hc[kMaxAxpy];
};

template <typename T>
__global__ void __launch_bounds__(kThreads) axpys_kernel(AxpyArgs<T> args, const double* __restrict__ dcoef, int K,
                                                         double sign, T* __restrict__ y, int64_t n,
                                                         const int* __restrict__ active) {
  if (active != nullptr && *active == 0) return;
  __shared__ double c[kMaxAxpy];
  if (threadIdx.x < K) c[threadIdx.x] = sign * (dcoef ? dcoef[threadIdx.x] : args.hc[threadIdx.x]);
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
    double acc = 0.0;
    for (int k = 0; k < K; ++k) acc = fma(c[k], (double)args.x[k][i], acc);
    y[i] = (T)((double)y[i] + acc);
  }
}

template <typename T>
void axpys_impl(int K, const double* dcoef, const double* hcoef, double sign, const T* const* x, T* y, int64_t n,
                cudaStream_t st, const int* active) {
  if (n == 0 || K == 0) return;
  const int grid = (int)std::min<int64_t>((n + kThreads - 1) / kThreads, (int64_t)num_sms() * 8);
  for (int k0 = 0; k0 < K; k0 += kMaxAxpy) {
    const int kc = std::min(kMaxAxpy, K - k0);
    AxpyArgs<T> args{};
    for (int k = 0; k < kc; ++k) {
      args.x[k] = x[k0 + k];
      args.hc[k] = hcoef ? hcoef[k0 + k] : 0.0;
    }
    axpys_kernel<T><<<grid, kThreads, 0, st>>>(args, dcoef ? dcoef + k0 : nullptr, kc, sign, y, n, active);
    BSGPU_CHECK_LAUNCH();
  }
}

// The same coefficients applied to two vector sets in one pass: y1 += sign*sum c_k x1_k, y2 += sign*sum c_k x2_k
// (the Gram-Schmidt update of a correction and of its image under the operator).
template <typename T>
struct Axpy2Args {
  const T* x1[kMaxAxpy];
  const T* x2[kMaxAxpy];
};

template <typename T>
__global__ void __launch_bounds__(kThreads) axpys2_kernel(Axpy2Args<T> args, const double* __restrict__ dcoef, int K,
                                                          double sign, T* __restrict__ y1, T* __restrict__ y2,
                                                          int64_t n) {
  __shared__ double c[kMaxAxpy];
  if (threadIdx.x < K) c[threadIdx.x] = sign * dcoef[threadIdx.x];
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += (int64_t)gridDim.x * kThreads) {
    double a1 = 0.0, a2 = 0.0;
    for (int k = 0; k < K; ++k) {
      a1 = fma(c[k], (double)args.x1[k][i], a1);
      a2 = fma(c[k], (double)args.x2[k][i], a2);
    }
    y1[i] = (T)((double)y1[i] + a1);
    y2[i] = (T)((double)y2[i] + a2);
  }
}

template <typename T>
void axpys2_impl(int K, const double* dcoef, double sign, const T* const* x1, T* y1, const T* const* x2, T* y2,
                 int64_t n, cudaStream_t st) {
  if (n == 0 || K == 0) return;
  const int grid = (int)std::min<int64_t>((n + kThreads - 1) / kThreads, (int64_t)num_sms() * 8);
  for (int k0 = 0; k0 < K; k0 += kMaxAxpy) {
    const int kc = std::min(kMaxAxpy, K - k0);
    Axpy2Args<T> args{};
    for (int k = 0; k < kc; ++k) {
      args.x1[k] = x1[k0 + k];
      args.x2[k] = x2[k0 + k];
    }
    axpys2_kernel<T><<<grid, kThreads, 0, st>>>(args, dcoef + k0, kc, sign, y1, y2, n);
    BSGPU_CHECK_LAUNCH();
  }
}

template <typename T>
__global__ void scale_inv2_kernel(const double* __restrict__ d, T* __restrict__ x, T* __restrict__ y, int64_t n,
                                  int* __restrict__ err, const int* __restrict__ active) {
  if (active != nullptr && *active == 0) return;
  const double v = d[0];
  if (!(v != 0.0) || !isfinite(v)) {
    if (blockIdx.x == 0 && threadIdx.x == 0 && err) *err = 1;
    return;
  }
  const double f = 1.0 / v;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    x[i] = (T)((double)x[i] * f);
    if (y) y[i] = (T)((double)y[i] * f);
  }
}

template <typename T>
__global__ void axpby_kernel(T alpha, const T* __restrict__ x, T beta, T* __restrict__ y, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = beta == T(0) ? alpha * x[i] : fma(alpha, x[i], beta * y[i]);
}

template <typename T>
__global__ void fill_kernel(T v, T* __restrict__ x, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = v;
}

template <typename TI, typename TO>
__global__ void convert_kernel(const TI* __restrict__ x, TO* __restrict__ y, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = (TO)x[i];
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

template <typename T>
__global__ void fill_random_kernel(T* __restrict__ x, int64_t n, uint64_t seed) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t h = splitmix64(seed * 0x100000001B3ull + (uint64_t)i);
    x[i] = (T)((double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0);
  }
}

template <typename T>
__global__ void gather_kernel(const T* __restrict__ full, T* __restrict__ sub, int64_t nsub, int Np, int keep,
                              const int64_t* __restrict__ map) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nsub; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t f = map ? map[t] : (t / keep) * Np + (t % keep);
    sub[t] = full[f];
  }
}

template <typename T>
__global__ void scatter_add_kernel(const T* __restrict__ sub, T* __restrict__ full, int64_t nsub, int Np, int keep,
                                   const int64_t* __restrict__ map) {
  for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nsub; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t f = map ? map[t] : (t / keep) * Np + (t % keep);
    full[f] += sub[t];
  }
}

__global__ void block_gemv_kernel(const double* __restrict__ M, const int64_t* __restrict__ moff,
                                  const int32_t* __restrict__ len, const int64_t* __restrict__ i0,
                                  const int32_t* __restrict__ row2blk, int uniformNp, int transpose,
                                  const double* __restrict__ x, double* __restrict__ y, int64_t N) {
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < N; g += (int64_t)gridDim.x * blockDim.x) {
    int64_t i, s0, o;
    int I;
    if (uniformNp > 0) {
      i = g / uniformNp;
      I = uniformNp;
      s0 = i * I;
      o = i * I * I;
    } else {
      i = row2blk[g];
      I = len[i];
      s0 = i0[i];
      o = moff[i];
    }
    const int r = (int)(g - s0);
    double s = 0.0;
    if (transpose)
      for (int c = 0; c < I; ++c) s = fma(M[o + (int64_t)c * I + r], x[s0 + c], s);
    else
      for (int c = 0; c < I; ++c) s = fma(M[o + (int64_t)r * I + c], x[s0 + c], s);
    y[g] = s;
  }
}

int elt_grid(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 8)); }

}  // namespace

void ReduceScratch::init() {
  grid = num_sms() * 4;
  partial.alloc((size_t)kMaxDots * grid);
  ticket.alloc(1);
  BSGPU_CUDA(cudaMemset(ticket.p, 0, sizeof(unsigned int)));
}

void dots(ReduceScratch& s, int K, const double* const* a, const double* const* b, int64_t n, double* out, int post,
          cudaStream_t st, const int* active) {
  dots_impl<double>(s, K, a, b, n, out, post, st, active);
}
void dots(ReduceScratch& s, int K, const float* const* a, const float* const* b, int64_t n, double* out, int post,
          cudaStream_t st, const int* active) {
  dots_impl<float>(s, K, a, b, n, out, post, st, active);
}
void axpys(int K, const double* dcoef, const double* hcoef, double sign, const double* const* x, double* y, int64_t n,
           cudaStream_t st, const int* active) {
  axpys_impl<double>(K, dcoef, hcoef, sign, x, y, n, st, active);
}
void axpys(int K, const double* dcoef, const double* hcoef, double sign, const float* const* x, float* y, int64_t n,
           cudaStream_t st, const int* active) {
  axpys_impl<float>(K, dcoef, hcoef, sign, x, y, n, st, active);
}
bool pcg_update(ReduceScratch& red, int NP, double* s, int* active, double* x, const double* p, const double* q,
                double* r, double* z, const double* dinv, int64_t nb, int mode, double tol, int max_iter,
                int min_iter, cudaStream_t st) {
  return pcg_update_impl<double>(red, NP, s, active, x, p, q, r, z, dinv, nb, mode, tol, max_iter, min_iter, st);
}
bool pcg_update(ReduceScratch& red, int NP, double* s, int* active, float* x, const float* p, const float* q,
                float* r, float* z, const float* dinv, int64_t nb, int mode, double tol, int max_iter, int min_iter,
                cudaStream_t st) {
  return pcg_update_impl<float>(red, NP, s, active, x, p, q, r, z, dinv, nb, mode, tol, max_iter, min_iter, st);
}
void axpys2(int K, const double* dcoef, double sign, const double* const* x1, double* y1, const double* const* x2,
            double* y2, int64_t n, cudaStream_t st) {
  axpys2_impl<double>(K, dcoef, sign, x1, y1, x2, y2, n, st);
}
void axpys2(int K, const double* dcoef, double sign, const float* const* x1, float* y1, const float* const* x2,
            float* y2, int64_t n, cudaStream_t st) {
  axpys2_impl<float>(K, dcoef, sign, x1, y1, x2, y2, n, st);
}
void scale_inv2(const double* d, double* x, double* y, int64_t n, int* err, cudaStream_t st, const int* active) {
  if (n == 0) return;
  scale_inv2_kernel<double><<<elt_grid(n), 256, 0, st>>>(d, x, y, n, err, active);
  BSGPU_CHECK_LAUNCH();
}
void scale_inv2(const double* d, float* x, float* y, int64_t n, int* err, cudaStream_t st, const int* active) {
  if (n == 0) return;
  scale_inv2_kernel<float><<<elt_grid(n), 256, 0, st>>>(d, x, y, n, err, active);
  BSGPU_CHECK_LAUNCH();
}
void axpby(double alpha, const double* x, double beta, double* y, int64_t n, cudaStream_t st) {
  if (n == 0) return;
  axpby_kernel<double><<<elt_grid(n), 256, 0, st>>>(alpha, x, beta, y, n);
  BSGPU_CHECK_LAUNCH();
}
void axpby(float alpha, const float* x, float beta, float* y, int64_t n, cudaStream_t st) {
  if (n == 0) return;
  axpby_kernel<float><<<elt_grid(n), 256, 0, st>>>(alpha, x, beta, y, n);
  BSGPU_CHECK_LAUNCH();
}
void fill(double v, double* x, int64_t n, cudaStream_t st) {
  if (n == 0) return;
  fill_kernel<double><<<elt_grid(n), 256, 0, st>>>(v, x, n);
  BSGPU_CHECK_LAUNCH();
}
void fill(float v, float* x, int64_t n, cudaStream_t st) {
  if (n == 0) return;
  fill_kernel<float><<<elt_grid(n), 256, 0, st>>>(v, x, n);
  BSGPU_CHECK_LAUNCH();
}
void convert(const double* x, float* y, int64_t n, cudaStream_t st) {
  if (n == 0) return;
  convert_kernel<double, float><<<elt_grid(n), 256, 0, st>>>(x, y, n);
  BSGPU_CHECK_LAUNCH();
}
void convert(const float* x, double* y, int64_t n, cudaStream_t st) {
  if (n == 0) return;
  convert_kernel<float, double><<<elt_grid(n), 256, 0, st>>>(x, y, n);
  BSGPU_CHECK_LAUNCH();
}
void fill_random(double* x, int64_t n, uint64_t seed, cudaStream_t st) {
  if (n == 0) return;
  fill_random_kernel<double><<<elt_grid(n), 256, 0, st>>>(x, n, seed);
  BSGPU_CHECK_LAUNCH();
}
void fill_random(float* x, int64_t n, uint64_t seed, cudaStream_t st) {
  if (n == 0) return;
  fill_random_kernel<float><<<elt_grid(n), 256, 0, st>>>(x, n, seed);
  BSGPU_CHECK_LAUNCH();
}
void restrict_gather(const double* full, double* sub, int64_t nsub, int Np, int keep, const int64_t* map,
                     cudaStream_t st) {
  if (nsub == 0) return;
  gather_kernel<double><<<elt_grid(nsub), 256, 0, st>>>(full, sub, nsub, Np, keep, map);
  BSGPU_CHECK_LAUNCH();
}
void restrict_gather(const float* full, float* sub, int64_t nsub, int Np, int keep, const int64_t* map,
                     cudaStream_t st) {
  if (nsub == 0) return;
  gather_kernel<float><<<elt_grid(nsub), 256, 0, st>>>(full, sub, nsub, Np, keep, map);
  BSGPU_CHECK_LAUNCH();
}
void restrict_scatter_add(const double* sub, double* full, int64_t nsub, int Np, int keep, const int64_t* map,
                          cudaStream_t st) {
  if (nsub == 0) return;
  scatter_add_kernel<double><<<elt_grid(nsub), 256, 0, st>>>(sub, full, nsub, Np, keep, map);
  BSGPU_CHECK_LAUNCH();
}
void restrict_scatter_add(const float* sub, float* full, int64_t nsub, int Np, int keep, const int64_t* map,
                          cudaStream_t st) {
  if (nsub == 0) return;
  scatter_add_kernel<float><<<elt_grid(nsub), 256, 0, st>>>(sub, full, nsub, Np, keep, map);
  BSGPU_CHECK_LAUNCH();
}
void block_gemv(const double* M, const int64_t* moff, const int32_t* len, const int64_t* i0, const int32_t* row2blk,
                int uniformNp, bool transpose, const double* x, double* y, int64_t N, cudaStream_t st) {
  if (N == 0) return;
  block_gemv_kernel<<<elt_grid(N), 256, 0, st>>>(M, moff, len, i0, row2blk, uniformNp, transpose ? 1 : 0, x, y, N);
  BSGPU_CHECK_LAUNCH();
}

}  // namespace bsgpu
