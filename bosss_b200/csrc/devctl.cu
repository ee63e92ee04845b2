// Device-side control flow of the graph-captured V-cycle (see devctl.cuh).
#include <algorithm>

#include "devctl.cuh"

namespace bsgpu {

namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 16;        // history vectors per chunk of the multi-dot
constexpr int kProducts = kChunk + 1;  // + the self product |m|^2

__device__ bool term_continue(const TermParams& t, int iter, double R0, double R) {
  const double eps = 2.2204460492503131e-16 * 1000;  // IterativeSolverConfig.MachineEpsilon
  if (t.mode == 2) return iter <= t.max_iter;
  if (t.mode == 3) {
    if (iter <= 1) return true;
    if (R < R0 * t.reduction) return false;
    if (iter > t.max_iter) return false;
    return true;
  }
  if (iter <= t.min_iter) return true;
  const bool ok = (t.mode == 0) ? (R < R0 * t.tol + t.tol) : (R < R0 * t.tol);
  if (ok) return false;
  if (iter > t.max_iter) return false;
  if (R0 < eps || R < eps) return false;
  return true;
}

// Term::operator() (solvers.cu) on the device: returns "continue", writes "converged".
__device__ bool term_eval(const TermParams& t, int iter, double R0, double R, bool* conv) {
  const double eps = 2.2204460492503131e-16 * 1000;
  *conv = false;
  if (t.mode == 2) {
    *conv = true;
    return iter <= t.max_iter;
  }
  if (t.mode == 3) {
    if (iter <= 1) return true;
    if (R < R0 * t.reduction) {
      *conv = true;
      return false;
    }
    return iter <= t.max_iter;
  }
  if (iter <= t.min_iter) return true;
  const bool ok = (t.mode == 0) ? (R < R0 * t.tol + t.tol) : (R < R0 * t.tol);
  if (ok) {
    *conv = true;
    return false;
  }
  if (iter > t.max_iter) return false;
  if (R0 < eps || R < eps) {
    *conv = true;
    return false;
  }
  return true;
}

__global__ void cond_set_kernel(cudaGraphConditionalHandle h, const int* a, const int* not_b, const int* k, int cap,
                                unsigned int* exec) {
  bool v = true;
  if (a != nullptr) v = v && (*a != 0);
  if (not_b != nullptr) v = v && (*not_b == 0);
  if (k != nullptr) v = v && (*k < cap);
  cudaGraphSetConditional(h, v ? 1u : 0u);
  if (v && exec != nullptr) *exec += 1u;
}

__global__ void positive_flag_kernel(const double* x, int* flag) { *flag = (*x > 0.0) ? 1 : 0; }

template <typename T> struct V16;
template <> struct V16<float> { using type = float4; static constexpr int W = 4; };
template <> struct V16<double> { using type = double2; static constexpr int W = 2; };

__device__ __forceinline__ double vdot(const float4& a, const float4& b) {
  return (double)a.x * b.x + (double)a.y * b.y + (double)a.z * b.z + (double)a.w * b.w;
}
__device__ __forceinline__ double vdot(const double2& a, const double2& b) { return fma(a.x, b.x, a.y * b.y); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Chunk blockIdx.y of the history (vectors 16*y .. 16*y+15 below *k) against m; chunk 0 also forms |m|^2.  Every
// CTA writes its per-product sums to `partial`; the last CTA of the chunk (atomic ticket) adds them in a fixed
// order.  Chunks with nothing to do return before touching the ticket (the decision is the same in all their CTAs).
template <typename T>
__global__ void __launch_bounds__(kThreads) hist_dots_kernel(const T* const* __restrict__ hist,
                                                             const int* __restrict__ kp, int kmax,
                                                             const T* __restrict__ m, int64_t n,
                                                             double* __restrict__ beta, double* __restrict__ self,
                                                             double* __restrict__ partial,
                                                             unsigned int* __restrict__ ticket) {
  using V = typename V16<T>::type;
  constexpr int W = V16<T>::W;
  const int k = min(*kp, kmax);
  const int j0 = blockIdx.y * kChunk;
  const int K = max(0, min(kChunk, k - j0));
  const bool do_self = self != nullptr && blockIdx.y == 0;
  if (K == 0 && !do_self) return;
  __shared__ const T* ptr[kChunk];
  if (threadIdx.x < K) ptr[threadIdx.x] = hist[j0 + threadIdx.x];
  __syncthreads();
  double acc[kProducts];
#pragma unroll
  for (int q = 0; q < kProducts; ++q) acc[q] = 0.0;
  const int64_t nv = n / W;
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  const V* mv = reinterpret_cast<const V*>(m);
  for (int64_t j = (int64_t)blockIdx.x * kThreads + threadIdx.x; j < nv; j += stride) {
    const V bb = __ldg(mv + j);
#pragma unroll
    for (int q = 0; q < kChunk; ++q)
      if (q < K) acc[q] += vdot(__ldcs(reinterpret_cast<const V*>(ptr[q]) + j), bb);
    if (do_self) acc[kChunk] += vdot(bb, bb);
  }
  for (int64_t i = nv * W + (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += stride) {
    const double b = (double)m[i];
#pragma unroll
    for (int q = 0; q < kChunk; ++q)
      if (q < K) acc[q] = fma((double)ptr[q][i], b, acc[q]);
    if (do_self) acc[kChunk] = fma(b, b, acc[kChunk]);
  }
  __shared__ double red[kThreads / 32][kProducts];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < kProducts; ++q) {
    const double v = warp_sum(acc[q]);
    if (lane == 0) red[warp][q] = v;
  }
  __syncthreads();
  const int64_t G = gridDim.x;
  double* part = partial + (int64_t)blockIdx.y * kProducts * G;
  if (threadIdx.x < kProducts) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) s += red[w][threadIdx.x];
    part[(int64_t)threadIdx.x * G + blockIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  __shared__ bool last;
  if (threadIdx.x == 0) last = (atomicAdd(ticket + blockIdx.y, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  // one warp per product, fixed summation order
  for (int q = warp; q < kProducts; q += kThreads / 32) {
    const bool wanted = (q < K) || (q == kChunk && do_self);
    if (!wanted) continue;
    double s = 0.0;
    for (int64_t b = lane; b < G; b += 32) s += __ldcg(part + (int64_t)q * G + b);
    s = warp_sum(s);
    if (lane == 0) {
      if (q < K)
        beta[j0 + q] = s;
      else
        *self = s;
    }
  }
  if (threadIdx.x == 0) ticket[blockIdx.y] = 0u;
}

template <typename T>
__global__ void __launch_bounds__(kThreads) hist_axpy2_kernel(const T* const* __restrict__ x1,
                                                              const T* const* __restrict__ x2,
                                                              const int* __restrict__ kp, int kmax,
                                                              const double* __restrict__ beta, T* __restrict__ y1,
                                                              T* __restrict__ y2, int64_t n) {
  using V = typename V16<T>::type;
  constexpr int W = V16<T>::W;
  const int k = min(*kp, min(kmax, kHistMax));
  if (k <= 0) return;
  __shared__ const T* p1[kHistMax];
  __shared__ const T* p2[kHistMax];
  __shared__ double c[kHistMax];
  for (int j = threadIdx.x; j < k; j += kThreads) {
    p1[j] = x1[j];
    p2[j] = x2[j];
    c[j] = beta[j];
  }
  __syncthreads();
  const int64_t nv = n / W;
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < nv; i += stride) {
    double a1[W], a2[W];
#pragma unroll
    for (int w = 0; w < W; ++w) a1[w] = a2[w] = 0.0;
    for (int j = 0; j < k; ++j) {
      const V u = __ldcs(reinterpret_cast<const V*>(p1[j]) + i);
      const V v = __ldcs(reinterpret_cast<const V*>(p2[j]) + i);
      const T* uu = reinterpret_cast<const T*>(&u);
      const T* vv = reinterpret_cast<const T*>(&v);
#pragma unroll
      for (int w = 0; w < W; ++w) {
        a1[w] = fma(c[j], (double)uu[w], a1[w]);
        a2[w] = fma(c[j], (double)vv[w], a2[w]);
      }
    }
    V o1 = reinterpret_cast<V*>(y1)[i];
    V o2 = reinterpret_cast<V*>(y2)[i];
    T* oo1 = reinterpret_cast<T*>(&o1);
    T* oo2 = reinterpret_cast<T*>(&o2);
#pragma unroll
    for (int w = 0; w < W; ++w) {
      oo1[w] = (T)((double)oo1[w] - a1[w]);
      oo2[w] = (T)((double)oo2[w] - a2[w]);
    }
    reinterpret_cast<V*>(y1)[i] = o1;
    reinterpret_cast<V*>(y2)[i] = o2;
  }
  for (int64_t i = nv * W + (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += stride) {
    double a1 = 0.0, a2 = 0.0;
    for (int j = 0; j < k; ++j) {
      a1 = fma(c[j], (double)p1[j][i], a1);
      a2 = fma(c[j], (double)p2[j][i], a2);
    }
    y1[i] = (T)((double)y1[i] - a1);
    y2[i] = (T)((double)y2[i] - a2);
  }
}

// After the first projection sweep: the norm of the correction's image before (nM) and after it, relative (rel),
// and whether a second sweep restores orthogonality (1e-5 < rel < 0.5, "twice is enough"; the cancellation bound
// 1e-5 of OrthonormalizationMultigrid.cs:263-337).  With an empty history there is nothing to project and rel = 1.
__global__ void ortho_decide1_kernel(OrthoState* s, const double* proj, int* err) {
  const double nM = sqrt(proj[1]);
  if (!isfinite(nM) || !isfinite(proj[0])) {
    atomicOr(err, kDevErrNaN);
    s->nM = 0.0;
    s->rel = 0.0;
    s->second = 0;
    return;
  }
  s->nM = nM;
  s->rel = nM > 0.0 ? proj[0] / nM : 0.0;
  s->second = (s->k > 0 && nM > 0.0 && s->rel > 1e-5 && s->rel < 0.5) ? 1 : 0;
}

__global__ void ortho_decide2_kernel(OrthoState* s, const double* proj) {
  s->rel = s->nM > 0.0 ? proj[0] / s->nM : 0.0;
}

// The correction is kept, normalised by its projected image norm, unless nothing independent of the history is
// left in it (rel <= 1e-5, or a zero correction); then it is dropped (stored as zero, which projects and minimises
// to nothing) and the level's post-smoothing loop ends, as after the reference's cancellation branch.
__global__ void ortho_final_kernel(OrthoState* s, const double* proj) {
  const bool keep = s->nM > 0.0 && s->rel > 1e-5 && proj[0] > 0.0;
  s->fac = keep ? 1.0 / proj[0] : 0.0;
  s->cancel = keep ? 0 : 1;
}

template <typename T>
__global__ void ortho_store_kernel(const OrthoState* __restrict__ s, T* __restrict__ W, T* __restrict__ MW,
                                   T* const* __restrict__ sol, T* const* __restrict__ mxx, int nslots, int64_t n,
                                   int* __restrict__ err) {
  const int k = s->k;
  if (k < 0 || k >= nslots) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(err, kDevErrSlots);
    return;
  }
  const double f = s->fac;
  T* S = sol[k];
  T* M = mxx[k];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const T w = (T)((double)W[i] * f);
    const T mw = (T)((double)MW[i] * f);
    W[i] = w;
    MW[i] = mw;
    S[i] = w;
    M[i] = mw;
  }
}

// RecalcResiPeriod (OrthonormalizationMultigrid.cs:179-190): recompute after a cancellation or every `period`
// history entries, else update.
__global__ void ortho_advance_kernel(OrthoState* s, int period, int nslots) {
  s->k = min(s->k + 1, nslots);
  const bool rec = period <= 1 || s->cancel != 0 || (s->k % period) == 0;
  s->recalc = rec ? 1 : 0;
  s->update = rec ? 0 : 1;
}

// MinimizeResidual's checks (OrthonormalizationMultigrid.cs:192-209): NaN and residual increase raise in the
// reference; here they set the error word (the host raises after the graph) and stop the level.
__global__ void minimize_check_kernel(OrthoState* s, const double* rn_new, TermParams tp, int* err) {
  const double rn = *rn_new;
  const double old = s->rn;
  s->rn = rn;
  if (!isfinite(rn)) {
    atomicOr(err, kDevErrNaN);
    s->active = 0;
    return;
  }
  const double tol = fmax(fmax(rn, old) * 0.2, 1.0e-7);
  if (rn > old + tol) {
    atomicOr(err, kDevErrResidualIncrease);
    s->active = 0;
    return;
  }
  if (s->active) s->active = term_continue(tp, s->iter, s->r0, rn) ? 1 : 0;
}

__global__ void level_begin_kernel(OrthoState* s, const double* r0_in, TermParams tp) {
  const double r0 = *r0_in;
  s->k = 0;
  s->cancel = 0;
  s->second = 0;
  s->recalc = 1;
  s->update = 0;
  s->restart = 0;
  s->iter = 1;
  s->iterations = 0;
  s->r0 = r0;
  s->rn = r0;
  s->active = (isfinite(r0) && term_continue(tp, 1, r0, r0)) ? 1 : 0;
}

__global__ void iter_begin_kernel(OrthoState* s, int cap) {
  s->restart = s->k >= cap ? 1 : 0;
  if (s->restart) s->k = 0;
  s->cancel = 0;
}

__global__ void iter_end_kernel(OrthoState* s, TermParams tp) {
  if (s->active) {
    s->iterations += 1;
    s->iter += 1;
    // the termination test ends every loop by its iteration limit; the hard bound keeps a recorded WHILE node
    // finite whatever the parameters
    s->active = (term_continue(tp, s->iter, s->r0, s->rn) && s->iter <= kMaxRecordedIterations) ? 1 : 0;
  }
}

template <typename T>
__global__ void copy_if_kernel(const T* __restrict__ x, T* __restrict__ y, int64_t n, const int* __restrict__ flag) {
  if (*flag == 0) return;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = x[i];
}

// ---- recorded FlexGMRES (FlexGMRES.cs:144-277) ----

__global__ void fg_begin_kernel(FgState* s, int nn_active, int has2) {
  s->j = 0;
  s->k1 = 1;
  s->kk = 0;
  s->iter = 0;
  s->outer = 0;
  s->inner = 0;
  s->use2 = 0;
  s->nn_active = nn_active;
  s->turn = 0;
  s->converged = 0;
  s->nhist = 0;
  s->stalled = 0;
  s->started = 0;
  s->has2 = has2;
  s->zero = 0;
  s->r0 = 0.0;
  s->est = 0.0;
  s->g_before = 0.0;
  s->inv = 0.0;
}

// The residual test at the top of every restart cycle (FlexGMRES.cs:168-182).
__global__ void fg_restart_kernel(FgState* s, FgArrays a, const double* rn, TermParams tp, int* err) {
  const double r = *rn;
  s->inner = 0;
  if (*err != 0) {  // an error raised inside the preconditioner ends the solve (the host raises it)
    s->outer = 0;
    return;
  }
  if (!isfinite(r)) {
    atomicOr(err, kDevErrKrylovNaN);
    s->outer = 0;
    return;
  }
  if (!s->started) {
    s->r0 = r;
    s->started = 1;
  }
  if (s->nhist < a.hcap) a.hist[s->nhist++] = r;
  bool conv = false;
  const bool cont = term_eval(tp, s->iter, s->r0, r, &conv) && s->iter < kMaxRecordedIterations;
  if (!cont) {
    s->converged = conv ? 1 : 0;
    s->outer = 0;
    return;
  }
  s->outer = 1;
  s->inner = 1;
  s->inv = r > 0.0 ? 1.0 / r : 0.0;
  a.g[0] = r;
  for (int i = 1; i <= a.m; ++i) a.g[i] = 0.0;
  s->j = 0;
  s->k1 = 1;
}

// Round-robin of the preconditioners (FlexGMRES.cs:196-199): every second step uses the second one while it is
// active.
__global__ void fg_step_begin_kernel(FgState* s, FgArrays a) {
  const int j = s->j;
  s->k1 = j + 1;
  s->use2 = (s->has2 && s->nn_active && (s->turn % 2 == 1)) ? 1 : 0;
  s->turn += 1;
  s->g_before = fabs(a.g[j]);
}

__global__ void fg_step_end_kernel(FgState* s, FgArrays a, const double* h1, const double* h2, const double* wn_p,
                                   TermParams tp, double stall, int* err) {
  const int j = s->j, m = a.m;
  const double wn = *wn_p;
  s->iter += 1;
  if (!isfinite(wn)) {
    atomicOr(err, kDevErrKrylovNaN);
    s->inner = 0;
    s->outer = 0;
    s->kk = 0;
    s->inv = 0.0;
    return;
  }
  double* H = a.H;
  for (int i = 0; i <= j; ++i) H[i * m + j] = h1[i] + h2[i];
  H[(j + 1) * m + j] = wn;
  s->inv = wn > 0.0 ? 1.0 / wn : 0.0;
  for (int i = 0; i < j; ++i) {
    const double a0 = H[i * m + j], b0 = H[(i + 1) * m + j];
    H[i * m + j] = a.cs[i] * a0 + a.sn[i] * b0;
    H[(i + 1) * m + j] = -a.sn[i] * a0 + a.cs[i] * b0;
  }
  const double a0 = H[j * m + j], b0 = H[(j + 1) * m + j];
  const double den = hypot(a0, b0);
  a.cs[j] = a0 / den;
  a.sn[j] = b0 / den;
  H[j * m + j] = den;
  H[(j + 1) * m + j] = 0.0;
  a.g[j + 1] = -a.sn[j] * a.g[j];
  a.g[j] = a.cs[j] * a.g[j];
  const double est = fabs(a.g[j + 1]);
  s->est = est;
  if (s->nhist < a.hcap) a.hist[s->nhist++] = est;
  if (s->use2 && est > stall * s->g_before) {
    s->nn_active = 0;  // the second preconditioner stalls: the first one for the rest of this solve
    s->stalled = 1;
  }
  bool conv = false;
  const bool cont = term_eval(tp, s->iter, s->r0, est, &conv);
  const bool stop = !cont || conv || wn == 0.0 || s->iter >= kMaxRecordedIterations || *err != 0;
  s->j = j + 1;
  s->kk = j + 1;
  s->inner = (!stop && j + 1 < m) ? 1 : 0;
}

__global__ void fg_backsub_kernel(FgState* s, FgArrays a) {
  const int kk = s->kk, m = a.m;
  for (int i = kk - 1; i >= 0; --i) {
    double v = a.g[i];
    for (int q = i + 1; q < kk; ++q) v += a.H[i * m + q] * a.ny[q];  // ny = -y
    a.ny[i] = -(v / a.H[i * m + i]);
  }
}

__global__ void slot_load_kernel(const double* const* __restrict__ tab, const int* __restrict__ idx,
                                 double* __restrict__ out, int64_t n) {
  const double* x = tab[idx ? *idx : 0];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = x[i];
}

__global__ void slot_store_kernel(const double* __restrict__ x, const double* __restrict__ scale,
                                  double* const* __restrict__ tab, const int* __restrict__ idx, int nslots, int64_t n,
                                  int* __restrict__ err) {
  const int k = idx ? *idx : 0;
  if (k < 0 || k >= nslots) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(err, kDevErrSlots);
    return;
  }
  const double f = scale ? *scale : 1.0;
  double* y = tab[k];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = x[i] * f;
}

// y -= sum_{j<k} beta[j] x[j] (FP64, one vector)
__global__ void __launch_bounds__(kThreads) hist_axpy1_kernel(const double* const* __restrict__ x,
                                                              const int* __restrict__ kp, int kmax,
                                                              const double* __restrict__ beta,
                                                              double* __restrict__ y, int64_t n) {
  const int k = min(*kp, min(kmax, kHistMax));
  if (k <= 0) return;
  __shared__ const double* p[kHistMax];
  __shared__ double c[kHistMax];
  for (int j = threadIdx.x; j < k; j += kThreads) {
    p[j] = x[j];
    c[j] = beta[j];
  }
  __syncthreads();
  const int64_t nv = n / 2;
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  for (int64_t i = (int64_t)blockIdx.x * kThreads + threadIdx.x; i < nv; i += stride) {
    double a0 = 0.0, a1 = 0.0;
    for (int j = 0; j < k; ++j) {
      const double2 u = __ldcs(reinterpret_cast<const double2*>(p[j]) + i);
      a0 = fma(c[j], u.x, a0);
      a1 = fma(c[j], u.y, a1);
    }
    double2 o = reinterpret_cast<double2*>(y)[i];
    o.x -= a0;
    o.y -= a1;
    reinterpret_cast<double2*>(y)[i] = o;
  }
  for (int64_t i = nv * 2 + (int64_t)blockIdx.x * kThreads + threadIdx.x; i < n; i += stride) {
    double a0 = 0.0;
    for (int j = 0; j < k; ++j) a0 = fma(c[j], p[j][i], a0);
    y[i] -= a0;
  }
}

__global__ void batch_copy_kernel(const double* const* __restrict__ src, double* const* __restrict__ dst,
                                  const int64_t* __restrict__ len, int count) {
  for (int b = blockIdx.y; b < count; b += gridDim.y) {
    const double* x = src[b];
    double* y = dst[b];
    const int64_t n = len[b];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      y[i] = x[i];
  }
}

int grid_for(int64_t n_work) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n_work + kThreads - 1) / kThreads, (int64_t)num_sms() * 2));
}

template <typename T>
void hist_dots_impl(HistScratch& s, const T* const* hist, const int* k, const T* m, int64_t n, double* beta,
                    double* self, cudaStream_t st) {
  require(s.chunks > 0, "history multi-dot: scratch not initialised");
  const int W = 16 / (int)sizeof(T);
  const int G = std::min(grid_for(std::max<int64_t>(n / W, 1)), s.grid);
  require((reinterpret_cast<uintptr_t>(m) & 15) == 0, "history multi-dot: unaligned vector");
  hist_dots_kernel<T><<<dim3(G, s.chunks), kThreads, 0, st>>>(hist, k, s.chunks * kChunk > s.slots ? s.slots : s.chunks * kChunk,
                                                                m, n, beta, self, s.partial.p, s.ticket.p);
  BSGPU_CHECK_LAUNCH();
}

template <typename T>
void hist_axpy2_impl(const T* const* x1, const T* const* x2, const int* k, int kmax, const double* beta, T* y1, T* y2,
                     int64_t n, cudaStream_t st) {
  const int W = 16 / (int)sizeof(T);
  require((reinterpret_cast<uintptr_t>(y1) & 15) == 0 && (reinterpret_cast<uintptr_t>(y2) & 15) == 0,
          "history multi-axpy: unaligned vector");
  require(kmax >= 1 && kmax <= kHistMax, "history multi-axpy: 1 <= slots <= 128");
  hist_axpy2_kernel<T><<<grid_for(std::max<int64_t>(n / W, 1)) * 2, kThreads, 0, st>>>(x1, x2, k, kmax, beta, y1, y2,
                                                                                       n);
  BSGPU_CHECK_LAUNCH();
}

template <typename T>
void store_impl(OrthoState* s, T* W, T* MW, T* const* sol, T* const* mxx, int nslots, int64_t n, int* err,
                cudaStream_t st) {
  ortho_store_kernel<T><<<grid_for(n) * 4, kThreads, 0, st>>>(s, W, MW, sol, mxx, nslots, n, err);
  BSGPU_CHECK_LAUNCH();
}

template <typename T>
void copy_if_impl(const T* x, T* y, int64_t n, const int* flag, cudaStream_t st) {
  copy_if_kernel<T><<<grid_for(n) * 4, kThreads, 0, st>>>(x, y, n, flag);
  BSGPU_CHECK_LAUNCH();
}

}  // namespace

void HistScratch::init(int cap) {
  require(cap >= 1 && cap <= kHistMax, "history length must be in 1..128");
  slots = cap;
  chunks = (cap + kChunk - 1) / kChunk;
  grid = num_sms() * 2;
  partial.alloc((size_t)chunks * kProducts * grid);
  ticket.alloc(chunks);
  BSGPU_CUDA(cudaMemset(ticket.p, 0, chunks * sizeof(unsigned int)));
}

void cond_set(cudaGraphConditionalHandle h, const int* a, const int* not_b, const int* k, int cap, unsigned int* exec,
              cudaStream_t st) {
  cond_set_kernel<<<1, 1, 0, st>>>(h, a, not_b, k, cap, exec);
  BSGPU_CHECK_LAUNCH();
}

void positive_flag(const double* x, int* flag, cudaStream_t st) {
  positive_flag_kernel<<<1, 1, 0, st>>>(x, flag);
  BSGPU_CHECK_LAUNCH();
}

void hist_dots(HistScratch& s, const double* const* hist, const int* k, const double* m, int64_t n, double* beta,
               double* self, cudaStream_t st) {
  hist_dots_impl<double>(s, hist, k, m, n, beta, self, st);
}
void hist_dots(HistScratch& s, const float* const* hist, const int* k, const float* m, int64_t n, double* beta,
               double* self, cudaStream_t st) {
  hist_dots_impl<float>(s, hist, k, m, n, beta, self, st);
}
void hist_axpy2(const double* const* x1, const double* const* x2, const int* k, int kmax, const double* beta,
                double* y1, double* y2, int64_t n, cudaStream_t st) {
  hist_axpy2_impl<double>(x1, x2, k, kmax, beta, y1, y2, n, st);
}
void hist_axpy2(const float* const* x1, const float* const* x2, const int* k, int kmax, const double* beta, float* y1,
                float* y2, int64_t n, cudaStream_t st) {
  hist_axpy2_impl<float>(x1, x2, k, kmax, beta, y1, y2, n, st);
}

void ortho_decide1(OrthoState* s, const double* proj, int* err, cudaStream_t st) {
  ortho_decide1_kernel<<<1, 1, 0, st>>>(s, proj, err);
  BSGPU_CHECK_LAUNCH();
}
void ortho_decide2(OrthoState* s, const double* proj, cudaStream_t st) {
  ortho_decide2_kernel<<<1, 1, 0, st>>>(s, proj);
  BSGPU_CHECK_LAUNCH();
}
void ortho_final(OrthoState* s, const double* proj, cudaStream_t st) {
  ortho_final_kernel<<<1, 1, 0, st>>>(s, proj);
  BSGPU_CHECK_LAUNCH();
}
void ortho_store(OrthoState* s, double* W, double* MW, double* const* sol, double* const* mxx, int nslots, int64_t n,
                 int* err, cudaStream_t st) {
  store_impl<double>(s, W, MW, sol, mxx, nslots, n, err, st);
}
void ortho_store(OrthoState* s, float* W, float* MW, float* const* sol, float* const* mxx, int nslots, int64_t n,
                 int* err, cudaStream_t st) {
  store_impl<float>(s, W, MW, sol, mxx, nslots, n, err, st);
}
void ortho_advance(OrthoState* s, int period, int nslots, cudaStream_t st) {
  ortho_advance_kernel<<<1, 1, 0, st>>>(s, period, nslots);
  BSGPU_CHECK_LAUNCH();
}
void minimize_check(OrthoState* s, const double* rn_new, TermParams tp, int* err, cudaStream_t st) {
  minimize_check_kernel<<<1, 1, 0, st>>>(s, rn_new, tp, err);
  BSGPU_CHECK_LAUNCH();
}
void level_begin(OrthoState* s, const double* r0_in, TermParams tp, cudaStream_t st) {
  level_begin_kernel<<<1, 1, 0, st>>>(s, r0_in, tp);
  BSGPU_CHECK_LAUNCH();
}
void iter_begin(OrthoState* s, int cap, cudaStream_t st) {
  iter_begin_kernel<<<1, 1, 0, st>>>(s, cap);
  BSGPU_CHECK_LAUNCH();
}
void iter_end(OrthoState* s, TermParams tp, cudaStream_t st) {
  iter_end_kernel<<<1, 1, 0, st>>>(s, tp);
  BSGPU_CHECK_LAUNCH();
}
void copy_if(const double* x, double* y, int64_t n, const int* flag, cudaStream_t st) {
  copy_if_impl<double>(x, y, n, flag, st);
}
void copy_if(const float* x, float* y, int64_t n, const int* flag, cudaStream_t st) {
  copy_if_impl<float>(x, y, n, flag, st);
}


void hist_axpy1(const double* const* x, const int* k, int kmax, const double* beta, double* y, int64_t n,
                cudaStream_t st) {
  require((reinterpret_cast<uintptr_t>(y) & 15) == 0, "history multi-axpy: unaligned vector");
  require(kmax >= 1 && kmax <= kHistMax, "history multi-axpy: 1 <= slots <= 128");
  hist_axpy1_kernel<<<grid_for(std::max<int64_t>(n / 2, 1)) * 2, kThreads, 0, st>>>(x, k, kmax, beta, y, n);
  BSGPU_CHECK_LAUNCH();
}

void fg_begin(FgState* s, int nn_active, int has2, cudaStream_t st) {
  fg_begin_kernel<<<1, 1, 0, st>>>(s, nn_active, has2);
  BSGPU_CHECK_LAUNCH();
}
void fg_restart(FgState* s, FgArrays a, const double* rn, TermParams tp, int* err, cudaStream_t st) {
  fg_restart_kernel<<<1, 1, 0, st>>>(s, a, rn, tp, err);
  BSGPU_CHECK_LAUNCH();
}
void fg_step_begin(FgState* s, FgArrays a, cudaStream_t st) {
  fg_step_begin_kernel<<<1, 1, 0, st>>>(s, a);
  BSGPU_CHECK_LAUNCH();
}
void fg_step_end(FgState* s, FgArrays a, const double* h1, const double* h2, const double* wn, TermParams tp,
                 double stall, int* err, cudaStream_t st) {
  fg_step_end_kernel<<<1, 1, 0, st>>>(s, a, h1, h2, wn, tp, stall, err);
  BSGPU_CHECK_LAUNCH();
}
void fg_backsub(FgState* s, FgArrays a, cudaStream_t st) {
  fg_backsub_kernel<<<1, 1, 0, st>>>(s, a);
  BSGPU_CHECK_LAUNCH();
}
void slot_load(const double* const* tab, const int* idx, double* out, int64_t n, cudaStream_t st) {
  slot_load_kernel<<<grid_for(n) * 4, kThreads, 0, st>>>(tab, idx, out, n);
  BSGPU_CHECK_LAUNCH();
}
void slot_store(const double* x, const double* scale, double* const* tab, const int* idx, int nslots, int64_t n,
                int* err, cudaStream_t st) {
  slot_store_kernel<<<grid_for(n) * 4, kThreads, 0, st>>>(x, scale, tab, idx, nslots, n, err);
  BSGPU_CHECK_LAUNCH();
}

void batch_copy(const double* const* src, double* const* dst, const int64_t* n, int count, cudaStream_t st) {
  if (count <= 0) return;
  batch_copy_kernel<<<dim3(32, std::min(count, 65535)), kThreads, 0, st>>>(src, dst, n, count);
  BSGPU_CHECK_LAUNCH();
}

}  // namespace bsgpu
