// Grid reductions in one launch: per-CTA sums into a scratch array, the last CTA to arrive (threadfence + atomic
// ticket) adds the partials in a fixed order, so a result does not depend on CTA scheduling.  256-thread CTAs.
#pragma once
#include "common.cuh"

namespace bsgpu {
namespace gridred {

constexpr int kRedThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Second half of every grid reduction: per-CTA sums of the K accumulators into `partial`, and the last CTA to
// arrive (threadfence + atomic ticket) adds the partials in a fixed order, so the result does not depend on CTA
// scheduling.
template <int KC>
__device__ __forceinline__ bool finish_dots(const double (&acc)[KC], int K, double* __restrict__ partial,
                                            unsigned int* __restrict__ ticket, double* __restrict__ out, int post) {
  __shared__ double red[kRedThreads / 32][KC];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < KC; ++k) {
    double v = warp_sum(acc[k]);
    if (lane == 0) red[warp][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < K) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kRedThreads / 32; ++w) s += red[w][threadIdx.x];
    partial[(int64_t)threadIdx.x * gridDim.x + blockIdx.x] = s;
  }
  __threadfence();
  __syncthreads();
  __shared__ bool last;
  if (threadIdx.x == 0) last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return false;
  __threadfence();
  for (int k = 0; k < K; ++k) {
    double s = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += kRedThreads) s += __ldcg(partial + (int64_t)k * gridDim.x + b);
    s = warp_sum(s);
    __syncthreads();
    if (lane == 0) red[warp][0] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kRedThreads / 32; ++w) t += red[w][0];
      out[k] = post == 1 ? sqrt(t) : t;
    }
  }
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

}  // namespace gridred
}  // namespace bsgpu
