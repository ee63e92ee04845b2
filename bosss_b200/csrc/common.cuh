// Shared helpers of the bsgpu library: status handling, CUDA error checks, device buffers.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/bsgpu.h"

namespace bsgpu {

// Exception carrying a bsgpu status code; converted to an int at the C boundary.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string& msg);

#define BSGPU_CUDA(call)                                                                             \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess) {                                                                         \
      if (e_ == cudaErrorMemoryAllocation)                                                           \
        throw ::bsgpu::Error(BSGPU_ERR_NOMEM, std::string(#call) + ": " + cudaGetErrorString(e_));    \
      throw ::bsgpu::Error(BSGPU_ERR_CUDA,                                                           \
                           std::string(__FILE__) + ":" + std::to_string(__LINE__) + " " + #call + ": " + \
                               cudaGetErrorString(e_));                                              \
    }                                                                                                \
  } while (0)

// Every kernel launch of the library is followed by this check, which also counts the launch (the count is
// exposed through bsgpu_get_launch_count for tracing).
void count_launch();
// Adjusts the counter for graph capture (kernels recorded into a graph run when the graph is replayed).
void add_launches(long long n);
unsigned long long launches_now();
#define BSGPU_CHECK_LAUNCH()          \
  do {                                \
    BSGPU_CUDA(cudaGetLastError());   \
    ::bsgpu::count_launch();          \
  } while (0)

inline void require(bool cond, const std::string& msg, int code = BSGPU_ERR_ARGUMENT) {
  if (!cond) throw Error(code, msg);
}

// Owning device buffer (cudaMalloc / cudaFree).
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  explicit DBuf(size_t count) { alloc(count); }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
    return *this;
  }
  ~DBuf() { release(); }
  void alloc(size_t count) {
    release();
    if (count) BSGPU_CUDA(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return n * sizeof(T); }
};

inline int num_sms() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms > 0 ? sms : 148;
}

inline cudaMemcpyKind kind_from_flags(int32_t flags) {
  return flags == BSGPU_DEVICE_POINTERS ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
}

}  // namespace bsgpu
