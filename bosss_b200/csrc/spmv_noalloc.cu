// Host-vector SpMV that allocates no device memory.
//
// bsgpu_matrix_spmv copies x and y through device buffers it obtains with cudaMalloc on every call.  Some
// callers cannot have that: a host program that has handed the GPU's memory to its own pool (or runs under a
// hard device-memory budget) must not see the library grow its footprint, and cudaMalloc/cudaFree may
// synchronise the whole device, which a caller on a latency-critical path cannot afford.  This variant stages x
// and y in one file-scope __device__ array instead.  That array is part of the module image: once the library's
// module is loaded on a GPU (at its first use there under CUDA's default lazy loading), that GPU holds the array
// (2 x 8 MiB) until the process exits, whether or not this entry point is ever called.  The device address is
// cached per device ordinal, so resetting a device's primary context (cudaDeviceReset) invalidates this entry
// point on that device for the rest of the process, as it invalidates every matrix handle.
#include <map>
#include <mutex>
#include <new>

#include "matrix.cuh"

namespace bsgpu {
const Matrix* matrix_from_handle(bsgpu_matrix_t A);
}

namespace {

// Largest number of rows (unknowns) the staging array can hold: x and y, FP64 each.
constexpr int64_t kNoAllocMaxRows = int64_t(1) << 20;

static __device__ __align__(256) double g_spmv_stage[2 * kNoAllocMaxRows];

// In host code g_spmv_stage only names a host-side stand-in of the array; a kernel handed that name would read
// the wrong memory.  The device address is looked up once per device (with that device current) and cached.
std::mutex g_stage_mutex;
std::map<int, double*> g_stage_addr;

double* stage_on_current_device() {
  int dev = 0;
  BSGPU_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(g_stage_mutex);
  auto it = g_stage_addr.find(dev);
  if (it != g_stage_addr.end()) return it->second;
  double* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_spmv_stage);
  if (e != cudaSuccess)
    throw bsgpu::Error(BSGPU_ERR_CUDA, std::string("cudaGetSymbolAddress(staging array): ") + cudaGetErrorString(e));
  g_stage_addr[dev] = p;
  return p;
}

}  // namespace

extern "C" BSGPU_API int bsgpu_matrix_spmv_noalloc(bsgpu_matrix_t A, double alpha, const double* x, double beta,
                                                   double* y) {
  try {
    const bsgpu::Matrix* M = bsgpu::matrix_from_handle(A);
    bsgpu::require(M != nullptr && x != nullptr && y != nullptr, "null argument");
    bsgpu::require(x != y, "In-Place computation is not supported.");
    bsgpu::require(!M->single, "FP64 matrices only");
    bsgpu::require(M->N <= kNoAllocMaxRows,
                   "bsgpu_matrix_spmv_noalloc: the matrix has " + std::to_string(M->N) +
                       " rows; the staging array holds at most " + std::to_string(kNoAllocMaxRows) +
                       " (use bsgpu_matrix_spmv)");
    if (M->N == 0) return BSGPU_OK;
    double* stage = stage_on_current_device();
    double* dx = stage;
    double* dy = stage + kNoAllocMaxRows;
    // The staging array keeps the previous call's contents; nothing in it has to start at zero: x is copied in
    // in full and y is either copied in (beta != 0) or not read (beta == 0).
    BSGPU_CUDA(cudaMemcpy(dx, x, M->N * sizeof(double), cudaMemcpyHostToDevice));
    if (beta != 0.0) BSGPU_CUDA(cudaMemcpy(dy, y, M->N * sizeof(double), cudaMemcpyHostToDevice));
    bsgpu::spmv(*M, alpha, dx, beta, beta != 0.0 ? dy : nullptr, dy, nullptr);
    BSGPU_CUDA(cudaMemcpy(y, dy, M->N * sizeof(double), cudaMemcpyDeviceToHost));
    return BSGPU_OK;
  } catch (const bsgpu::Error& e) {
    bsgpu::set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    bsgpu::set_last_error("host allocation failed");
    return BSGPU_ERR_NOMEM;
  } catch (const std::exception& e) {
    bsgpu::set_last_error(e.what());
    return BSGPU_ERR_ARGUMENT;
  }
}
