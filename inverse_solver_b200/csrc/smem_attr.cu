// The dynamic shared-memory limit of the tile kernels, raised once per
// (kernel, device) to the device's opt-in maximum.  Setting the limit to each
// launch's own size, as a per-launch call would, races when two host threads
// (two solvers of different grids in the request loop) launch the same
// kernel with different sizes: one lowers the limit between the other's
// setting and its launch, which then fails.
#include <cuda_runtime.h>

#include <mutex>
#include <set>
#include <utility>

#include "cbs_kernels.cuh"

namespace odt {

cudaError_t raise_smem_limit(const void* kernel, size_t bytes) {
  if (bytes <= 48 * 1024) return cudaSuccess;
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int optin = 0;
  e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  if (bytes > (size_t)optin) return cudaErrorInvalidValue;
  std::lock_guard<std::mutex> lk(mu);
  if (done.count({kernel, dev})) return cudaSuccess;
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
  if (e == cudaSuccess) done.insert({kernel, dev});
  return e;
}

}  // namespace odt
