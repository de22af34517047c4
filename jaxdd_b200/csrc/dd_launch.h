// Host-side helpers of the C ABI's entry points: the device check and the launch status.
#pragma once

#include <cuda_runtime.h>

#include "../../include/jaxdd_b200.h"

namespace dd {

// DD_OK when the current device is an sm_100 part (compute capability 10.x), DD_ERR_DEVICE when
// it is another part or there is no usable device. Reads attributes only. An error raised by
// the query itself is cleared so that it does not surface in the caller's next
// cudaGetLastError; an error the caller left pending is not touched when the query succeeds.
inline int device_status() {
  int dev = -1, major = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return DD_ERR_DEVICE;
  }
  if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) {
    cudaGetLastError();
    return DD_ERR_DEVICE;
  }
  return major == 10 ? DD_OK : DD_ERR_DEVICE;
}

// Launch `kernel` with the given arguments (each passed by reference, of the kernel's own
// parameter types) and return this launch's own status: cudaLaunchKernel returns the error of
// the launch it makes, so an error left by an earlier, unrelated call is neither reported as
// this launch's nor cleared.
template <typename... P, typename... A>
inline int launch(void (*kernel)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                  A&... args) {
  static_assert(sizeof...(P) == sizeof...(A), "one argument per kernel parameter");
  void* ptrs[] = {static_cast<void*>(&args)...};
  return cudaLaunchKernel(reinterpret_cast<const void*>(kernel), grid, block, ptrs, smem, s) ==
                 cudaSuccess
             ? DD_OK
             : DD_ERR_LAUNCH;
}

}  // namespace dd
