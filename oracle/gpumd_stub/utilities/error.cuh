// Test infrastructure only (oracle): GPUMD's error macros as the reference's
// SUS2-SH engine uses them.  A failed CUDA call prints and exits, as GPUMD's
// do.  gpumd_stub_host_memory() is the driver's loader-only switch: while it
// is set, GPU_Vector keeps host memory and cudaMemcpyToSymbol (which the
// engine's constructor calls for some graph layouts) does nothing, so the
// constructor runs without a GPU.
#pragma once
#include "gpu_macro.cuh"
#include <cstdio>
#include <cstdlib>

inline bool& gpumd_stub_host_memory() {
  static bool host = false;
  return host;
}

#define CHECK(call)                                                                     \
  do {                                                                                  \
    const cudaError_t stub_err_ = (call);                                               \
    if (stub_err_ != cudaSuccess) {                                                     \
      std::printf("CUDA Error:\n    File: %s\n    Line: %d\n    Error text: %s\n",      \
                  __FILE__, __LINE__, cudaGetErrorString(stub_err_));                    \
      std::exit(1);                                                                     \
    }                                                                                   \
  } while (0)

#define GPU_CHECK_KERNEL { CHECK(cudaGetLastError()); }

#define PRINT_INPUT_ERROR(text)                                                         \
  do {                                                                                  \
    std::printf("Input Error:\n    File: %s\n    Line: %d\n    Error text: %s\n",        \
                __FILE__, __LINE__, text);                                              \
    std::exit(1);                                                                       \
  } while (0)

template <class Symbol>
cudaError_t gpumd_stub_memcpy_to_symbol(const Symbol& symbol, const void* src, size_t count, size_t offset = 0) {
  if (gpumd_stub_host_memory()) return cudaSuccess;
  return cudaMemcpyToSymbol(symbol, src, count, offset, cudaMemcpyHostToDevice);
}
#define cudaMemcpyToSymbol gpumd_stub_memcpy_to_symbol
