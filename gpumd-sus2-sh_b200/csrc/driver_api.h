// CUDA driver entry points through the runtime's cudaGetDriverEntryPoint, so
// the library loads NVRTC-built modules without linking libcuda.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

namespace sus2sh {
namespace drv {

using PFN_load = CUresult (*)(CUmodule*, const void*);
using PFN_get = CUresult (*)(CUfunction*, CUmodule, const char*);
using PFN_launch = CUresult (*)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                                CUstream, void**, void**);
using PFN_unload = CUresult (*)(CUmodule);
using PFN_set_attr = CUresult (*)(CUfunction, CUfunction_attribute, int);
using PFN_get_attr = CUresult (*)(int*, CUfunction_attribute, CUfunction);

template <typename F>
F entry(const char* name) {
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint(name, &fn, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
    return nullptr;
  return reinterpret_cast<F>(fn);
}

}  // namespace drv
}  // namespace sus2sh
