// Test infrastructure only (oracle): the gpu* aliases of GPUMD's portability
// header that the reference's SUS2-SH engine uses, mapped to the CUDA runtime.
#pragma once
#include <cuda_runtime.h>

#define gpuError_t cudaError_t
#define gpuSuccess cudaSuccess
#define gpuGetLastError cudaGetLastError
#define gpuGetErrorString cudaGetErrorString
#define gpuDeviceSynchronize cudaDeviceSynchronize
#define gpuMemset cudaMemset
#define gpuMemcpy cudaMemcpy
#define gpuMemcpyHostToDevice cudaMemcpyHostToDevice
#define gpuMemcpyDeviceToHost cudaMemcpyDeviceToHost
#define gpuMemcpyDeviceToDevice cudaMemcpyDeviceToDevice
