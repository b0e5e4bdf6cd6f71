// Test infrastructure only (oracle): a minimal stand-in for GPUMD's owning
// device array, with the members the reference's SUS2-SH engine and the
// engine's GPUMD shim call (resize, copy_from_host, copy_to_host, fill, data,
// size).  resize discards the
// contents, as GPUMD's does.  When gpumd_stub_host_memory() is set (the
// driver's loader-only mode) the storage is host memory, so the engine's
// constructor (model reading and graph set-up) runs without a GPU.
#pragma once
#include "error.cuh"
#include <cstddef>
#include <cstdlib>
#include <cstring>

template <typename T>
class GPU_Vector {
public:
  GPU_Vector() = default;
  explicit GPU_Vector(size_t n) { resize(n); }
  GPU_Vector(const GPU_Vector&) = delete;
  GPU_Vector& operator=(const GPU_Vector&) = delete;
  ~GPU_Vector() { release(); }

  void resize(size_t n) {
    if (n == size_ && data_) return;
    release();
    size_ = n;
    if (n == 0) return;
    host_ = gpumd_stub_host_memory();
    if (host_) data_ = static_cast<T*>(std::malloc(n * sizeof(T)));
    else CHECK(cudaMalloc(reinterpret_cast<void**>(&data_), n * sizeof(T)));
  }
  void copy_from_host(const T* h) { copy_from_host(h, size_); }
  void copy_from_host(const T* h, size_t n) {
    if (n == 0) return;
    if (host_) std::memcpy(data_, h, n * sizeof(T));
    else CHECK(cudaMemcpy(data_, h, n * sizeof(T), cudaMemcpyHostToDevice));
  }
  void copy_to_host(T* h) const { copy_to_host(h, size_); }
  void copy_to_host(T* h, size_t n) const {
    if (n == 0) return;
    if (host_) std::memcpy(h, data_, n * sizeof(T));
    else CHECK(cudaMemcpy(h, data_, n * sizeof(T), cudaMemcpyDeviceToHost));
  }
  // Sets every element to value (device arrays: a kernel on the default stream).
  void fill(T value);
  T* data() { return data_; }
  const T* data() const { return data_; }
  size_t size() const { return size_; }

private:
  void release() {
    if (data_) {
      if (host_) std::free(data_);
      else cudaFree(data_);
    }
    data_ = nullptr;
    size_ = 0;
  }
  T* data_ = nullptr;
  size_t size_ = 0;
  bool host_ = false;
};

#ifdef __CUDACC__
template <typename T>
__global__ void gpumd_stub_fill(T* p, size_t n, T value) {
  const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) p[i] = value;
}

template <typename T>
void GPU_Vector<T>::fill(T value) {
  if (size_ == 0) return;
  if (host_) {
    for (size_t i = 0; i < size_; ++i) data_[i] = value;
    return;
  }
  gpumd_stub_fill<T><<<static_cast<unsigned>((size_ + 255) / 256), 256>>>(data_, size_, value);
  CHECK(cudaGetLastError());
}
#endif
