// sus2sh_cg_energy_noalloc: the CG product graph (forward, site energy,
// adjoint) on caller-provided basic moments, allocating no device memory.
//
// Why it exists: some callers cannot call cudaMalloc at the moment they need
// the contraction.  MD codes that reserve all device memory up front in their
// own pools forbid allocations during a run (a cudaMalloc there can fail
// once the pool holds the GPU's memory, and it bypasses their accounting);
// real-time loops cannot take the device-wide synchronisation an allocation
// or free may imply.  The handle's model tables are created once by
// sus2sh_create; this entry point then needs only the caller's input/output
// arrays plus the fixed work area below.
//
// The work area (the per-atom value/adjoint slots of the CG program, laid out
// [slot][N]) is one file-scope __device__ array of kNoAllocScratchBytes
// (16 MiB).  Every GPU that loads this library holds it until the process
// exits.  All calls share it, so calls that overlap on the GPU (different
// streams, or different host threads) race and must be serialised by the
// caller.  The kernel zeroes the adjoint slots it uses itself; leftover
// contents of earlier calls are never read.
#include "../../include/sus2sh.h"
#include "engine.cuh"

#include <mutex>
#include <string>

namespace sus2sh {

// Program tables of a handle (defined next to the handle in capi.cu).
bool cg_view(const sus2sh_handle* h, CgView* out);
void set_last_error(const std::string& msg);

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_cg_scratch[kNoAllocScratchBytes];

namespace {

// Host-side device address of g_cg_scratch per device.  In host code the
// symbol g_cg_scratch is only a host stand-in, never a device address.
std::mutex g_scratch_mutex;
void* g_scratch_addr[kMaxDevices] = {};

// Same row machine as the engine's HBM-slot product kernel, reading the
// species from `type` and the basics from `B` in the model's
// alpha_index_basic order, writing the adjoints in that order.
template <typename T>
__global__ void __launch_bounds__(128)
    k_cg_noalloc(int N, const ProgramDev p, const int* __restrict__ type, const T* __restrict__ B,
                 T* __restrict__ G, T* __restrict__ scratch, const double* __restrict__ shift_coeffs,
                 const double* __restrict__ species_coeffs, int species, double* __restrict__ pe) {
  const int atom = blockIdx.x * blockDim.x + threadIdx.x;
  if (atom >= N) return;
  T* S = scratch + atom;
  const size_t stride = static_cast<size_t>(N);
  const int gofs = p.nvalue;
  for (int b = 0; b < p.nbasic; ++b) S[b * stride] = B[static_cast<size_t>(b) * N + atom];
  for (int v = 0; v < p.nvalue; ++v) S[(gofs + v) * stride] = T(0);
  const uint32_t* __restrict__ code = p.code;
  const T* __restrict__ cf = reinterpret_cast<const T*>(p.coef);
  double E = 0.0;
  for (int r = 0; r < p.nrows; ++r) {
    const uint32_t h = __ldg(code++);
    const int kind = h >> 30;
    const int nt = (h >> 16) & 0x3FFF;
    const int dst = h & 0xFFFF;
    if (kind == 0) {
      T acc = T(0);
      for (int t = 0; t < nt; ++t) {
        const uint32_t w = __ldg(code + t);
        acc = fma(__ldg(cf + t) * S[(w & 0xFFFF) * stride], S[(w >> 16) * stride], acc);
      }
      S[dst * stride] = acc;
    } else if (kind == 1) {
      T acc = T(0);
      for (int t = 0; t < nt; ++t) {
        const uint32_t w = __ldg(code + t);
        const int ia = w & 0xFFFF, ib = w >> 16;
        const T c = __ldg(cf + t);
        const T va = S[ia * stride], vb = S[ib * stride];
        acc = fma(c * va, vb, acc);
        S[(gofs + ia) * stride] += c * vb;
        S[(gofs + ib) * stride] += c * va;
      }
      E += static_cast<double>(acc);
    } else if (kind == 2) {
      const int ia = __ldg(code) & 0xFFFF;
      const T c = __ldg(cf);
      E += static_cast<double>(c * S[ia * stride]);
      S[(gofs + ia) * stride] += c;
    } else {
      T acc = T(0);
      for (int t = 0; t < nt; ++t) {
        const uint32_t w = __ldg(code + t);
        acc = fma(__ldg(cf + t) * S[(gofs + (w & 0xFFFF)) * stride], S[(w >> 16) * stride], acc);
      }
      S[(gofs + dst) * stride] += acc;
    }
    code += nt;
    cf += nt;
  }
  const int ti = type[atom];
  if (ti < 0 || ti >= species) {
    // A species outside the model: the atom's energy and adjoints are NaN, so
    // the caller sees the bad input instead of another species' numbers.
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    pe[atom] = nan;
    for (int b = 0; b < p.nbasic; ++b) G[static_cast<size_t>(b) * N + atom] = static_cast<T>(nan);
    return;
  }
  const double ct = species_coeffs[ti];
  pe[atom] = shift_coeffs[ti] + ct + ct * E;
  const T sc = static_cast<T>(ct);
  for (int b = 0; b < p.nbasic; ++b) G[static_cast<size_t>(b) * N + atom] = sc * S[(gofs + b) * stride];
}

}  // namespace
}  // namespace sus2sh

extern "C" int sus2sh_cg_energy_noalloc(const sus2sh_handle* h, int N, const int* type, const void* basics,
                                        double* potential, void* basic_adjoint, void* stream) {
  using namespace sus2sh;
  CgView v;
  if (!h || !type || !basics || !potential || !basic_adjoint || N <= 0 || !cg_view(h, &v)) {
    set_last_error("sus2sh_cg_energy_noalloc: invalid argument");
    return SUS2SH_E_ARG;
  }
  const size_t elem = v.use_float ? sizeof(float) : sizeof(double);
  const size_t need = 2ull * static_cast<size_t>(v.prog.nvalue) * static_cast<size_t>(N) * elem;
  if (need > kNoAllocScratchBytes) {
    set_last_error("sus2sh_cg_energy_noalloc: N=" + std::to_string(N) + " needs " + std::to_string(need) +
                   " bytes of work area; the fixed maximum is " + std::to_string(kNoAllocScratchBytes) +
                   " bytes (N <= " + std::to_string(kNoAllocScratchBytes / (2ull * v.prog.nvalue * elem)) +
                   " for this model and precision)");
    return SUS2SH_E_ARG;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    set_last_error("sus2sh_cg_energy_noalloc: no usable current device");
    return SUS2SH_E_CUDA;
  }
  if (dev != v.device) {
    // the model tables live on the handle's device; the work area and the
    // launch would be on the current one
    set_last_error("sus2sh_cg_energy_noalloc: the current device (" + std::to_string(dev) +
                   ") is not the device the handle was created on (" + std::to_string(v.device) + ")");
    return SUS2SH_E_ARG;
  }
  void* scratch = nullptr;
  {
    // First call on each device: resolve the device address of the array
    // with that device current.
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      const cudaError_t rc = cudaGetSymbolAddress(&p, g_cg_scratch);
      if (rc != cudaSuccess || !p) {
        set_last_error(std::string("sus2sh_cg_energy_noalloc: cudaGetSymbolAddress failed: ") +
                       cudaGetErrorString(rc));
        return SUS2SH_E_CUDA;
      }
      g_scratch_addr[dev] = p;
    }
    scratch = g_scratch_addr[dev];
  }
  // cudaLaunchKernelEx returns this launch's own status; an error the caller
  // left pending from earlier work stays pending for the caller to read.
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((N + 127) / 128);
  cfg.blockDim = dim3(128);
  cfg.stream = static_cast<cudaStream_t>(stream);
  cudaError_t rc;
  if (v.use_float) {
    rc = cudaLaunchKernelEx(&cfg, k_cg_noalloc<float>, N, v.prog, type, static_cast<const float*>(basics),
                            static_cast<float*>(basic_adjoint), static_cast<float*>(scratch), v.shift, v.species,
                            v.species_count, potential);
  } else {
    rc = cudaLaunchKernelEx(&cfg, k_cg_noalloc<double>, N, v.prog, type, static_cast<const double*>(basics),
                            static_cast<double*>(basic_adjoint), static_cast<double*>(scratch), v.shift,
                            v.species, v.species_count, potential);
  }
  if (rc != cudaSuccess) {
    set_last_error(std::string("sus2sh_cg_energy_noalloc: launch failed: ") + cudaGetErrorString(rc));
    return SUS2SH_E_CUDA;
  }
  return SUS2SH_OK;
}
