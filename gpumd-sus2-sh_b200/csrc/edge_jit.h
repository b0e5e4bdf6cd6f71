// Per-edge kernels (k_basic, k_force of edge_kernels.cuh) compiled with NVRTC
// for sm_100a when the model is loaded, for any shape the model format allows
// (sh_l_max <= 6, radial_funcs_count <= 48, radial_basis_size <= 16).  The
// ahead-of-time library covers the common shapes; this covers the rest with
// the same kernel templates, so every model the reference loads runs.
#pragma once

#include <memory>
#include <string>
#include <vector>

namespace sus2sh {

struct EdgeJitBinary {
  std::vector<char> cubin;
  std::string basic_name, force_name;  // lowered (mangled) kernel names
  std::string basic_gate_name, force_gate_name;  // GATE variants (gate models only)
  std::string log;                     // NVRTC + ptxas report
  int basic_registers = -1, force_registers = -1;
  double compile_ms = 0.0;
};

// Compiles k_basic<T, L, K, RB, BLOCK> and k_force<...> (T = float if fp32,
// else double), and their GATE variants when gate is set.  Results are cached for the life of the process; throws
// InputError with the compiler log on failure.
std::shared_ptr<const EdgeJitBinary> compile_edge_kernels(bool fp32, int l_max, int k_max, int rb, int block,
                                                          bool gate);

// Module of one compiled shape, loaded into the current context.
class EdgeJitModule {
 public:
  EdgeJitModule() = default;
  ~EdgeJitModule();
  EdgeJitModule(const EdgeJitModule&) = delete;
  EdgeJitModule& operator=(const EdgeJitModule&) = delete;
  bool load(const EdgeJitBinary& bin, std::string* err);
  bool loaded() const { return basic_ != nullptr; }
  // args: pointer to the host EdgeArgs<T> passed by value to the kernel.
  bool launch_basic(void* stream, int N, int block, size_t smem, const void* args, void* B, bool gate,
                    std::string* err);
  bool launch_force(void* stream, int N, int block, size_t smem, const void* args, const void* G,
                    const double* weight, void* ftmp, double* force, double* virial, double sign, bool gate,
                    std::string* err);

 private:
  bool set_smem(void* fn, size_t smem, int* have, std::string* err);
  void* module_ = nullptr;
  void* basic_ = nullptr;
  void* force_ = nullptr;
  void* basic_gate_ = nullptr;
  void* force_gate_ = nullptr;
  int basic_smem_ = 48 * 1024, force_smem_ = 48 * 1024, basic_gate_smem_ = 48 * 1024,
      force_gate_smem_ = 48 * 1024;
};

}  // namespace sus2sh
