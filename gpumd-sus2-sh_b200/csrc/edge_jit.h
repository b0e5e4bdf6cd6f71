// Per-edge kernels (k_basic, k_force of edge_kernels.cuh) compiled with NVRTC
// for sm_100a when the model is loaded:
//  * for any shape the model format allows (sh_l_max <= 6, radial_funcs_count
//    <= 48, radial_basis_size <= 16): the ahead-of-time library covers the
//    common shapes, this covers the rest with the same kernel templates, so
//    every model the reference loads runs;
//  * specialised to one FP32 model: the radial coefficients and their
//    derivative series compiled in, so each is an immediate operand of its
//    multiply-add instead of a constant load per edge.
#pragma once

#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace sus2sh {

struct EdgeJitBinary {
  std::vector<std::vector<char>> cubins;              // one per NVRTC program
  std::vector<int> blocks;                            // CTA sizes compiled
  std::vector<std::string> basic_names, force_names;  // lowered (mangled) names, one per CTA size
  std::vector<int> basic_cubin, force_cubin;          // the cubin holding each of them
  std::string basic_gate_name, force_gate_name;       // GATE variants (gate models only, 128 threads, cubin 0)
  std::string log;                                    // NVRTC + ptxas report
  int basic_registers = -1, force_registers = -1;     // of the first CTA size
  long long global_bytes = -1;                        // module data in global memory ("bytes gmem")
  bool model_coef = false;                            // coefficients compiled in
  double compile_ms = 0.0;
};

// Compiles k_basic<T, L, K, RB, BLOCK> and k_force<...> (T = float if fp32,
// else double), and their GATE variants when gate is set, for the Chebyshev
// radial kinds (read at run time) or, with radial_kind = kRadialLaguerre, for
// the Laguerre basis.  Results are cached for the life of the process; throws
// InputError with the compiler log on failure.
std::shared_ptr<const EdgeJitBinary> compile_edge_kernels(bool fp32, int l_max, int k_max, int rb, int block,
                                                          bool gate, int radial_kind = 0);

// FP32 k_basic / k_force of one model at 64, 128 and 256 threads per CTA,
// with `coef` (the kernels' coefficient table: c[mu][n], then the derivative
// series when it fits, as EdgeArgs::coef holds them), whether the radial
// functions of a pair share one argument, and the radial basis kind compiled in:
// six NVRTC programs built on parallel host threads.  Cached per process by
// shape, table and radial setup.
std::shared_ptr<const EdgeJitBinary> compile_model_edge_kernels(int l_max, int k_max, int rb,
                                                                const std::vector<float>& coef, bool shared_xi,
                                                                int radial_kind);

// The fused batch kernel k_batch_fused<L, K, RB, BLOCK, MIN_BLOCKS>
// (batch_fused.cuh) of one FP32 model: the radial coefficients, shared-
// argument flag and radial kind compiled in as for
// compile_model_edge_kernels, and cg_fn, the model's straight-line CG
// contraction as a device function (CgSource::device_fn).  One NVRTC program
// with a kernel per (BLOCK, MIN_BLOCKS) variant; cached per process by its
// source.
struct FusedJitBinary {
  std::vector<char> cubin;
  std::vector<std::string> names;  // lowered kernel names, one per variant
  std::vector<int> blocks, min_blocks, registers;
  std::string log;
  double compile_ms = 0.0;
};
std::shared_ptr<const FusedJitBinary> compile_batch_fused(int l_max, int k_max, int rb, const std::vector<float>& coef,
                                                          bool shared_xi, int radial_kind, const std::string& cg_fn,
                                                          const std::vector<std::pair<int, int>>& variants);

// Module of one compiled shape, loaded into the current context.
class EdgeJitModule {
 public:
  EdgeJitModule() = default;
  ~EdgeJitModule();
  EdgeJitModule(const EdgeJitModule&) = delete;
  EdgeJitModule& operator=(const EdgeJitModule&) = delete;
  bool load(const EdgeJitBinary& bin, std::string* err);
  bool loaded() const { return !modules_.empty(); }
  // args: pointer to the host EdgeArgs<T> passed by value to the kernel;
  // block: a CTA size the binary was compiled for (gate variants: 128).
  bool launch_basic(void* stream, int N, int block, size_t smem, const void* args, void* B, bool gate,
                    std::string* err);
  bool launch_force(void* stream, int N, int block, size_t smem, const void* args, const void* G,
                    const double* weight, void* ftmp, double* force, double* virial, double sign, bool gate,
                    std::string* err);

 private:
  struct Fn {
    void* fn = nullptr;
    int smem = 48 * 1024;  // dynamic shared memory the function is opted into
  };
  Fn* find(bool force, bool gate, int block);
  bool set_smem(Fn& f, size_t smem, std::string* err);
  bool launch(Fn* f, const char* what, void* stream, int N, int block, size_t smem, void** params, std::string* err);
  std::vector<void*> modules_;
  std::vector<int> blocks_;
  std::vector<Fn> basic_, force_;
  Fn basic_gate_, force_gate_;
};

}  // namespace sus2sh
