// Model-specialised CG product kernels: the saved product graph of one model
// emitted as straight-line CUDA (every moment and adjoint a named scalar, so
// they live in registers) and compiled at model load with NVRTC for sm_100a.
//
// The generated kernel does what k_product does for one centre atom per
// thread -- forward contraction, site energy, adjoint of the basic moments --
// with the rows scheduled so that each intermediate is produced right before
// its consumers and back-propagated as soon as its last consumer has run
// (short live ranges), terminal scalar rows fused into the energy, and every
// coefficient an immediate.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "mtp_model.h"

namespace sus2sh {

struct CgSource {
  std::string code;
  std::string kernel_name;
  long long fp_terms = 0;  // emitted multiply-add terms (size estimate)
};

// Emits the kernel source.  basic_canon[b] is the canonical [k*C + l*l+l+m]
// row of model basic b in the B/G arrays; ncanon = K*C.
CgSource generate_cg_source(const HostModel& m, const Layered& lay, bool use_float,
                            const std::vector<int>& basic_canon, int ncanon);

struct CgBinary {
  std::vector<char> cubin;
  std::string log;
  int registers = -1;  // parsed from the ptxas report, -1 if unknown
};

// NVRTC compile for sm_100a; throws InputError with the log on failure.
CgBinary compile_cg_source(const CgSource& src);

// Loaded module of a compiled kernel on the current device (driver API
// through cudaGetDriverEntryPoint, so the library needs no libcuda link).
class CgModule {
 public:
  CgModule() = default;
  ~CgModule();
  CgModule(const CgModule&) = delete;
  CgModule& operator=(const CgModule&) = delete;
  // Loads the cubin into the current context once; returns false on error.
  bool load(const CgBinary& bin, const std::string& kernel_name, std::string* err);
  bool loaded() const { return func_ != nullptr; }
  // Launches with params: N, pos4, B, G, shift, species, pe, pe_assign.
  bool launch(void* stream, int N, const void* pos4, const void* B, void* G, const double* shift,
              const double* species, double* pe, int pe_assign, std::string* err);

 private:
  void* module_ = nullptr;
  void* func_ = nullptr;
};

}  // namespace sus2sh
