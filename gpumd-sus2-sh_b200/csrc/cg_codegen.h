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
  std::string code;                // the whole program as one translation unit
  std::vector<std::string> units;  // split kernels: the same program as separately
                                   // compiled units (kernel first), linked by nvJitLink
  std::string kernel_name;
  long long fp_terms = 0;  // emitted multiply-add terms (size estimate)
  // launch shape: threads per CTA (lane = atom) and dynamic shared memory
  int block = 128;
  size_t smem_bytes = 0;
  bool split = false;      // component-split kernel (generate_cg_split_source)
  int functions = 1;       // device functions in the program
  int components = 0;      // independent components (split kernels)
  // straight-line kernels only: the same contraction as a device function
  // sus2sh::batch::cg_atom(const T (&B)[ncanon], T (&G)[ncanon], T sc) ->
  // sum of the weighted moments, on the normalised basics B and writing
  // G = sc * dE/dB (canonical order), for the fused batch kernel
  std::string device_fn;
};

// Device helpers at the head of every generated kernel: sus2_pol() (an L2
// evict-first cache policy), sus2_ld(p, pol) and sus2_st(p, v, pol) for the
// basic moments read and their adjoints written, so that these streams do not
// evict the kernel's own code from L2 (see edge::l2_evict_first).  Defined for
// the device compiler only.
extern const char* const kCgStreamHelpers;

// Emits the kernel source.  basic_canon[b] is the canonical [k*C + l*l+l+m]
// row of model basic b in the B/G arrays; ncanon = K*C.
CgSource generate_cg_source(const HostModel& m, const Layered& lay, bool use_float,
                            const std::vector<int>& basic_canon, int ncanon);

// Component-split kernel for graphs too large for one straight-line
// function: the local intermediates (those feeding terminal scalar rows only)
// are grouped into the connected components of the terminal terms, each
// evaluated by its own __noinline__ function with its values in registers;
// basic moments, shared intermediates and all their adjoints live in
// lane-private shared memory.  Same kernel parameters as
// generate_cg_source.  Returns false with the reason in *why when the graph
// does not split into components of at most 160 values or its shared-memory
// slots do not fit.
bool generate_cg_split_source(const HostModel& m, const Layered& lay, bool use_float,
                              const std::vector<int>& basic_canon, int ncanon, CgSource* out,
                              std::string* why);

// Forward-over-reverse (dual-number) version of generate_cg_source for the
// parameter gradients.  Kernel parameters: N, pos4, B, Bd (basic tangents),
// species, ew (dL/dE_i, may be NULL), Galpha, Gbeta ([K*C][N] outputs:
// c_t (ew a - b) and c_t a) and contrib ([scalar_count][N]:
// c_t (ew M_s - dM_s), summed over atoms into dL/dw_s by the caller).
CgSource generate_pg_source(const HostModel& m, const Layered& lay, bool use_float,
                            const std::vector<int>& basic_canon, int ncanon);

struct CgBinary {
  std::vector<char> cubin;
  std::string log;
  int registers = -1;      // parsed from the ptxas report, -1 if unknown
  bool whole = false;      // compiled as one program (every device function with its callers)
  bool from_disk = false;  // read from the on-disk cache of whole-program builds
};

// How a component-split kernel is compiled.  The straight-line kernels are
// always one program.
//  * kWhole: the whole source as one NVRTC program.  ptxas then sees every
//    device function together with the kernel that calls it and gives the
//    calls no ABI (no callee-saved registers spilled to the stack around
//    each call): on the l4k4 body-5 graph the cubin is 2.31 MB instead of
//    3.67 MB and the kernel, bound by instruction fetch, runs 3.07 instead of
//    3.77 ms on 262,144 atoms (the same results, bit for bit).  The compile
//    is one thread (about 70 s for that graph), so its result is kept on
//    disk (cg_cache_dir) and later loads of the same kernel read it back
//    (every one-program build, straight-line kernels included, goes through
//    that cache).
//  * kParallel: the units compiled in parallel threads as relocatable code
//    and joined by nvJitLink (about 8 s for that graph).
enum class CgBuild { kParallel, kWhole };

// NVRTC compile for sm_100a; cached per process by source and build.  Throws
// InputError with the log on failure.
CgBinary compile_cg_source(const CgSource& src, CgBuild build = CgBuild::kWhole);

// Directory of the on-disk cache of whole-program builds: $SUS2SH_CACHE_DIR
// ("" or "off" disables the cache), else $XDG_CACHE_HOME/sus2sh, else
// $HOME/.cache/sus2sh; "" when there is none.
std::string cg_cache_dir();

// Loaded module of a compiled kernel on the current device (driver API
// through cudaGetDriverEntryPoint, so the library needs no libcuda link).
class CgModule {
 public:
  CgModule() = default;
  ~CgModule();
  CgModule(const CgModule&) = delete;
  CgModule& operator=(const CgModule&) = delete;
  // Loads the cubin into the current context once (and raises the kernel's
  // dynamic shared-memory limit to smem_bytes); returns false on error.
  bool load(const CgBinary& bin, const std::string& kernel_name, std::string* err, size_t smem_bytes = 0);
  bool loaded() const { return func_ != nullptr; }
  // Registers per thread and local memory (spill + stack) bytes per thread of
  // the loaded kernel, call tree included (-1 before load).
  int registers() const { return regs_; }
  int local_bytes() const { return local_; }
  // Resident CTAs per SM of the loaded kernel at this CTA size and dynamic
  // shared memory (0 on error).
  int max_active_blocks(int block, size_t smem_bytes) const;
  // Launches with an explicit parameter array.
  bool launch_args(void* stream, unsigned grid, unsigned block, size_t smem_bytes, void** args, std::string* err);
  // Launches with params: N, pos4, B, G, shift, species, pe, pe_assign, on
  // ceil(N / block) CTAs of `block` threads with smem_bytes dynamic shared memory.
  bool launch(void* stream, int N, const void* pos4, const void* B, void* G, const double* shift,
              const double* species, double* pe, int pe_assign, std::string* err, int block = 128,
              size_t smem_bytes = 0);

 private:
  void* module_ = nullptr;
  void* func_ = nullptr;
  int regs_ = -1, local_ = -1;
};

}  // namespace sus2sh
