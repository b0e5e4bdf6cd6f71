// NVRTC build of the per-edge kernels for model shapes without an
// ahead-of-time instantiation.
#include "edge_jit.h"

#include <nvrtc.h>

#include <chrono>
#include <cstdlib>
#include <map>
#include <mutex>

#include "driver_api.h"
#include "mtp_model.h"

namespace sus2sh {
namespace {

#include "edge_jit_sources.inc"

std::string shape_key(bool fp32, int l, int k, int rb, int block, bool gate) {
  return std::string(fp32 ? "f" : "d") + "/" + std::to_string(l) + "/" + std::to_string(k) + "/" +
         std::to_string(rb) + "/" + std::to_string(block) + (gate ? "/gate" : "");
}

// "Used N registers" following "Compiling entry function '<name>'" in the
// ptxas report.
int registers_of(const std::string& log, const std::string& name) {
  const size_t p = log.find("Compiling entry function '" + name + "'");
  if (p == std::string::npos) return -1;
  const size_t u = log.find("Used ", p);
  if (u == std::string::npos) return -1;
  return std::atoi(log.c_str() + u + 5);
}

std::shared_ptr<const EdgeJitBinary> build(bool fp32, int l, int k, int rb, int block, bool gate) {
  const auto t0 = std::chrono::steady_clock::now();
  const std::string T = fp32 ? "float" : "double";
  const std::string targs = "<" + T + ", " + std::to_string(l) + ", " + std::to_string(k) + ", " +
                            std::to_string(rb) + ", " + std::to_string(block) + ">";
  const std::string basic_expr = "&sus2sh::edge::k_basic" + targs;
  const std::string force_expr = "&sus2sh::edge::k_force" + targs;
  const std::string gargs = "<" + T + ", " + std::to_string(l) + ", " + std::to_string(k) + ", " +
                            std::to_string(rb) + ", 128, true>";
  const std::string basic_gate_expr = "&sus2sh::edge::k_basic" + gargs;
  const std::string force_gate_expr = "&sus2sh::edge::k_force" + gargs;
  const char* src = "#include \"edge_kernels.cuh\"\n";
  nvrtcProgram prog;
  if (nvrtcCreateProgram(&prog, src, "sus2sh_edge.cu", kJitHeaderCount, kJitHeaderSources, kJitHeaderNames) !=
      NVRTC_SUCCESS)
    throw InputError("NVRTC could not create the edge-kernel program.");
  nvrtcAddNameExpression(prog, basic_expr.c_str());
  nvrtcAddNameExpression(prog, force_expr.c_str());
  if (gate) {
    nvrtcAddNameExpression(prog, basic_gate_expr.c_str());
    nvrtcAddNameExpression(prog, force_gate_expr.c_str());
  }
  const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "--fmad=true", "--ptxas-options=--verbose",
                        "--generate-line-info"};
  const nvrtcResult rc = nvrtcCompileProgram(prog, 5, opts);
  auto out = std::make_shared<EdgeJitBinary>();
  size_t log_size = 0;
  nvrtcGetProgramLogSize(prog, &log_size);
  if (log_size > 1) {
    out->log.resize(log_size);
    nvrtcGetProgramLog(prog, &out->log[0]);
  }
  if (rc != NVRTC_SUCCESS) {
    nvrtcDestroyProgram(&prog);
    throw InputError("NVRTC failed to compile the edge kernels (" + targs + "): " + out->log.substr(0, 2000));
  }
  const char* lowered = nullptr;
  nvrtcGetLoweredName(prog, basic_expr.c_str(), &lowered);
  out->basic_name = lowered ? lowered : "";
  lowered = nullptr;
  nvrtcGetLoweredName(prog, force_expr.c_str(), &lowered);
  out->force_name = lowered ? lowered : "";
  if (gate) {
    lowered = nullptr;
    nvrtcGetLoweredName(prog, basic_gate_expr.c_str(), &lowered);
    out->basic_gate_name = lowered ? lowered : "";
    lowered = nullptr;
    nvrtcGetLoweredName(prog, force_gate_expr.c_str(), &lowered);
    out->force_gate_name = lowered ? lowered : "";
  }
  size_t n = 0;
  nvrtcGetCUBINSize(prog, &n);
  out->cubin.resize(n);
  nvrtcGetCUBIN(prog, out->cubin.data());
  nvrtcDestroyProgram(&prog);
  out->basic_registers = registers_of(out->log, out->basic_name);
  out->force_registers = registers_of(out->log, out->force_name);
  out->compile_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return out;
}

}  // namespace

std::shared_ptr<const EdgeJitBinary> compile_edge_kernels(bool fp32, int l_max, int k_max, int rb, int block,
                                                          bool gate) {
  static std::mutex mu;
  static std::map<std::string, std::shared_ptr<const EdgeJitBinary>> cache;
  const std::string key = shape_key(fp32, l_max, k_max, rb, block, gate);
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  auto bin = build(fp32, l_max, k_max, rb, block, gate);
  std::lock_guard<std::mutex> lock(mu);
  return cache.emplace(key, bin).first->second;
}

using namespace drv;

EdgeJitModule::~EdgeJitModule() {
  if (module_) {
    if (auto unload = entry<PFN_unload>("cuModuleUnload")) unload(static_cast<CUmodule>(module_));
  }
}

bool EdgeJitModule::load(const EdgeJitBinary& bin, std::string* err) {
  if (basic_) return true;
  cudaFree(nullptr);  // make the primary context current on this thread
  auto load_data = entry<PFN_load>("cuModuleLoadData");
  auto get_fn = entry<PFN_get>("cuModuleGetFunction");
  if (!load_data || !get_fn) {
    if (err) *err = "driver entry points unavailable";
    return false;
  }
  CUmodule mod = nullptr;
  if (load_data(&mod, bin.cubin.data()) != CUDA_SUCCESS) {
    if (err) *err = "cuModuleLoadData failed for the edge kernels";
    return false;
  }
  CUfunction fb = nullptr, ff = nullptr, gb = nullptr, gf = nullptr;
  bool ok = get_fn(&fb, mod, bin.basic_name.c_str()) == CUDA_SUCCESS &&
            get_fn(&ff, mod, bin.force_name.c_str()) == CUDA_SUCCESS;
  if (ok && !bin.basic_gate_name.empty())
    ok = get_fn(&gb, mod, bin.basic_gate_name.c_str()) == CUDA_SUCCESS &&
         get_fn(&gf, mod, bin.force_gate_name.c_str()) == CUDA_SUCCESS;
  if (!ok) {
    if (auto unload = entry<PFN_unload>("cuModuleUnload")) unload(mod);
    if (err) *err = "cuModuleGetFunction failed for the edge kernels";
    return false;
  }
  module_ = mod;
  basic_ = fb;
  force_ = ff;
  basic_gate_ = gb;
  force_gate_ = gf;
  return true;
}

bool EdgeJitModule::set_smem(void* fn, size_t smem, int* have, std::string* err) {
  if (static_cast<int>(smem) <= *have) return true;
  static PFN_set_attr set_attr = entry<PFN_set_attr>("cuFuncSetAttribute");
  if (!set_attr || set_attr(static_cast<CUfunction>(fn), CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES,
                            static_cast<int>(smem)) != CUDA_SUCCESS) {
    if (err) *err = "cuFuncSetAttribute failed for the edge kernels";
    return false;
  }
  *have = static_cast<int>(smem);
  return true;
}

bool EdgeJitModule::launch_basic(void* stream, int N, int block, size_t smem, const void* args, void* B, bool gate,
                                 std::string* err) {
  static PFN_launch launch_fn = entry<PFN_launch>("cuLaunchKernel");
  void* fn = gate ? basic_gate_ : basic_;
  if (!launch_fn || !fn) {
    if (err) *err = "edge kernels not loaded";
    return false;
  }
  if (!set_smem(fn, smem, gate ? &basic_gate_smem_ : &basic_smem_, err)) return false;
  void* params[] = {const_cast<void*>(args), &B};
  const unsigned grid = static_cast<unsigned>((N + block - 1) / block);
  if (launch_fn(static_cast<CUfunction>(fn), grid, 1, 1, static_cast<unsigned>(block), 1, 1,
                static_cast<unsigned>(smem), static_cast<CUstream>(stream), params, nullptr) != CUDA_SUCCESS) {
    if (err) *err = "cuLaunchKernel failed for k_basic";
    return false;
  }
  return true;
}

bool EdgeJitModule::launch_force(void* stream, int N, int block, size_t smem, const void* args, const void* G,
                                 const double* weight, void* ftmp, double* force, double* virial, double sign,
                                 bool gate, std::string* err) {
  static PFN_launch launch_fn = entry<PFN_launch>("cuLaunchKernel");
  void* fn = gate ? force_gate_ : force_;
  if (!launch_fn || !fn) {
    if (err) *err = "edge kernels not loaded";
    return false;
  }
  if (!set_smem(fn, smem, gate ? &force_gate_smem_ : &force_smem_, err)) return false;
  void* params[] = {const_cast<void*>(args), &G, &weight, &ftmp, &force, &virial, &sign};
  const unsigned grid = static_cast<unsigned>((N + block - 1) / block);
  if (launch_fn(static_cast<CUfunction>(fn), grid, 1, 1, static_cast<unsigned>(block), 1, 1,
                static_cast<unsigned>(smem), static_cast<CUstream>(stream), params, nullptr) != CUDA_SUCCESS) {
    if (err) *err = "cuLaunchKernel failed for k_force";
    return false;
  }
  return true;
}

}  // namespace sus2sh
