// NVRTC build of the per-edge kernels for model shapes without an
// ahead-of-time instantiation.
#include "edge_jit.h"
#include "sh_math.cuh"

#include <nvrtc.h>

#include <algorithm>
#include <cctype>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>

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

// "N bytes gmem" of the ptxas report (module data in global memory).
long long global_bytes_of(const std::string& log) {
  const size_t p = log.find(" bytes gmem");
  if (p == std::string::npos) return -1;
  size_t q = p;
  while (q > 0 && std::isdigit(static_cast<unsigned char>(log[q - 1]))) --q;
  return std::atoll(log.c_str() + q);
}

// The coefficient table as an exact hexadecimal float initializer of
// model_coef(), declared ahead of the kernel headers that call it.
std::string coef_prelude(const std::vector<float>& coef, bool shared_xi, int radial_kind) {
  std::string s = "#define SUS2_MODEL_COEF 1\n#define SUS2_MODEL_SHARED_XI " + std::to_string(shared_xi ? 1 : 0) +
                  "\n#define SUS2_MODEL_RADIAL_KIND " + std::to_string(radial_kind) +
                  "\nnamespace sus2sh {\nnamespace edge {\n"
                  "__device__ __forceinline__ float model_coef(int i) {\n  constexpr float c[" +
                  std::to_string(std::max<size_t>(coef.size(), 1)) + "] = {";
  char buf[48];
  for (size_t i = 0; i < coef.size(); ++i) {
    std::snprintf(buf, sizeof(buf), "%s%af", i ? ", " : "", static_cast<double>(coef[i]));
    s += buf;
  }
  if (coef.empty()) s += "0.0f";
  s += "};\n  return c[i];\n}\n}  // namespace edge\n}  // namespace sus2sh\n";
  return s;
}

// One NVRTC program: k_basic (which & 1) and k_force (which & 2) at the CTA
// sizes `blocks`, the GATE variants when gate is set, the coefficient table
// compiled in when coef is given.
std::shared_ptr<EdgeJitBinary> build(bool fp32, int l, int k, int rb, const std::vector<int>& blocks, bool gate,
                                     const std::vector<float>* coef, int which = 3, bool shared_xi = true,
                                     int radial_kind = 0) {
  const auto t0 = std::chrono::steady_clock::now();
  const std::string T = fp32 ? "float" : "double";
  const std::string shape = T + ", " + std::to_string(l) + ", " + std::to_string(k) + ", " + std::to_string(rb);
  std::vector<std::string> basic_expr, force_expr;
  for (int b : blocks) {
    basic_expr.push_back("&sus2sh::edge::k_basic<" + shape + ", " + std::to_string(b) + ">");
    force_expr.push_back("&sus2sh::edge::k_force<" + shape + ", " + std::to_string(b) + ">");
  }
  const std::string basic_gate_expr = "&sus2sh::edge::k_basic<" + shape + ", 128, true>";
  const std::string force_gate_expr = "&sus2sh::edge::k_force<" + shape + ", 128, true>";
  // a shape build for the Laguerre basis compiles it in; otherwise the
  // Chebyshev kinds are read at run time
  const std::string src = (coef ? coef_prelude(*coef, shared_xi, radial_kind)
                                : (radial_kind == kRadialLaguerre ? "#define SUS2_SHAPE_RADIAL_KIND 2\n" : "")) +
                          std::string("#include \"edge_kernels.cuh\"\n");
  nvrtcProgram prog;
  if (nvrtcCreateProgram(&prog, src.c_str(), "sus2sh_edge.cu", kJitHeaderCount, kJitHeaderSources,
                         kJitHeaderNames) != NVRTC_SUCCESS)
    throw InputError("NVRTC could not create the edge-kernel program.");
  for (size_t b = 0; b < blocks.size(); ++b) {
    if (which & 1) nvrtcAddNameExpression(prog, basic_expr[b].c_str());
    if (which & 2) nvrtcAddNameExpression(prog, force_expr[b].c_str());
  }
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
    out->log.resize(std::strlen(out->log.c_str()));  // up to its NUL: logs of several programs are joined
  }
  if (rc != NVRTC_SUCCESS) {
    nvrtcDestroyProgram(&prog);
    throw InputError("NVRTC failed to compile the edge kernels (<" + shape + ">): " + out->log.substr(0, 2000));
  }
  auto lowered_name = [&](const std::string& expr) {
    const char* lowered = nullptr;
    nvrtcGetLoweredName(prog, expr.c_str(), &lowered);
    return std::string(lowered ? lowered : "");
  };
  out->blocks = blocks;
  for (size_t b = 0; b < blocks.size(); ++b) {
    out->basic_names.push_back((which & 1) ? lowered_name(basic_expr[b]) : std::string());
    out->force_names.push_back((which & 2) ? lowered_name(force_expr[b]) : std::string());
    out->basic_cubin.push_back(0);
    out->force_cubin.push_back(0);
  }
  if (gate) {
    out->basic_gate_name = lowered_name(basic_gate_expr);
    out->force_gate_name = lowered_name(force_gate_expr);
  }
  size_t n = 0;
  nvrtcGetCUBINSize(prog, &n);
  out->cubins.emplace_back(n);
  nvrtcGetCUBIN(prog, out->cubins.back().data());
  nvrtcDestroyProgram(&prog);
  out->basic_registers = (which & 1) ? registers_of(out->log, out->basic_names[0]) : -1;
  out->force_registers = (which & 2) ? registers_of(out->log, out->force_names[0]) : -1;
  out->global_bytes = global_bytes_of(out->log);
  out->model_coef = coef != nullptr;
  out->compile_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return out;
}

std::mutex& cache_mutex() {
  static std::mutex mu;
  return mu;
}
std::map<std::string, std::shared_ptr<const EdgeJitBinary>>& cache() {
  static std::map<std::string, std::shared_ptr<const EdgeJitBinary>> c;
  return c;
}

template <typename Build>
std::shared_ptr<const EdgeJitBinary> cached(const std::string& key, Build&& make) {
  {
    std::lock_guard<std::mutex> lock(cache_mutex());
    auto it = cache().find(key);
    if (it != cache().end()) return it->second;
  }
  std::shared_ptr<const EdgeJitBinary> bin = make();
  std::lock_guard<std::mutex> lock(cache_mutex());
  return cache().emplace(key, bin).first->second;
}

}  // namespace

std::shared_ptr<const EdgeJitBinary> compile_edge_kernels(bool fp32, int l_max, int k_max, int rb, int block,
                                                          bool gate, int radial_kind) {
  const bool lag = radial_kind == kRadialLaguerre;
  return cached(shape_key(fp32, l_max, k_max, rb, block, gate) + (lag ? "/laguerre" : ""),
                [&] { return build(fp32, l_max, k_max, rb, {block}, gate, nullptr, 3, true, lag ? radial_kind : 0); });
}

std::shared_ptr<const EdgeJitBinary> compile_model_edge_kernels(int l_max, int k_max, int rb,
                                                                const std::vector<float>& coef, bool shared_xi,
                                                                int radial_kind) {
  // FNV-1a of the table's bytes
  unsigned long long h = 1469598103934665603ull;
  const unsigned char* b = reinterpret_cast<const unsigned char*>(coef.data());
  for (size_t i = 0; i < coef.size() * sizeof(float); ++i) h = (h ^ b[i]) * 1099511628211ull;
  const std::string key = shape_key(true, l_max, k_max, rb, 0, false) + "/model/" + std::to_string(coef.size()) +
                          "/" + std::to_string(h) + (shared_xi ? "/shared" : "/per-function") +
                          "/kind" + std::to_string(radial_kind);
  return cached(key, [&] {
    const auto t0 = std::chrono::steady_clock::now();
    const int blocks[3] = {64, 128, 256};
    std::shared_ptr<EdgeJitBinary> part[6];
    std::string failure[6];
    std::vector<std::thread> pool;
    for (int p = 0; p < 6; ++p)
      pool.emplace_back([&, p] {
        try {
          part[p] = build(true, l_max, k_max, rb, {blocks[p / 2]}, false, &coef, p % 2 ? 2 : 1, shared_xi, radial_kind);
        } catch (const std::exception& e) {
          failure[p] = e.what();
        }
      });
    for (std::thread& t : pool) t.join();
    for (const std::string& f : failure)
      if (!f.empty()) throw InputError(f);
    auto out = std::make_shared<EdgeJitBinary>();
    out->model_coef = true;
    out->blocks = {64, 128, 256};
    for (int p = 0; p < 6; ++p) {
      out->cubins.push_back(std::move(part[p]->cubins[0]));
      out->log += part[p]->log;
      out->global_bytes = std::max(out->global_bytes, part[p]->global_bytes);
      if (p % 2 == 0) {
        out->basic_names.push_back(part[p]->basic_names[0]);
        out->basic_cubin.push_back(p);
      } else {
        out->force_names.push_back(part[p]->force_names[0]);
        out->force_cubin.push_back(p);
      }
    }
    out->basic_registers = part[0]->basic_registers;
    out->force_registers = part[1]->force_registers;
    out->compile_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return std::shared_ptr<const EdgeJitBinary>(out);
  });
}

std::shared_ptr<const FusedJitBinary> compile_batch_fused(int l_max, int k_max, int rb, const std::vector<float>& coef,
                                                          bool shared_xi, int radial_kind, const std::string& cg_fn,
                                                          const std::vector<std::pair<int, int>>& variants) {
  static std::mutex mu;
  static std::map<std::string, std::shared_ptr<const FusedJitBinary>> done;
  const std::string src = coef_prelude(coef, shared_xi, radial_kind) + "#include \"edge_kernels.cuh\"\n" + cg_fn +
                          "#include \"batch_fused.cuh\"\n";
  std::vector<std::string> expr;
  for (const auto& v : variants)
    expr.push_back("&sus2sh::batch::k_batch_fused<" + std::to_string(l_max) + ", " + std::to_string(k_max) + ", " +
                   std::to_string(rb) + ", " + std::to_string(v.first) + ", " + std::to_string(v.second) + ">");
  std::string key = src;
  for (const std::string& e : expr) key += "\n" + e;
  std::lock_guard<std::mutex> lock(mu);  // one build at a time; later handles of the model reuse it
  auto it = done.find(key);
  if (it != done.end()) return it->second;
  const auto t0 = std::chrono::steady_clock::now();
  nvrtcProgram prog;
  if (nvrtcCreateProgram(&prog, src.c_str(), "sus2sh_batch_fused.cu", kJitHeaderCount, kJitHeaderSources,
                         kJitHeaderNames) != NVRTC_SUCCESS)
    throw InputError("NVRTC could not create the fused batch program.");
  for (const std::string& e : expr) nvrtcAddNameExpression(prog, e.c_str());
  const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "--fmad=true", "--ptxas-options=--verbose",
                        "--generate-line-info"};
  const nvrtcResult rc = nvrtcCompileProgram(prog, 5, opts);
  auto out = std::make_shared<FusedJitBinary>();
  size_t log_size = 0;
  nvrtcGetProgramLogSize(prog, &log_size);
  if (log_size > 1) {
    out->log.resize(log_size);
    nvrtcGetProgramLog(prog, &out->log[0]);
    out->log.resize(std::strlen(out->log.c_str()));
  }
  if (rc != NVRTC_SUCCESS) {
    nvrtcDestroyProgram(&prog);
    throw InputError("NVRTC failed to compile the fused batch kernel: " + out->log.substr(0, 2000));
  }
  for (size_t v = 0; v < variants.size(); ++v) {
    const char* lowered = nullptr;
    nvrtcGetLoweredName(prog, expr[v].c_str(), &lowered);
    out->names.push_back(lowered ? lowered : "");
    out->blocks.push_back(variants[v].first);
    out->min_blocks.push_back(variants[v].second);
    out->registers.push_back(registers_of(out->log, out->names.back()));
  }
  size_t n = 0;
  nvrtcGetCUBINSize(prog, &n);
  out->cubin.resize(n);
  nvrtcGetCUBIN(prog, out->cubin.data());
  nvrtcDestroyProgram(&prog);
  out->compile_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return done.emplace(key, out).first->second;
}

using namespace drv;

EdgeJitModule::~EdgeJitModule() {
  if (auto unload = entry<PFN_unload>("cuModuleUnload"))
    for (void* m : modules_) unload(static_cast<CUmodule>(m));
}

bool EdgeJitModule::load(const EdgeJitBinary& bin, std::string* err) {
  if (!modules_.empty()) return true;
  cudaFree(nullptr);  // make the primary context current on this thread
  auto load_data = entry<PFN_load>("cuModuleLoadData");
  auto get_fn = entry<PFN_get>("cuModuleGetFunction");
  auto unload = entry<PFN_unload>("cuModuleUnload");
  if (!load_data || !get_fn || !unload) {
    if (err) *err = "driver entry points unavailable";
    return false;
  }
  std::vector<CUmodule> mods;
  bool ok = true;
  for (const std::vector<char>& c : bin.cubins) {
    CUmodule mod = nullptr;
    ok = ok && load_data(&mod, c.data()) == CUDA_SUCCESS;
    if (mod) mods.push_back(mod);
  }
  std::vector<Fn> basic(bin.blocks.size()), force(bin.blocks.size());
  Fn gb, gf;
  auto get = [&](Fn& f, const std::string& name, int m) {
    CUfunction fn = nullptr;
    ok = ok && m < static_cast<int>(mods.size()) && get_fn(&fn, mods[m], name.c_str()) == CUDA_SUCCESS;
    f.fn = fn;
  };
  for (size_t b = 0; ok && b < bin.blocks.size(); ++b) {
    get(basic[b], bin.basic_names[b], bin.basic_cubin[b]);
    get(force[b], bin.force_names[b], bin.force_cubin[b]);
  }
  if (ok && !bin.basic_gate_name.empty()) {
    get(gb, bin.basic_gate_name, 0);
    get(gf, bin.force_gate_name, 0);
  }
  if (!ok) {
    for (CUmodule m : mods) unload(m);
    if (err) *err = "loading the edge-kernel modules failed";
    return false;
  }
  for (CUmodule m : mods) modules_.push_back(m);
  blocks_ = bin.blocks;
  basic_ = std::move(basic);
  force_ = std::move(force);
  basic_gate_ = gb;
  force_gate_ = gf;
  return true;
}

EdgeJitModule::Fn* EdgeJitModule::find(bool force, bool gate, int block) {
  if (gate) {
    Fn* f = force ? &force_gate_ : &basic_gate_;
    return block == 128 && f->fn ? f : nullptr;
  }
  for (size_t b = 0; b < blocks_.size(); ++b)
    if (blocks_[b] == block) return force ? &force_[b] : &basic_[b];
  return nullptr;
}

bool EdgeJitModule::set_smem(Fn& f, size_t smem, std::string* err) {
  if (static_cast<int>(smem) <= f.smem) return true;
  static PFN_set_attr set_attr = entry<PFN_set_attr>("cuFuncSetAttribute");
  if (!set_attr || set_attr(static_cast<CUfunction>(f.fn), CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES,
                            static_cast<int>(smem)) != CUDA_SUCCESS) {
    if (err) *err = "cuFuncSetAttribute failed for the edge kernels";
    return false;
  }
  f.smem = static_cast<int>(smem);
  return true;
}

bool EdgeJitModule::launch(Fn* f, const char* what, void* stream, int N, int block, size_t smem, void** params,
                           std::string* err) {
  static PFN_launch launch_fn = entry<PFN_launch>("cuLaunchKernel");
  if (!launch_fn || !f || !f->fn) {
    if (err) *err = std::string(what) + ": no compiled kernel for " + std::to_string(block) + "-thread CTAs";
    return false;
  }
  if (!set_smem(*f, smem, err)) return false;
  const unsigned grid = static_cast<unsigned>((N + block - 1) / block);
  if (launch_fn(static_cast<CUfunction>(f->fn), grid, 1, 1, static_cast<unsigned>(block), 1, 1,
                static_cast<unsigned>(smem), static_cast<CUstream>(stream), params, nullptr) != CUDA_SUCCESS) {
    if (err) *err = std::string("cuLaunchKernel failed for ") + what;
    return false;
  }
  return true;
}

bool EdgeJitModule::launch_basic(void* stream, int N, int block, size_t smem, const void* args, void* B, bool gate,
                                 std::string* err) {
  void* params[] = {const_cast<void*>(args), &B};
  return launch(find(false, gate, block), "k_basic", stream, N, block, smem, params, err);
}

bool EdgeJitModule::launch_force(void* stream, int N, int block, size_t smem, const void* args, const void* G,
                                 const double* weight, void* ftmp, double* force, double* virial, double sign,
                                 bool gate, std::string* err) {
  void* params[] = {const_cast<void*>(args), &G, &weight, &ftmp, &force, &virial, &sign};
  return launch(find(true, gate, block), "k_force", stream, N, block, smem, params, err);
}

}  // namespace sus2sh
