// Straight-line CG product kernels generated per model and compiled with
// NVRTC (see cg_codegen.h).
#include "cg_codegen.h"
#include "driver_api.h"

#include <cuda.h>
#include <cuda_runtime.h>
#include <nvrtc.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <set>
#include <sstream>

namespace sus2sh {
namespace {

std::string lit(double c, bool f32) {
  char buf[64];
  if (f32) std::snprintf(buf, sizeof(buf), "%.9ef", static_cast<double>(static_cast<float>(c)));
  else std::snprintf(buf, sizeof(buf), "%.17e", c);
  return buf;
}

unsigned long long fnv1a(const std::string& s) {
  unsigned long long h = 1469598103934665603ull;
  for (unsigned char ch : s) {
    h ^= ch;
    h *= 1099511628211ull;
  }
  return h;
}

}  // namespace

CgSource generate_cg_source(const HostModel& m, const Layered& lay, bool use_float,
                            const std::vector<int>& basic_canon, int ncanon) {
  const int M = m.moments, Bb = m.basic_count;
  const char* T = use_float ? "float" : "double";
  const char* FMA = use_float ? "fmaf" : "fma";
  // target -> row index
  std::vector<int> row_of(M, -1);
  for (size_t r = 0; r < lay.rows.size(); ++r) row_of[lay.rows[r].target] = static_cast<int>(r);
  std::vector<double> weight(M, 0.0);
  std::vector<char> is_scalar(M, 0);
  for (int s = 0; s < m.scalar_count; ++s) {
    weight[m.moment_mapping[s]] += m.moment_coeffs[s];
    is_scalar[m.moment_mapping[s]] = 1;
  }
  // liveness: a row is live if its target feeds the energy
  std::vector<char> live(M, 0);
  for (int r = static_cast<int>(lay.rows.size()) - 1; r >= 0; --r) {
    // rows are sorted by layer ascending, so walking backwards visits
    // consumers before producers
    const Row& row = lay.rows[r];
    if (is_scalar[row.target] && weight[row.target] != 0.0) live[row.target] = 1;
    if (!live[row.target]) continue;
    for (size_t t = 0; t < row.left.size(); ++t) {
      live[row.left[t]] = 1;
      live[row.right[t]] = 1;
    }
  }
  // live consumers of every moment (unique rows)
  std::vector<std::vector<int>> consumers(M);
  for (const Row& row : lay.rows) {
    if (!live[row.target]) continue;
    std::set<int> ops(row.left.begin(), row.left.end());
    ops.insert(row.right.begin(), row.right.end());
    for (int o : ops) consumers[o].push_back(row.target);
  }
  std::vector<int> pending(M, 0);
  for (int x = 0; x < M; ++x) pending[x] = static_cast<int>(consumers[x].size());
  std::vector<char> terminal(M, 0);
  for (const Row& row : lay.rows)
    if (live[row.target] && consumers[row.target].empty()) terminal[row.target] = 1;

  std::ostringstream body;
  long long terms = 0;
  std::vector<char> emitted(M, 0);
  for (int b = 0; b < Bb; ++b) emitted[b] = 1;

  auto v = [](int x) { return "v" + std::to_string(x); };
  auto a = [](int x) { return "a" + std::to_string(x); };

  std::function<void(int)> ensure = [&](int x) {
    if (emitted[x]) return;
    const Row& row = lay.rows[row_of[x]];
    for (size_t t = 0; t < row.left.size(); ++t) {
      ensure(row.left[t]);
      ensure(row.right[t]);
    }
    body << "  " << T << " " << v(x) << " = " << lit(row.coeff[0], use_float) << " * " << v(row.left[0]) << " * "
         << v(row.right[0]) << ";\n";
    for (size_t t = 1; t < row.left.size(); ++t)
      body << "  " << v(x) << " = " << FMA << "(" << lit(row.coeff[t], use_float) << " * " << v(row.left[t])
           << ", " << v(row.right[t]) << ", " << v(x) << ");\n";
    terms += static_cast<long long>(row.left.size());
    body << "  " << T << " " << a(x) << " = " << (weight[x] != 0.0 ? lit(weight[x], use_float) : (use_float ? "0.0f" : "0.0"))
         << ";\n";
    if (is_scalar[x] && weight[x] != 0.0)
      body << "  E += (double)(" << lit(weight[x], use_float) << " * " << v(x) << ");\n";
    emitted[x] = 1;
  };

  std::function<void(int)> back = [&](int x) {
    const Row& row = lay.rows[row_of[x]];
    body << "  {\n";
    for (size_t t = 0; t < row.left.size(); ++t) {
      body << "    const " << T << " q" << t << " = " << lit(row.coeff[t], use_float) << " * " << a(x) << ";\n";
      body << "    " << a(row.left[t]) << " = " << FMA << "(q" << t << ", " << v(row.right[t]) << ", "
           << a(row.left[t]) << ");\n";
      body << "    " << a(row.right[t]) << " = " << FMA << "(q" << t << ", " << v(row.left[t]) << ", "
           << a(row.right[t]) << ");\n";
    }
    body << "  }\n";
    terms += 2 * static_cast<long long>(row.left.size());
    std::set<int> ops(row.left.begin(), row.left.end());
    ops.insert(row.right.begin(), row.right.end());
    for (int o : ops) {
      if (o < Bb) continue;
      if (--pending[o] == 0) back(o);
    }
  };

  // terminal rows, ordered by their latest-defined operand
  std::vector<int> term_rows;
  std::vector<int> order(M, 0);
  for (size_t r = 0; r < lay.rows.size(); ++r) order[lay.rows[r].target] = static_cast<int>(r) + 1;
  for (const Row& row : lay.rows)
    if (terminal[row.target]) term_rows.push_back(row.target);
  auto key = [&](int t) {
    const Row& row = lay.rows[row_of[t]];
    int k = 0;
    for (size_t i = 0; i < row.left.size(); ++i) k = std::max({k, order[row.left[i]], order[row.right[i]]});
    return k;
  };
  std::stable_sort(term_rows.begin(), term_rows.end(), [&](int x, int y) { return key(x) < key(y); });

  for (int t : term_rows) {
    const Row& row = lay.rows[row_of[t]];
    for (size_t i = 0; i < row.left.size(); ++i) {
      ensure(row.left[i]);
      ensure(row.right[i]);
    }
    const double w = weight[t];
    body << "  {\n    " << T << " t = " << (use_float ? "0.0f" : "0.0") << ";\n";
    for (size_t i = 0; i < row.left.size(); ++i) {
      const std::string c = lit(row.coeff[i] * w, use_float);
      body << "    { const " << T << " p = " << c << " * " << v(row.left[i]) << ";\n";
      body << "      t = " << FMA << "(p, " << v(row.right[i]) << ", t);\n";
      body << "      " << a(row.right[i]) << " += p;\n";
      body << "      " << a(row.left[i]) << " = " << FMA << "(" << c << ", " << v(row.right[i]) << ", "
           << a(row.left[i]) << "); }\n";
    }
    body << "    E += (double)t;\n  }\n";
    terms += 2 * static_cast<long long>(row.left.size());
    std::set<int> ops(row.left.begin(), row.left.end());
    ops.insert(row.right.begin(), row.right.end());
    for (int o : ops) {
      if (o < Bb) continue;
      if (--pending[o] == 0) back(o);
    }
  }

  std::ostringstream src;
  const std::string tag = std::to_string(fnv1a(body.str()) ^ (use_float ? 0x1234ull : 0x4321ull));
  CgSource out;
  out.kernel_name = "sus2sh_cg_" + tag;
  src << "// generated SUS2-SH CG product kernel (" << (use_float ? "FP32" : "FP64") << ")\n"
      << "struct D4 { double x, y, z, w; };\n"
      << "extern \"C\" __global__ void __launch_bounds__(128) " << out.kernel_name
      << "(int N, const D4* __restrict__ pos4, const " << T << "* __restrict__ B, " << T
      << "* __restrict__ G, const double* __restrict__ shift, const double* __restrict__ species, "
         "double* __restrict__ pe, int pe_assign) {\n"
      << "  const int i = blockIdx.x * blockDim.x + threadIdx.x;\n"
      << "  if (i >= N) return;\n"
      << "  const size_t n = (size_t)N;\n"
      << "  double E = 0.0;\n";
  for (int b = 0; b < Bb; ++b) {
    src << "  const " << T << " " << v(b) << " = __ldg(B + " << basic_canon[b] << " * n + i);\n";
    src << "  " << T << " " << a(b) << " = " << (weight[b] != 0.0 ? lit(weight[b], use_float) : (use_float ? "0.0f" : "0.0"))
        << ";\n";
    if (is_scalar[b] && weight[b] != 0.0)
      src << "  E += (double)(" << lit(weight[b], use_float) << " * " << v(b) << ");\n";
  }
  src << body.str();
  src << "  const int ti = (int)__double_as_longlong(pos4[i].w);\n"
      << "  const double ct = species[ti];\n"
      << "  const double site = shift[ti] + ct + ct * E;\n"
      << "  if (pe) pe[i] = pe_assign ? site : pe[i] + site;\n"
      << "  const " << T << " sc = (" << T << ")ct;\n";
  std::vector<int> canon_basic(ncanon, -1);
  for (int b = 0; b < Bb; ++b) canon_basic[basic_canon[b]] = b;
  for (int c = 0; c < ncanon; ++c) {
    if (canon_basic[c] >= 0) src << "  G[" << c << " * n + i] = sc * " << a(canon_basic[c]) << ";\n";
    else src << "  G[" << c << " * n + i] = (" << T << ")0;\n";
  }
  src << "}\n";
  out.code = src.str();
  out.fp_terms = terms;
  return out;
}

CgBinary compile_cg_source(const CgSource& src) {
  nvrtcProgram prog;
  if (nvrtcCreateProgram(&prog, src.code.c_str(), "sus2sh_cg.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS)
    throw InputError("NVRTC could not create the CG program.");
  const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "--ptxas-options=--verbose",
                        "--fmad=true"};
  const nvrtcResult rc = nvrtcCompileProgram(prog, 4, opts);
  CgBinary out;
  size_t log_size = 0;
  nvrtcGetProgramLogSize(prog, &log_size);
  if (log_size > 1) {
    out.log.resize(log_size);
    nvrtcGetProgramLog(prog, &out.log[0]);
  }
  if (rc != NVRTC_SUCCESS) {
    nvrtcDestroyProgram(&prog);
    throw InputError("NVRTC failed to compile the CG program: " + out.log.substr(0, 2000));
  }
  size_t n = 0;
  nvrtcGetCUBINSize(prog, &n);
  out.cubin.resize(n);
  nvrtcGetCUBIN(prog, out.cubin.data());
  nvrtcDestroyProgram(&prog);
  const size_t p = out.log.find("Used ");
  if (p != std::string::npos) out.registers = std::atoi(out.log.c_str() + p + 5);
  return out;
}

// ---------------------------------------------------------------------------
// driver API through the runtime's entry-point query
// ---------------------------------------------------------------------------
using namespace drv;

CgModule::~CgModule() {
  if (module_) {
    if (auto unload = entry<PFN_unload>("cuModuleUnload")) unload(static_cast<CUmodule>(module_));
  }
}

bool CgModule::load(const CgBinary& bin, const std::string& kernel_name, std::string* err) {
  if (func_) return true;
  cudaFree(nullptr);  // make the primary context current on this thread
  auto load_data = entry<PFN_load>("cuModuleLoadData");
  auto get_fn = entry<PFN_get>("cuModuleGetFunction");
  if (!load_data || !get_fn) {
    if (err) *err = "driver entry points unavailable";
    return false;
  }
  CUmodule mod = nullptr;
  if (load_data(&mod, bin.cubin.data()) != CUDA_SUCCESS) {
    if (err) *err = "cuModuleLoadData failed for the CG kernel";
    return false;
  }
  CUfunction f = nullptr;
  if (get_fn(&f, mod, kernel_name.c_str()) != CUDA_SUCCESS) {
    if (err) *err = "cuModuleGetFunction failed for the CG kernel";
    return false;
  }
  module_ = mod;
  func_ = f;
  return true;
}

bool CgModule::launch(void* stream, int N, const void* pos4, const void* B, void* G, const double* shift,
                      const double* species, double* pe, int pe_assign, std::string* err) {
  static PFN_launch launch_fn = entry<PFN_launch>("cuLaunchKernel");
  if (!launch_fn || !func_) {
    if (err) *err = "CG kernel not loaded";
    return false;
  }
  void* args[] = {&N, &pos4, &B, &G, &shift, &species, &pe, &pe_assign};
  const unsigned grid = static_cast<unsigned>((N + 127) / 128);
  if (launch_fn(static_cast<CUfunction>(func_), grid, 1, 1, 128, 1, 1, 0, static_cast<CUstream>(stream), args,
                nullptr) != CUDA_SUCCESS) {
    if (err) *err = "cuLaunchKernel failed for the CG kernel";
    return false;
  }
  return true;
}

}  // namespace sus2sh
