// Straight-line CG product kernels generated per model and compiled with
// NVRTC (see cg_codegen.h).
#include "cg_codegen.h"
#include "driver_api.h"

#include <cuda.h>
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <sys/stat.h>
#include <unistd.h>
#include <nvJitLink.h>
#include <nvrtc.h>

#include <algorithm>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
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

const char* const kCgStreamHelpers = R"(#ifdef __CUDA_ARCH__
__device__ __forceinline__ unsigned long long sus2_pol() {
  unsigned long long p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ float sus2_ld(const float* a, unsigned long long pol) {
  float v;
  asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ double sus2_ld(const double* a, unsigned long long pol) {
  double v;
  asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ void sus2_st(float* a, float v, unsigned long long pol) {
  asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(a), "f"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void sus2_st(double* a, double v, unsigned long long pol) {
  asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(a), "d"(v), "l"(pol) : "memory");
}
#endif
)";

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
      << kCgStreamHelpers
      << "extern \"C\" __global__ void __launch_bounds__(128) " << out.kernel_name
      << "(int N, const D4* __restrict__ pos4, const " << T << "* __restrict__ B, " << T
      << "* __restrict__ G, const double* __restrict__ shift, const double* __restrict__ species, "
         "double* __restrict__ pe, int pe_assign) {\n"
      << "  const int i = blockIdx.x * blockDim.x + threadIdx.x;\n"
      << "  if (i >= N) return;\n"
      << "  const size_t n = (size_t)N;\n"
      << "  const unsigned long long pol = sus2_pol();\n"
      << "  double E = 0.0;\n";
  for (int b = 0; b < Bb; ++b) {
    src << "  const " << T << " " << v(b) << " = sus2_ld(B + " << basic_canon[b] << " * n + i, pol);\n";
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
    if (canon_basic[c] >= 0) src << "  sus2_st(G + " << c << " * n + i, sc * " << a(canon_basic[c]) << ", pol);\n";
    else src << "  sus2_st(G + " << c << " * n + i, (" << T << ")0, pol);\n";
  }
  src << "}\n";
  out.code = src.str();
  out.fp_terms = terms;
  // the same body as a device function on register arrays (canonical order)
  // for kernels that produce the basics and consume the adjoints themselves
  std::ostringstream fn;
  fn << "namespace sus2sh {\nnamespace batch {\n"
     << "__device__ __forceinline__ double cg_atom(const " << T << " (&B)[" << ncanon << "], " << T << " (&G)["
     << ncanon << "], " << T << " sc) {\n"
     << "  double E = 0.0;\n";
  for (int b = 0; b < Bb; ++b) {
    fn << "  const " << T << " " << v(b) << " = B[" << basic_canon[b] << "];\n";
    fn << "  " << T << " " << a(b) << " = " << (weight[b] != 0.0 ? lit(weight[b], use_float) : (use_float ? "0.0f" : "0.0"))
       << ";\n";
    if (is_scalar[b] && weight[b] != 0.0)
      fn << "  E += (double)(" << lit(weight[b], use_float) << " * " << v(b) << ");\n";
  }
  fn << body.str();
  for (int c = 0; c < ncanon; ++c) {
    if (canon_basic[c] >= 0) fn << "  G[" << c << "] = sc * " << a(canon_basic[c]) << ";\n";
    else fn << "  G[" << c << "] = (" << T << ")0;\n";
  }
  fn << "  return E;\n}\n}  // namespace batch\n}  // namespace sus2sh\n";
  out.device_fn = fn.str();
  return out;
}

// Forward-over-reverse CG product for the parameter gradients: every moment
// carries its value v and tangent w (the derivative along the position
// perturbation of the force-matching term), every adjoint its value a and
// tangent b.  Same row schedule as generate_cg_source; every scalar is kept
// (a weight of zero still has a gradient).  Per atom the kernel writes
// contrib[s] = c_t (ew M_s - dM_s) for the reduction of dL/dw_s, and the
// basic adjoints alpha = c_t (ew a - b), beta = c_t a for the radial pass.
CgSource generate_pg_source(const HostModel& m, const Layered& lay, bool use_float,
                            const std::vector<int>& basic_canon, int ncanon) {
  const int M = m.moments, Bb = m.basic_count;
  const char* T = use_float ? "float" : "double";
  const char* FMA = use_float ? "fmaf" : "fma";
  const std::string zero = use_float ? "0.0f" : "0.0";
  std::vector<int> row_of(M, -1);
  for (size_t r = 0; r < lay.rows.size(); ++r) row_of[lay.rows[r].target] = static_cast<int>(r);
  std::vector<double> weight(M, 0.0);
  std::vector<char> is_scalar(M, 0);
  std::vector<std::vector<int>> scalars_of(M);
  for (int s = 0; s < m.scalar_count; ++s) {
    weight[m.moment_mapping[s]] += m.moment_coeffs[s];
    is_scalar[m.moment_mapping[s]] = 1;
    scalars_of[m.moment_mapping[s]].push_back(s);
  }
  std::vector<char> live(M, 0);
  for (int r = static_cast<int>(lay.rows.size()) - 1; r >= 0; --r) {
    const Row& row = lay.rows[r];
    if (is_scalar[row.target]) live[row.target] = 1;
    if (!live[row.target]) continue;
    for (size_t t = 0; t < row.left.size(); ++t) live[row.left[t]] = live[row.right[t]] = 1;
  }
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
  auto w = [](int x) { return "w" + std::to_string(x); };
  auto a = [](int x) { return "a" + std::to_string(x); };
  auto bt = [](int x) { return "b" + std::to_string(x); };
  auto contrib = [&](std::ostringstream& o, int x, const std::string& val, const std::string& tan) {
    for (int s : scalars_of[x])
      o << "  contrib[" << s << " * n + i] = (" << T << ")(ct * (ak * (double)" << val << " - (double)" << tan
        << "));\n";
  };

  std::function<void(int)> ensure = [&](int x) {
    if (emitted[x]) return;
    const Row& row = lay.rows[row_of[x]];
    for (size_t t = 0; t < row.left.size(); ++t) {
      ensure(row.left[t]);
      ensure(row.right[t]);
    }
    body << "  " << T << " " << v(x) << " = " << zero << ", " << w(x) << " = " << zero << ";\n";
    for (size_t t = 0; t < row.left.size(); ++t) {
      const int l = row.left[t], r = row.right[t];
      const std::string c = lit(row.coeff[t], use_float);
      body << "  { const " << T << " cl = " << c << " * " << v(l) << ";\n"
           << "    " << v(x) << " = " << FMA << "(cl, " << v(r) << ", " << v(x) << ");\n"
           << "    " << w(x) << " = " << FMA << "(cl, " << w(r) << ", " << FMA << "(" << c << " * " << w(l) << ", "
           << v(r) << ", " << w(x) << ")); }\n";
    }
    terms += 3 * static_cast<long long>(row.left.size());
    body << "  " << T << " " << a(x) << " = " << (weight[x] != 0.0 ? lit(weight[x], use_float) : zero) << ", "
         << bt(x) << " = " << zero << ";\n";
    contrib(body, x, v(x), w(x));
    emitted[x] = 1;
  };

  std::function<void(int)> back = [&](int x) {
    const Row& row = lay.rows[row_of[x]];
    for (size_t t = 0; t < row.left.size(); ++t) {
      const int l = row.left[t], r = row.right[t];
      const std::string c = lit(row.coeff[t], use_float);
      body << "  { const " << T << " q = " << c << " * " << a(x) << ", qd = " << c << " * " << bt(x) << ";\n"
           << "    " << bt(l) << " = " << FMA << "(qd, " << v(r) << ", " << FMA << "(q, " << w(r) << ", " << bt(l)
           << "));\n"
           << "    " << bt(r) << " = " << FMA << "(qd, " << v(l) << ", " << FMA << "(q, " << w(l) << ", " << bt(r)
           << "));\n"
           << "    " << a(l) << " = " << FMA << "(q, " << v(r) << ", " << a(l) << ");\n"
           << "    " << a(r) << " = " << FMA << "(q, " << v(l) << ", " << a(r) << "); }\n";
    }
    terms += 6 * static_cast<long long>(row.left.size());
    std::set<int> ops(row.left.begin(), row.left.end());
    ops.insert(row.right.begin(), row.right.end());
    for (int o : ops) {
      if (o < Bb) continue;
      if (--pending[o] == 0) back(o);
    }
  };

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
    const double wt = weight[t];
    body << "  {\n    " << T << " t = " << zero << ", td = " << zero << ";\n";
    for (size_t i = 0; i < row.left.size(); ++i) {
      const int l = row.left[i], r = row.right[i];
      const std::string c = lit(row.coeff[i], use_float);
      body << "    { const " << T << " cl = " << c << " * " << v(l) << ";\n"
           << "      t = " << FMA << "(cl, " << v(r) << ", t);\n"
           << "      td = " << FMA << "(cl, " << w(r) << ", " << FMA << "(" << c << " * " << w(l) << ", " << v(r)
           << ", td)); }\n";
      if (wt != 0.0) {
        const std::string p = lit(row.coeff[i] * wt, use_float);
        body << "    " << a(l) << " = " << FMA << "(" << p << ", " << v(r) << ", " << a(l) << ");\n"
             << "    " << a(r) << " = " << FMA << "(" << p << ", " << v(l) << ", " << a(r) << ");\n"
             << "    " << bt(l) << " = " << FMA << "(" << p << ", " << w(r) << ", " << bt(l) << ");\n"
             << "    " << bt(r) << " = " << FMA << "(" << p << ", " << w(l) << ", " << bt(r) << ");\n";
      }
    }
    std::ostringstream cb;
    contrib(cb, t, "t", "td");
    body << cb.str() << "  }\n";
    terms += static_cast<long long>(row.left.size()) * (wt != 0.0 ? 7 : 3);
    std::set<int> ops(row.left.begin(), row.left.end());
    ops.insert(row.right.begin(), row.right.end());
    for (int o : ops) {
      if (o < Bb) continue;
      if (--pending[o] == 0) back(o);
    }
  }

  std::ostringstream src;
  const std::string tag = std::to_string(fnv1a(body.str()) ^ (use_float ? 0x9e37ull : 0x79b9ull));
  CgSource out;
  out.kernel_name = "sus2sh_pg_" + tag;
  src << "// generated SUS2-SH forward-over-reverse CG product kernel (" << (use_float ? "FP32" : "FP64") << ")\n"
      << "struct D4 { double x, y, z, w; };\n"
      << "extern \"C\" __global__ void __launch_bounds__(128) " << out.kernel_name
      << "(int N, const D4* __restrict__ pos4, const " << T << "* __restrict__ B, const " << T
      << "* __restrict__ Bd, const double* __restrict__ species, const double* __restrict__ ew, " << T
      << "* __restrict__ Galpha, " << T << "* __restrict__ Gbeta, " << T << "* __restrict__ contrib) {\n"
      << "  const int i = blockIdx.x * blockDim.x + threadIdx.x;\n"
      << "  if (i >= N) return;\n"
      << "  const size_t n = (size_t)N;\n"
      << "  const double ct = species[(int)__double_as_longlong(pos4[i].w)];\n"
      << "  const double ak = ew ? ew[i] : 0.0;\n";
  for (int b = 0; b < Bb; ++b) {
    src << "  const " << T << " " << v(b) << " = __ldg(B + " << basic_canon[b] << " * n + i), " << w(b)
        << " = __ldg(Bd + " << basic_canon[b] << " * n + i);\n";
    src << "  " << T << " " << a(b) << " = " << (weight[b] != 0.0 ? lit(weight[b], use_float) : zero) << ", "
        << bt(b) << " = " << zero << ";\n";
    contrib(src, b, v(b), w(b));
  }
  src << body.str();
  src << "  const " << T << " sc = (" << T << ")ct, sa = (" << T << ")(ct * ak);\n";
  std::vector<int> canon_basic(ncanon, -1);
  for (int b = 0; b < Bb; ++b) canon_basic[basic_canon[b]] = b;
  for (int c = 0; c < ncanon; ++c) {
    if (canon_basic[c] >= 0) {
      const int b = canon_basic[c];
      src << "  Galpha[" << c << " * n + i] = " << FMA << "(sa, " << a(b) << ", -sc * " << bt(b) << ");\n"
          << "  Gbeta[" << c << " * n + i] = sc * " << a(b) << ";\n";
    } else {
      src << "  Galpha[" << c << " * n + i] = (" << T << ")0;\n  Gbeta[" << c << " * n + i] = (" << T << ")0;\n";
    }
  }
  src << "}\n";
  out.code = src.str();
  out.fp_terms = terms;
  return out;
}

namespace {

struct UnitResult {
  std::vector<char> cubin;
  std::string log;
  std::string error;
};

// One NVRTC program for sm_100a (relocatable when rdc), ptxas report kept.
UnitResult compile_unit(const std::string& code, bool rdc) {
  UnitResult out;
  nvrtcProgram prog;
  if (nvrtcCreateProgram(&prog, code.c_str(), "sus2sh_cg.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) {
    out.error = "NVRTC could not create the CG program.";
    return out;
  }
  std::vector<const char*> opts = {"--gpu-architecture=sm_100a", "--std=c++17", "--ptxas-options=--verbose",
                                   "--fmad=true"};
  if (rdc) opts.push_back("--relocatable-device-code=true");
  // extra NVRTC options for tuning runs (whitespace separated), e.g.
  // SUS2SH_NVRTC_OPTIONS="--ptxas-options=--device-function-maxrregcount=255"
  std::vector<std::string> extra;
  if (const char* env = std::getenv("SUS2SH_NVRTC_OPTIONS")) {
    std::istringstream is(env);
    for (std::string w; is >> w;) extra.push_back(w);
  }
  for (const std::string& w : extra) opts.push_back(w.c_str());
  const nvrtcResult rc = nvrtcCompileProgram(prog, static_cast<int>(opts.size()), opts.data());
  size_t log_size = 0;
  nvrtcGetProgramLogSize(prog, &log_size);
  if (log_size > 1) {
    out.log.resize(log_size);
    nvrtcGetProgramLog(prog, &out.log[0]);
  }
  if (rc != NVRTC_SUCCESS) {
    nvrtcDestroyProgram(&prog);
    out.error = "NVRTC failed to compile the CG program: " + out.log.substr(0, 2000);
    return out;
  }
  size_t n = 0;
  nvrtcGetCUBINSize(prog, &n);
  out.cubin.resize(n);
  nvrtcGetCUBIN(prog, out.cubin.data());
  nvrtcDestroyProgram(&prog);
  return out;
}

// nvJitLink 12.9, opened by path at first use.  The library is not linked:
// a process that loaded an older libnvJitLink.so.12 first (PyTorch wheels
// bundle one) would otherwise fail to resolve the 12.9 entry points.
struct JitLinkApi {
  decltype(&__nvJitLinkCreate_12_9) create = nullptr;
  decltype(&__nvJitLinkDestroy_12_9) destroy = nullptr;
  decltype(&__nvJitLinkAddData_12_9) add_data = nullptr;
  decltype(&__nvJitLinkComplete_12_9) complete = nullptr;
  decltype(&__nvJitLinkGetLinkedCubinSize_12_9) cubin_size = nullptr;
  decltype(&__nvJitLinkGetLinkedCubin_12_9) cubin = nullptr;
  decltype(&__nvJitLinkGetErrorLogSize_12_9) error_size = nullptr;
  decltype(&__nvJitLinkGetErrorLog_12_9) error_log = nullptr;
  bool ok = false;
};

const JitLinkApi& jitlink() {
  static const JitLinkApi api = [] {
    JitLinkApi a;
    std::vector<std::string> paths;
    if (const char* home = std::getenv("CUDA_HOME")) paths.push_back(std::string(home) + "/lib64/libnvJitLink.so.12");
    paths.push_back("/usr/local/cuda/lib64/libnvJitLink.so.12");
    paths.push_back("libnvJitLink.so.12");
    for (const std::string& p : paths) {
      void* h = dlopen(p.c_str(), RTLD_NOW | RTLD_LOCAL);
      if (!h) continue;
      a.create = reinterpret_cast<decltype(a.create)>(dlsym(h, "__nvJitLinkCreate_12_9"));
      a.destroy = reinterpret_cast<decltype(a.destroy)>(dlsym(h, "__nvJitLinkDestroy_12_9"));
      a.add_data = reinterpret_cast<decltype(a.add_data)>(dlsym(h, "__nvJitLinkAddData_12_9"));
      a.complete = reinterpret_cast<decltype(a.complete)>(dlsym(h, "__nvJitLinkComplete_12_9"));
      a.cubin_size = reinterpret_cast<decltype(a.cubin_size)>(dlsym(h, "__nvJitLinkGetLinkedCubinSize_12_9"));
      a.cubin = reinterpret_cast<decltype(a.cubin)>(dlsym(h, "__nvJitLinkGetLinkedCubin_12_9"));
      a.error_size = reinterpret_cast<decltype(a.error_size)>(dlsym(h, "__nvJitLinkGetErrorLogSize_12_9"));
      a.error_log = reinterpret_cast<decltype(a.error_log)>(dlsym(h, "__nvJitLinkGetErrorLog_12_9"));
      a.ok = a.create && a.destroy && a.add_data && a.complete && a.cubin_size && a.cubin && a.error_size &&
             a.error_log;
      if (a.ok) break;
      dlclose(h);
      a = JitLinkApi{};
    }
    return a;
  }();
  return api;
}

// Largest "Used N registers" in a ptxas report (-1 if none).
int max_registers(const std::string& log) {
  int best = -1;
  for (size_t p = log.find("Used "); p != std::string::npos; p = log.find("Used ", p + 5))
    best = std::max(best, std::atoi(log.c_str() + p + 5));
  return best;
}

CgBinary build_one_program(const std::string& code) {
  CgBinary out;
  UnitResult u = compile_unit(code, false);
  if (!u.error.empty()) throw InputError(u.error);
  out.cubin = std::move(u.cubin);
  out.log = std::move(u.log);
  out.registers = max_registers(out.log);
  out.whole = true;
  return out;
}

CgBinary build_binary(const CgSource& src, CgBuild build) {
  const JitLinkApi& jl = jitlink();
  if (src.units.size() < 2 || build == CgBuild::kWhole || !jl.ok) {
    // one program (also the fallback when nvJitLink 12.9 is not available)
    return build_one_program(src.code);
  }
  CgBinary out;
  // component-split kernel: the units compile in parallel as relocatable
  // code and nvJitLink joins them
  std::vector<UnitResult> res(src.units.size());
  const size_t hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nthreads = std::min(src.units.size(), std::min<size_t>(hw, 32));
  std::vector<std::thread> pool;
  std::mutex mu;
  size_t next = 0;
  for (size_t t = 0; t < nthreads; ++t)
    pool.emplace_back([&] {
      for (;;) {
        size_t k;
        {
          std::lock_guard<std::mutex> lock(mu);
          if (next >= src.units.size()) return;
          k = next++;
        }
        res[k] = compile_unit(src.units[k], true);
      }
    });
  for (std::thread& th : pool) th.join();
  for (const UnitResult& u : res) {
    if (!u.error.empty()) throw InputError(u.error);
    out.log += u.log;
  }
  nvJitLinkHandle h = nullptr;
  const char* lopts[] = {"-arch=sm_100a"};
  if (jl.create(&h, 1, lopts) != NVJITLINK_SUCCESS) throw InputError("nvJitLink could not be created.");
  auto link_error = [&](const char* what) {
    size_t n = 0;
    std::string log;
    if (jl.error_size(h, &n) == NVJITLINK_SUCCESS && n > 1) {
      log.resize(n);
      jl.error_log(h, &log[0]);
    }
    jl.destroy(&h);
    throw InputError(std::string(what) + " " + log.substr(0, 2000));
  };
  for (size_t k = 0; k < res.size(); ++k) {
    const std::string name = "unit" + std::to_string(k);
    if (jl.add_data(h, NVJITLINK_INPUT_CUBIN, res[k].cubin.data(), res[k].cubin.size(), name.c_str()) !=
        NVJITLINK_SUCCESS)
      link_error("nvJitLink rejected a CG unit:");
  }
  if (jl.complete(h) != NVJITLINK_SUCCESS) link_error("nvJitLink failed to link the CG kernel:");
  size_t n = 0;
  jl.cubin_size(h, &n);
  out.cubin.resize(n);
  jl.cubin(h, out.cubin.data());
  jl.destroy(&h);
  out.registers = max_registers(out.log);
  return out;
}

// ---- on-disk cache of whole-program builds
//
// One file per kernel source: a 64-byte header (magic, format, source size,
// two independent 64-bit hashes of the source, NVRTC version, log and cubin
// sizes), the ptxas report, the cubin.  Written to a temporary name and
// renamed, so readers never see a partial file; a file that does not match
// its header is ignored and rewritten.
constexpr char kCacheMagic[8] = {'S', 'U', 'S', '2', 'C', 'G', 'B', '1'};

struct CacheHeader {
  char magic[8];
  uint64_t code_size, h1, h2;
  int32_t nvrtc_major, nvrtc_minor;
  uint64_t log_size, cubin_size;
  uint64_t reserved;
};
static_assert(sizeof(CacheHeader) == 64, "cache header layout");

uint64_t hash2(const std::string& s) {
  // a second, independent hash (64-bit multiply-xorshift over 8-byte words)
  uint64_t h = 0x9E3779B97F4A7C15ull ^ s.size();
  size_t i = 0;
  for (; i + 8 <= s.size(); i += 8) {
    uint64_t w;
    std::memcpy(&w, s.data() + i, 8);
    h = (h ^ w) * 0xBF58476D1CE4E5B9ull;
    h ^= h >> 31;
  }
  for (; i < s.size(); ++i) h = (h ^ static_cast<unsigned char>(s[i])) * 0x94D049BB133111EBull;
  return h ^ (h >> 29);
}

std::string cache_path(const std::string& dir, const std::string& code, CacheHeader* hdr) {
  std::memcpy(hdr->magic, kCacheMagic, 8);
  hdr->code_size = code.size();
  hdr->h1 = fnv1a(code);
  hdr->h2 = hash2(code);
  int major = 0, minor = 0;
  nvrtcVersion(&major, &minor);
  hdr->nvrtc_major = major;
  hdr->nvrtc_minor = minor;
  hdr->log_size = hdr->cubin_size = hdr->reserved = 0;
  char name[160];
  std::snprintf(name, sizeof(name), "/cg_%016llx_%016llx_nvrtc%d.%d_sm100a.cubin",
                static_cast<unsigned long long>(hdr->h1), static_cast<unsigned long long>(hdr->h2), major, minor);
  return dir + name;
}

bool cache_read(const std::string& path, const CacheHeader& want, CgBinary* out) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  CacheHeader h;
  bool ok = std::fread(&h, sizeof(h), 1, f) == 1 && std::memcmp(h.magic, want.magic, 8) == 0 &&
            h.code_size == want.code_size && h.h1 == want.h1 && h.h2 == want.h2 &&
            h.nvrtc_major == want.nvrtc_major && h.nvrtc_minor == want.nvrtc_minor && h.cubin_size > 0 &&
            h.cubin_size < (1ull << 31) && h.log_size < (1ull << 26);
  if (ok) {
    out->log.resize(h.log_size);
    out->cubin.resize(h.cubin_size);
    ok = (h.log_size == 0 || std::fread(&out->log[0], 1, h.log_size, f) == h.log_size) &&
         std::fread(out->cubin.data(), 1, h.cubin_size, f) == h.cubin_size && std::fgetc(f) == EOF;
  }
  std::fclose(f);
  if (!ok) return false;
  out->registers = max_registers(out->log);
  out->whole = true;
  out->from_disk = true;
  return true;
}

bool make_dirs(const std::string& dir) {
  for (size_t p = 1; p <= dir.size(); ++p) {
    if (p < dir.size() && dir[p] != '/') continue;
    const std::string sub = dir.substr(0, p);
    if (mkdir(sub.c_str(), 0755) != 0 && errno != EEXIST) return false;
  }
  struct stat st;
  return stat(dir.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}

void cache_write(const std::string& dir, const std::string& path, CacheHeader hdr, const CgBinary& bin) {
  if (!make_dirs(dir)) return;
  hdr.log_size = bin.log.size();
  hdr.cubin_size = bin.cubin.size();
  char suffix[64];
  std::snprintf(suffix, sizeof(suffix), ".tmp%ld_%zu", static_cast<long>(getpid()),
                std::hash<std::thread::id>()(std::this_thread::get_id()));
  const std::string tmp = path + suffix;
  FILE* f = std::fopen(tmp.c_str(), "wb");
  if (!f) return;
  bool ok = std::fwrite(&hdr, sizeof(hdr), 1, f) == 1 &&
            (bin.log.empty() || std::fwrite(bin.log.data(), 1, bin.log.size(), f) == bin.log.size()) &&
            std::fwrite(bin.cubin.data(), 1, bin.cubin.size(), f) == bin.cubin.size();
  ok = std::fclose(f) == 0 && ok;
  if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) std::remove(tmp.c_str());
}

}  // namespace

std::string cg_cache_dir() {
  if (const char* d = std::getenv("SUS2SH_CACHE_DIR")) {
    const std::string s = d;
    if (s.empty() || s == "off" || s == "0") return "";
    return s;
  }
  if (const char* x = std::getenv("XDG_CACHE_HOME"))
    if (*x) return std::string(x) + "/sus2sh";
  if (const char* home = std::getenv("HOME"))
    if (*home) return std::string(home) + "/.cache/sus2sh";
  return "";
}

CgBinary compile_cg_source(const CgSource& src, CgBuild build) {
  // binaries are cached per process: models of the same graph (or the same
  // model loaded twice) compile once
  static std::mutex* mu = new std::mutex;  // never destroyed: safe at process exit
  static auto* cache = new std::map<std::string, std::shared_ptr<const CgBinary>>;
  const bool whole = build == CgBuild::kWhole || src.units.size() < 2;
  const std::string key = src.kernel_name + ":" + std::to_string(src.code.size()) + ":" +
                          std::to_string(fnv1a(src.code)) + (whole ? ":whole" : ":units");
  {
    std::lock_guard<std::mutex> lock(*mu);
    auto it = cache->find(key);
    if (it != cache->end()) return *it->second;
  }
  std::shared_ptr<const CgBinary> bin;
  if (whole) {
    // one-program builds go through the disk cache
    const std::string dir = cg_cache_dir();
    CacheHeader hdr;
    const std::string path = dir.empty() ? std::string() : cache_path(dir, src.code, &hdr);
    CgBinary b;
    if (!path.empty() && cache_read(path, hdr, &b)) {
      bin = std::make_shared<const CgBinary>(std::move(b));
    } else {
      bin = std::make_shared<const CgBinary>(build_one_program(src.code));
      if (!path.empty()) cache_write(dir, path, hdr, *bin);
    }
  } else {
    bin = std::make_shared<const CgBinary>(build_binary(src, build));
  }
  std::lock_guard<std::mutex> lock(*mu);
  return *cache->emplace(key, bin).first->second;
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

bool CgModule::load(const CgBinary& bin, const std::string& kernel_name, std::string* err, size_t smem_bytes) {
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
  if (smem_bytes > 0) {
    auto set_attr = entry<PFN_set_attr>("cuFuncSetAttribute");
    if (!set_attr || set_attr(f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, static_cast<int>(smem_bytes)) !=
                         CUDA_SUCCESS) {
      if (err) *err = "cuFuncSetAttribute failed for the CG kernel's shared memory";
      return false;
    }
  }
  if (auto get_attr = entry<PFN_get_attr>("cuFuncGetAttribute")) {
    get_attr(&regs_, CU_FUNC_ATTRIBUTE_NUM_REGS, f);
    get_attr(&local_, CU_FUNC_ATTRIBUTE_LOCAL_SIZE_BYTES, f);
  }
  module_ = mod;
  func_ = f;
  return true;
}

int CgModule::max_active_blocks(int block, size_t smem_bytes) const {
  using PFN_occ = CUresult (*)(int*, CUfunction, int, size_t);
  static PFN_occ occ = entry<PFN_occ>("cuOccupancyMaxActiveBlocksPerMultiprocessor");
  int n = 0;
  if (!occ || !func_ || occ(&n, static_cast<CUfunction>(func_), block, smem_bytes) != CUDA_SUCCESS) return 0;
  return n;
}

bool CgModule::launch_args(void* stream, unsigned grid, unsigned block, size_t smem_bytes, void** args,
                           std::string* err) {
  static PFN_launch launch_fn = entry<PFN_launch>("cuLaunchKernel");
  if (!launch_fn || !func_) {
    if (err) *err = "CG kernel not loaded";
    return false;
  }
  if (launch_fn(static_cast<CUfunction>(func_), grid, 1, 1, block, 1, 1, static_cast<unsigned>(smem_bytes),
                static_cast<CUstream>(stream), args, nullptr) != CUDA_SUCCESS) {
    if (err) *err = "cuLaunchKernel failed for a generated kernel";
    return false;
  }
  return true;
}

bool CgModule::launch(void* stream, int N, const void* pos4, const void* B, void* G, const double* shift,
                      const double* species, double* pe, int pe_assign, std::string* err, int block,
                      size_t smem_bytes) {
  static PFN_launch launch_fn = entry<PFN_launch>("cuLaunchKernel");
  if (!launch_fn || !func_) {
    if (err) *err = "CG kernel not loaded";
    return false;
  }
  void* args[] = {&N, &pos4, &B, &G, &shift, &species, &pe, &pe_assign};
  const unsigned grid = static_cast<unsigned>((N + block - 1) / block);
  if (launch_fn(static_cast<CUfunction>(func_), grid, 1, 1, static_cast<unsigned>(block), 1, 1,
                static_cast<unsigned>(smem_bytes), static_cast<CUstream>(stream), args, nullptr) != CUDA_SUCCESS) {
    if (err) *err = "cuLaunchKernel failed for the CG kernel";
    return false;
  }
  return true;
}

}  // namespace sus2sh
