// libsus2sh_tools.so: helpers around the engine that are not part of it.
//
// In a real run GPUMD provides the structure and the integrator, and a
// trained model comes from the fitting code; the tests and the benchmark need
// seeded stand-ins for all three, plus a measurement of the FP32/FP64
// CUDA-core peak that the roofline of the SIMT kernels is quoted against.
// They live in this library so that libsus2sh.so holds the engine and its
// C-ABI only.  The model writer and the graph counts reuse the engine's
// standard-graph builder (linked from libsus2sh.so).
#include "../../include/sus2sh.h"
#include "../../include/sus2sh_tools.h"
#include "../csrc/mtp_model.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <string>
#include <vector>

namespace {

std::string g_tools_error;

template <typename F>
int tools_guarded(F&& f) {
  try {
    f();
    return SUS2SH_OK;
  } catch (const sus2sh::InputError& ex) {
    g_tools_error = ex.what();
    return SUS2SH_E_INPUT;
  } catch (const std::exception& ex) {
    g_tools_error = ex.what();
    return SUS2SH_E_ARG;
  }
}

struct SynthSpec {
  int species = 2;
  int l_max = 3;
  int k_max = 3;
  int body_order = 4;
  int rb_size = 8;
  double r_min = 2.0;
  double rc = 5.0;
  int rational = 0;                  // radial basis: 0 Chebyshev-sss, 1 its rational map, 2 Laguerre-log1p
  std::vector<int> body_l_max_list;  // empty: none written
  std::vector<double> shift;         // [S] site energy shifts
  double radial_sigma = 0.1;
  double moment_sigma = 0.01;
  double scal = 1.0;     // radial tanh scale
  double rshift = -1.0;  // radial shift (Laguerre: rho); <0 -> (r_min+rc)/2
  double radial_type_coeff = 1.0;
  unsigned long long seed = 0;
};

// A standard graph plus seeded random coefficients, in the text layout the
// reference's reader accepts (src/force/sus2_sh.cu:2105-2482).
void write_synthetic_model(const std::string& path, const SynthSpec& sp) {
  using namespace sus2sh;
  if (sp.species <= 0 || sp.l_max < 0 || sp.l_max > 6 || sp.k_max <= 0 || sp.body_order < 2 ||
      sp.body_order > 6 || sp.rb_size <= 0 || sp.rb_size > 16 ||
      static_cast<int>(sp.shift.size()) != sp.species)
    throw InputError("Invalid synthetic model specification.");
  std::vector<int> blmax = default_body_l_max(sp.l_max);
  if (!sp.body_l_max_list.empty())
    for (size_t i = 0; i < sp.body_l_max_list.size(); ++i) blmax[2 + i] = sp.body_l_max_list[i];
  const StandardGraph g = build_standard_graph(sp.l_max, sp.k_max, sp.body_order, blmax);
  const int S = sp.species, kmu = sp.k_max * (sp.l_max + 1);
  std::mt19937_64 rng(sp.seed);
  std::normal_distribution<double> nrm(0.0, 1.0);
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) throw InputError("Cannot write synthetic model: " + path);
  auto list = [&](const char* key, const std::vector<double>& v) {
    std::fprintf(f, "%s = {", key);
    for (size_t i = 0; i < v.size(); ++i) std::fprintf(f, "%s%.17g", i ? ", " : "", v[i]);
    std::fprintf(f, "}\n");
  };
  std::fprintf(f, "MTP\nversion = 1.1.0\npotential_name = SUS2-SH synthetic\n");
  std::fprintf(f, "potential_tag = SUS2-SH\nscaling = 1.0\nscaling_map = LK\n");
  std::fprintf(f, "species_count = %d\n", S);
  std::fprintf(f, "sh_l_max = %d\nsh_k_max = %d\nsh_body_order = %d\nsh_parity = even\n", sp.l_max, sp.k_max,
               sp.body_order);
  if (!sp.body_l_max_list.empty()) {
    std::fprintf(f, "sh_body_l_max = {");
    for (size_t i = 0; i < sp.body_l_max_list.size(); ++i)
      std::fprintf(f, "%s%d", i ? ", " : "", sp.body_l_max_list[i]);
    std::fprintf(f, "}\n");
  }
  std::fprintf(f, "radial_basis_type = %s\n",
               sp.rational == 2 ? "RBLaguerre_log1p" : (sp.rational ? "RBChebyshev_sss_rational" : "RBChebyshev_sss"));
  std::fprintf(f, "\tmin_dist = %.17g\n\tmax_dist = %.17g\n", sp.r_min, sp.rc);
  std::fprintf(f, "\tradial_basis_size = %d\n\tradial_funcs_count = %d\n", sp.rb_size, kmu);
  list("shift_coeffs", sp.shift);
  std::vector<double> scal(2 * S * S * kmu);
  const double rshift = sp.rshift < 0.0 ? 0.5 * (sp.r_min + sp.rc) : sp.rshift;
  for (int mu = 0; mu < kmu; ++mu)
    for (int p = 0; p < S * S; ++p) {
      scal[2 * mu * S * S + p] = sp.scal;
      scal[2 * mu * S * S + S * S + p] = rshift;
    }
  list("scal_coeffs", scal);
  std::fprintf(f, "\tradial_coeffs\n");
  for (int mu = 0; mu < kmu; ++mu) {
    std::fprintf(f, "\t\t{");
    for (int n = 0; n < sp.rb_size; ++n) std::fprintf(f, "%s%.17g", n ? ", " : "", sp.radial_sigma * nrm(rng));
    for (int t = 0; t < S; ++t) std::fprintf(f, ", %.17g", sp.radial_type_coeff);
    std::fprintf(f, "}\n");
  }
  std::fprintf(f, "alpha_moments_count = %d\n", g.node_count);
  std::fprintf(f, "alpha_index_basic_count = %d\nalpha_index_basic = {", static_cast<int>(g.basic_k.size()));
  for (size_t i = 0; i < g.basic_k.size(); ++i)
    std::fprintf(f, "%s{%d, %d, %d}", i ? ", " : "", g.basic_k[i], g.basic_l[i], g.basic_m[i]);
  std::fprintf(f, "}\n");
  std::fprintf(f, "sh_product_count = %d\nsh_products = {", static_cast<int>(g.products.size()));
  for (size_t p = 0; p < g.products.size(); ++p)
    std::fprintf(f, "%s{%d, %d, %d, %.17g}", p ? ", " : "", g.products[p].left, g.products[p].right,
                 g.products[p].target, g.products[p].coeff);
  std::fprintf(f, "}\n");
  std::fprintf(f, "alpha_scalar_moments = %d\nalpha_moment_mapping = {", static_cast<int>(g.scalars.size()));
  for (size_t s = 0; s < g.scalars.size(); ++s) std::fprintf(f, "%s%d", s ? ", " : "", g.scalars[s]);
  std::fprintf(f, "}\n");
  std::fprintf(f, "sh_scalar_info_count = %d\nsh_scalar_info = {", static_cast<int>(g.scalars.size()));
  for (size_t s = 0; s < g.scalar_body.size(); ++s) std::fprintf(f, "%s{%d}", s ? ", " : "", g.scalar_body[s]);
  std::fprintf(f, "}\n");
  list("species_coeffs", std::vector<double>(S, 1.0));
  std::vector<double> w(g.scalars.size());
  for (double& x : w) x = sp.moment_sigma * nrm(rng);
  list("moment_coeffs", w);
  std::fclose(f);
}

// ---- velocity Verlet (units A, fs, amu, eV) ----------------------------------
constexpr double kAccel = 9.648533212331002e-3;  // (eV/A/amu) -> A/fs^2

// Half kick + drift; the force (and optionally energy/virial) arrays are
// zeroed after use so the next accumulating force call starts from zero.
__global__ void k_kick_drift(int N, double dt, const double* __restrict__ inv_mass_type,
                             const int* __restrict__ type, double* __restrict__ f, double* __restrict__ v,
                             double* __restrict__ x, double* __restrict__ pe, double* __restrict__ vir) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double a = 0.5 * dt * kAccel * inv_mass_type[type[i]];
  for (int d = 0; d < 3; ++d) {
    const double vv = v[i + d * N] + a * f[i + d * N];
    v[i + d * N] = vv;
    x[i + d * N] += dt * vv;
    f[i + d * N] = 0.0;
  }
  if (pe) pe[i] = 0.0;
  if (vir)
    for (int q = 0; q < 9; ++q) vir[static_cast<size_t>(q) * N + i] = 0.0;
}

__global__ void k_kick(int N, double dt, const double* __restrict__ inv_mass_type, const int* __restrict__ type,
                       const double* __restrict__ f, double* __restrict__ v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double a = 0.5 * dt * kAccel * inv_mass_type[type[i]];
  for (int d = 0; d < 3; ++d) v[i + d * N] += a * f[i + d * N];
}

// Sum of per-atom energy (out[0]) and virial (out[1..9]): warp shuffles, one
// FP64 atomic per block and component.
__global__ void k_tools_reduce(int N, const double* __restrict__ pe, const double* __restrict__ vir,
                               double* __restrict__ out) {
  __shared__ double red[10][8];
  double v[10];
  for (int q = 0; q < 10; ++q) v[q] = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    v[0] += pe[i];
    if (vir)
      for (int q = 0; q < 9; ++q) v[q + 1] += vir[static_cast<size_t>(q) * N + i];
  }
  for (int q = 0; q < 10; ++q) {
    double x = v[q];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x < 10) {
    double x = 0.0;
    for (int w = 0; w < (blockDim.x >> 5); ++w) x += red[threadIdx.x][w];
    atomicAdd(out + threadIdx.x, x);
  }
}

// FMA throughput probe: 8 independent dependency chains per thread, each
// thread writes only its own output slot.
template <typename T>
__global__ void __launch_bounds__(256) k_fma_peak(int iters, T seed, T* __restrict__ out) {
  T a0 = seed + threadIdx.x, a1 = a0 + T(1), a2 = a0 + T(2), a3 = a0 + T(3);
  T a4 = a0 + T(4), a5 = a0 + T(5), a6 = a0 + T(6), a7 = a0 + T(7);
  const T m = T(0.9999), c = T(1e-4);
  for (int k = 0; k < iters; ++k) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
      a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
    }
  }
  out[blockIdx.x * blockDim.x + threadIdx.x] = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
}

inline int blocks_for(int n, int b) { return (n + b - 1) / b; }

double measure_fma_tflops(bool fp64) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int blocks = sms * 8, threads = 256, iters = fp64 ? 512 : 2048;
  void* out = nullptr;
  if (cudaMalloc(&out, sizeof(double) * blocks * threads) != cudaSuccess) return -1.0;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 6; ++rep) {
    cudaEventRecord(e0);
    if (fp64) k_fma_peak<double><<<blocks, threads>>>(iters, 1.0, static_cast<double*>(out));
    else k_fma_peak<float><<<blocks, threads>>>(iters, 1.0f, static_cast<float*>(out));
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best) best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (cudaGetLastError() != cudaSuccess) return -1.0;
  const double flops = 2.0 * 8.0 * 16.0 * iters * static_cast<double>(blocks) * threads;
  return flops / (best * 1e-3) / 1e12;
}

}  // namespace

extern "C" {

const char* sus2sh_tools_last_error(void) { return g_tools_error.c_str(); }

int sus2sh_write_synthetic_model(const char* path, int species, int l_max, int k_max, int body_order,
                                 const int* body_l_max, int n_body_l_max, int rb_size, double r_min, double rc,
                                 int rational, const double* shift_coeffs, double radial_sigma,
                                 double moment_sigma, double scal, double rshift, unsigned long long seed) {
  if (!path || !shift_coeffs) return SUS2SH_E_ARG;
  return tools_guarded([&] {
    SynthSpec sp;
    sp.species = species;
    sp.l_max = l_max;
    sp.k_max = k_max;
    sp.body_order = body_order;
    sp.rb_size = rb_size;
    sp.r_min = r_min;
    sp.rc = rc;
    sp.rational = rational;
    if (body_l_max)
      for (int i = 0; i < n_body_l_max; ++i) sp.body_l_max_list.push_back(body_l_max[i]);
    sp.shift.assign(shift_coeffs, shift_coeffs + species);
    sp.radial_sigma = radial_sigma;
    sp.moment_sigma = moment_sigma;
    sp.scal = scal;
    sp.rshift = rshift;
    sp.seed = seed;
    write_synthetic_model(path, sp);
  });
}

int sus2sh_standard_graph_counts(int l_max, int k_max, int body_order, const int* body_l_max, int n_body_l_max,
                                 int* out) {
  if (!out) return SUS2SH_E_ARG;
  return tools_guarded([&] {
    std::vector<int> bl = sus2sh::default_body_l_max(l_max);
    if (body_l_max)
      for (int i = 0; i < n_body_l_max && 2 + i < 7; ++i) bl[2 + i] = body_l_max[i];
    const sus2sh::StandardGraph g = sus2sh::build_standard_graph(l_max, k_max, body_order, bl);
    out[0] = g.node_count;
    out[1] = static_cast<int>(g.basic_k.size());
    out[2] = static_cast<int>(g.products.size());
    out[3] = static_cast<int>(g.scalars.size());
    out[4] = g.tensor_blocks;
    out[5] = g.cg_blocks;
    out[6] = g.cg_terms;
    out[7] = g.max_layer;
  });
}

int sus2sh_md_kick_drift(int N, double dt, const double* inv_mass_type, const int* type, double* force,
                         double* velocity, double* position, double* potential, double* virial, void* stream) {
  if (N <= 0) return SUS2SH_OK;
  k_kick_drift<<<blocks_for(N, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      N, dt, inv_mass_type, type, force, velocity, position, potential, virial);
  return cudaPeekAtLastError() == cudaSuccess ? SUS2SH_OK : SUS2SH_E_CUDA;
}

int sus2sh_md_kick(int N, double dt, const double* inv_mass_type, const int* type, const double* force,
                   double* velocity, void* stream) {
  if (N <= 0) return SUS2SH_OK;
  k_kick<<<blocks_for(N, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(N, dt, inv_mass_type, type, force,
                                                                           velocity);
  return cudaPeekAtLastError() == cudaSuccess ? SUS2SH_OK : SUS2SH_E_CUDA;
}

int sus2sh_reduce(int N, const double* potential, const double* virial, double* out, void* stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (cudaMemsetAsync(out, 0, 10 * sizeof(double), s) != cudaSuccess) return SUS2SH_E_CUDA;
  const int grid = std::max(1, std::min(592, blocks_for(N, 256)));
  k_tools_reduce<<<grid, 256, 0, s>>>(N, potential, virial, out);
  return cudaPeekAtLastError() == cudaSuccess ? SUS2SH_OK : SUS2SH_E_CUDA;
}

int sus2sh_measure_fma_peak(int fp64, double* tflops) {
  if (!tflops) return SUS2SH_E_ARG;
  *tflops = measure_fma_tflops(fp64 != 0);
  return *tflops > 0 ? SUS2SH_OK : SUS2SH_E_CUDA;
}

int sus2sh_random_insertion(int N, double lx, double ly, double lz, double dmin, unsigned long long seed,
                            double* position) {
  if (N <= 0 || !position || !(dmin > 0.0)) return SUS2SH_E_ARG;
  // grid of cells >= dmin; each cell holds few points
  const int nx = std::max(1, static_cast<int>(lx / dmin)), ny = std::max(1, static_cast<int>(ly / dmin)),
            nz = std::max(1, static_cast<int>(lz / dmin));
  const double cx = lx / nx, cy = ly / ny, cz = lz / nz;
  std::vector<std::vector<int>> cells(static_cast<size_t>(nx) * ny * nz);
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  const double d2 = dmin * dmin;
  long long attempts = 0;
  const long long budget = 2000LL * N + 1000000LL;
  int placed = 0;
  while (placed < N) {
    if (++attempts > budget) return -5;
    const double x = U(rng) * lx, y = U(rng) * ly, z = U(rng) * lz;
    const int ix = std::min(nx - 1, static_cast<int>(x / cx)), iy = std::min(ny - 1, static_cast<int>(y / cy)),
              iz = std::min(nz - 1, static_cast<int>(z / cz));
    bool ok = true;
    for (int oz = -1; oz <= 1 && ok; ++oz)
      for (int oy = -1; oy <= 1 && ok; ++oy)
        for (int ox = -1; ox <= 1 && ok; ++ox) {
          const int jx = (ix + ox + nx) % nx, jy = (iy + oy + ny) % ny, jz = (iz + oz + nz) % nz;
          for (int p : cells[(static_cast<size_t>(jz) * ny + jy) * nx + jx]) {
            double dx = position[p] - x, dy = position[p + N] - y, dz = position[p + 2 * N] - z;
            dx -= lx * std::round(dx / lx);
            dy -= ly * std::round(dy / ly);
            dz -= lz * std::round(dz / lz);
            if (dx * dx + dy * dy + dz * dz < d2) {
              ok = false;
              break;
            }
          }
        }
    if (!ok) continue;
    position[placed] = x;
    position[placed + N] = y;
    position[placed + 2 * N] = z;
    cells[(static_cast<size_t>(iz) * ny + iy) * nx + ix].push_back(placed);
    ++placed;
  }
  return SUS2SH_OK;
}

}  // extern "C"
