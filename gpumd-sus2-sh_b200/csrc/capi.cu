// Handle, CG-program compiler and the extern "C" entry points of sus2sh.h /
// sus2sh_diag.h.
#include "../../include/sus2sh.h"
#include "../../include/sus2sh_diag.h"
#include "cg_codegen.h"
#include "edge_jit.h"
#include "engine.cuh"
#include "mtp_model.h"
#include "sh_math.cuh"
#include "zbl.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <future>
#include <map>
#include <memory>
#include <random>
#include <string>
#include <type_traits>
#include <vector>

namespace sus2sh {
namespace {

thread_local std::string g_last_error;

// Graphs up to this many saved products get one straight-line CG function
// (above it ptxas spills: 7.5 KB at 5,475 products, 83 KB and a 4-minute
// compile at 10,993); larger graphs get the component-split kernel, and
// graphs that split into no small components run the row interpreter.
constexpr long long kCgSingleMaxProducts = 3000;

// Margin (A) of the inner neighbour list the basic-moment kernel walks: the
// listed pairs within rc + margin, refiltered from the full list whenever an
// atom has moved more than margin / 2 since the last build.
constexpr double kInnerMargin = 0.2;

// The CG kernel source the engine builds for a model: the single straight-line
// function, the component-split kernel (split: -1 auto, 0 never, 1 always), or
// none (false; the row interpreter runs, *why says why).
bool choose_cg_source(const HostModel& m, const Layered& lay, const std::vector<int>& basic_canon, int ncanon,
                      bool use_float, int split, CgSource* out, std::string* why) {
  long long terms = 0;
  for (const Row& r : lay.rows) terms += static_cast<long long>(r.left.size());
  const bool single_ok = terms <= kCgSingleMaxProducts;
  if (split == 1 || (split < 0 && !single_ok)) {
    if (generate_cg_split_source(m, lay, use_float, basic_canon, ncanon, out, why)) return true;
  }
  if (single_ok) {
    *out = generate_cg_source(m, lay, use_float, basic_canon, ncanon);
    return true;
  }
  if (why && why->empty()) *why = "graph above the single-function limit and the split kernel is disabled";
  return false;
}

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string& m) : std::runtime_error(m) {}
};

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  void resize(size_t count) {
    if (count == n) return;
    release();
    if (count) ck(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc");
    n = count;
  }
  void upload(const std::vector<T>& v) {
    resize(v.size());
    if (!v.empty()) ck(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "upload");
  }
};

// Derivative series of Chebyshev expansions: for every mu,
// sum_n c[mu][n] T_n'(x) = sum_n d[mu][n] T_n(x) with d[mu][rb-1] = 0, by the
// recurrence d_{n-1} = d_{n+1} + 2 n c_n (n = rb-1 .. 1) and d_0 halved.  The
// force kernel evaluates R' from these instead of a dT_n recurrence.
std::vector<double> chebyshev_derivative(const std::vector<double>& c, int kmu, int rb) {
  std::vector<double> d(c.size(), 0.0);
  for (int mu = 0; mu < kmu; ++mu) {
    const double* cm = &c[static_cast<size_t>(mu) * rb];
    double* dm = &d[static_cast<size_t>(mu) * rb];
    double next2 = 0.0, next1 = 0.0;  // d_{n+1}, d_n while walking down
    for (int n = rb - 1; n >= 1; --n) {
      const double v = next2 + 2.0 * n * cm[n];  // d_{n-1}
      dm[n - 1] = v;
      next2 = next1;
      next1 = v;
    }
    if (rb > 1) dm[0] *= 0.5;
  }
  return d;
}

// Derivative series of Laguerre expansions: L_n' = -(L_0 + ... + L_{n-1}), so
// sum_n c[mu][n] L_n'(u) = sum_k d[mu][k] L_k(u) with d[mu][k] = -sum_{n>k}
// c[mu][n] (d[mu][rb-1] = 0).
std::vector<double> laguerre_derivative(const std::vector<double>& c, int kmu, int rb) {
  std::vector<double> d(c.size(), 0.0);
  for (int mu = 0; mu < kmu; ++mu) {
    const double* cm = &c[static_cast<size_t>(mu) * rb];
    double* dm = &d[static_cast<size_t>(mu) * rb];
    double acc = 0.0;
    for (int k = rb - 2; k >= 0; --k) {
      acc -= cm[k + 1];
      dm[k] = acc;
    }
  }
  return d;
}

// The derivative series of the model's radial basis.
std::vector<double> radial_derivative(RadialMap kind, const std::vector<double>& c, int kmu, int rb) {
  return kind == RadialMap::LaguerreLog1p ? laguerre_derivative(c, kmu, rb) : chebyshev_derivative(c, kmu, rb);
}

// ---------------------------------------------------------------------------
// CG program: the layered rows of the saved sh_products compiled to the
// slot machine executed by k_product (see engine.cu for the row kinds).
// Forward rows follow build_explicit_sh_graph_metadata's layers
// (sus2_sh.cu:1913-2093); terminal scalar rows are fused into the energy and
// seed their sources directly (terminal-scalar fusion, sus2_sh.cu:5674-5778,
// 8149-8196); back rows are grouped by source per layer with duplicate
// (target, other) terms merged (sus2_sh.cu:2050-2092, 8966-8981).
// ---------------------------------------------------------------------------
struct ProgramHost {
  std::vector<uint32_t> code;
  std::vector<double> coef;
  int nrows = 0, nvalue = 0, nbasic = 0, ncanon = 0;
  std::vector<int> basic_canon, canon_basic;
  int terminal_rows = 0;
};

uint32_t header(int kind, size_t nt, int dst) {
  if (nt >= (1u << 14)) throw InputError("SUS2_SH product row has too many terms for the program.");
  return (static_cast<uint32_t>(kind) << 30) | (static_cast<uint32_t>(nt) << 16) |
         static_cast<uint32_t>(dst);
}

uint32_t pack2(int a, int b) { return static_cast<uint32_t>(a) | (static_cast<uint32_t>(b) << 16); }

ProgramHost compile_program(const HostModel& m, const Layered& lay) {
  ProgramHost P;
  const int M = m.moments, B = m.basic_count;
  const int C = (m.l_max + 1) * (m.l_max + 1);
  P.nbasic = B;
  P.ncanon = m.k_max * C;
  P.canon_basic.assign(P.ncanon, -1);
  for (int b = 0; b < B; ++b) {
    const int l = m.basic_l[b];
    const int k = (m.basic_mu[b] - l) / (m.l_max + 1);
    const int c = k * C + l * l + l + m.basic_m[b];
    if (P.canon_basic[c] >= 0) throw InputError("SUS2_SH alpha_index_basic lists a (k,l,m) twice.");
    P.canon_basic[c] = b;
    P.basic_canon.push_back(c);
  }
  // weight of every moment = sum of its scalar coefficients
  std::vector<double> weight(M, 0.0);
  std::vector<char> is_scalar(M, 0);
  for (int s = 0; s < m.scalar_count; ++s) {
    weight[m.moment_mapping[s]] += m.moment_coeffs[s];
    is_scalar[m.moment_mapping[s]] = 1;
  }
  std::vector<char> used(M, 0);
  for (const Row& r : lay.rows)
    for (size_t t = 0; t < r.left.size(); ++t) used[r.left[t]] = used[r.right[t]] = 1;
  // value slots: basics, then non-terminal live targets in row order
  std::vector<int> slot(M, -1);
  for (int b = 0; b < B; ++b) slot[b] = b;
  int nv = B;
  for (const Row& r : lay.rows)
    if (!lay.terminal[r.target] && (used[r.target] || is_scalar[r.target])) slot[r.target] = nv++;
  P.nvalue = nv;
  if (2 * nv >= 65536) throw InputError("SUS2_SH product graph exceeds 32767 live moments.");

  auto emit = [&](int kind, int dst, const std::vector<int>& a, const std::vector<int>& b,
                  const std::vector<double>& c) {
    P.code.push_back(header(kind, a.size(), dst));
    for (size_t t = 0; t < a.size(); ++t) {
      P.code.push_back(pack2(a[t], b[t]));
      P.coef.push_back(c[t]);
    }
    ++P.nrows;
  };
  // forward rows
  for (const Row& r : lay.rows) {
    if (slot[r.target] < 0) continue;
    std::vector<int> a, b;
    for (size_t t = 0; t < r.left.size(); ++t) {
      a.push_back(slot[r.left[t]]);
      b.push_back(slot[r.right[t]]);
    }
    emit(0, slot[r.target], a, b, r.coeff);
  }
  // terminal scalar rows: energy + seeds of their sources
  for (const Row& r : lay.rows) {
    if (!lay.terminal[r.target]) continue;
    const double w = weight[r.target];
    if (w == 0.0) continue;
    std::vector<int> a, b;
    std::vector<double> c;
    for (size_t t = 0; t < r.left.size(); ++t) {
      a.push_back(slot[r.left[t]]);
      b.push_back(slot[r.right[t]]);
      c.push_back(r.coeff[t] * w);
    }
    emit(1, 0, a, b, c);
    ++P.terminal_rows;
  }
  // seeds of non-terminal scalars (basics included)
  for (int mm = 0; mm < M; ++mm) {
    if (!is_scalar[mm] || lay.terminal[mm] || weight[mm] == 0.0) continue;
    emit(2, 0, {slot[mm]}, {0}, {weight[mm]});
  }
  // back rows, layers descending, grouped by source, duplicates merged
  for (int layer = lay.max_layer; layer >= 1; --layer) {
    std::map<int, std::vector<std::pair<std::pair<int, int>, double>>> by_src;
    for (const Row& r : lay.rows) {
      if (r.layer != layer || slot[r.target] < 0 || lay.terminal[r.target]) continue;
      for (size_t t = 0; t < r.left.size(); ++t) {
        by_src[r.left[t]].push_back({{r.target, r.right[t]}, r.coeff[t]});
        by_src[r.right[t]].push_back({{r.target, r.left[t]}, r.coeff[t]});
      }
    }
    for (auto& kv : by_src) {
      std::vector<int> a, b;
      std::vector<double> c;
      std::map<std::pair<int, int>, size_t> seen;
      for (auto& term : kv.second) {
        auto it = seen.find(term.first);
        if (it != seen.end()) {
          c[it->second] += term.second;
          continue;
        }
        seen[term.first] = c.size();
        a.push_back(slot[term.first.first]);
        b.push_back(slot[term.first.second]);
        c.push_back(term.second);
      }
      emit(3, slot[kv.first], a, b, c);
    }
  }
  return P;
}

// ---------------------------------------------------------------------------
// box geometry
// ---------------------------------------------------------------------------
void invert3(const double* h, double* inv) {
  const double det = h[0] * (h[4] * h[8] - h[5] * h[7]) - h[1] * (h[3] * h[8] - h[5] * h[6]) +
                     h[2] * (h[3] * h[7] - h[4] * h[6]);
  if (!(std::abs(det) > 0.0)) throw InputError("SUS2_SH box matrix is singular.");
  const double id = 1.0 / det;
  inv[0] = (h[4] * h[8] - h[5] * h[7]) * id;
  inv[1] = (h[2] * h[7] - h[1] * h[8]) * id;
  inv[2] = (h[1] * h[5] - h[2] * h[4]) * id;
  inv[3] = (h[5] * h[6] - h[3] * h[8]) * id;
  inv[4] = (h[0] * h[8] - h[2] * h[6]) * id;
  inv[5] = (h[2] * h[3] - h[0] * h[5]) * id;
  inv[6] = (h[3] * h[7] - h[4] * h[6]) * id;
  inv[7] = (h[1] * h[6] - h[0] * h[7]) * id;
  inv[8] = (h[0] * h[4] - h[1] * h[3]) * id;
}

// Cell grid with cells at least `cutoff` thick in every direction.
int make_geometry(const double* h, const int* pbc, double cutoff, int N, BoxGeom& g) {
  std::memcpy(g.h, h, sizeof(g.h));
  invert3(h, g.hinv);
  const double a[3] = {h[0], h[3], h[6]}, b[3] = {h[1], h[4], h[7]}, c[3] = {h[2], h[5], h[8]};
  auto cross_norm = [](const double* u, const double* v) {
    const double x = u[1] * v[2] - u[2] * v[1], y = u[2] * v[0] - u[0] * v[2], z = u[0] * v[1] - u[1] * v[0];
    return std::sqrt(x * x + y * y + z * z);
  };
  const double vol = std::abs(a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) +
                              a[2] * (b[0] * c[1] - b[1] * c[0]));
  const double thick[3] = {vol / cross_norm(b, c), vol / cross_norm(c, a), vol / cross_norm(a, b)};
  long long total = 1;
  for (int d = 0; d < 3; ++d) {
    g.pbc[d] = pbc[d] ? 1 : 0;
    int n = static_cast<int>(std::floor(thick[d] / cutoff));
    n = std::max(1, std::min(n, 1024));
    g.ncell[d] = n;
    total *= n;
  }
  const long long limit = std::max<long long>(64, 4LL * N);
  while (total > limit) {
    int d = 0;
    for (int e = 1; e < 3; ++e)
      if (g.ncell[e] > g.ncell[d]) d = e;
    total /= g.ncell[d];
    g.ncell[d] = std::max(1, g.ncell[d] / 2);
    total *= g.ncell[d];
  }
  for (int d = 0; d < 3; ++d) {
    const double w = thick[d] / g.ncell[d];
    int r = static_cast<int>(std::ceil(cutoff / w - 1e-12));
    r = std::max(1, r);
    if (!g.pbc[d]) r = std::min(r, std::max(1, g.ncell[d] - 1));
    if (g.pbc[d] && r > 2)
      throw InputError("SUS2_SH periodic box is thinner than half the neighbour cutoff (rc + skin).");
    g.reach[d] = r;
  }
  for (int r = 0; r < 3; ++r)
    for (int d = 0; d < 3; ++d) g.cellvec[3 * r + d] = h[3 * r + d] / g.ncell[d];
  for (int tx = -2; tx <= 2; ++tx)
    for (int ty = -2; ty <= 2; ++ty)
      for (int tz = -2; tz <= 2; ++tz) {
        const int code = (tx + 2) * 25 + (ty + 2) * 5 + (tz + 2);
        for (int k = 0; k < 3; ++k) g.shift[code][k] = tx * a[k] + ty * b[k] + tz * c[k];
      }
  return static_cast<int>(total);
}

}  // namespace

// ---------------------------------------------------------------------------
// the handle
// ---------------------------------------------------------------------------
struct Engine {
  HostModel model;
  Options opt;
  Layered lay;
  ProgramHost prog;
  bool use_float = true;
  RadialSetup rs{};
  std::vector<double> coef;        // [kmu][rb] unscaled
  std::vector<double> dcoef;       // [kmu][rb] derivative series of coef (radial_derivative)
  std::vector<double> pair_table;  // [S*S][stride]

  // model on device
  DevBuf<uint32_t> d_code;
  DevBuf<float> d_coef_f;
  DevBuf<double> d_coef_d;
  DevBuf<int> d_basic_canon, d_canon_basic;
  DevBuf<double> d_shift, d_species;
  DevBuf<float> d_pair_f;
  DevBuf<double> d_pair_d;

  // per-size work
  int N = 0, cap = 0, ncells = 0, cells_alloc = 0;
  BoxGeom geom{};
  BoxGeom* h_geom = nullptr;  // pinned staging
  DevBuf<BoxGeom> d_geom;
  double last_h[9] = {0};
  int last_pbc[3] = {-1, -1, -1};
  bool have_ref = false;
  bool force_next = true;
  int calls_since_build = 0;
  DevBuf<double4> pos4, ref4;
  DevBuf<int> nbr, ncount, cell_count, cell_start, cell_atoms, atom_cell, atom_rank;
  DevBuf<float4> cell_rel;  // positions in cell_atoms order, relative to their cell's corner (FP32)
  // the per-call neighbour work after the rebuild decision as one CUDA graph
  // with IF nodes (rebuilt when a size or buffer it holds changes); off for
  // good after any graph error, the plain launches then do the same work
  bool nbr_graph_ok = true;
  cudaStream_t nbr_capture = nullptr;
  cudaGraph_t nbr_graph = nullptr;
  cudaGraphExec_t nbr_exec = nullptr;
  NeighborGraphArgs nbr_args;
  // in-cutoff sub-list of the current positions, written by the basic-moment
  // kernel and walked by the force kernel (cut_valid: written since the last
  // change of positions or list)
  DevBuf<int> cut_nbr, cut_count;
  bool cut_valid = false;
  // inner list: listed pairs within rc + kInnerMargin (single boxes with a
  // skin above the margin), walked by the basic-moment kernel
  DevBuf<int> inner_nbr, inner_count;
  bool inner_valid = false;
  DevBuf<unsigned char> Bbuf, Gbuf, scratch, ftmp;
  DevBuf<Status> d_status;
  Status* h_status = nullptr;  // pinned
  int device = -1;             // the device current at creation; all tables live there
  cudaStream_t last_stream = nullptr;
  size_t prod_smem = 0;
  int prod_tile = 32;
  bool prod_global = false;
  // host-buffer path: the site energies go to the host on a second stream
  // while the forces are computed (created at the first such call)
  DevBuf<double> io_pos, io_pe, io_f, io_vir, io_red;
  DevBuf<int> io_type;
  cudaStream_t io_side = nullptr;
  cudaEvent_t io_pe_ready = nullptr, io_pe_copied = nullptr;
  // forward state
  int fwd_N = 0;
  // stage profiler (CUDA events on the caller's stream; the reference's
  // sus2_sh_profile stages neighbor/basic/product/force/accumulate,
  // sus2_sh.cu:67-80, timed there with device syncs)
  bool profile = false;
  struct EvSet {
    cudaEvent_t e[6];
  };
  std::vector<EvSet> ev_used, ev_free;
  double prof_ms[5] = {0, 0, 0, 0, 0};
  long long prof_calls = 0;
  long long launches = 0;  // kernels launched by this handle
  // ZBL tables
  DevBuf<int> d_zbl_z;
  DevBuf<double> d_zbl_in, d_zbl_out;
  double list_cutoff = 0.0;  // max(rc, largest ZBL outer cutoff)
  // batches of cells
  bool batch_active = false;
  int batch_ncells = 0;
  DevBuf<double> d_cell_hinv, d_cell_shift;
  DevBuf<int> d_cell_reach, d_batch_cell;
  // flat products + scalars (parameter gradients)
  DevBuf<int> d_fl, d_fr, d_ft, d_smap;
  DevBuf<double> d_fc, d_sw;
  DevBuf<unsigned char> pg_buf;
  // tile autotuner: CTA sizes of the edge kernels, timed on the first call
  int basic_block = 128, force_block = 128;
  bool tuned = false;
  // two-layer gate models
  bool gate = false;
  std::vector<double> gate_coef;  // [kmu][rb] first-layer radial coefficients
  std::vector<double> gate_dcoef;  // their derivative series
  GateProgDev gprog{};
  DevBuf<int> d_g_basic, d_g_prod, d_g_qslot, d_g_qbody;
  DevBuf<double> d_g_coef, d_g_w, d_g_mix, d_g_add;
  DevBuf<char> Bg, Gg, gslots, gmult, gderiv, gadj;
  // edge kernels built with NVRTC at load (shapes without an ahead-of-time build)
  // edge kernels: 0 ahead-of-time build, 1 NVRTC build of the shape (shapes
  // without an ahead-of-time build, sus2_sh_edge_jit=1, FP64 and gate models),
  // 2 NVRTC build specialised to this FP32 model's radial coefficients
  int edge_jit = 0;
  std::shared_ptr<const EdgeJitBinary> ejit_bin;
  EdgeJitModule ejit_mod;
  // model-specialised CG kernel (NVRTC); empty cubin -> interpreter
  CgSource cg_src;
  CgBinary cg_bin;
  CgModule cg_mod;
  // forward-over-reverse product kernel of the parameter gradients (first use)
  bool pg_tried = false;
  CgSource pg_src;
  CgBinary pg_bin;
  CgModule pg_mod;
  double cg_compile_ms = 0.0;
  // fused persistent batch kernel (batch_fused.cuh, option
  // sus2_sh_batch_fused=1): FP32 models with the straight-line CG kernel and
  // model-specialised edge kernels, no gate and no ZBL; built, and its
  // variant and tile size picked by timing, at the first batch call.  On the
  // 4096-cell l3k3 batch it runs 3.53 ms per evaluation against 2.13 ms for
  // the stage kernels (12 warps per SM at 168 registers, CTAs waiting at the
  // per-tile barriers, lanes idle in a tile's last partial block), so the
  // stage kernels are the default
  std::vector<float> model_table;  // coefficient table of the model-specialised edge build
  bool fused_tried = false;
  std::shared_ptr<const FusedJitBinary> fused_bin;
  std::vector<std::unique_ptr<CgModule>> fused_mods;  // one per compiled variant
  int fused_variant = 0, fused_tile = 512;
  bool fused_tuned = false;
  double fused_compile_ms = 0.0;
  DevBuf<int> d_tile_ctr;
  int sm_count = 0;

  ~Engine() {
    if (nbr_exec) cudaGraphExecDestroy(nbr_exec);
    if (nbr_graph) cudaGraphDestroy(nbr_graph);
    if (nbr_capture) cudaStreamDestroy(nbr_capture);
    if (io_side) {
      cudaStreamSynchronize(io_side);
      cudaStreamDestroy(io_side);
      cudaEventDestroy(io_pe_ready);
      cudaEventDestroy(io_pe_copied);
    }
    if (h_geom) cudaFreeHost(h_geom);
    if (h_status) cudaFreeHost(h_status);
    for (auto& v : {&ev_used, &ev_free})
      for (EvSet& es : *v)
        for (cudaEvent_t e : es.e) cudaEventDestroy(e);
  }

  EvSet* ev_begin(cudaStream_t s) {
    if (!profile) return nullptr;
    if (ev_free.empty()) {
      EvSet es;
      for (cudaEvent_t& e : es.e) ck(cudaEventCreate(&e), "cudaEventCreate");
      ev_free.push_back(es);
    }
    ev_used.push_back(ev_free.back());
    ev_free.pop_back();
    ck(cudaEventRecord(ev_used.back().e[0], s), "cudaEventRecord");
    return &ev_used.back();
  }
  void mark(EvSet* ev, int k, cudaStream_t s) {
    if (ev) ck(cudaEventRecord(ev->e[k], s), "cudaEventRecord");
  }
  // Waits for recorded calls and folds their stage times into prof_ms.
  void profile_collect() {
    for (EvSet& es : ev_used) {
      ck(cudaEventSynchronize(es.e[5]), "cudaEventSynchronize");
      for (int k = 0; k < 5; ++k) {
        float ms = 0.0f;
        ck(cudaEventElapsedTime(&ms, es.e[k], es.e[k + 1]), "cudaEventElapsedTime");
        prof_ms[k] += ms;
      }
      ++prof_calls;
      ev_free.push_back(es);
    }
    ev_used.clear();
  }

  size_t elem() const { return use_float ? sizeof(float) : sizeof(double); }

  void init(const char* path, int num_atoms, int nopts, const char** opts) {
    model = load_model(path);
    opt = parse_options(model, nopts, opts);
    use_float = opt.use_float;
    profile = opt.profile;
    lay = layer_products(model);
    prog = compile_program(model, lay);
    gate = model.gate.enabled;
    list_cutoff = model.rc;
    if (model.zbl_enabled) {
      // atomic numbers from the model, else from the element symbols after the
      // file name (SUS2_SH constructor, sus2_sh.cu:7824-7860)
      std::vector<int> z = model.zbl_atomic_numbers;
      if (z.empty()) {
        if (nopts < model.species_count)
          throw InputError(
              "SUS2_SH ZBL model requires zbl_atomic_numbers metadata or element symbols after the model file.");
        for (int t = 0; t < model.species_count; ++t) {
          const std::string sym = opts[t] ? opts[t] : "";
          const int an = zbl::atomic_number(sym);
          if (an <= 0) throw InputError("SUS2_SH ZBL cannot map element symbol to an atomic number: " + sym);
          z.push_back(an);
        }
      }
      if (static_cast<int>(z.size()) != model.species_count)
        throw InputError("SUS2_SH ZBL metadata should provide one atomic number per species.");
      std::vector<double> pin, pout;
      const std::string err = zbl::pair_cutoffs(z, model.zbl_inner, model.zbl_outer, model.zbl_typewise,
                                                model.zbl_typewise ? model.zbl_typewise_factor : 0.0, pin, pout);
      if (!err.empty()) throw InputError("SUS2_SH ZBL metadata error: " + err);
      d_zbl_z.upload(z);
      d_zbl_in.upload(pin);
      d_zbl_out.upload(pout);
      for (double o : pout) list_cutoff = std::max(list_cutoff, o);
    }
    const int S = model.species_count, kmu = model.radial_funcs, rb = model.rb_size;
    // radial tables: unscaled c[mu][n] uniform; per-pair (scal, shift) and
    // the LK scale scaling*rtc[zi]*rtc[zj] (sus2_sh.cu:2484-2517)
    coef = model.radial_coeffs;
    rs.species = S;
    rs.kmu = kmu;
    rs.rb = rb;
    rs.kind = static_cast<int>(model.radial_map);
    rs.pair_stride = 2 * kmu + 1;
    rs.rc = model.rc;
    bool shared = true;
    pair_table.assign(static_cast<size_t>(S) * S * rs.pair_stride, 0.0);
    for (int zi = 0; zi < S; ++zi)
      for (int zj = 0; zj < S; ++zj) {
        const int pair = zi * S + zj;
        double* row = &pair_table[static_cast<size_t>(pair) * rs.pair_stride];
        for (int mu = 0; mu < kmu; ++mu) {
          const int off = 2 * mu * S * S + S * zi + zj;
          row[2 * mu] = model.scal_coeffs[off];
          row[2 * mu + 1] = model.scal_coeffs[off + S * S];
          if (row[2 * mu] != row[0] || row[2 * mu + 1] != row[1]) shared = false;
        }
        row[2 * kmu] = model.scaling * model.radial_type_coeffs[zi] * model.radial_type_coeffs[zj];
      }
    rs.shared_xi = shared;
    if (gate) gate_coef = model.gate.radial_coeffs;
    if (opt.reference_rounding) {
      // the reference's FP32 radial tables (sus2_sh.cu:2499-2512)
      for (double& x : gate_coef) x = static_cast<double>(static_cast<float>(x));
      for (double& x : coef) x = static_cast<double>(static_cast<float>(x));
      for (double& x : pair_table) x = static_cast<double>(static_cast<float>(x));
    }
    if (pair_table.size() > static_cast<size_t>(kMaxPairTable))
      throw InputError("SUS2_SH radial pair table too large (species_count^2 * (2*radial_funcs+1) > 8192).");
    dcoef = radial_derivative(model.radial_map, coef, kmu, rb);
    if (gate) gate_dcoef = radial_derivative(model.radial_map, gate_coef, kmu, rb);
    // edge kernels from NVRTC now: specialised to the model (FP32, non-gate),
    // or for the shape when it has no ahead-of-time build (or on request)
    if (opt.edge_jit) {
      edge_jit = 1;
    } else if (use_float && !gate && opt.model_edges) {
      edge_jit = 2;
    } else if (!shape_supported(model.l_max, model.k_max, model.rb_size) || rs.kind == kRadialLaguerre) {
      // the ahead-of-time kernels carry the Chebyshev bases only
      edge_jit = 1;
    }
    std::future<std::shared_ptr<const EdgeJitBinary>> model_edges;
    if (edge_jit == 2) {
      // built on host threads while the CG kernel below compiles
      std::vector<float> table(kMaxCoef);
      table.resize(fill_coef(coef, dcoef, table.data()));
      model_table = table;
      model_edges = std::async(std::launch::async, [l = model.l_max, k = model.k_max, rb = model.rb_size, table,
                                                    shared_xi = rs.shared_xi != 0, kind = rs.kind] {
        return compile_model_edge_kernels(l, k, rb, table, shared_xi, kind);
      });
    } else if (edge_jit == 1) {
      ejit_bin = compile_edge_kernels(use_float, model.l_max, model.k_max, model.rb_size, 128, gate, rs.kind);
    }
    // device uploads
    d_code.upload(prog.code);
    if (use_float) {
      d_coef_f.upload(std::vector<float>(prog.coef.begin(), prog.coef.end()));
      d_pair_f.upload(std::vector<float>(pair_table.begin(), pair_table.end()));
    } else {
      d_coef_d.upload(prog.coef);
      d_pair_d.upload(pair_table);
    }
    d_basic_canon.upload(prog.basic_canon);
    if (gate) build_gate_program();
    d_canon_basic.upload(prog.canon_basic);
    d_shift.upload(model.shift_coeffs);
    d_species.upload(model.species_coeffs);
    {
      std::vector<int> l, r, t;
      std::vector<double> c;
      for (const Product& p : model.products) {
        l.push_back(p.left);
        r.push_back(p.right);
        t.push_back(p.target);
        c.push_back(p.coeff);
      }
      d_fl.upload(l);
      d_fr.upload(r);
      d_ft.upload(t);
      d_fc.upload(c);
      d_smap.upload(model.moment_mapping);
      d_sw.upload(model.moment_coeffs);
    }
    ck(cudaGetDevice(&device), "cudaGetDevice");
    ck(cudaMallocHost(&h_geom, sizeof(BoxGeom)), "cudaMallocHost");
    ck(cudaMallocHost(&h_status, sizeof(Status)), "cudaMallocHost");
    std::memset(h_status, 0, sizeof(Status));
    d_geom.resize(1);
    d_status.resize(1);
    ck(cudaMemset(d_status.p, 0, sizeof(Status)), "cudaMemset");
    // product kernel launch shape: lane = atom, slots in shared memory when
    // they fit, else in an HBM scratch [slot][N]
    const size_t per_atom = 2ull * prog.nvalue * elem();
    int best_tile = 0, best_threads = 0;
    for (int tile : {32, 64, 128}) {
      const size_t bytes = per_atom * tile;
      if (bytes > 227 * 1024) continue;
      const int ctas = std::min<int>(static_cast<int>((227 * 1024) / bytes), 2048 / tile);
      if (ctas * tile > best_threads) {
        best_threads = ctas * tile;
        best_tile = tile;
      }
    }
    prod_global = best_tile == 0;
    prod_tile = best_tile ? best_tile : 128;
    prod_smem = per_atom * prod_tile;
    // model-specialised CG kernel (straight-line or component-split)
    if (opt.cg_jit) {
      const auto t0 = std::chrono::steady_clock::now();
      std::string why;
      if (choose_cg_source(model, lay, prog.basic_canon, prog.ncanon, use_float, opt.cg_split, &cg_src, &why))
        cg_bin = compile_cg_source(cg_src, opt.cg_whole ? CgBuild::kWhole : CgBuild::kParallel);
      cg_compile_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    if (model_edges.valid()) {
      // a failed model-specialised build falls back to the kernels that read
      // the coefficients from their parameters (ahead of time, or built for
      // the shape)
      try {
        ejit_bin = model_edges.get();
      } catch (const std::exception&) {
        ejit_bin.reset();
        edge_jit = shape_supported(model.l_max, model.k_max, model.rb_size) && rs.kind != kRadialLaguerre ? 0 : 1;
        if (edge_jit == 1)
          ejit_bin = compile_edge_kernels(use_float, model.l_max, model.k_max, model.rb_size, 128, gate, rs.kind);
      }
    }
    if (num_atoms > 0) ensure_size(num_atoms);
  }

  void ensure_size(int n) {
    if (n == N) return;
    if (n <= 0 || n >= (1 << 24)) throw InputError("SUS2_SH engine supports 1 <= N < 16777216 atoms.");
    if (last_stream) cudaStreamSynchronize(last_stream);
    N = n;
    const size_t nb = static_cast<size_t>(model.k_max) * (model.l_max + 1) * (model.l_max + 1);
    pos4.resize(N);
    ref4.resize(N);
    ncount.resize(N);
    atom_cell.resize(N);
    atom_rank.resize(N);
    cell_atoms.resize(N);
    cell_rel.resize(N);
    Bbuf.resize(nb * N * elem());
    Gbuf.resize(nb * N * elem());
    ftmp.resize(static_cast<size_t>(N) * (use_float ? sizeof(float4) : sizeof(double4)));
    if (prod_global) scratch.resize(2ull * prog.nvalue * N * elem());
    if (gate) {
      const size_t kmu = static_cast<size_t>(model.radial_funcs);
      Bg.resize(nb * N * elem());
      Gg.resize(nb * N * elem());
      gslots.resize(2ull * gprog.nslots * N * elem());
      gmult.resize(kmu * N * elem());
      gderiv.resize(kmu * N * elem());
      gadj.resize(kmu * N * elem());
    }
    cap = 0;
    nbr.release();
    cut_nbr.release();
    cut_count.resize(N);
    cut_valid = false;
    inner_nbr.release();
    inner_count.resize(N);
    inner_valid = false;
    have_ref = false;
    force_next = true;
  }

  template <typename T>
  EdgeArgs<T> edge_args() const {
    EdgeArgs<T> a{};
    a.N = N;
    a.cap = cap;
    a.l_max = model.l_max;
    a.k_max = model.k_max;
    a.rs = rs;
    a.pos4 = pos4.p;
    a.nbr = nbr.p;
    a.ncount = ncount.p;
    a.cut_nbr = cut_nbr.p;
    a.cut_count = cut_count.p;
    a.use_cut = 0;
    a.inner_nbr = inner_valid ? inner_nbr.p : nullptr;
    a.inner_count = inner_count.p;
    a.pair_table = use_float ? static_cast<const void*>(d_pair_f.p) : static_cast<const void*>(d_pair_d.p);
    if (batch_active) {
      a.shift = reinterpret_cast<const double(*)[3]>(d_cell_shift.p);
      a.atom_cell = d_batch_cell.p;
    } else {
      a.shift = d_geom.p->shift;
      a.atom_cell = nullptr;
    }
    fill_coef(coef, dcoef, a.coef);
    return a;
  }

  // The edge kernels' coefficient table: c[mu][n], then the derivative series
  // when both fit kMaxCoef.  Returns the entries written.
  template <typename T>
  static size_t fill_coef(const std::vector<double>& c, const std::vector<double>& d, T* out) {
    for (size_t k = 0; k < c.size(); ++k) out[k] = static_cast<T>(c[k]);
    if (2 * c.size() > static_cast<size_t>(kMaxCoef)) return c.size();
    for (size_t k = 0; k < d.size(); ++k) out[c.size() + k] = static_cast<T>(d[k]);
    return c.size() + d.size();
  }

  // EdgeArgs of the gate's first layer: same pair tables, gate coefficients.
  template <typename T>
  EdgeArgs<T> edge_args_gate() const {
    EdgeArgs<T> a = edge_args<T>();
    fill_coef(gate_coef, gate_dcoef, a.coef);
    return a;
  }

  // Slots for the moments the gate signals need (basics first), the needed
  // products below the gate's product limit in file order, and the signal maps.
  void build_gate_program() {
    const GateModel& g = model.gate;
    if (model.radial_funcs > 48) throw InputError("SUS2_SH gate supports radial_funcs_count <= 48.");
    std::vector<int> slot(model.moments, -1);
    std::vector<int> bcanon;
    int ns = 0;
    for (int b = 0; b < model.basic_count; ++b)
      if (g.needed[b]) {
        slot[b] = ns++;
        bcanon.push_back(prog.basic_canon[b]);
      }
    const int nbasic = ns;
    for (int m = model.basic_count; m < model.moments; ++m)
      if (g.needed[m]) slot[m] = ns++;
    std::vector<int> qslot, qbody;
    for (size_t q = 0; q < g.moment_of.size(); ++q) {
      int& sl = slot[g.moment_of[q]];
      if (sl < 0) sl = ns++;  // zero-weight signal: a zero slot keeps every read in bounds
      qslot.push_back(sl);
      qbody.push_back(g.body_of[q]);
    }
    std::vector<int> pr;
    std::vector<double> pc;
    for (int p = 0; p < g.product_limit; ++p) {
      const Product& x = model.products[p];
      if (!g.needed[x.target]) continue;
      pr.push_back(slot[x.left]);
      pr.push_back(slot[x.right]);
      pr.push_back(slot[x.target]);
      pc.push_back(x.coeff);
    }
    d_g_basic.upload(bcanon);
    d_g_prod.upload(pr);
    d_g_coef.upload(pc);
    d_g_qslot.upload(qslot);
    d_g_qbody.upload(qbody);
    d_g_w.upload(g.weights);
    d_g_mix.upload(g.body_mix.empty() ? std::vector<double>(1, 0.0) : g.body_mix);
    d_g_add.upload(g.additive);
    gprog = GateProgDev{};
    gprog.nslots = ns;
    gprog.nbasic = nbasic;
    gprog.basic_canon = d_g_basic.p;
    gprog.nprod = static_cast<int>(pc.size());
    gprog.prod = d_g_prod.p;
    gprog.coef = d_g_coef.p;
    gprog.nq = static_cast<int>(qslot.size());
    gprog.q_slot = d_g_qslot.p;
    gprog.q_body = d_g_qbody.p;
    gprog.kmu = model.radial_funcs;
    gprog.nbody = g.body_count;
    gprog.mode = g.mode == GateMode::MuBodyLinearCombo ? 1 : 2;
    gprog.amplitude = g.amplitude;
    gprog.weights = d_g_w.p;
    gprog.body_mix = d_g_mix.p;
    gprog.additive = d_g_add.p;
  }

  ProgramDev program_dev() const {
    ProgramDev p{};
    p.nrows = prog.nrows;
    p.nvalue = prog.nvalue;
    p.nbasic = prog.nbasic;
    p.ncanon = prog.ncanon;
    p.code = d_code.p;
    p.coef = use_float ? static_cast<const void*>(d_coef_f.p) : static_cast<const void*>(d_coef_d.p);
    p.basic_canon = d_basic_canon.p;
    p.canon_basic = d_canon_basic.p;
    return p;
  }

  // Batch of independent cells: geometry tables, packing and a fresh
  // neighbour list (cutoff rc, no skin) on every call.  After the first call
  // with a given (N, ncells) nothing synchronises or allocates, so the call
  // can be captured in a CUDA graph.
  void prepare_batch(cudaStream_t s, int n, int ncells, const int* off, const double* cell_h, const int* cell_pbc,
                     const int* type, const double* x, bool fill_lists = true) {
    inner_valid = false;  // the batch list holds only pairs within rc
    cut_valid = false;  // new positions
    if (ncells <= 0) throw InputError("sus2sh batch: ncells must be positive.");
    ensure_size(n);
    last_stream = s;
    if (ncells != batch_ncells) {
      d_cell_hinv.resize(9ull * ncells);
      d_cell_reach.resize(3ull * ncells);
      d_cell_shift.resize(375ull * ncells);
      batch_ncells = ncells;
      cap = 0;
    }
    d_batch_cell.resize(N);
    batch_active = true;
    have_ref = false;  // the single-box list is no longer current
    force_next = true;
    launch_batch_geometry(s, ncells, cell_h, cell_pbc, list_cutoff, d_cell_hinv.p, d_cell_reach.p,
                          reinterpret_cast<double(*)[3]>(d_cell_shift.p), &d_status.p->thin_cell);
    launch_batch_pack(s, N, ncells, off, x, type, cell_h, d_cell_hinv.p, cell_pbc, model.species_count,
                      d_batch_cell.p, pos4.p, d_status.p);
    launches += 2;
    const double cutoff2 = list_cutoff * list_cutoff;
    if (cap == 0) {
      ck(cudaMemsetAsync(&d_status.p->max_count, 0, sizeof(int), s), "memset");
      launch_batch_fill(s, N, ncells, off, d_batch_cell.p, pos4.p, cell_h, d_cell_reach.p, cutoff2, nullptr,
                        ncount.p, 0, 1, d_status.p);
      Status st{};
      ck(cudaMemcpyAsync(&st, d_status.p, sizeof(Status), cudaMemcpyDeviceToHost, s), "status");
      ck(cudaStreamSynchronize(s), "cudaStreamSynchronize");
      if (st.thin_cell) throw InputError("sus2sh batch: a periodic cell is thinner than half the cutoff.");
      grow_capacity(st.max_count);
      launches += 2;
    }
    if (fill_lists) {  // (the fused batch kernel fills them itself)
      launch_batch_fill(s, N, ncells, off, d_batch_cell.p, pos4.p, cell_h, d_cell_reach.p, cutoff2, nbr.p,
                        ncount.p, cap, 0, d_status.p);
      launches += 2;
    }
    ck(cudaGetLastError(), "batch neighbour build launch");
  }

  // The fused batch kernel for this model, built at the first batch call;
  // false (stage kernels) when the model is not of the kind it covers, the
  // option turns it off or its build fails.
  bool fused_available() {
    if (fused_tried) return fused_bin != nullptr;
    fused_tried = true;
    if (!opt.batch_fused || !use_float || gate || model.zbl_enabled || edge_jit != 2 || !ejit_bin ||
        !ejit_bin->model_coef || cg_bin.cubin.empty() || cg_src.split || cg_src.device_fn.empty())
      return false;
    try {
      const std::vector<std::pair<int, int>> variants = {{128, 3}, {128, 2}};
      auto bin = compile_batch_fused(model.l_max, model.k_max, model.rb_size, model_table, rs.shared_xi != 0, rs.kind,
                                     cg_src.device_fn, variants);
      std::vector<std::unique_ptr<CgModule>> mods;
      for (size_t v = 0; v < bin->names.size(); ++v) {
        CgBinary cb;
        cb.cubin = bin->cubin;
        auto mod = std::make_unique<CgModule>();
        std::string err;
        if (!mod->load(cb, bin->names[v], &err, fused_smem(kFusedMaxTile))) throw CudaError(err);
        mods.push_back(std::move(mod));
      }
      cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device);
      d_tile_ctr.resize(1);
      fused_mods = std::move(mods);
      fused_compile_ms = bin->compile_ms;
      fused_bin = bin;
    } catch (const std::exception&) {
      fused_bin.reset();
      fused_mods.clear();
    }
    return fused_bin != nullptr;
  }

  // Largest tile the timing picks from, and the shared memory of a tile size:
  // the pair table and an FP32 force buffer of 2 tiles + 1024 atoms (a tile
  // holds at most tile - 1 atoms plus its last cell).
  static constexpr int kFusedMaxTile = 1024;
  static int fused_buf_atoms(int tile) { return 2 * tile + 1024; }
  size_t fused_smem(int tile) const {
    return (edge_smem<float>() + 15) / 16 * 16 + 3 * sizeof(float) * static_cast<size_t>(fused_buf_atoms(tile));
  }

  void launch_fused(cudaStream_t s, int variant, int tile, int ncells, const int* off, const double* cell_h,
                    double* pe, double* force, double* virial, double* cell_energy, double* cell_virial) {
    EdgeArgs<float> a = edge_args<float>();
    a.cut_nbr = nullptr;  // the batch list holds pairs within rc only
    a.use_cut = 0;
    batch::FusedArgs f{};
    f.ncells = ncells;
    f.ntiles = N / tile + 1;
    f.tile_atoms = tile;
    f.buf_atoms = fused_buf_atoms(tile);
    f.off = off;
    f.shift_coeffs = d_shift.p;
    f.species_coeffs = d_species.p;
    f.pe = pe;
    f.force = force;
    f.virial = virial;
    f.cell_energy = cell_energy;
    f.cell_virial = cell_virial;
    f.tile_counter = d_tile_ctr.p;
    f.fill = 1;
    f.cell_h = cell_h;
    f.cell_reach = d_cell_reach.p;
    f.cutoff2 = list_cutoff * list_cutoff;
    f.nbr = nbr.p;
    f.ncount = ncount.p;
    f.cap = cap;
    f.st = d_status.p;
    CgModule& mod = *fused_mods[variant];
    const int block = fused_bin->blocks[variant];
    const size_t smem = fused_smem(tile);
    const int per_sm = std::max(1, mod.max_active_blocks(block, smem));
    const unsigned grid = static_cast<unsigned>(std::min<long long>(f.ntiles, static_cast<long long>(per_sm) * sm_count));
    void* args[] = {&a, &f};
    std::string err;
    ck(cudaMemsetAsync(d_tile_ctr.p, 0, sizeof(int), s), "memset");
    if (!mod.launch_args(s, grid, static_cast<unsigned>(block), smem, args, &err)) throw CudaError(err);
    launches += 1;
  }

  // Variant and tile size of the fused kernel, timed once per handle on the
  // first batch (scratch outputs; this call synchronises anyway, for the
  // neighbour capacity); sus2_sh_batch_tile fixes the tile size.
  void tune_fused(cudaStream_t s, int ncells, const int* off, const double* cell_h) {
    DevBuf<double> pe_s, f_s, w_s, ce_s, cw_s;
    pe_s.resize(N);
    f_s.resize(3ull * N);
    w_s.resize(9ull * N);
    ce_s.resize(ncells);
    cw_s.resize(9ull * ncells);
    cudaEvent_t e0, e1;
    ck(cudaEventCreate(&e0), "cudaEventCreate");
    ck(cudaEventCreate(&e1), "cudaEventCreate");
    std::vector<int> tiles = {256, 512, kFusedMaxTile};
    if (opt.batch_tile > 0) tiles = {std::min(opt.batch_tile, kFusedMaxTile)};
    float best = 1e30f;
    for (size_t v = 0; v < fused_mods.size(); ++v)
      for (int tile : tiles) {
        auto run = [&] {
          launch_fused(s, static_cast<int>(v), tile, ncells, off, cell_h, pe_s.p, f_s.p, w_s.p, ce_s.p, cw_s.p);
        };
        run();  // warm
        ck(cudaEventRecord(e0, s), "cudaEventRecord");
        run();
        ck(cudaEventRecord(e1, s), "cudaEventRecord");
        ck(cudaEventSynchronize(e1), "cudaEventSynchronize");
        float ms = 0.0f;
        ck(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
        if (ms < best) {
          best = ms;
          fused_variant = static_cast<int>(v);
          fused_tile = tile;
        }
      }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ck(cudaGetLastError(), "fused batch tuning");
  }

  // Positions -> pos4, conditional neighbour build.
  void prepare(cudaStream_t s, int n, const double* h, const int* pbc, const int* type, const double* x) {
    cut_valid = false;  // new positions
    ensure_size(n);
    last_stream = s;
    batch_active = false;
    bool box_changed = false;
    for (int k = 0; k < 9; ++k) box_changed |= h[k] != last_h[k];
    for (int k = 0; k < 3; ++k) box_changed |= (pbc[k] ? 1 : 0) != last_pbc[k];
    const double cutoff = list_cutoff + opt.skin;
    if (box_changed) {
      ncells = make_geometry(h, pbc, cutoff, N, geom);
      std::memcpy(last_h, h, sizeof(last_h));
      for (int k = 0; k < 3; ++k) last_pbc[k] = pbc[k] ? 1 : 0;
      if (ncells + 1 > cells_alloc) {
        // counts plus one scan block sum per 1024 cells
        cell_count.resize(ncells + 1 + (ncells + 1023) / 1024);
        cell_start.resize(ncells + 1);
        cells_alloc = ncells + 1;
      }
      // the pinned staging buffer may still feed an earlier queued copy
      ck(cudaStreamSynchronize(s), "cudaStreamSynchronize");
      *h_geom = geom;
      ck(cudaMemcpyAsync(d_geom.p, h_geom, sizeof(BoxGeom), cudaMemcpyHostToDevice, s), "geom upload");
      force_next = true;
    }
    bool force = force_next;
    if (opt.rebuild_interval > 0 && calls_since_build + 1 >= opt.rebuild_interval) force = true;
    ck(cudaMemsetAsync(&d_status.p->maxdisp2_bits, 0, sizeof(unsigned int), s), "memset");
    launch_pack(s, N, x, type, ref4.p, pos4.p, d_geom.p, have_ref ? 1 : 0, model.species_count, d_status.p);
    launches += 1;
    const float half_skin2 = static_cast<float>(0.25 * opt.skin * opt.skin);
    const double cutoff2 = cutoff * cutoff;
    if (cap == 0) {
      // first build: count pass, size the list, then fill
      ck(cudaMemsetAsync(&d_status.p->max_count, 0, sizeof(int), s), "memset");
      launch_build(s, N, 1, half_skin2, cutoff2, geom, d_geom.p, pos4.p, ref4.p, cell_count.p, cell_start.p,
                   cell_atoms.p, cell_rel.p, atom_cell.p, atom_rank.p, ncells, nullptr, ncount.p, 0, 1, d_status.p);
      launches += 8;
      Status st{};
      ck(cudaMemcpyAsync(&st, d_status.p, sizeof(Status), cudaMemcpyDeviceToHost, s), "status");
      ck(cudaStreamSynchronize(s), "cudaStreamSynchronize");
      grow_capacity(st.max_count);
      force = true;
    }
    const bool use_inner = opt.skin > kInnerMargin;
    const double inner = model.rc + kInnerMargin;
    inner_valid = false;
    const float half_margin2 = static_cast<float>(0.25 * kInnerMargin * kInnerMargin);
    bool graphed = false;
    // (a caller capturing this stream into its own graph gets the plain launches)
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &capturing) != cudaSuccess) capturing = cudaStreamCaptureStatusActive;
    if (opt.neighbor_graph && nbr_graph_ok && capturing == cudaStreamCaptureStatusNone) {
      NeighborGraphArgs g;
      g.N = N;
      g.ncells = ncells;
      g.cap = cap;
      g.use_inner = use_inner ? 1 : 0;
      g.cutoff2 = cutoff2;
      g.inner2 = inner * inner;
      g.half_margin2 = half_margin2;
      g.geom = d_geom.p;
      g.pos4 = pos4.p;
      g.ref4 = ref4.p;
      g.cell_count = cell_count.p;
      g.cell_start = cell_start.p;
      g.cell_atoms = cell_atoms.p;
      g.atom_cell = atom_cell.p;
      g.atom_rank = atom_rank.p;
      g.nbr = nbr.p;
      g.ncount = ncount.p;
      g.inner_nbr = inner_nbr.p;
      g.inner_count = inner_count.p;
      g.cell_rel = cell_rel.p;
      g.st = d_status.p;
      if (!nbr_exec || !(g == nbr_args)) {
        if (nbr_exec) cudaGraphExecDestroy(nbr_exec);
        if (nbr_graph) cudaGraphDestroy(nbr_graph);
        nbr_exec = nullptr;
        nbr_graph = nullptr;
        if (!nbr_capture) ck(cudaStreamCreateWithFlags(&nbr_capture, cudaStreamNonBlocking), "cudaStreamCreate");
        if (build_neighbor_graph(nbr_capture, g, &nbr_graph, &nbr_exec) == cudaSuccess) {
          nbr_args = g;
        } else {
          cudaGetLastError();  // the plain launches below do the same work
          nbr_graph_ok = false;
        }
      }
      if (nbr_exec) {
        launch_decide(s, d_status.p, force ? 1 : 0, half_skin2);
        ck(cudaGraphLaunch(nbr_exec, s), "neighbour graph launch");
        launches += 2 + (force ? 8 : 0);  // k_decide, k_cond and, when the host forced a build, its kernels
        graphed = true;
      }
    }
    if (!graphed) {
      launch_build(s, N, force ? 1 : 0, half_skin2, cutoff2, geom, d_geom.p, pos4.p, ref4.p, cell_count.p,
                   cell_start.p, cell_atoms.p, cell_rel.p, atom_cell.p, atom_rank.p, ncells, nbr.p, ncount.p, cap, 0,
                   d_status.p);
      launches += 8;
      if (use_inner) {
        launch_inner(s, N, d_status.p, half_margin2, inner * inner, pos4.p, nbr.p, ncount.p, cap, d_geom.p,
                     inner_nbr.p, inner_count.p);
        launches += 1;
      }
    }
    if (use_inner) inner_valid = true;
    ck(cudaGetLastError(), "neighbour build launch");
    have_ref = true;
    force_next = false;
    calls_since_build = force ? 0 : calls_since_build + 1;
  }

  void grow_capacity(int max_count) {
    int c = static_cast<int>(std::ceil(max_count * 1.25)) + 8;
    c = (c + 3) & ~3;
    if (c <= cap) return;
    cap = c;
    nbr.resize(static_cast<size_t>(cap) * N);
    cut_nbr.resize(static_cast<size_t>(cap) * N);
    inner_nbr.resize(static_cast<size_t>(cap) * N);
    cut_valid = false;
  }

  ZblTables zbl_tables() const {
    ZblTables z{};
    z.species = model.species_count;
    z.z = d_zbl_z.p;
    z.inner = d_zbl_in.p;
    z.outer = d_zbl_out.p;
    return z;
  }

  // Tile autotuner: times every supported CTA size of k_basic and k_force on
  // the live neighbour list (scratch outputs, so the caller's arrays are not
  // touched) and keeps the fastest.  Runs once per handle, at the first
  // evaluation, where the neighbour-list sizing already synchronises.
  template <typename T>
  size_t edge_smem() const {
    return sizeof(T) * static_cast<size_t>(rs.species) * rs.species * rs.pair_stride;
  }

  // CTA size of an NVRTC launch: the requested one when the module has it
  // (the model-specialised build has 64, 128 and 256), else its first.
  int jit_block(int block, bool gated) const {
    if (gated) return 128;
    for (int b : ejit_bin->blocks)
      if (b == block) return block;
    return ejit_bin->blocks.front();
  }

  // k_basic / k_force through the ahead-of-time build or the NVRTC module.
  template <typename T>
  void run_basic(cudaStream_t s, const EdgeArgs<T>& a, void* out, bool gated, int block) {
    if (edge_jit) {
      std::string err;
      if (!ejit_mod.load(*ejit_bin, &err) ||
          !ejit_mod.launch_basic(s, a.N, jit_block(block, gated), edge_smem<T>(), &a, out, gated, &err))
        throw CudaError(err);
      cut_valid = true;
      return;
    }
    if (launch_basic<T>(s, a, reinterpret_cast<T*>(out), gated ? 128 : block, gated) != 0)
      throw InputError("SUS2_SH basic kernel shape not compiled.");
    cut_valid = true;
  }

  template <typename T>
  void run_force(cudaStream_t s, const EdgeArgs<T>& a_in, const void* G, bool gated, const double* weight,
                 double* force, double* virial, double sign, int block) {
    EdgeArgs<T> a = a_in;
    a.use_cut = cut_valid ? 1 : 0;
    if (edge_jit) {
      std::string err;
      if (!ejit_mod.load(*ejit_bin, &err) ||
          !ejit_mod.launch_force(s, a.N, jit_block(block, gated), edge_smem<T>(), &a, G, weight, ftmp.p, force,
                                 virial, sign, gated, &err))
        throw CudaError(err);
      return;
    }
    if (launch_force<T>(s, a, reinterpret_cast<const T*>(G), weight, ftmp.p, force, virial, sign,
                        gated ? 128 : block, gated) != 0)
      throw InputError("SUS2_SH force kernel shape not compiled.");
  }

  template <typename T>
  void autotune(cudaStream_t s, const EdgeArgs<T>& a) {
    tuned = true;
    if (!opt.autotune || sizeof(T) != 4 || edge_jit == 1 || gate) return;
    DevBuf<double> f_scratch, w_scratch;
    f_scratch.resize(3ull * N);
    w_scratch.resize(9ull * N);
    ck(cudaMemsetAsync(Gbuf.p, 0, Gbuf.n, s), "memset");
    cudaEvent_t e0, e1;
    ck(cudaEventCreate(&e0), "cudaEventCreate");
    ck(cudaEventCreate(&e1), "cudaEventCreate");
    auto time_it = [&](auto&& launch) {
      launch();  // warm
      ck(cudaEventRecord(e0, s), "cudaEventRecord");
      launch();
      ck(cudaEventRecord(e1, s), "cudaEventRecord");
      ck(cudaEventSynchronize(e1), "cudaEventSynchronize");
      float ms = 0.0f;
      ck(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime");
      return ms;
    };
    float best_b = 1e30f, best_f = 1e30f;
    for (int block : {64, 128, 256}) {
      const float tb = time_it([&] { run_basic<T>(s, a, Bbuf.p, false, block); });
      const float tf = time_it([&] {
        // the basic launches above wrote the in-cutoff sub-list
        run_force<T>(s, a, Gbuf.p, false, nullptr, f_scratch.p, w_scratch.p, 1.0, block);
      });
      launches += 4;
      if (tb < best_b) {
        best_b = tb;
        basic_block = block;
      }
      if (tf < best_f) {
        best_f = tf;
        force_block = block;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ck(cudaGetLastError(), "autotune");
  }

  template <typename T>
  void forward_impl(cudaStream_t s, double* pe, int pe_assign, EvSet* ev = nullptr) {
    EdgeArgs<T> a = edge_args<T>();
    if (!tuned) autotune<T>(s, a);
    mark(ev, 1, s);
    if (gate) {
      const EdgeArgs<T> ag = edge_args_gate<T>();
      run_basic<T>(s, ag, Bg.p, false, basic_block);
      launch_gate_forward<T>(s, N, gprog, pos4.p, reinterpret_cast<const T*>(Bg.p), reinterpret_cast<T*>(gslots.p),
                             reinterpret_cast<T*>(gmult.p), reinterpret_cast<T*>(gderiv.p));
      a.gate_mult = reinterpret_cast<const T*>(gmult.p);
      run_basic<T>(s, a, Bbuf.p, true, 128);
      launches += 3;
    } else {
      run_basic<T>(s, a, Bbuf.p, false, basic_block);
    }
    mark(ev, 2, s);
    if (!cg_bin.cubin.empty()) {
      std::string err;
      if (!cg_mod.load(cg_bin, cg_src.kernel_name, &err, cg_src.smem_bytes) ||
          !cg_mod.launch(s, N, pos4.p, Bbuf.p, Gbuf.p, d_shift.p, d_species.p, pe, pe_assign, &err, cg_src.block,
                         cg_src.smem_bytes))
        throw CudaError(err);
    } else {
      launch_product<T>(s, N, program_dev(), pos4.p, reinterpret_cast<const T*>(Bbuf.p),
                        reinterpret_cast<T*>(Gbuf.p),
                        prod_global ? reinterpret_cast<T*>(scratch.p) : nullptr, prod_smem, prod_tile,
                        d_shift.p, d_species.p, pe, pe_assign);
    }
    launches += 2;
    if (model.zbl_enabled && pe) {
      launch_zbl(s, 0, N, cap, pos4.p, nbr.p, ncount.p, a.shift, a.atom_cell, zbl_tables(), nullptr, pe, nullptr,
                 nullptr, 1.0);
      launches += 1;
    }
  }

  template <typename T>
  void backward_impl(cudaStream_t s, const double* weight, double* force, double* virial, double sign,
                     EvSet* ev = nullptr) {
    EdgeArgs<T> a = edge_args<T>();
    ck(cudaMemsetAsync(ftmp.p, 0, ftmp.n, s), "memset");
    mark(ev, 3, s);
    if (gate) {
      // main pass (gate multipliers, dE/dh), gate back-propagation, first-layer
      // pass; the per-atom weights are folded into dE/dh by the main pass
      ck(cudaMemsetAsync(gadj.p, 0, gadj.n, s), "memset");
      ck(cudaMemsetAsync(Gg.p, 0, Gg.n, s), "memset");
      a.gate_mult = reinterpret_cast<const T*>(gmult.p);
      a.gate_deriv = reinterpret_cast<const T*>(gderiv.p);
      a.gate_adj = reinterpret_cast<T*>(gadj.p);
      run_force<T>(s, a, Gbuf.p, true, weight, force, virial, sign, 128);
      T* M = reinterpret_cast<T*>(gslots.p);
      launch_gate_backward<T>(s, N, gprog, M, M + static_cast<size_t>(gprog.nslots) * N,
                              reinterpret_cast<const T*>(gadj.p), reinterpret_cast<T*>(Gg.p));
      const EdgeArgs<T> ag = edge_args_gate<T>();
      run_force<T>(s, ag, Gg.p, false, nullptr, force, virial, sign, force_block);
      launches += 2;
    } else {
      run_force<T>(s, a, Gbuf.p, false, weight, force, virial, sign, force_block);
    }
    if (model.zbl_enabled) {
      launch_zbl(s, 1, N, cap, pos4.p, nbr.p, ncount.p, a.shift, a.atom_cell, zbl_tables(), weight, nullptr, force,
                 virial, sign);
      launches += 1;
    }
    mark(ev, 4, s);
    launch_finalize<T>(s, N, ftmp.p, force, sign);
    mark(ev, 5, s);
    launches += 2;
  }

  // dL/dw and dL/dc of a loss with upstream weights ew = dL/dE_i, fw = dL/dF_i.
  template <typename T>
  void param_grad_impl(cudaStream_t s, const double* ew, const double* fw, double* grad_w, double* grad_c) {
    if (gate) throw InputError("SUS2_SH parameter gradients do not cover two-layer gate models.");
    if (!pg_tried) {
      // model-specialised forward-over-reverse product kernel, built at the
      // first gradient call for graphs of the straight-line size
      pg_tried = true;
      long long terms = 0;
      for (const Row& r : lay.rows) terms += static_cast<long long>(r.left.size());
      if (opt.cg_jit && terms <= kCgSingleMaxProducts) {
        pg_src = generate_pg_source(model, lay, use_float, prog.basic_canon, prog.ncanon);
        pg_bin = compile_cg_source(pg_src);
      }
    }
    const bool generated = !pg_bin.cubin.empty();
    const size_t nb = static_cast<size_t>(prog.ncanon) * N;
    // generated kernel: per-atom scalar terms [scalar][N] and 64 partial sums
    // (doubles) per scalar; interpreter: its [4 M][N] scratch
    const size_t ns = static_cast<size_t>(std::max(model.scalar_count, 1));
    // the partial sums start on a 256-byte boundary (FP64 loads and stores)
    const size_t partial_at = ((4 * nb + ns * N) * sizeof(T) + 255) / 256 * 256 / sizeof(T);
    const size_t total = generated ? partial_at + (ns * 64 * sizeof(double)) / sizeof(T)
                                   : 4 * nb + 4ull * model.moments * N;
    pg_buf.resize(total * sizeof(T));
    T* base = reinterpret_cast<T*>(pg_buf.p);
    T *B = base, *Bd = base + nb, *Galpha = base + 2 * nb, *Gbeta = base + 3 * nb, *X = base + 4 * nb;
    const EdgeArgs<T> a = edge_args<T>();
    if (launch_pg_basic<T>(s, a, fw, B, Bd, grad_c) != 0)
      throw InputError("SUS2_SH parameter gradients are built ahead of time for the common shapes only; "
                       "this model shape (sh_l_max, sh_k_max, radial_basis_size) has none.");
    if (generated) {
      std::string err;
      int n = N;
      const void* p4 = pos4.p;
      const void* sp = d_species.p;
      void* args[] = {&n, &p4, &B, &Bd, &sp, &ew, &Galpha, &Gbeta, &X};
      if (!pg_mod.load(pg_bin, pg_src.kernel_name, &err) ||
          !pg_mod.launch_args(s, static_cast<unsigned>((N + 127) / 128), 128, 0, args, &err))
        throw CudaError(err);
      launch_pg_reduce<T>(s, model.scalar_count, N, X, reinterpret_cast<double*>(base + partial_at), grad_w);
    } else {
      FlatProgram fp{};
      fp.nprod = static_cast<int>(model.products.size());
      fp.nbasic = prog.nbasic;
      fp.ncanon = prog.ncanon;
      fp.nscalar = model.scalar_count;
      fp.left = d_fl.p;
      fp.right = d_fr.p;
      fp.target = d_ft.p;
      fp.coeff = d_fc.p;
      fp.basic_canon = d_basic_canon.p;
      fp.scalar_map = d_smap.p;
      fp.scalar_w = d_sw.p;
      launch_pg_product<T>(s, N, fp, model.moments, pos4.p, d_species.p, ew, B, Bd, X, Galpha, Gbeta, grad_w);
    }
    launch_pg_radial<T>(s, a, fw, Galpha, Gbeta, grad_c);
    launches += generated ? 5 : 3;
  }

  void finish(cudaStream_t s) {
    ck(cudaMemcpyAsync(h_status, d_status.p, sizeof(Status), cudaMemcpyDeviceToHost, s), "status");
    ck(cudaGetLastError(), "kernel launch");
  }

  // One energy/force/virial evaluation.  between(s), when given, is called on
  // the host between the energy and the force passes (the site energies are
  // final on stream s from that point).
  template <typename Between = std::nullptr_t>
  void compute(cudaStream_t s, int n, const double* h, const int* pbc, const int* type, const double* x,
               double* pe, double* f, double* vir, Between between = nullptr) {
    EvSet* ev = ev_begin(s);
    prepare(s, n, h, pbc, type, x);
    if (use_float) {
      forward_impl<float>(s, pe, 0, ev);
      if constexpr (!std::is_same_v<Between, std::nullptr_t>) between(s);
      backward_impl<float>(s, nullptr, f, vir, 1.0, ev);
    } else {
      forward_impl<double>(s, pe, 0, ev);
      if constexpr (!std::is_same_v<Between, std::nullptr_t>) between(s);
      backward_impl<double>(s, nullptr, f, vir, 1.0, ev);
    }
    finish(s);
  }

  int sync(int* flags) {
    if (last_stream) ck(cudaStreamSynchronize(last_stream), "cudaStreamSynchronize");
    else ck(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    int f = 0;
    if (h_status->overflow) {
      f |= SUS2SH_STATUS_OVERFLOW;
      grow_capacity(h_status->max_count);
      const int zero = 0;
      ck(cudaMemcpy(&d_status.p->overflow, &zero, sizeof(int), cudaMemcpyHostToDevice), "status reset");
      h_status->overflow = 0;
      force_next = true;
    }
    if (h_status->thin_cell) f |= SUS2SH_STATUS_THIN_CELL;
    if (h_status->bad_type) {
      f |= SUS2SH_STATUS_BAD_TYPE;
      const int zero = 0;
      ck(cudaMemcpy(&d_status.p->bad_type, &zero, sizeof(int), cudaMemcpyHostToDevice), "status reset");
      h_status->bad_type = 0;
    }
    if (flags) *flags = f;
    if (f & SUS2SH_STATUS_BAD_TYPE) {
      g_last_error = "species index outside [0, species_count) (treated as species 0)";
      return SUS2SH_E_ARG;
    }
    return (f & SUS2SH_STATUS_OVERFLOW) ? SUS2SH_E_NEIGHBOR : SUS2SH_OK;
  }
};

}  // namespace sus2sh

struct sus2sh_handle {
  sus2sh::Engine e;
};

namespace sus2sh {
bool cg_view(const sus2sh_handle* h, CgView* out) {
  if (!h || !out) return false;
  out->prog = h->e.program_dev();
  out->shift = h->e.d_shift.p;
  out->species = h->e.d_species.p;
  out->species_count = h->e.model.species_count;
  out->use_float = h->e.use_float ? 1 : 0;
  out->device = h->e.device;
  return true;
}
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace sus2sh

using sus2sh::CudaError;
using sus2sh::InputError;

namespace {
template <typename F>
int guarded(F&& f) {
  try {
    f();
    return SUS2SH_OK;
  } catch (const InputError& ex) {
    sus2sh::g_last_error = ex.what();
    return SUS2SH_E_INPUT;
  } catch (const CudaError& ex) {
    sus2sh::g_last_error = ex.what();
    return SUS2SH_E_CUDA;
  } catch (const std::exception& ex) {
    sus2sh::g_last_error = ex.what();
    return SUS2SH_E_ARG;
  }
}

bool check_box(const double* h, const int* pbc) {
  if (!h || !pbc) {
    sus2sh::g_last_error = "box_h and pbc must not be NULL";
    return false;
  }
  return true;
}
}  // namespace

namespace {
template <int L>
void real_sh_host(double x, double y, double z, double* Y, const double* G, double* V) {
  sus2sh::sh_values<L, double>(x, y, z, Y);
  if (G && V) sus2sh::sh_grad_contract<L, double>(x, y, z, G, V[0], V[1], V[2]);
}
}  // namespace

extern "C" {

int sus2sh_is_sus2_sh_file(const char* path) {
  return path && sus2sh::is_sus2_sh_file(path) ? 1 : 0;
}

int sus2sh_create(const char* path, int num_atoms, int nopts, const char** opts, sus2sh_handle** out) {
  if (!path || !out) {
    sus2sh::g_last_error = "sus2sh_create: NULL path or output handle";
    return SUS2SH_E_ARG;
  }
  *out = nullptr;
  std::unique_ptr<sus2sh_handle> h(new sus2sh_handle());
  const int rc = guarded([&] { h->e.init(path, num_atoms, nopts, opts); });
  if (rc == SUS2SH_OK) *out = h.release();
  return rc;
}

int sus2sh_compute(sus2sh_handle* h, int N, const double box_h[9], const int pbc[3], const int* type,
                   const double* position, double* potential, double* force, double* virial, void* stream) {
  if (!h || !type || !position || !potential || !force || !virial || N <= 0) {
    sus2sh::g_last_error = "sus2sh_compute: invalid argument";
    return SUS2SH_E_ARG;
  }
  if (!check_box(box_h, pbc)) return SUS2SH_E_ARG;
  return guarded([&] {
    h->e.compute(static_cast<cudaStream_t>(stream), N, box_h, pbc, type, position, potential, force, virial);
  });
}

int sus2sh_forward(sus2sh_handle* h, int N, const double box_h[9], const int pbc[3], const int* type,
                   const double* position, double* potential, void* stream) {
  if (!h || !type || !position || !potential || N <= 0) {
    sus2sh::g_last_error = "sus2sh_forward: invalid argument";
    return SUS2SH_E_ARG;
  }
  if (!check_box(box_h, pbc)) return SUS2SH_E_ARG;
  return guarded([&] {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    h->e.prepare(s, N, box_h, pbc, type, position);
    if (h->e.use_float) h->e.forward_impl<float>(s, potential, 1);
    else h->e.forward_impl<double>(s, potential, 1);
    h->e.finish(s);
    h->e.fwd_N = N;
  });
}

int sus2sh_backward(sus2sh_handle* h, const double* grad_potential, double* grad_position, double* virial,
                    void* stream) {
  if (!h || !grad_position || h->e.fwd_N != h->e.N || h->e.N == 0) {
    sus2sh::g_last_error = "sus2sh_backward: invalid argument or no matching forward";
    return SUS2SH_E_ARG;
  }
  return guarded([&] {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int N = h->e.N;
    sus2sh::ck(cudaMemsetAsync(grad_position, 0, sizeof(double) * 3 * N, s), "memset");
    if (virial) sus2sh::ck(cudaMemsetAsync(virial, 0, sizeof(double) * 9 * N, s), "memset");
    if (h->e.use_float) h->e.backward_impl<float>(s, grad_potential, grad_position, virial, -1.0);
    else h->e.backward_impl<double>(s, grad_potential, grad_position, virial, -1.0);
    h->e.finish(s);
  });
}

int sus2sh_param_grad(sus2sh_handle* h, int N, const double box_h[9], const int pbc[3], const int* type,
                      const double* position, const double* energy_weight, const double* force_weight,
                      double* grad_moment_coeffs, double* grad_radial_coeffs, void* stream) {
  if (!h || !type || !position || !grad_moment_coeffs || !grad_radial_coeffs || N <= 0) {
    sus2sh::g_last_error = "sus2sh_param_grad: invalid argument";
    return SUS2SH_E_ARG;
  }
  if (!check_box(box_h, pbc)) return SUS2SH_E_ARG;
  return guarded([&] {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    h->e.prepare(s, N, box_h, pbc, type, position);
    if (h->e.use_float)
      h->e.param_grad_impl<float>(s, energy_weight, force_weight, grad_moment_coeffs, grad_radial_coeffs);
    else
      h->e.param_grad_impl<double>(s, energy_weight, force_weight, grad_moment_coeffs, grad_radial_coeffs);
    h->e.finish(s);
  });
}

int sus2sh_compute_batch(sus2sh_handle* h, int N, int ncells, const int* cell_offset, const double* cell_h,
                         const int* cell_pbc, const int* type, const double* position, double* potential,
                         double* force, double* virial, double* cell_energy, double* cell_virial, void* stream) {
  if (!h || !cell_offset || !cell_h || !type || !position || !potential || !force || !virial || N <= 0 ||
      ncells <= 0) {
    sus2sh::g_last_error = "sus2sh_compute_batch: invalid argument";
    return SUS2SH_E_ARG;
  }
  return guarded([&] {
    sus2sh::Engine& e = h->e;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const bool fused = e.fused_available();
    e.prepare_batch(s, N, ncells, cell_offset, cell_h, cell_pbc, type, position, !fused);
    if (fused) {
      // one persistent launch: neighbour fill, moments, CG products, forces,
      // per-cell sums
      if (!e.fused_tuned) {
        e.fused_tuned = true;
        e.tune_fused(s, ncells, cell_offset, cell_h);
      }
      e.launch_fused(s, e.fused_variant, e.fused_tile, ncells, cell_offset, cell_h, potential, force, virial,
                     cell_energy, cell_virial);
      e.finish(s);
      return;
    }
    if (e.use_float) {
      e.forward_impl<float>(s, potential, 0);
      e.backward_impl<float>(s, nullptr, force, virial, 1.0);
    } else {
      e.forward_impl<double>(s, potential, 0);
      e.backward_impl<double>(s, nullptr, force, virial, 1.0);
    }
    if (cell_energy || cell_virial) {
      sus2sh::launch_cell_reduce(s, ncells, N, cell_offset, potential, cell_virial ? virial : nullptr, cell_energy,
                                 cell_virial);
      e.launches += 1;
    }
    e.finish(s);
  });
}

int sus2sh_param_grad_batch(sus2sh_handle* h, int N, int ncells, const int* cell_offset, const double* cell_h,
                            const int* cell_pbc, const int* type, const double* position, const double* energy_weight,
                            const double* force_weight, double* grad_moment_coeffs, double* grad_radial_coeffs,
                            void* stream) {
  if (!h || !cell_offset || !cell_h || !type || !position || !grad_moment_coeffs || !grad_radial_coeffs ||
      N <= 0 || ncells <= 0) {
    sus2sh::g_last_error = "sus2sh_param_grad_batch: invalid argument";
    return SUS2SH_E_ARG;
  }
  return guarded([&] {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    h->e.prepare_batch(s, N, ncells, cell_offset, cell_h, cell_pbc, type, position);
    if (h->e.use_float)
      h->e.param_grad_impl<float>(s, energy_weight, force_weight, grad_moment_coeffs, grad_radial_coeffs);
    else
      h->e.param_grad_impl<double>(s, energy_weight, force_weight, grad_moment_coeffs, grad_radial_coeffs);
    h->e.finish(s);
  });
}

int sus2sh_compute_host(sus2sh_handle* h, int N, const double box_h[9], const int pbc[3], const int* type,
                        const double* position, double* potential, double* force, double* virial_total,
                        void* stream) {
  if (!h || !type || !position || !potential || !force || N <= 0) {
    sus2sh::g_last_error = "sus2sh_compute_host: invalid argument";
    return SUS2SH_E_ARG;
  }
  if (!check_box(box_h, pbc)) return SUS2SH_E_ARG;
  return guarded([&] {
    sus2sh::Engine& e = h->e;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    e.io_pos.resize(3ull * N);
    e.io_type.resize(N);
    e.io_pe.resize(N);
    e.io_f.resize(3ull * N);
    e.io_vir.resize(9ull * N);
    e.io_red.resize(10);
    using sus2sh::ck;
    ck(cudaMemcpyAsync(e.io_pos.p, position, sizeof(double) * 3 * N, cudaMemcpyHostToDevice, s), "H2D");
    ck(cudaMemcpyAsync(e.io_type.p, type, sizeof(int) * N, cudaMemcpyHostToDevice, s), "H2D");
    ck(cudaMemsetAsync(e.io_pe.p, 0, sizeof(double) * N, s), "memset");
    ck(cudaMemsetAsync(e.io_f.p, 0, sizeof(double) * 3 * N, s), "memset");
    ck(cudaMemsetAsync(e.io_vir.p, 0, sizeof(double) * 9 * N, s), "memset");
    if (!e.io_side) {
      ck(cudaStreamCreateWithFlags(&e.io_side, cudaStreamNonBlocking), "cudaStreamCreate");
      ck(cudaEventCreateWithFlags(&e.io_pe_ready, cudaEventDisableTiming), "cudaEventCreate");
      ck(cudaEventCreateWithFlags(&e.io_pe_copied, cudaEventDisableTiming), "cudaEventCreate");
    }
    // the site energies leave on the side stream while the force pass runs
    e.compute(s, N, box_h, pbc, e.io_type.p, e.io_pos.p, e.io_pe.p, e.io_f.p, e.io_vir.p, [&](cudaStream_t cs) {
      ck(cudaEventRecord(e.io_pe_ready, cs), "cudaEventRecord");
      ck(cudaStreamWaitEvent(e.io_side, e.io_pe_ready, 0), "cudaStreamWaitEvent");
      ck(cudaMemcpyAsync(potential, e.io_pe.p, sizeof(double) * N, cudaMemcpyDeviceToHost, e.io_side), "D2H");
      ck(cudaEventRecord(e.io_pe_copied, e.io_side), "cudaEventRecord");
    });
    sus2sh::launch_reduce(s, N, e.io_pe.p, e.io_vir.p, e.io_red.p);
    e.launches += 1;
    ck(cudaMemcpyAsync(force, e.io_f.p, sizeof(double) * 3 * N, cudaMemcpyDeviceToHost, s), "D2H");
    ck(cudaStreamWaitEvent(s, e.io_pe_copied, 0), "cudaStreamWaitEvent");
    if (virial_total) {
      double red[10];
      ck(cudaMemcpyAsync(red, e.io_red.p, sizeof(red), cudaMemcpyDeviceToHost, s), "D2H");
      ck(cudaStreamSynchronize(s), "cudaStreamSynchronize");
      std::memcpy(virial_total, red + 1, 9 * sizeof(double));
    } else {
      ck(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    }
  });
}

void sus2sh_destroy(sus2sh_handle* h) {
  if (!h) return;
  if (h->e.last_stream) cudaStreamSynchronize(h->e.last_stream);
  delete h;
}

double sus2sh_cutoff(const sus2sh_handle* h) { return h ? h->e.model.rc : 0.0; }

const char* sus2sh_last_error(void) { return sus2sh::g_last_error.c_str(); }

int sus2sh_sync(sus2sh_handle* h, int* status_flags) {
  if (!h) return SUS2SH_E_ARG;
  int rc = SUS2SH_OK;
  const int g = guarded([&] { rc = h->e.sync(status_flags); });
  return g != SUS2SH_OK ? g : rc;
}

int sus2sh_model_info(const sus2sh_handle* h, int* out, int n) {
  if (!h || !out) return 0;
  const sus2sh::Engine& e = h->e;
  const int v[41] = {e.model.species_count, e.model.l_max, e.model.k_max, e.model.body_order,
                     e.model.rb_size, e.model.basic_count, e.model.moments,
                     static_cast<int>(e.model.products.size()), e.model.scalar_count,
                     static_cast<int>(e.lay.rows.size()), e.lay.max_layer, e.prog.terminal_rows,
                     e.prog.nvalue, e.prog.nrows, e.model.standard_graph_matched ? 1 : 0,
                     e.use_float ? 1 : 0, e.cap, e.h_status ? e.h_status->builds : 0,
                     static_cast<int>(e.launches & 0x7fffffff), e.rs.shared_xi, e.prod_global ? 1 : 0,
                     e.cg_bin.cubin.empty() ? 0 : 1, e.cg_bin.registers, static_cast<int>(e.cg_compile_ms),
                     e.basic_block, e.force_block, e.edge_jit,
                     e.ejit_bin ? e.ejit_bin->basic_registers : -1, e.ejit_bin ? e.ejit_bin->force_registers : -1,
                     e.ejit_bin ? static_cast<int>(e.ejit_bin->compile_ms) : 0,
                     e.gate ? static_cast<int>(e.model.gate.mode) : 0,
                     e.cg_bin.cubin.empty() ? 0 : (e.cg_src.split ? 2 : 1),
                     e.cg_mod.registers(), e.cg_mod.local_bytes(),
                     e.cg_bin.cubin.empty() ? 0 : (e.cg_bin.whole ? 1 : 2), e.cg_bin.from_disk ? 1 : 0,
                     e.fused_bin ? 1 : 0,
                     e.fused_bin ? e.fused_bin->registers[e.fused_variant] : -1,
                     e.fused_bin ? e.fused_bin->blocks[e.fused_variant] * 100 + e.fused_bin->min_blocks[e.fused_variant] : 0,
                     e.fused_bin ? e.fused_tile : 0, static_cast<int>(e.fused_compile_ms)};
  const int k = std::min(n, 41);
  for (int i = 0; i < k; ++i) out[i] = v[i];
  return k;
}

int sus2sh_profile(sus2sh_handle* h, int enable) {
  if (!h) return SUS2SH_E_ARG;
  return guarded([&] {
    h->e.profile_collect();
    h->e.profile = enable != 0;
    for (double& v : h->e.prof_ms) v = 0.0;
    h->e.prof_calls = 0;
  });
}

int sus2sh_profile_read(sus2sh_handle* h, double* out, int n) {
  if (!h || !out) return SUS2SH_E_ARG;
  int rc = guarded([&] { h->e.profile_collect(); });
  if (rc != SUS2SH_OK) return rc;
  const double v[6] = {h->e.prof_ms[0], h->e.prof_ms[1], h->e.prof_ms[2], h->e.prof_ms[3], h->e.prof_ms[4],
                       static_cast<double>(h->e.prof_calls)};
  for (int i = 0; i < n && i < 6; ++i) out[i] = v[i];
  return SUS2SH_OK;
}

int sus2sh_cg_kernel_info(const char* path, int use_float, int split, int* info, char* text, size_t text_size) {
  if (!path || !info) return SUS2SH_E_ARG;
  return guarded([&] {
    const sus2sh::HostModel m = sus2sh::load_model(path);
    const sus2sh::Layered lay = sus2sh::layer_products(m);
    const sus2sh::ProgramHost prog = sus2sh::compile_program(m, lay);
    const auto t0 = std::chrono::steady_clock::now();
    sus2sh::CgSource src;
    std::string why;
    if (split == 2) {
      src = sus2sh::generate_pg_source(m, lay, use_float != 0, prog.basic_canon, prog.ncanon);
    } else if (!sus2sh::choose_cg_source(m, lay, prog.basic_canon, prog.ncanon, use_float != 0,
                                         split == 3 ? 1 : split, &src, &why)) {
      throw InputError("no CG kernel for this graph (" + why + "); the row interpreter runs it");
    }
    const sus2sh::CgBinary bin =
        sus2sh::compile_cg_source(src, split == 3 ? sus2sh::CgBuild::kParallel : sus2sh::CgBuild::kWhole);
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    int spill = 0;
    const size_t p = bin.log.find("bytes spill stores");
    if (p != std::string::npos) {
      size_t q = p;
      while (q > 0 && bin.log[q - 1] == ' ') --q;
      while (q > 0 && std::isdigit(static_cast<unsigned char>(bin.log[q - 1]))) --q;
      spill = std::atoi(bin.log.c_str() + q);
    }
    info[0] = bin.registers;
    info[1] = spill;
    info[2] = static_cast<int>(src.fp_terms);
    info[3] = static_cast<int>(ms);
    info[4] = static_cast<int>(bin.cubin.size());
    info[5] = src.split ? 1 : 0;
    info[6] = src.functions;
    info[7] = src.components;
    info[8] = src.block;
    info[9] = static_cast<int>(src.smem_bytes);
    if (text && text_size) {
      const std::string& t = use_float < 0 ? src.code : bin.log;
      const size_t k = std::min(text_size - 1, t.size());
      std::memcpy(text, t.data(), k);
      text[k] = 0;
    }
  });
}

int sus2sh_real_sh(int l_max, double x, double y, double z, double* Y, const double* G, double* V) {
  if (!Y) return SUS2SH_E_ARG;
  switch (l_max) {
    case 0: real_sh_host<0>(x, y, z, Y, G, V); break;
    case 1: real_sh_host<1>(x, y, z, Y, G, V); break;
    case 2: real_sh_host<2>(x, y, z, Y, G, V); break;
    case 3: real_sh_host<3>(x, y, z, Y, G, V); break;
    case 4: real_sh_host<4>(x, y, z, Y, G, V); break;
    case 5: real_sh_host<5>(x, y, z, Y, G, V); break;
    case 6: real_sh_host<6>(x, y, z, Y, G, V); break;
    default: return SUS2SH_E_ARG;
  }
  return SUS2SH_OK;
}

int sus2sh_edge_kernel_info(int fp32, int l_max, int k_max, int rb, int* basic_registers, int* force_registers,
                            double* compile_ms, char* log, size_t log_len) {
  return guarded([&] {
    if (l_max < 0 || l_max > 6 || k_max <= 0 || k_max * (l_max + 1) > 48 || rb <= 0 || rb > 16)
      throw sus2sh::InputError("SUS2_SH edge-kernel shape out of range.");
    const auto bin = sus2sh::compile_edge_kernels(fp32 != 0, l_max, k_max, rb, 128, false);
    if (basic_registers) *basic_registers = bin->basic_registers;
    if (force_registers) *force_registers = bin->force_registers;
    if (compile_ms) *compile_ms = bin->compile_ms;
    if (log && log_len) {
      std::strncpy(log, bin->log.c_str(), log_len - 1);
      log[log_len - 1] = '\0';
    }
  });
}

}  // extern "C"

namespace {
// The model-specialised edge build's inputs for a model file, as the engine
// derives them at load: the coefficient table (c[mu][n], then the derivative
// series when it fits) and whether every radial function of every pair has
// the (scal, shift) of the pair's first function.
void model_edge_inputs(const sus2sh::HostModel& m, std::vector<float>* table, bool* shared) {
  const std::vector<double> dc = sus2sh::radial_derivative(m.radial_map, m.radial_coeffs, m.radial_funcs, m.rb_size);
  table->assign(sus2sh::kMaxCoef, 0.0f);
  table->resize(sus2sh::Engine::fill_coef(m.radial_coeffs, dc, table->data()));
  const int S = m.species_count, kmu = m.radial_funcs;
  *shared = true;
  for (int p = 0; p < S * S; ++p)
    for (int mu = 0; mu < kmu; ++mu)
      *shared = *shared && m.scal_coeffs[2 * mu * S * S + p] == m.scal_coeffs[p] &&
                m.scal_coeffs[2 * mu * S * S + S * S + p] == m.scal_coeffs[S * S + p];
}
}  // namespace

extern "C" {

int sus2sh_model_edge_kernel_info(const char* path, int* info, char* log, size_t log_len) {
  if (!path || !info) return SUS2SH_E_ARG;
  return guarded([&] {
    const sus2sh::HostModel m = sus2sh::load_model(path);
    std::vector<float> table;
    bool shared = true;
    model_edge_inputs(m, &table, &shared);
    const auto bin = sus2sh::compile_model_edge_kernels(m.l_max, m.k_max, m.rb_size, table, shared,
                                                        static_cast<int>(m.radial_map));
    info[0] = bin->basic_registers;
    info[1] = bin->force_registers;
    info[2] = static_cast<int>(bin->compile_ms);
    info[3] = static_cast<int>(bin->global_bytes);
    info[4] = static_cast<int>(table.size());
    size_t bytes = 0;
    for (const auto& c : bin->cubins) bytes += c.size();
    info[5] = static_cast<int>(bytes);
    if (log && log_len) {
      std::strncpy(log, bin->log.c_str(), log_len - 1);
      log[log_len - 1] = '\0';
    }
  });
}

int sus2sh_batch_kernel_info(const char* path, int* info, char* log, size_t log_len) {
  if (!path || !info) return SUS2SH_E_ARG;
  return guarded([&] {
    const sus2sh::HostModel m = sus2sh::load_model(path);
    const sus2sh::Layered lay = sus2sh::layer_products(m);
    const sus2sh::ProgramHost prog = sus2sh::compile_program(m, lay);
    sus2sh::CgSource src;
    std::string why;
    if (!sus2sh::choose_cg_source(m, lay, prog.basic_canon, prog.ncanon, true, -1, &src, &why) || src.split ||
        src.device_fn.empty())
      throw sus2sh::InputError("no fused batch kernel for this model: its CG graph takes the component-split kernel");
    std::vector<float> table;
    bool shared = true;
    model_edge_inputs(m, &table, &shared);
    const auto bin = sus2sh::compile_batch_fused(m.l_max, m.k_max, m.rb_size, table, shared,
                                                 static_cast<int>(m.radial_map), src.device_fn, {{128, 3}, {128, 2}});
    info[0] = bin->registers[0];
    info[1] = bin->registers[1];
    info[2] = static_cast<int>(bin->compile_ms);
    info[3] = static_cast<int>(bin->cubin.size());
    if (log && log_len) {
      std::strncpy(log, bin->log.c_str(), log_len - 1);
      log[log_len - 1] = '\0';
    }
  });
}

int sus2sh_zbl_pair(int zi, int zj, double r, double inner, double outer, double* energy, double* dEdr) {
  if (!energy || !dEdr) return SUS2SH_E_ARG;
  const sus2sh::zbl::PairValue v = sus2sh::zbl::pair(zi, zj, r, inner, outer);
  *energy = v.energy;
  *dEdr = v.dEdr;
  return SUS2SH_OK;
}

}  // extern "C"
