// SUS2-SH model description on the host: the .mtp reader, the real
// Clebsch-Gordan standard graph builder and the run.in option parser.
//
// Reference interfaces restated here (hu-yanxiao/GPUMD-SUS2-SH):
//   load_sh_model                     src/force/sus2_sh.cu:2105-2482
//   SHStandardGraphBuilderHost        src/force/sus2_sh.cu:1227-1706
//   standard_sh_graph_matches         src/force/sus2_sh.cu:1872-1911
//   build_explicit_sh_graph_metadata  src/force/sus2_sh.cu:1913-2093
//   parse_sh_float                    src/force/sus2_sh.cu:520-536
// Input errors throw sus2sh::InputError; the C-ABI turns them into return
// codes (the reference prints and calls exit(1), sus2_sh.cu:269-273).
#pragma once

#include <stdexcept>
#include <string>
#include <vector>

namespace sus2sh {

struct InputError : std::runtime_error {
  explicit InputError(const std::string& m) : std::runtime_error(m) {}
};

struct Product {
  int left = 0, right = 0, target = 0;
  double coeff = 0.0;
};

// The radial basis of the file (kRadial* kinds of sh_math.cuh): Chebyshev of
// the tanh map, of the rational map, or Laguerre of log(1 + r / rho).
enum class RadialMap { Tanh = 0, Rational = 1, LaguerreLog1p = 2 };

enum class GateMode { MuBodyLinearCombo = 1, MuScalarFull = 2 };

struct GateModel {
  bool enabled = false;
  GateMode mode = GateMode::MuScalarFull;
  double amplitude = 0.8;              // A in G = 1 + A tanh(a h)
  int body_count = 0;                  // two_layer_gate_body_order_max - 1 (= K)
  std::vector<double> radial_coeffs;   // [Kmu][rb] gate radial coefficients
  std::vector<double> additive;        // [S] a per species of the gated atom
  std::vector<int> scalar_indices;     // [Q] scalar ids
  std::vector<double> weights;         // full: [Kmu][Q]; combo: [Q]
  std::vector<double> body_mix;        // combo: [Kmu][body_count]
  // derived
  std::vector<int> moment_of;          // [Q] moment id of each gate scalar
  std::vector<int> body_of;            // [Q] body id (body order - 2)
  std::vector<unsigned char> needed;   // [moments] needed by the gate signals
  int product_limit = 0;               // products [0, limit) can feed a needed moment
};

struct HostModel {
  int species_count = 0;
  int l_max = 0;
  int k_max = 0;
  int body_order = 0;
  int rb_size = 0;
  int radial_funcs = 0;     // K (L+1)
  int moments = 0;          // alpha_moments_count
  int basic_count = 0;      // alpha_index_basic_count
  int scalar_count = 0;     // alpha_scalar_moments
  double scaling = 1.0;
  double rc = 0.0;          // max_dist
  RadialMap radial_map = RadialMap::Tanh;
  std::string radial_basis_type;
  std::vector<int> body_l_max;          // indexed by body order, size 7
  std::vector<double> shift_coeffs;     // [S] site energy shift
  std::vector<double> scal_coeffs;      // [Kmu][2][S][S]: scal block then shift block
  std::vector<double> species_coeffs;   // [S]
  std::vector<double> moment_coeffs;    // [scalars]
  std::vector<int> moment_mapping;      // [scalars] -> moment id
  std::vector<int> basic_mu, basic_l, basic_m;  // [basics]
  std::vector<Product> products;
  std::vector<double> radial_coeffs;    // [Kmu][rb]
  std::vector<double> radial_type_coeffs;  // [S]
  bool standard_graph_matched = false;
  // ZBL short-range term (load_sh_model, sus2_sh.cu:2132-2147)
  bool zbl_enabled = false;
  double zbl_inner = 0.7;
  double zbl_outer = 1.4;
  bool zbl_typewise = false;
  double zbl_typewise_factor = 0.7;
  std::vector<int> zbl_atomic_numbers;  // empty: from the element symbols
  // body order of each scalar (sh_scalar_info, sus2_sh.cu:2354-2378), empty if absent
  std::vector<int> scalar_body;
  // Two-layer mu-body gate (load_sh_model, sus2_sh.cu:2153-2268; metadata
  // :2412-2478).  Neighbour site mode, shared radial (scal, shift) tables.
  GateModel gate;
};

// Parses a SUS2-SH v1.1.0 .mtp file with the reference reader's semantics.
HostModel load_model(const std::string& path);
// True when the file contains "potential_tag = SUS2-SH" (sus2_sh.cu:7771-7780).
bool is_sus2_sh_file(const std::string& path);

// ---- standard graph -------------------------------------------------------
struct StandardGraph {
  int node_count = 0;
  int max_layer = 0;
  std::vector<int> basic_k, basic_l, basic_m;
  std::vector<Product> products;
  std::vector<int> scalars;
  std::vector<int> scalar_body;  // body order of each scalar
  int tensor_blocks = 0;
  int cg_blocks = 0;
  int cg_terms = 0;
};

// Body-order indexed l limits (size 7), default l_max everywhere.
std::vector<int> default_body_l_max(int l_max);
StandardGraph build_standard_graph(int l_max, int k_max, int body_order,
                                   const std::vector<int>& body_l_max);
double real_cg(int l1, int m1, int l2, int m2, int L, int M);

// ---- explicit layered rows (build_explicit_sh_graph_metadata) -------------
struct Row {
  int layer = 0;
  int target = 0;
  std::vector<int> left, right;
  std::vector<double> coeff;
};
struct Layered {
  int max_layer = 0;
  std::vector<Row> rows;            // sorted by (layer, target)
  std::vector<int> node_layer;      // per moment
  std::vector<char> terminal;       // scalar target consumed by no product
  std::vector<int> scalar_of;       // moment -> scalar index (last wins), -1
};
Layered layer_products(const HostModel& m);

// ---- run.in options ---------------------------------------------------------
struct Options {
  bool use_float = true;        // sus2_float / sus2_sh_float / SUS2_GPUMD_FLOAT
  double skin = 1.0;            // sus2_sh_skin= (Angstrom)
  int rebuild_interval = 0;     // sus2_sh_rebuild_interval= (0: displacement only)
  bool reference_rounding = false;  // sus2_sh_reference_rounding=
  bool profile = false;             // sus2_sh_profile / sus2_profile / SUS2_SH_GPUMD_PROFILE
  bool cg_jit = true;               // sus2_sh_cg_jit=0 runs the CG row interpreter instead
  int cg_split = -1;                // sus2_sh_cg_split=0|1: never / always the component-split
                                    // CG kernel (-1: graphs above the single-function limit)
  bool cg_whole = true;             // sus2_sh_cg_whole=0 compiles a component-split CG kernel as
                                    // parallel relocatable units (fast load, slower kernel)
                                    // instead of one program (disk-cached)
  bool autotune = true;             // sus2_sh_autotune=0 keeps 128-thread edge-kernel CTAs
  bool edge_jit = false;            // sus2_sh_edge_jit=1 compiles the edge kernels at load even
                                    // for a shape built ahead of time
  bool model_edges = true;          // sus2_sh_model_edges=0 keeps the FP32 edge kernels that read
                                    // the radial coefficients from their parameters
  bool neighbor_graph = true;       // sus2_sh_neighbor_graph=0 launches the neighbour-build kernels
                                    // on every call instead of a graph that skips them
  bool batch_fused = false;         // sus2_sh_batch_fused=1 evaluates batches of cells with the
                                    // fused persistent kernel instead of the stage kernels
                                    // (measured slower on the 4096-cell batch: 3.53 vs 2.13 ms)
  int batch_tile = 0;               // sus2_sh_batch_tile=<atoms>: tile size of the fused batch
                                    // kernel (0: picked by timing at the first batch call)
};
// Options start after the species symbols (sus2_sh.cu:527); unknown tokens of
// the reference's tuning switches are accepted and ignored.
Options parse_options(const HostModel& m, int nopts, const char** opts);


}  // namespace sus2sh
