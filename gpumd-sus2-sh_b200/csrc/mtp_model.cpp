// .mtp reader, standard real-CG graph builder, layered-row compiler, option
// parser and seeded synthetic-model writer.  See mtp_model.h for the
// reference functions each part restates.
#include "mtp_model.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <functional>
#include <map>
#include <sstream>
#include <tuple>
#include <unordered_map>

namespace sus2sh {
namespace {

// ---------------------------------------------------------------------------
// text helpers (semantics of sus2_sh.cu:275-477)
// ---------------------------------------------------------------------------
std::string slurp(const std::string& path) {
  std::ifstream in(path);
  if (!in) throw InputError("Failed to open SUS2-SH model file: " + path);
  std::ostringstream ss;
  ss << in.rdbuf();
  return ss.str();
}

std::string strip(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace(static_cast<unsigned char>(s[a]))) ++a;
  while (b > a && std::isspace(static_cast<unsigned char>(s[b - 1]))) --b;
  return s.substr(a, b - a);
}

size_t locate(const std::string& text, const std::string& tok, size_t from = 0) {
  size_t p = text.find(tok, from);
  if (p == std::string::npos) throw InputError("Missing token in SUS2-SH model file: " + tok);
  return p;
}

bool contains(const std::string& text, const std::string& tok) {
  return text.find(tok) != std::string::npos;
}

// Rest of the line after the first occurrence of `tok`, trimmed.
std::string value_of(const std::string& text, const std::string& tok) {
  size_t p = locate(text, tok) + tok.size();
  size_t e = text.find('\n', p);
  return strip(text.substr(p, e == std::string::npos ? std::string::npos : e - p));
}

int int_of(const std::string& text, const std::string& tok) {
  const std::string v = value_of(text, tok);
  try {
    return std::stoi(v);
  } catch (...) {
    throw InputError("Invalid integer in SUS2-SH model file for " + tok + ": " + v);
  }
}

double double_of(const std::string& text, const std::string& tok) {
  const std::string v = value_of(text, tok);
  try {
    return std::stod(v);
  } catch (...) {
    throw InputError("Invalid number in SUS2-SH model file for " + tok + ": " + v);
  }
}

// First balanced {...} after `tok`, braces included.
std::string braced(const std::string& text, const std::string& tok) {
  size_t p = locate(text, tok);
  p = locate(text, "{", p);
  int depth = 0;
  size_t start = p;
  for (size_t i = p; i < text.size(); ++i) {
    if (text[i] == '{') {
      if (depth == 0) start = i;
      ++depth;
    } else if (text[i] == '}') {
      if (--depth == 0) return text.substr(start, i - start + 1);
    }
  }
  throw InputError("Unterminated braced section in SUS2-SH model file: " + tok);
}

// Groups one level inside the outer braces: "{{a},{b}}" -> {a},{b}.
std::vector<std::string> inner_groups(const std::string& text) {
  std::vector<std::string> out;
  int depth = 0;
  size_t start = 0;
  for (size_t i = 0; i < text.size(); ++i) {
    if (text[i] == '{') {
      if (depth == 1) start = i;
      ++depth;
    } else if (text[i] == '}') {
      if (depth == 2) out.push_back(text.substr(start, i - start + 1));
      --depth;
    }
  }
  return out;
}

// Every top-level {...} group in `text`.
std::vector<std::string> outer_groups(const std::string& text) {
  std::vector<std::string> out;
  int depth = 0;
  size_t start = 0;
  for (size_t i = 0; i < text.size(); ++i) {
    if (text[i] == '{') {
      if (depth == 0) start = i;
      ++depth;
    } else if (text[i] == '}') {
      if (--depth == 0) out.push_back(text.substr(start, i - start + 1));
    }
  }
  return out;
}

template <typename T>
std::vector<T> numbers(const std::string& text) {
  std::string s = text;
  for (char& c : s)
    if (c == '{' || c == '}' || c == ',') c = ' ';
  std::istringstream in(s);
  std::vector<T> v;
  T x;
  while (in >> x) v.push_back(x);
  return v;
}

bool parse_bool(const std::string& v, const std::string& name) {
  if (v == "1" || v == "true" || v == "TRUE" || v == "yes" || v == "on") return true;
  if (v == "0" || v == "false" || v == "FALSE" || v == "no" || v == "off") return false;
  throw InputError("Invalid boolean value for " + name + ": " + v);
}

}  // namespace

bool is_sus2_sh_file(const std::string& path) {
  std::ifstream in(path);
  if (!in) return false;
  std::ostringstream ss;
  ss << in.rdbuf();
  return contains(ss.str(), "potential_tag = SUS2-SH");
}

// ---------------------------------------------------------------------------
// Reader (load_sh_model, sus2_sh.cu:2105-2482).  The two-layer gate and ZBL
// fields are outside this engine and are rejected explicitly.
// ---------------------------------------------------------------------------
namespace {
// Gate keys (sus2_sh.cu:2153-2268), validated in the reference's order with its
// messages.  Only the neighbour-site, shared-radial mu-body modes exist.
void parse_gate(const std::string& text, HostModel& m) {
  GateModel& g = m.gate;
  g.enabled = true;
  std::string mode = contains(text, "two_layer_gate_mode =") ? value_of(text, "two_layer_gate_mode =") : "legacy";
  if (mode == "mu-body-linear-combo") {
    g.mode = GateMode::MuBodyLinearCombo;
  } else if (mode == "mu-scalar-full" || mode == "mu-body-order") {
    g.mode = GateMode::MuScalarFull;
  } else if (mode == "legacy") {
    throw InputError(
        "GPUMD SUS2_SH mu-body-order branch requires two_layer_gate_mode = "
        "mu-body-linear-combo or mu-scalar-full; legacy gate models are not supported here.");
  } else {
    throw InputError("Unsupported SUS2_SH two_layer_gate_mode in GPUMD: " + mode);
  }
  if (contains(text, "two_layer_gate_include_one_body =") &&
      parse_bool(value_of(text, "two_layer_gate_include_one_body ="), "two_layer_gate_include_one_body ="))
    throw InputError("GPUMD SUS2_SH gate backend requires two_layer_gate_include_one_body = false.");
  if (contains(text, "two_layer_gate_scale_mode ="))
    throw InputError("GPUMD SUS2_SH mu-body gate does not support two_layer_gate_scale_mode.");
  if (contains(text, "two_layer_gate_bias ="))
    throw InputError("GPUMD SUS2_SH mu-body gate does not support two_layer_gate_bias.");
  if (contains(text, "two_layer_residual_enabled =") &&
      parse_bool(value_of(text, "two_layer_residual_enabled ="), "two_layer_residual_enabled ="))
    throw InputError("GPUMD SUS2_SH mu-body gate does not support residual gate fields.");
  if (contains(text, "two_layer_gate_site_mode =")) {
    const std::string site = value_of(text, "two_layer_gate_site_mode =");
    if (site == "double")
      throw InputError(
          "GPUMD SUS2_SH mu-body gate currently supports two_layer_gate_site_mode = neighbor. "
          "Double-site gate will be added after the single-gate CUDA path is verified.");
    if (site != "neighbor") throw InputError("Unsupported SUS2_SH two_layer_gate_site_mode in GPUMD: " + site);
  }
  if (contains(text, "two_layer_gate_tanh_amplitude ="))
    g.amplitude = double_of(text, "two_layer_gate_tanh_amplitude =");
  if (!std::isfinite(g.amplitude) || g.amplitude < 0.0 || g.amplitude > 1.0)
    throw InputError("SUS2_SH two_layer_gate_tanh_amplitude should be finite and in [0,1].");
  const std::string radial_mode =
      contains(text, "two_layer_gate_radial_mode =") ? value_of(text, "two_layer_gate_radial_mode =") : "";
  if (radial_mode != "shared-radial")
    throw InputError("GPUMD SUS2_SH gate backend currently requires shared-radial gate mode.");
  const int body_max = int_of(text, "two_layer_gate_body_order_max =");
  if (body_max != m.k_max + 1) throw InputError("SUS2_SH two_layer_gate_body_order_max should equal sh_k_max + 1.");
  g.body_count = body_max - 1;
  const int radial_count = int_of(text, "two_layer_gate_radial_coeff_count =");
  if (radial_count != m.radial_funcs * m.rb_size)
    throw InputError("SUS2_SH two-layer gate radial coefficient count is inconsistent.");
  g.radial_coeffs = numbers<double>(braced(text, "two_layer_gate_radial_coeffs ="));
  if (static_cast<int>(g.radial_coeffs.size()) != radial_count)
    throw InputError("SUS2_SH two-layer gate radial coeff list has wrong size.");
  if (contains(text, "two_layer_gate_additive_coeff_count =")) {
    const int n = int_of(text, "two_layer_gate_additive_coeff_count =");
    if (n != m.species_count) throw InputError("SUS2_SH two-layer gate additive coefficient count is inconsistent.");
    g.additive = numbers<double>(braced(text, "two_layer_gate_additive_coeffs ="));
    if (static_cast<int>(g.additive.size()) != n)
      throw InputError("SUS2_SH two-layer gate additive coeff list has wrong size.");
  } else {
    g.additive.assign(m.species_count, 1.0);
  }
  const int weight_count = int_of(text, "two_layer_gate_weight_count =");
  if (weight_count <= 0) throw InputError("SUS2_SH two-layer gate should contain at least one scalar weight.");
  g.scalar_indices = numbers<int>(braced(text, "two_layer_gate_scalar_indices ="));
  g.weights = numbers<double>(braced(text, "two_layer_gate_weights ="));
  const int nq = static_cast<int>(g.scalar_indices.size());
  if (nq <= 0) throw InputError("SUS2_SH two-layer gate scalar index list is empty.");
  const int expected = g.mode == GateMode::MuScalarFull ? m.radial_funcs * nq : nq;
  if (weight_count != expected || static_cast<int>(g.weights.size()) != expected)
    throw InputError("SUS2_SH two-layer gate scalar index/weight dimensions are inconsistent.");
  if (g.mode == GateMode::MuBodyLinearCombo) {
    const int n = int_of(text, "two_layer_gate_body_mix_weight_count =");
    if (n != m.radial_funcs * g.body_count)
      throw InputError("SUS2_SH two-layer gate body-mix weight count is inconsistent.");
    g.body_mix = numbers<double>(braced(text, "two_layer_gate_body_mix_weights ="));
    if (static_cast<int>(g.body_mix.size()) != n)
      throw InputError("SUS2_SH two-layer gate body-mix weight list has wrong size.");
  } else if (contains(text, "two_layer_gate_body_mix_weights =") ||
             contains(text, "two_layer_gate_body_mix_weight_count =")) {
    throw InputError("SUS2_SH mu-scalar-full gate should not contain body-mix weights.");
  }
}

// Gate scalar -> moment and body bucket, the moments the gate signals need and
// the last product that can feed one (sus2_sh.cu:2412-2478).
void gate_metadata(HostModel& m) {
  GateModel& g = m.gate;
  const int nq = static_cast<int>(g.scalar_indices.size());
  g.moment_of.assign(nq, 0);
  g.body_of.assign(nq, 0);
  g.needed.assign(m.moments, 0);
  std::vector<unsigned char> present(g.body_count, 0);
  for (int q = 0; q < nq; ++q) {
    const int s = g.scalar_indices[q];
    if (s < 0 || s >= m.scalar_count) throw InputError("SUS2_SH two-layer gate scalar index is out of range.");
    const int body = m.scalar_body[s] - 2;
    if (body < 0 || body >= g.body_count)
      throw InputError("SUS2_SH two-layer gate scalar body order is outside the gate range.");
    g.body_of[q] = body;
    present[body] = 1;
    const int mom = m.moment_mapping[s];
    if (mom < 0 || mom >= m.moments) throw InputError("SUS2_SH two-layer gate mapped moment index is out of range.");
    g.moment_of[q] = mom;
    bool effective = false;
    if (g.mode == GateMode::MuScalarFull) {
      for (int mu = 0; mu < m.radial_funcs && !effective; ++mu) effective = g.weights[mu * nq + q] != 0.0;
    } else if (g.weights[q] != 0.0) {
      for (int mu = 0; mu < m.radial_funcs && !effective; ++mu)
        effective = g.body_mix[mu * g.body_count + body] != 0.0;
    }
    if (effective) g.needed[mom] = 1;
  }
  for (int b = 0; b < g.body_count; ++b)
    if (!present[b]) throw InputError("SUS2_SH two-layer gate scalar list misses a required body-order bucket.");
  g.product_limit = 0;
  for (int p = static_cast<int>(m.products.size()) - 1; p >= 0; --p) {
    const Product& pr = m.products[p];
    if (!g.needed[pr.target]) continue;
    g.needed[pr.left] = 1;
    g.needed[pr.right] = 1;
    if (g.product_limit == 0) g.product_limit = p + 1;
  }
}
}  // namespace

HostModel load_model(const std::string& path) {
  const std::string text = slurp(path);
  HostModel m;
  if (value_of(text, "version =") != "1.1.0")
    throw InputError("SUS2_SH currently supports only version = 1.1.0.");
  if (value_of(text, "potential_tag =") != "SUS2-SH")
    throw InputError("SUS2_SH selected for a non-SUS2-SH model.");
  m.scaling = double_of(text, "scaling =");
  const std::string scaling_map = value_of(text, "scaling_map =");
  m.species_count = int_of(text, "species_count =");
  m.l_max = int_of(text, "sh_l_max =");
  m.k_max = int_of(text, "sh_k_max =");
  m.body_order = int_of(text, "sh_body_order =");
  if (contains(text, "sh_parity =") && value_of(text, "sh_parity =") != "even")
    throw InputError("SUS2_SH GPUMD backend currently supports even parity models only.");
  m.radial_basis_type = value_of(text, "radial_basis_type =");
  if (m.radial_basis_type == "RBChebyshev_sss" || m.radial_basis_type == "RBChebyshev_sss_lmp") {
    m.radial_map = RadialMap::Tanh;
  } else if (m.radial_basis_type == "RBLaguerre_log1p" || m.radial_basis_type == "RBLaguerre_log1p_lmp") {
    m.radial_map = RadialMap::LaguerreLog1p;
  } else if (m.radial_basis_type == "RBChebyshev_sss_rational" ||
             m.radial_basis_type == "RBChebyshev_sss_rational_lmp") {
    m.radial_map = RadialMap::Rational;
  } else {
    throw InputError("Unsupported SUS2_SH radial_basis_type: " + m.radial_basis_type +
                     ". Supported: RBChebyshev_sss[_lmp], RBLaguerre_log1p[_lmp], "
                     "RBChebyshev_sss_rational[_lmp].");
  }
  m.rc = double_of(text, "max_dist =");
  m.zbl_enabled = contains(text, "zbl_enabled =") && parse_bool(value_of(text, "zbl_enabled ="), "zbl_enabled =");
  if (m.zbl_enabled) {
    if (contains(text, "zbl_inner =")) m.zbl_inner = double_of(text, "zbl_inner =");
    if (contains(text, "zbl_outer =")) m.zbl_outer = double_of(text, "zbl_outer =");
    m.zbl_typewise = contains(text, "zbl_typewise_cutoff_enabled =")
                         ? parse_bool(value_of(text, "zbl_typewise_cutoff_enabled ="), "zbl_typewise_cutoff_enabled =")
                         : contains(text, "zbl_typewise_cutoff_factor =");
    if (contains(text, "zbl_typewise_cutoff_factor ="))
      m.zbl_typewise_factor = double_of(text, "zbl_typewise_cutoff_factor =");
    if (contains(text, "zbl_atomic_numbers ="))
      m.zbl_atomic_numbers = numbers<int>(braced(text, "zbl_atomic_numbers ="));
  }
  m.rb_size = int_of(text, "radial_basis_size =");
  m.radial_funcs = int_of(text, "radial_funcs_count =");
  m.moments = int_of(text, "alpha_moments_count =");
  m.basic_count = int_of(text, "alpha_index_basic_count =");
  m.scalar_count = int_of(text, "alpha_scalar_moments =");
  if (contains(text, "two_layer_gate_enabled =") &&
      parse_bool(value_of(text, "two_layer_gate_enabled ="), "two_layer_gate_enabled ="))
    parse_gate(text, m);

  if (scaling_map != "LK") throw InputError("SUS2_SH requires scaling_map = LK.");
  if (m.l_max < 0 || m.l_max > 6)
    throw InputError("SUS2_SH supports sh_l_max in [0,6].");
  if (m.body_order < 2 || m.body_order > 6)
    throw InputError("SUS2_SH supports sh_body_order in [2,6].");
  if (m.k_max <= 0 || m.radial_funcs != m.k_max * (m.l_max + 1))
    throw InputError("SUS2_SH inconsistent sh_k_max/radial_funcs_count.");
  if (m.rb_size <= 0 || m.rb_size > 16 || m.radial_funcs > 48)
    throw InputError("SUS2_SH GPU scratch limit exceeded: rb_size<=16, radial_funcs_count<=48.");
  if (m.basic_count <= 0 || m.basic_count > 320)
    throw InputError("SUS2_SH GPU scratch limit exceeded: alpha_index_basic_count<=320.");
  if (m.species_count <= 0 || m.species_count > 16)
    throw InputError("SUS2_SH engine supports species_count in [1,16].");
  if (!(m.rc > 0.0)) throw InputError("SUS2_SH max_dist must be positive.");

  m.body_l_max = default_body_l_max(m.l_max);
  if (contains(text, "sh_body_l_max =")) {
    const auto vals = numbers<int>(braced(text, "sh_body_l_max ="));
    const int expected = m.body_order >= 6 ? 5 : 4;
    if (static_cast<int>(vals.size()) != expected)
      throw InputError("Unexpected SUS2_SH sh_body_l_max size.");
    for (int b = 2; b <= 1 + expected; ++b) m.body_l_max[b] = vals[b - 2];
  }
  for (int b = 2; b <= m.body_order; ++b)
    if (m.body_l_max[b] < 0 || m.body_l_max[b] > m.l_max)
      throw InputError("SUS2_SH sh_body_l_max entry is out of range.");

  m.shift_coeffs = numbers<double>(braced(text, "shift_coeffs ="));
  m.scal_coeffs = numbers<double>(braced(text, "scal_coeffs ="));
  m.species_coeffs = numbers<double>(braced(text, "species_coeffs ="));
  m.moment_coeffs = numbers<double>(braced(text, "moment_coeffs ="));
  m.moment_mapping = numbers<int>(braced(text, "alpha_moment_mapping ="));

  const auto raw = numbers<int>(braced(text, "alpha_index_basic ="));
  if (static_cast<int>(raw.size()) != 3 * m.basic_count)
    throw InputError("Unexpected SUS2_SH alpha_index_basic size.");
  for (int i = 0; i < m.basic_count; ++i) {
    const int k = raw[3 * i], l = raw[3 * i + 1], mm = raw[3 * i + 2];
    if (k < 0 || k >= m.k_max || l < 0 || l > m.l_max || std::abs(mm) > l)
      throw InputError("Invalid SUS2_SH alpha_index_basic entry.");
    m.basic_mu.push_back(k * (m.l_max + 1) + l);
    m.basic_l.push_back(l);
    m.basic_m.push_back(mm);
  }

  const int nprod = int_of(text, "sh_product_count =");
  const auto groups = inner_groups(braced(text, "sh_products ="));
  if (static_cast<int>(groups.size()) != nprod)
    throw InputError("Unexpected SUS2_SH sh_products size.");
  m.products.resize(nprod);
  for (int p = 0; p < nprod; ++p) {
    const auto v = numbers<double>(groups[p]);
    if (v.size() != 4) throw InputError("Invalid SUS2_SH product entry.");
    Product& pr = m.products[p];
    pr.left = static_cast<int>(v[0]);
    pr.right = static_cast<int>(v[1]);
    pr.target = static_cast<int>(v[2]);
    pr.coeff = v[3];
    if (pr.left < 0 || pr.left >= m.moments || pr.right < 0 || pr.right >= m.moments ||
        pr.target < 0 || pr.target >= m.moments)
      throw InputError("SUS2_SH product index out of range.");
  }

  if (contains(text, "sh_scalar_info_count =")) {
    const int count = int_of(text, "sh_scalar_info_count =");
    if (count != m.scalar_count) throw InputError("SUS2_SH sh_scalar_info_count should equal alpha_scalar_moments.");
    const auto info = inner_groups(braced(text, "sh_scalar_info ="));
    if (static_cast<int>(info.size()) != count) throw InputError("Unexpected SUS2_SH sh_scalar_info size.");
    m.scalar_body.assign(count, 0);
    for (int q = 0; q < count; ++q) {
      const auto v = numbers<int>(info[q]);
      if (v.empty()) throw InputError("Invalid SUS2_SH sh_scalar_info entry.");
      if (v[0] < 2 || v[0] > m.body_order) throw InputError("SUS2_SH sh_scalar_info body order is out of range.");
      m.scalar_body[q] = v[0];
    }
  } else if (m.gate.enabled) {
    throw InputError("GPUMD SUS2_SH mu-body gate requires sh_scalar_info metadata.");
  }

  m.radial_coeffs.assign(static_cast<size_t>(m.radial_funcs) * m.rb_size, 0.0);
  m.radial_type_coeffs.assign(m.species_count, 1.0);
  const size_t r0 = locate(text, "radial_coeffs");
  const size_t r1 = locate(text, "alpha_moments_count", r0);
  const auto rgroups = outer_groups(text.substr(r0, r1 - r0));
  if (static_cast<int>(rgroups.size()) < m.radial_funcs)
    throw InputError("Unexpected SUS2_SH radial_coeffs section.");
  for (int mu = 0; mu < m.radial_funcs; ++mu) {
    const auto v = numbers<double>(rgroups[mu]);
    if (static_cast<int>(v.size()) != m.rb_size + m.species_count)
      throw InputError("Unexpected SUS2_SH radial_coeffs row size.");
    for (int n = 0; n < m.rb_size; ++n) m.radial_coeffs[mu * m.rb_size + n] = v[n];
    if (mu == 0)
      for (int t = 0; t < m.species_count; ++t) m.radial_type_coeffs[t] = v[m.rb_size + t];
  }

  const int S = m.species_count;
  if (static_cast<int>(m.shift_coeffs.size()) != S ||
      static_cast<int>(m.species_coeffs.size()) != S ||
      static_cast<int>(m.scal_coeffs.size()) != 2 * S * S * m.radial_funcs ||
      static_cast<int>(m.moment_mapping.size()) != m.scalar_count ||
      static_cast<int>(m.moment_coeffs.size()) != m.scalar_count)
    throw InputError("Unexpected SUS2_SH coefficient dimensions.");

  if (m.gate.enabled) gate_metadata(m);

  // Standard-graph match is informational (prepare_sh_graph_metadata,
  // sus2_sh.cu:2095-2103); execution always follows the saved products.
  {
    const StandardGraph g = build_standard_graph(m.l_max, m.k_max, m.body_order, m.body_l_max);
    bool ok = g.node_count == m.moments && static_cast<int>(g.basic_k.size()) == m.basic_count &&
              g.products.size() == m.products.size() && g.scalars.size() == m.moment_mapping.size();
    for (int i = 0; ok && i < m.basic_count; ++i)
      ok = m.basic_mu[i] == g.basic_k[i] * (m.l_max + 1) + g.basic_l[i] &&
           m.basic_l[i] == g.basic_l[i] && m.basic_m[i] == g.basic_m[i];
    for (size_t p = 0; ok && p < m.products.size(); ++p) {
      const Product& e = g.products[p];
      const Product& a = m.products[p];
      ok = a.left == e.left && a.right == e.right && a.target == e.target &&
           std::abs(a.coeff - e.coeff) <= 2.0e-10 * (1.0 + std::abs(e.coeff));
    }
    for (size_t s = 0; ok && s < g.scalars.size(); ++s) ok = g.scalars[s] == m.moment_mapping[s];
    m.standard_graph_matched = ok;
  }
  // Explicit-graph validation (sus2_sh.cu:1913-2006) happens in layer_products.
  (void)layer_products(m);
  return m;
}

// ---------------------------------------------------------------------------
// Real Clebsch-Gordan coefficients (sus2_sh.cu:1107-1218)
// ---------------------------------------------------------------------------
namespace {
double fact(int n) {
  if (n < 0) return 0.0;
  double v = 1.0;
  for (int i = 2; i <= n; ++i) v *= i;
  return v;
}

bool triangle(int a, int b, int c) { return std::abs(a - b) <= c && c <= a + b; }

double complex_cg(int j1, int m1, int j2, int m2, int j, int m) {
  if (m != m1 + m2 || !triangle(j1, j2, j) || std::abs(m1) > j1 || std::abs(m2) > j2 ||
      std::abs(m) > j)
    return 0.0;
  const double a = std::sqrt((2.0 * j + 1.0) * fact(j1 + j2 - j) * fact(j1 - j2 + j) *
                             fact(-j1 + j2 + j) / fact(j1 + j2 + j + 1));
  const double b = std::sqrt(fact(j1 + m1) * fact(j1 - m1) * fact(j2 + m2) * fact(j2 - m2) *
                             fact(j + m) * fact(j - m));
  double s = 0.0;
  for (int k = 0; k <= j1 + j2 + j + 1; ++k) {
    const int e1 = j1 + j2 - j - k, e2 = j1 - m1 - k, e3 = j2 + m2 - k;
    const int e4 = j - j2 + m1 + k, e5 = j - j1 - m2 + k;
    if (e1 < 0 || e2 < 0 || e3 < 0 || e4 < 0 || e5 < 0) continue;
    s += ((k & 1) ? -1.0 : 1.0) / (fact(k) * fact(e1) * fact(e2) * fact(e3) * fact(e4) * fact(e5));
  }
  return a * b * s;
}

// Row `real_m`, column `complex_m` of the unitary map taking complex to real
// harmonics (sus2_sh.cu:1149-1170).
std::complex<double> u_real_complex(int rm, int cm) {
  const double h = 1.0 / std::sqrt(2.0);
  if (rm == 0) return cm == 0 ? 1.0 : 0.0;
  const int a = std::abs(rm);
  if (std::abs(cm) != a) return 0.0;
  const double par = (a & 1) ? -1.0 : 1.0;
  if (rm > 0) return cm == a ? std::complex<double>(h * par, 0.0) : std::complex<double>(h, 0.0);
  return cm == a ? std::complex<double>(0.0, -h * par) : std::complex<double>(0.0, h);
}
}  // namespace

double real_cg(int l1, int m1, int l2, int m2, int L, int M) {
  std::complex<double> s = 0.0;
  for (int cM = -L; cM <= L; ++cM) {
    const std::complex<double> uo = std::conj(u_real_complex(M, cM));
    if (std::abs(uo) == 0.0) continue;
    for (int c1 = -l1; c1 <= l1; ++c1) {
      const std::complex<double> u1 = u_real_complex(m1, c1);
      if (std::abs(u1) == 0.0) continue;
      for (int c2 = -l2; c2 <= l2; ++c2) {
        const std::complex<double> u2 = u_real_complex(m2, c2);
        if (std::abs(u2) == 0.0) continue;
        const double cg = complex_cg(l1, c1, l2, c2, L, cM);
        if (std::abs(cg) < 1.0e-14) continue;
        s += uo * cg * u1 * u2;
      }
    }
  }
  static const std::complex<double> phase[4] = {{1, 0}, {0, 1}, {-1, 0}, {0, -1}};
  s *= phase[(l1 + l2 - L) & 3];
  if (std::abs(s.imag()) > 1.0e-10)
    throw InputError("SUS2_SH standard graph produced a non-real CG coefficient.");
  return s.real();
}

std::vector<int> default_body_l_max(int l_max) { return std::vector<int>(7, l_max); }

// ---------------------------------------------------------------------------
// Standard graph builder (SHStandardGraphBuilderHost, sus2_sh.cu:1227-1706).
// Node numbering, product order, key de-duplication and the 1e-12 pruning
// follow the reference exactly so that saved graphs compare element-wise.
// ---------------------------------------------------------------------------
namespace {
class GraphBuilder {
 public:
  GraphBuilder(int lmax, int kmax) : lmax_(lmax), kmax_(kmax) {}

  StandardGraph build(int body_order, const std::vector<int>& body_lmax) {
    body_lmax_ = body_lmax;
    for (int l = lmax_; l >= 0; --l)
      for (int k = kmax_ - 1; k >= 0; --k) q_.push_back({l, k});
    collect_specs(body_order);
    for (size_t qi = 0; qi < q_.size(); ++qi)
      if (required_[qi]) basic_tensor(static_cast<int>(qi));
    StandardGraph g;
    for (const Spec& s : specs_) {
      const int node = build_scalar(s);
      if (node >= 0) {
        g.scalars.push_back(node);
        g.scalar_body.push_back(s.body);
      }
    }
    for (const Product& p : products_)
      if (std::abs(p.coeff) >= 1.0e-12) g.products.push_back(p);
    g.node_count = nodes_;
    g.basic_k = bk_;
    g.basic_l = bl_;
    g.basic_m = bm_;
    g.tensor_blocks = tensor_blocks_;
    g.cg_blocks = cg_blocks_;
    g.cg_terms = cg_terms_;
    g.max_layer = max_layer_;
    return g;
  }

 private:
  struct Tensor {
    int l = 0, layer = 0;
    bool zero = false;
    std::vector<int> node;
  };
  struct Spec {
    int body;
    int q[5];
    int inter;
  };
  struct Q {
    int l, k;
  };

  int lookup_or(const std::string& key) const {
    auto it = lookup_.find(key);
    return it == lookup_.end() ? -1 : it->second;
  }
  int store(const std::string& key, Tensor t) {
    tensors_.push_back(std::move(t));
    keys_.push_back(key);
    const int id = static_cast<int>(tensors_.size()) - 1;
    lookup_[key] = id;
    return id;
  }

  int basic_tensor(int qi) {
    const std::string key = "q" + std::to_string(q_[qi].k * (lmax_ + 1) + q_[qi].l) + "_l" +
                            std::to_string(q_[qi].l) + "_k" + std::to_string(q_[qi].k);
    const int found = lookup_or(key);
    if (found >= 0) return found;
    Tensor t;
    t.l = q_[qi].l;
    for (int m = -t.l; m <= t.l; ++m) {
      t.node.push_back(nodes_++);
      bk_.push_back(q_[qi].k);
      bl_.push_back(t.l);
      bm_.push_back(m);
    }
    ++tensor_blocks_;
    return store(key, std::move(t));
  }

  void add_product(int a, int b, int target, double c) {
    if (std::abs(c) < 1.0e-12) return;
    if (b < a) std::swap(a, b);
    const auto key = std::make_tuple(a, b, target);
    auto it = product_lookup_.find(key);
    if (it != product_lookup_.end()) {
      products_[it->second].coeff += c;
      return;
    }
    product_lookup_[key] = static_cast<int>(products_.size());
    products_.push_back({a, b, target, c});
  }

  // Couples two tensors to total angular momentum L (sus2_sh.cu:1292-1449).
  int couple(int li, int ri, int L) {
    const std::string key = "(" + keys_[li] + "x" + keys_[ri] + ")->" + std::to_string(L);
    const int found = lookup_or(key);
    if (found >= 0) return found;
    const Tensor left = tensors_[li], right = tensors_[ri];
    Tensor out;
    out.l = L;
    out.layer = 1 + std::max(left.layer, right.layer);
    if (left.zero || right.zero) {
      out.zero = true;
      return store(key, std::move(out));
    }
    std::vector<std::tuple<int, int, int, double>> local;  // insertion ordered
    std::map<std::tuple<int, int, int>, int> local_ix;
    std::vector<double> logical;
    std::map<std::tuple<int, int, int>, int> logical_ix;
    for (int m1 = -left.l; m1 <= left.l; ++m1)
      for (int m2 = -right.l; m2 <= right.l; ++m2)
        for (int M = -L; M <= L; ++M) {
          const double c = cached_cg(left.l, m1, right.l, m2, L, M);
          if (std::abs(c) < 1.0e-12) continue;
          const int lc = m1 + left.l, rc = m2 + right.l, tc = M + L;
          auto lk = std::make_tuple(lc, rc, tc);
          auto lit = logical_ix.find(lk);
          if (lit == logical_ix.end()) {
            logical_ix[lk] = static_cast<int>(logical.size());
            logical.push_back(c);
          } else {
            logical[lit->second] += c;
          }
          int a = left.node[lc], b = right.node[rc];
          if (b < a) std::swap(a, b);
          auto pk = std::make_tuple(a, b, tc);
          auto pit = local_ix.find(pk);
          if (pit == local_ix.end()) {
            local_ix[pk] = static_cast<int>(local.size());
            local.emplace_back(a, b, tc, c);
          } else {
            std::get<3>(local[pit->second]) += c;
          }
        }
    int kept = 0;
    for (const auto& t : local)
      if (std::abs(std::get<3>(t)) >= 1.0e-12) ++kept;
    if (kept == 0) {
      out.zero = true;
      return store(key, std::move(out));
    }
    for (int M = -L; M <= L; ++M) out.node.push_back(nodes_++);
    ++tensor_blocks_;
    ++cg_blocks_;
    for (double c : logical)
      if (std::abs(c) >= 1.0e-12) ++cg_terms_;
    max_layer_ = std::max(max_layer_, out.layer);
    const std::vector<int> out_nodes = out.node;
    const int id = store(key, std::move(out));
    for (const auto& t : local)
      if (std::abs(std::get<3>(t)) >= 1.0e-12)
        add_product(std::get<0>(t), std::get<1>(t), out_nodes[std::get<2>(t)], std::get<3>(t));
    return id;
  }

  double cached_cg(int l1, int m1, int l2, int m2, int L, int M) {
    const auto key = std::make_tuple(l1, m1, l2, m2, L, M);
    auto it = cg_cache_.find(key);
    if (it != cg_cache_.end()) return it->second;
    const double v = real_cg(l1, m1, l2, m2, L, M);
    cg_cache_[key] = v;
    return v;
  }

  bool allowed(int qi, int body) const { return q_[qi].l <= body_lmax_[body]; }

  // Tuples of q indices with non-increasing l and non-increasing k
  // (sus2_sh.cu:1472-1494).
  void tuples(int count, int body, const std::function<void(const std::vector<int>&)>& cb) {
    std::vector<int> tup;
    std::function<void(int, int, int)> rec = [&](int pos, int max_l, int max_k) {
      if (pos == count) {
        cb(tup);
        return;
      }
      for (int qi = 0; qi < static_cast<int>(q_.size()); ++qi) {
        if (!allowed(qi, body) || q_[qi].l > max_l || q_[qi].k > max_k) continue;
        tup.push_back(qi);
        rec(pos + 1, q_[qi].l, q_[qi].k);
        tup.pop_back();
      }
    };
    rec(0, lmax_, kmax_ - 1);
  }

  void add_spec(int body, const std::vector<int>& qs, int inter) {
    Spec s{body, {-1, -1, -1, -1, -1}, inter};
    for (size_t i = 0; i < qs.size(); ++i) s.q[i] = qs[i];
    specs_.push_back(s);
    for (int i = 0; i < body - 1; ++i) required_[s.q[i]] = 1;
  }

  // Scalar specifications per body order (sus2_sh.cu:1523-1587).
  void collect_specs(int body_order) {
    required_.assign(q_.size(), 0);
    auto l = [&](int qi) { return q_[qi].l; };
    if (body_order >= 2)
      tuples(1, 2, [&](const std::vector<int>& t) {
        if (l(t[0]) == 0) add_spec(2, t, 0);
      });
    if (body_order >= 3)
      tuples(2, 3, [&](const std::vector<int>& t) {
        if (l(t[0]) == l(t[1])) add_spec(3, t, 0);
      });
    if (body_order >= 4)
      tuples(3, 4, [&](const std::vector<int>& t) {
        const int a = l(t[0]), b = l(t[1]), c = l(t[2]);
        if ((a + b + c) % 2 == 0 && triangle(a, b, c)) add_spec(4, t, c);
      });
    if (body_order >= 5)
      tuples(4, 5, [&](const std::vector<int>& t) {
        const int a = l(t[0]), b = l(t[1]), c = l(t[2]), d = l(t[3]);
        if ((a + b + c + d) % 2 != 0) return;
        const int lo = std::max(std::abs(a - b), std::abs(c - d));
        const int hi = std::min(a + b, c + d);
        for (int L = lo; L <= hi; ++L) add_spec(5, t, L);
      });
    if (body_order >= 6)
      tuples(5, 6, [&](const std::vector<int>& t) {
        const int a = l(t[0]), b = l(t[1]), c = l(t[2]), d = l(t[3]), e = l(t[4]);
        if ((a + b + c + d + e) % 2 != 0) return;
        const int lo = std::max(std::abs(a - b), std::abs(c - d));
        const int hi = std::min(a + b, c + d);
        for (int L = lo; L <= hi; ++L)
          if (triangle(L, e, L)) add_spec(6, t, L);
      });
  }

  int scalar_node(int t) const {
    return tensors_[t].zero ? -1 : tensors_[t].node[0];
  }

  // sus2_sh.cu:1589-1629
  int build_scalar(const Spec& s) {
    const int t0 = basic_tensor(s.q[0]);
    if (s.body == 2) return tensors_[t0].node[0];
    const int t1 = basic_tensor(s.q[1]);
    if (s.body == 3) return scalar_node(couple(t0, t1, 0));
    const int t2 = basic_tensor(s.q[2]);
    if (s.body == 4) {
      const int pair = couple(t0, t1, s.inter);
      if (tensors_[pair].zero) return -1;
      return scalar_node(couple(pair, t2, 0));
    }
    const int t3 = basic_tensor(s.q[3]);
    const int left = couple(t0, t1, s.inter);
    const int right_pair = couple(t2, t3, s.inter);
    if (s.body == 6) {
      const int t4 = basic_tensor(s.q[4]);
      if (tensors_[left].zero || tensors_[right_pair].zero) return -1;
      const int right = couple(right_pair, t4, s.inter);
      if (tensors_[right].zero) return -1;
      return scalar_node(couple(left, right, 0));
    }
    if (tensors_[left].zero || tensors_[right_pair].zero) return -1;
    return scalar_node(couple(left, right_pair, 0));
  }

  int lmax_, kmax_;
  int nodes_ = 0, tensor_blocks_ = 0, cg_blocks_ = 0, cg_terms_ = 0, max_layer_ = 0;
  std::vector<int> body_lmax_;
  std::vector<Q> q_;
  std::vector<Tensor> tensors_;
  std::vector<std::string> keys_;
  std::unordered_map<std::string, int> lookup_;
  std::map<std::tuple<int, int, int>, int> product_lookup_;
  std::vector<Product> products_;
  std::vector<char> required_;
  std::vector<Spec> specs_;
  std::vector<int> bk_, bl_, bm_;
  std::map<std::tuple<int, int, int, int, int, int>, double> cg_cache_;
};
}  // namespace

StandardGraph build_standard_graph(int l_max, int k_max, int body_order,
                                   const std::vector<int>& body_l_max) {
  if (l_max < 0 || k_max <= 0 || body_order < 2 || body_order > 6 || body_l_max.size() < 7)
    throw InputError("Invalid standard graph specification.");
  GraphBuilder b(l_max, k_max);
  return b.build(body_order, body_l_max);
}

// ---------------------------------------------------------------------------
// Layered rows (build_explicit_sh_graph_metadata, sus2_sh.cu:1913-2093) and
// terminal-scalar flags (sus2_sh.cu:8149-8196).
// ---------------------------------------------------------------------------
Layered layer_products(const HostModel& m) {
  const int M = m.moments, B = m.basic_count;
  if (M <= 0 || B <= 0 || B > M) throw InputError("SUS2_SH invalid explicit product graph dimensions.");
  std::vector<int> last_def(M, -1);
  std::vector<std::vector<int>> by_target(M);
  for (size_t p = 0; p < m.products.size(); ++p) {
    const Product& pr = m.products[p];
    if (pr.target < B) throw InputError("SUS2_SH explicit product graph writes into a basic moment.");
    by_target[pr.target].push_back(static_cast<int>(p));
    last_def[pr.target] = static_cast<int>(p);
  }
  for (size_t p = 0; p < m.products.size(); ++p) {
    const Product& pr = m.products[p];
    for (int s : {pr.left, pr.right}) {
      if (s >= B && last_def[s] < 0)
        throw InputError("SUS2_SH explicit product graph references an undefined moment.");
      if (s >= B && last_def[s] >= static_cast<int>(p))
        throw InputError("SUS2_SH explicit product graph is not topologically ordered.");
    }
  }
  std::vector<char> defined(M, 0);
  for (int i = 0; i < B; ++i) defined[i] = 1;
  std::vector<int> targets;
  for (int t = B; t < M; ++t)
    if (!by_target[t].empty()) {
      targets.push_back(t);
      defined[t] = 1;
    }
  std::sort(targets.begin(), targets.end(), [&](int a, int b) {
    return last_def[a] != last_def[b] ? last_def[a] < last_def[b] : a < b;
  });
  for (int s = 0; s < m.scalar_count; ++s) {
    const int mm = m.moment_mapping[s];
    if (mm < 0 || mm >= M || !defined[mm])
      throw InputError("SUS2_SH alpha_moment_mapping references an undefined moment.");
  }
  Layered out;
  out.node_layer.assign(M, 0);
  for (int t : targets) {
    int src = 0;
    for (int p : by_target[t])
      src = std::max({src, out.node_layer[m.products[p].left], out.node_layer[m.products[p].right]});
    out.node_layer[t] = src + 1;
    out.max_layer = std::max(out.max_layer, src + 1);
  }
  std::vector<std::vector<int>> per_layer(out.max_layer + 1);
  for (int t : targets) per_layer[out.node_layer[t]].push_back(t);
  std::vector<char> used(M, 0);
  for (int layer = 1; layer <= out.max_layer; ++layer) {
    std::sort(per_layer[layer].begin(), per_layer[layer].end());
    for (int t : per_layer[layer]) {
      Row r;
      r.layer = layer;
      r.target = t;
      for (int p : by_target[t]) {
        r.left.push_back(m.products[p].left);
        r.right.push_back(m.products[p].right);
        r.coeff.push_back(m.products[p].coeff);
        used[m.products[p].left] = used[m.products[p].right] = 1;
      }
      out.rows.push_back(std::move(r));
    }
  }
  out.scalar_of.assign(M, -1);
  for (int s = 0; s < m.scalar_count; ++s) out.scalar_of[m.moment_mapping[s]] = s;
  out.terminal.assign(M, 0);
  for (const Row& r : out.rows)
    if (out.scalar_of[r.target] >= 0 && !used[r.target]) out.terminal[r.target] = 1;
  return out;
}

// ---------------------------------------------------------------------------
// Options (parse_sh_float, sus2_sh.cu:520-536).  Tokens before index
// species_count are element symbols.
// ---------------------------------------------------------------------------
Options parse_options(const HostModel& m, int nopts, const char** opts) {
  Options o;
  if (const char* env = std::getenv("SUS2_GPUMD_FLOAT")) o.use_float = parse_bool(env, "SUS2_GPUMD_FLOAT");
  {
    const char* env = std::getenv("SUS2_SH_GPUMD_PROFILE");
    if (!env) env = std::getenv("SUS2_GPUMD_PROFILE");
    if (env) o.profile = parse_bool(env, "SUS2_SH_GPUMD_PROFILE");
  }
  const int begin = std::min(nopts, m.species_count);
  for (int i = begin; i < nopts; ++i) {
    const std::string s = opts[i] ? opts[i] : "";
    const size_t eq = s.find('=');
    const std::string key = eq == std::string::npos ? s : s.substr(0, eq);
    const std::string val = eq == std::string::npos ? "" : s.substr(eq + 1);
    if (key == "sus2_float" || key == "sus2_sh_float") {
      o.use_float = parse_bool(val, key);
    } else if (key == "sus2_sh_skin") {
      o.skin = std::atof(val.c_str());
      if (!(o.skin >= 0.0)) throw InputError("sus2_sh_skin must be >= 0.");
    } else if (key == "sus2_sh_rebuild_interval") {
      o.rebuild_interval = std::atoi(val.c_str());
    } else if (key == "sus2_sh_profile" || key == "sus2_profile") {
      o.profile = parse_bool(val, key);
    } else if (key == "sus2_sh_autotune") {
      o.autotune = parse_bool(val, key);
    } else if (key == "sus2_sh_edge_jit") {
      o.edge_jit = parse_bool(val, key);
    } else if (key == "sus2_sh_model_edges") {
      o.model_edges = parse_bool(val, key);
    } else if (key == "sus2_sh_neighbor_graph") {
      o.neighbor_graph = parse_bool(val, key);
    } else if (key == "sus2_sh_batch_fused") {
      o.batch_fused = parse_bool(val, key);
    } else if (key == "sus2_sh_batch_tile") {
      o.batch_tile = std::atoi(val.c_str());
      if (o.batch_tile < 0 || o.batch_tile > (1 << 20))
        throw InputError("sus2_sh_batch_tile must be between 0 and 1048576 atoms.");
    } else if (key == "sus2_sh_cg_jit") {
      o.cg_jit = parse_bool(val, key);
    } else if (key == "sus2_sh_cg_split") {
      o.cg_split = parse_bool(val, key) ? 1 : 0;
    } else if (key == "sus2_sh_cg_whole") {
      o.cg_whole = parse_bool(val, key);
    } else if (key == "sus2_sh_reference_rounding") {
      o.reference_rounding = parse_bool(val, key);
    } else if (key == "sus2_radial_direct" || key == "sus2_sh_radial_direct" || key == "radial_direct") {
      if (!parse_bool(val, key))
        throw InputError("SUS2_SH first backend currently requires direct radial evaluation.");
    } else if (key == "sus2_sh_factor_pruning" || key == "sus2_factor_pruning" || key == "sh_factor_pruning") {
      if (val != "legacy" && val != "Legacy" && val != "LEGACY" && val != "q-total" &&
          val != "q_total" && val != "total" && val != "QTotal" && val != "QTOTAL")
        throw InputError("Invalid SUS2_SH factor pruning mode: " + val + " (expected legacy or q-total).");
    }
    // Every other token (the reference's A/B tuning switches) is accepted and
    // ignored: this engine has a single execution plan.
  }
  return o;
}

}  // namespace sus2sh
