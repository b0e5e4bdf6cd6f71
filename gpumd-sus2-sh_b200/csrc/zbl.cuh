// Universal ZBL short-range pair term (Ziegler-Biersack-Littmark screened
// Coulomb) with a cosine switch, as the reference adds it to SUS2-SH models
// with `zbl_enabled = 1` (src/force/sus2_zbl_common.cuh:18-225, applied by
// gpu_sh_apply_zbl, src/force/sus2_sh.cu:7522-7627):
//
//   E(r) = S(r) k Zi Zj phi(r / a) / r,  1/a = 2.134563 (Zi^0.23 + Zj^0.23),
//   phi(x) = 0.18175 e^{-3.1998 x} + 0.50986 e^{-0.94229 x}
//          + 0.28022 e^{-0.4029 x} + 0.02817 e^{-0.20162 x},
//   S = 1 (r <= r_in), (1 + cos(pi (r - r_in)/(r_out - r_in)))/2 (r_in < r < r_out),
//   0 beyond, k = 14.3996454784255 eV A.
// The constants and the covalent-radius table are the reference's (they
// define the model), restated here; evaluation is FP64 in both engines.
#pragma once

#include <cmath>
#include <string>
#include <vector>

#if defined(__CUDACC__)
#define SUS2_ZBL_FN __host__ __device__ __forceinline__
#else
#define SUS2_ZBL_FN inline
#endif

namespace sus2sh {
namespace zbl {

constexpr double kDefaultInner = 0.7;
constexpr double kDefaultOuter = 1.4;
constexpr double kDefaultTypewiseFactor = 0.7;
constexpr int kMaxZ = 94;

struct PairValue {
  double energy;
  double dEdr;
};

// Energy and dE/dr of one pair at distance r (0 outside (0, outer)).
SUS2_ZBL_FN PairValue pair(int zi, int zj, double r, double inner, double outer) {
  PairValue out{0.0, 0.0};
  if (zi <= 0 || zj <= 0 || r <= 0.0 || outer <= 0.0 || r >= outer) return out;
  const double ainv = 2.134563 * (pow(static_cast<double>(zi), 0.23) + pow(static_cast<double>(zj), 0.23));
  const double x = ainv * r;
  const double c[4] = {0.18175, 0.50986, 0.28022, 0.02817};
  const double b[4] = {3.1998, 0.94229, 0.4029, 0.20162};
  double phi = 0.0, dphi = 0.0;
  for (int q = 0; q < 4; ++q) {
    const double e = exp(-b[q] * x);
    phi += c[q] * e;
    dphi -= c[q] * b[q] * ainv * e;
  }
  const double k = 14.3996454784255 * static_cast<double>(zi) * static_cast<double>(zj);
  const double e0 = k * phi / r;
  const double de0 = k * (dphi / r - phi / (r * r));
  double s = 1.0, ds = 0.0;
  if (r > inner) {
    const double w = 3.141592653589793238462643383279502884 / (outer - inner);
    s = 0.5 * cos(w * (r - inner)) + 0.5;
    ds = -0.5 * w * sin(w * (r - inner));
  }
  out.energy = s * e0;
  out.dEdr = s * de0 + ds * e0;
  return out;
}

// Covalent radius (A) used by the typewise cutoffs; 0 outside 1..94.
inline double covalent_radius(int z) {
  static const double r[kMaxZ] = {
      0.426667, 0.613333, 1.6,      1.25333,  1.02667,  1.0,      0.946667, 0.84,     0.853333, 0.893333,
      1.86667,  1.66667,  1.50667,  1.38667,  1.46667,  1.36,     1.32,     1.28,     2.34667,  2.05333,
      1.77333,  1.62667,  1.61333,  1.46667,  1.42667,  1.38667,  1.33333,  1.32,     1.34667,  1.45333,
      1.49333,  1.45333,  1.53333,  1.46667,  1.52,     1.56,     2.52,     2.22667,  1.96,     1.85333,
      1.76,     1.65333,  1.53333,  1.50667,  1.50667,  1.44,     1.53333,  1.64,     1.70667,  1.68,
      1.68,     1.64,     1.76,     1.74667,  2.78667,  2.34667,  2.16,     1.96,     2.10667,  2.09333,
      2.08,     2.06667,  2.01333,  2.02667,  2.01333,  2.0,      1.98667,  1.98667,  1.97333,  2.04,
      1.94667,  1.82667,  1.74667,  1.64,     1.57333,  1.54667,  1.48,     1.49333,  1.50667,  1.76,
      1.73333,  1.73333,  1.81333,  1.74667,  1.84,     1.89333,  2.68,     2.41333,  2.22667,  2.10667,
      2.02667,  2.04,     2.05333,  2.06667};
  return (z >= 1 && z <= kMaxZ) ? r[z - 1] : 0.0;
}

// Atomic number of an element symbol, 0 if unknown.
inline int atomic_number(const std::string& symbol) {
  static const char* const sym[kMaxZ] = {
      "H",  "He", "Li", "Be", "B",  "C",  "N",  "O",  "F",  "Ne", "Na", "Mg", "Al", "Si", "P",  "S",
      "Cl", "Ar", "K",  "Ca", "Sc", "Ti", "V",  "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn", "Ga", "Ge",
      "As", "Se", "Br", "Kr", "Rb", "Sr", "Y",  "Zr", "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd",
      "In", "Sn", "Sb", "Te", "I",  "Xe", "Cs", "Ba", "La", "Ce", "Pr", "Nd", "Pm", "Sm", "Eu", "Gd",
      "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu", "Hf", "Ta", "W",  "Re", "Os", "Ir", "Pt", "Au", "Hg",
      "Tl", "Pb", "Bi", "Po", "At", "Rn", "Fr", "Ra", "Ac", "Th", "Pa", "U",  "Np", "Pu"};
  for (int z = 0; z < kMaxZ; ++z)
    if (symbol == sym[z]) return z + 1;
  return 0;
}

// Per species pair (i*S + j) inner/outer cutoffs: global (inner, outer), or
// typewise inner 0 and outer min(factor (r_cov,i + r_cov,j), outer).  Returns
// an error message, empty on success.
inline std::string pair_cutoffs(const std::vector<int>& z, double inner, double outer, bool typewise,
                                double factor, std::vector<double>& pin, std::vector<double>& pout) {
  const int S = static_cast<int>(z.size());
  if (S <= 0) return "ZBL requires one atomic number per model species.";
  if (inner < 0.0) return "ZBL inner cutoff should be non-negative.";
  if (outer <= 0.0) return "ZBL outer cutoff should be positive.";
  if (typewise) {
    if (factor < 0.5) return "ZBL typewise cutoff factor should be at least 0.5.";
  } else if (outer <= inner) {
    return "ZBL cutoffs should satisfy 0 <= inner < outer.";
  }
  pin.assign(static_cast<size_t>(S) * S, 0.0);
  pout.assign(static_cast<size_t>(S) * S, 0.0);
  for (int a = 0; a < S; ++a)
    for (int b = 0; b < S; ++b) {
      if (z[a] <= 0 || z[b] <= 0 || (typewise && (covalent_radius(z[a]) <= 0.0 || covalent_radius(z[b]) <= 0.0)))
        return "ZBL atomic numbers should be in [1, 94].";
      double i_cut = inner, o_cut = outer;
      if (typewise) {
        i_cut = 0.0;
        const double t = factor * (covalent_radius(z[a]) + covalent_radius(z[b]));
        o_cut = t < outer ? t : outer;
      }
      if (o_cut <= i_cut) return "ZBL pair cutoffs should satisfy inner < outer.";
      pin[static_cast<size_t>(a) * S + b] = i_cut;
      pout[static_cast<size_t>(a) * S + b] = o_cut;
    }
  return "";
}

}  // namespace zbl
}  // namespace sus2sh

#undef SUS2_ZBL_FN
