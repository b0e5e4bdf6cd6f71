// Test infrastructure only: a C-ABI harness around the reference's own ZBL
// header (src/force/sus2_zbl_common.cuh), compiled from the reference tree by
// oracle/build_ref.py into oracle/_ref/libref_zbl.so.  Tests use it to pin the
// oracle's ZBL restatement and the engine's pair function; nothing else loads
// it.
#include <cstring>
#include <string>
#include <vector>

#include "src/force/sus2_zbl_common.cuh"

extern "C" {

void ref_zbl_pair(int zi, int zj, double r, double inner, double outer, double* energy, double* dEdr) {
  const SUS2ZBLPairValue v = sus2_zbl_pair(zi, zj, r, inner, outer);
  *energy = v.energy;
  *dEdr = v.dEdr;
}

double ref_zbl_covalent_radius(int z) { return sus2_zbl_covalent_radius(z); }

int ref_zbl_atomic_number(const char* symbol) { return sus2_zbl_atomic_number_from_symbol(symbol); }

double ref_zbl_typewise_outer(int zi, int zj, double outer, double factor) {
  return sus2_zbl_typewise_outer_cutoff(zi, zj, outer, factor);
}

// 1 on success (tables filled), 0 with the reference's message in err.
int ref_zbl_tables(int species, const int* z, double inner, double outer, int typewise, double factor, double* pin,
                   double* pout, double* pout_sq, char* err, int errlen) {
  std::vector<int> zv(z, z + (species > 0 ? species : 0));
  std::vector<double> a, b, c;
  std::string msg;
  const bool ok = sus2_zbl_fill_pair_cutoff_tables(zv, inner, outer, typewise != 0, factor, a, b, c, &msg);
  if (!ok) {
    if (err && errlen > 0) {
      std::strncpy(err, msg.c_str(), static_cast<size_t>(errlen) - 1);
      err[errlen - 1] = '\0';
    }
    return 0;
  }
  for (size_t k = 0; k < a.size(); ++k) {
    pin[k] = a[k];
    pout[k] = b[k];
    pout_sq[k] = c[k];
  }
  return 1;
}

void ref_zbl_defaults(double* inner, double* outer, double* factor) {
  *inner = sus2_zbl_default_inner_cutoff();
  *outer = sus2_zbl_default_outer_cutoff();
  *factor = sus2_zbl_default_typewise_cutoff_factor();
}

}  // extern "C"
