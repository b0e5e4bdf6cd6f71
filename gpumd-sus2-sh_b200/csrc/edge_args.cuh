// Arguments of the per-edge kernels (k_basic, k_force and the parameter-
// gradient edge kernels), shared by the ahead-of-time build and the NVRTC
// build of model shapes compiled at load (no host headers here).
#pragma once

namespace sus2sh {

constexpr int kMaxPairTable = 8192;  // floats of per-pair radial table
constexpr int kMaxCoef = 48 * 16;

// Radial table: per pair p = t_i*S + t_j: [KMU] (scal, shift) pairs then the
// pair scale; shared_xi means every mu of a pair uses the same (scal, shift).
// kind: 0 Chebyshev basis of the tanh map, 1 of the rational map, 2 Laguerre
// basis of log(1 + r / rho) (kRadial* in sh_math.cuh; shift holds rho).
struct RadialSetup {
  int species;
  int kmu;
  int rb;
  int kind;
  int shared_xi;
  int pair_stride;  // floats per pair in the table
  double rc;
};

template <typename T>
struct EdgeArgs {
  int N;
  int cap;
  int l_max, k_max;
  RadialSetup rs;
  const double4* pos4;
  const int* nbr;
  const int* ncount;
  // in-cutoff sub-list [cap][N] / counts [N]: k_basic writes it (when
  // cut_nbr is set) in the order of the full list, k_force then walks only
  // those pairs (when use_cut is set) instead of testing every listed pair
  int* cut_nbr;
  int* cut_count;
  int use_cut;
  // inner list (pairs within rc + a margin, list order) walked by k_basic
  // instead of nbr / ncount when set
  const int* inner_nbr;
  const int* inner_count;
  const void* pair_table;   // T[S*S][pair_stride]
  const double (*shift)[3];  // image vectors [cells][125][3] (one box: BoxGeom::shift)
  const int* atom_cell;      // cell of each atom in a batch of boxes, NULL for one box
  // two-layer gate models only (kernels instantiated with GATE = true):
  const T* gate_mult;        // [Kmu][N] G_{j,mu} = 1 + A tanh(a_j h_{j,mu})
  const T* gate_deriv;       // [Kmu][N] dG/dh
  T* gate_adj;               // [Kmu][N] dE/dh accumulated by k_force (atomics)
  // c[mu][n] (uniform across lanes), then, when 2 kmu rb <= kMaxCoef, the
  // derivative series d[mu][n] at offset kmu rb:
  // sum_n c[mu][n] P_n'(x) = sum_n d[mu][n] P_n(x), d[mu][rb-1] = 0, for the
  // basis polynomials P_n of the kind (Chebyshev T_n or Laguerre L_n).
  // One array keeps the FP32 kernel parameters under 4 KB, where every
  // coefficient is an immediate constant-bank operand.
  T coef[kMaxCoef];
};

// Neighbour and input status flags of one engine handle (device, sticky).
struct Status {
  unsigned int maxdisp2_bits;  // max |u - ref|^2 since last build (float bits)
  int rebuilt;                 // a build happened in this call
  int overflow;                // neighbour capacity exceeded (sticky)
  int max_count;               // largest neighbour count seen at a build
  int builds;                  // number of builds
  int bad_type;                // a species index outside [0, species_count) was seen (sticky)
  int thin_cell;               // a batch cell thinner than half the cutoff (sticky)
  int pad;
};

namespace batch {

// Arguments of the fused batch kernel (batch_fused.cuh) beside its EdgeArgs.
struct FusedArgs {
  int ncells;
  int ntiles;      // N / tile_atoms + 1
  int tile_atoms;  // TA
  int buf_atoms;   // capacity of the shared-memory force buffer (atoms)
  const int* off;  // cell offsets [ncells + 1]
  const double* shift_coeffs;    // per-species energy shift
  const double* species_coeffs;  // per-species c_t
  double* pe;                    // [N], accumulated
  double* force;                 // [3][N], accumulated
  double* virial;                // [9][N], accumulated (may be NULL)
  double* cell_energy;           // [ncells], assigned (may be NULL)
  double* cell_virial;           // [9 ncells], assigned (may be NULL)
  int* tile_counter;             // next tile to draw; zeroed before every launch
  // fill = 1: each tile first builds its cells' neighbour lists (the batch
  // fill of batch_fill.cuh, into nbr / ncount with capacity cap, cutoff^2
  // cutoff2, status flags in st); 0: the lists are already built
  int fill;
  const double* cell_h;          // [9 ncells]
  const int* cell_reach;         // [3 ncells]
  double cutoff2;
  int* nbr;                      // [cap][N]
  int* ncount;                   // [N]
  int cap;
  Status* st;
};

}  // namespace batch

}  // namespace sus2sh
