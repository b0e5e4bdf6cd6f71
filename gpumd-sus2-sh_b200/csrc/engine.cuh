// Device-side data layout and kernel launchers of the SUS2-SH engine.
//
// HBM layout (N atoms):
//   pos4   double4[N]   unwrapped position (x,y,z) + species in .w (int bits)
//   ref4   double4[N]   wrapped position at the last neighbour build
//   nbr    int32[cap][N] neighbour j (bits 0-23) | image code (bits 24-31)
//   ncount int32[N]
//   B, G   T[K*C][N]    basic moments and their adjoints, canonical order
//                        k*C + l*l + l + m, C = (L+1)^2
//   ftmp   float4/double [N]  scatter target for F_j -= dE
// Every launch goes to the caller's stream; no host synchronisation happens
// in the steady state.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "edge_args.cuh"

namespace sus2sh {


// Box and cell grid for one neighbour build (host computed).
struct BoxGeom {
  double h[9];      // column vectors a=(h0,h3,h6), b=(h1,h4,h7), c=(h2,h5,h8)
  double hinv[9];
  int pbc[3];
  int ncell[3];     // cells per fractional direction
  int reach[3];     // cell offsets scanned per direction (1 or 2)
  double cellvec[9];  // h with column d divided by ncell[d]: cell (cx,cy,cz)'s corner is cellvec (cx,cy,cz)
  double shift[125][3];  // Cartesian image vectors of codes (base 5, -2..2)
};

struct ProgramDev {
  int nrows;
  int nvalue;         // value slots; grad slot of v is v + nvalue
  int nbasic;
  int ncanon;         // K*C
  const uint32_t* code;
  const void* coef;   // T[]
  const int* basic_canon;  // [nbasic] canonical index of model basic b
  const int* canon_basic;  // [ncanon] model basic or -1
};

// The saved products in file order (flat form) and the scalar weights, for
// the parameter-gradient pass.
struct FlatProgram {
  int nprod, nbasic, ncanon, nscalar;
  const int* left;
  const int* right;
  const int* target;
  const double* coeff;
  const int* basic_canon;
  const int* scalar_map;
  const double* scalar_w;
};

// Parameter gradients (param_grad.cu): weights ew = dL/dE_i (N, may be NULL)
// and fw = dL/dF_i (3N SoA, may be NULL).  Passes: launch_pg_basic (B and its
// tangent Bd, zeroes grad_c), then the product pass -- the generated
// forward-over-reverse kernel followed by launch_pg_reduce over its
// [nscalar][N] per-atom terms, or the flat interpreter launch_pg_product
// (scratch work [4 M][N]) -- then launch_pg_radial (grad_c [kmu*rb],
// accumulated).  grad_w [nscalar] is assigned.  B, Bd, Galpha, Gbeta:
// [K*C][N].  The edge passes return -1 for shapes without an ahead-of-time
// build.
template <typename T>
int launch_pg_basic(cudaStream_t s, const EdgeArgs<T>& a, const double* fw, T* B, T* Bd, double* grad_c);
template <typename T>
void launch_pg_product(cudaStream_t s, int N, const FlatProgram& p, int M, const double4* pos4,
                       const double* species_coeffs, const double* ew, const T* B, const T* Bd, T* work, T* Galpha,
                       T* Gbeta, double* grad_w);
// partial: nscalar * 64 doubles of scratch.
template <typename T>
void launch_pg_reduce(cudaStream_t s, int nscalar, int N, const T* contrib, double* partial, double* grad_w);
template <typename T>
int launch_pg_radial(cudaStream_t s, const EdgeArgs<T>& a, const double* fw, const T* Galpha, const T* Gbeta,
                     double* grad_c);

// Program tables of a handle, for kernels outside the handle's own path.
struct CgView {
  ProgramDev prog;
  const double* shift;
  const double* species;
  int species_count;
  int use_float;
  int device;  // device the handle's tables were created on
};

// ---- launchers (engine.cu) ----------------------------------------------
void launch_pack(cudaStream_t s, int N, const double* x, const int* type, const double4* ref4,
                 double4* pos4, const BoxGeom* geom_dev, int have_ref, int species, Status* st);
// Inner list of the listed pairs within sqrt(inner2) (k_inner); runs when the
// list was rebuilt in this call or the largest displacement since the build
// exceeds sqrt(half_margin2).
void launch_inner(cudaStream_t s, int N, const Status* st, float half_margin2, double inner2, const double4* pos4,
                  const int* nbr, const int* ncount, int cap, const BoxGeom* geom_dev, int* inner_nbr,
                  int* inner_count);
// The neighbour build in two parts: the rebuild decision (k_decide) and the
// rebuild kernels (each returns at once when no rebuild was decided).
void launch_decide(cudaStream_t s, Status* st, int force, float half_skin2);
void launch_rebuild(cudaStream_t s, int N, double cutoff2, const BoxGeom* geom_dev, double4* pos4, double4* ref4,
                    int* cell_count, int* cell_start, int* cell_atoms, float4* cell_rel, int* atom_cell,
                    int* atom_rank, int ncells, int* nbr, int* ncount, int cap, int count_only, Status* st);

// Everything the per-call neighbour work after the decision needs.
struct NeighborGraphArgs {
  int N = 0, ncells = 0, cap = 0, use_inner = 0;
  double cutoff2 = 0.0, inner2 = 0.0;
  float half_margin2 = 0.0f;
  const BoxGeom* geom = nullptr;
  double4 *pos4 = nullptr, *ref4 = nullptr;
  int *cell_count = nullptr, *cell_start = nullptr, *cell_atoms = nullptr, *atom_cell = nullptr,
      *atom_rank = nullptr, *nbr = nullptr, *ncount = nullptr, *inner_nbr = nullptr, *inner_count = nullptr;
  float4* cell_rel = nullptr;
  Status* st = nullptr;
  bool operator==(const NeighborGraphArgs& o) const {
    return N == o.N && ncells == o.ncells && cap == o.cap && use_inner == o.use_inner && cutoff2 == o.cutoff2 &&
           inner2 == o.inner2 && half_margin2 == o.half_margin2 && geom == o.geom && pos4 == o.pos4 &&
           ref4 == o.ref4 && cell_count == o.cell_count && cell_start == o.cell_start &&
           cell_atoms == o.cell_atoms && atom_cell == o.atom_cell && atom_rank == o.atom_rank && nbr == o.nbr &&
           ncount == o.ncount && inner_nbr == o.inner_nbr && inner_count == o.inner_count &&
           cell_rel == o.cell_rel && st == o.st;
  }
};

// The per-call neighbour work after launch_decide as one CUDA graph: a
// one-thread kernel sets two IF conditions from the decision, so the rebuild
// kernels run only when a build is due and k_inner only when the inner list
// needs a refresh (a step without a rebuild launches neither).  The body
// graphs are captured on `capture`.
cudaError_t build_neighbor_graph(cudaStream_t capture, const NeighborGraphArgs& args, cudaGraph_t* graph,
                                 cudaGraphExec_t* exec);

void launch_build(cudaStream_t s, int N, int force, float half_skin2, double cutoff2, const BoxGeom& g,
                  const BoxGeom* geom_dev, double4* pos4, double4* ref4, int* cell_count, int* cell_start,
                  int* cell_atoms, float4* cell_rel, int* atom_cell, int* atom_rank, int ncells, int* nbr,
                  int* ncount, int cap, int count_only, Status* st);

// Edge kernels with CTA size `block` (64, 128 or 256 for FP32; 128 for FP64);
// gate = true selects the gate-model main-pass variants (128 only).
template <typename T>
int launch_basic(cudaStream_t s, const EdgeArgs<T>& a, T* B, int block, bool gate = false);
template <typename T>
int launch_force(cudaStream_t s, const EdgeArgs<T>& a, const T* G, const double* weight,
                 void* ftmp, double* force, double* virial, double sign, int block, bool gate = false);
bool block_supported(int block, bool fp32);

// Two-layer gate: the first-layer graph program (needed moments only) and the
// signal -> multiplier map (gate.cu).
struct GateProgDev {
  int nslots;             // needed moments; basics first
  int nbasic;             // needed basics: slot b <-> canonical row basic_canon[b]
  const int* basic_canon;
  int nprod;              // needed products in file order
  const int* prod;        // [nprod][3] left, right, target slot
  const double* coef;     // [nprod]
  int nq;                 // gate scalars
  const int* q_slot;      // [nq]
  const int* q_body;      // [nq]
  int kmu, nbody, mode;   // mode 1 mu-body-linear-combo, 2 mu-scalar-full
  double amplitude;
  const double* weights;  // full [kmu][nq], combo [nq]
  const double* body_mix; // combo [kmu][nbody]
  const double* additive; // [S]
};
// Gate signals from the first-layer basics Bg: slots M (value scratch
// [nslots][N]), G and dG/dh ([kmu][N]).
template <typename T>
void launch_gate_forward(cudaStream_t s, int N, const GateProgDev& p, const double4* pos4, const T* Bg, T* M,
                         T* gmult, T* gderiv);
// dE/dh ([kmu][N]) -> first-layer basic adjoints Gg (canonical rows, written
// for the needed basics; the caller zeroes Gg), grads scratch gM [nslots][N].
template <typename T>
void launch_gate_backward(cudaStream_t s, int N, const GateProgDev& p, const T* M, T* gM, const T* adjh, T* Gg);
// Sums per-atom energy and virial into out[0] and out[1..9] (FP64 atomics).
void launch_reduce(cudaStream_t s, int N, const double* pe, const double* virial, double* out);
template <typename T>
void launch_product(cudaStream_t s, int N, const ProgramDev& p, const double4* pos4, const T* B,
                    T* G, T* scratch, size_t smem_tile_bytes, int tile, const double* shift_coeffs,
                    const double* species_coeffs, double* pe, int pe_assign);
template <typename T>
void launch_finalize(cudaStream_t s, int N, const void* ftmp, double* force, double sign);

// Batches of independent periodic boxes (cells) evaluated in one pass.
// Cell c holds atoms [off[c], off[c+1]); box columns cell_h[9c..9c+8].
void launch_batch_geometry(cudaStream_t s, int ncells, const double* cell_h, const int* cell_pbc,
                           double cutoff, double* cell_hinv, int* cell_reach, double (*cell_shift)[3],
                           int* status_error);
void launch_batch_pack(cudaStream_t s, int N, int ncells, const int* off, const double* x, const int* type,
                       const double* cell_h, const double* cell_hinv, const int* cell_pbc, int species,
                       int* atom_cell, double4* pos4, Status* st);
void launch_batch_fill(cudaStream_t s, int N, int ncells, const int* off, const int* atom_cell, const double4* pos4,
                       const double* cell_h, const int* cell_reach, double cutoff2, int* nbr, int* ncount,
                       int cap, int count_only, Status* st);
void launch_cell_reduce(cudaStream_t s, int ncells, int N, const int* off, const double* pe, const double* virial,
                        double* cell_energy, double* cell_virial);

// ZBL pair term over the neighbour list (FP64).  mode 0: pe[i] += E_i;
// mode 1: weighted forces (force[i] += sign w_i sum dE, force[j] -= sign w_i dE
// by FP64 atomics) and, if virial != NULL, virial[i] -= w_i r_ij (x) dE.
struct ZblTables {
  int species;
  const int* z;         // [S] atomic numbers
  const double* inner;  // [S*S]
  const double* outer;  // [S*S]
};
void launch_zbl(cudaStream_t s, int mode, int N, int cap, const double4* pos4, const int* nbr, const int* ncount,
                const double (*shift)[3], const int* atom_cell, const ZblTables& z, const double* weight,
                double* pe, double* force, double* virial, double sign);

bool shape_supported(int l_max, int k_max, int rb);

}  // namespace sus2sh
