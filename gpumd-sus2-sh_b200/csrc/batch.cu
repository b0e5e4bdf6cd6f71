// Batches of small independent periodic boxes ("cells") evaluated together:
// geometry tables per cell, packing, per-cell neighbour lists (batch_fill.cuh)
// and per-cell reductions.  The edge, product and force kernels are the
// engine's own; they read each atom's image vectors from its cell's table
// (EdgeArgs::atom_cell).
#include "batch_fill.cuh"
#include "edge_common.cuh"
#include "engine.cuh"

namespace sus2sh {
namespace {
using namespace edge;

__device__ __forceinline__ void inv3(const double* h, double* o) {
  const double det = h[0] * (h[4] * h[8] - h[5] * h[7]) - h[1] * (h[3] * h[8] - h[5] * h[6]) +
                     h[2] * (h[3] * h[7] - h[4] * h[6]);
  const double id = 1.0 / det;
  o[0] = (h[4] * h[8] - h[5] * h[7]) * id;
  o[1] = (h[2] * h[7] - h[1] * h[8]) * id;
  o[2] = (h[1] * h[5] - h[2] * h[4]) * id;
  o[3] = (h[5] * h[6] - h[3] * h[8]) * id;
  o[4] = (h[0] * h[8] - h[2] * h[6]) * id;
  o[5] = (h[2] * h[3] - h[0] * h[5]) * id;
  o[6] = (h[3] * h[7] - h[4] * h[6]) * id;
  o[7] = (h[1] * h[6] - h[0] * h[7]) * id;
  o[8] = (h[0] * h[4] - h[1] * h[3]) * id;
}

// One block per cell: inverse, image reach and the 125 image vectors.
__global__ void k_batch_geometry(int ncells, const double* __restrict__ cell_h, const int* __restrict__ cell_pbc,
                                 double cutoff, double* __restrict__ cell_hinv, int* __restrict__ cell_reach,
                                 double (*__restrict__ cell_shift)[3], int* __restrict__ err) {
  const int c = blockIdx.x;
  if (c >= ncells) return;
  const double* h = cell_h + 9 * c;
  if (threadIdx.x == 0) {
    double inv[9];
    inv3(h, inv);
    for (int k = 0; k < 9; ++k) cell_hinv[9 * c + k] = inv[k];
    const double a[3] = {h[0], h[3], h[6]}, b[3] = {h[1], h[4], h[7]}, cc[3] = {h[2], h[5], h[8]};
    const double* u[3] = {b, cc, a};
    const double* v[3] = {cc, a, b};
    const double vol = fabs(a[0] * (b[1] * cc[2] - b[2] * cc[1]) - a[1] * (b[0] * cc[2] - b[2] * cc[0]) +
                            a[2] * (b[0] * cc[1] - b[1] * cc[0]));
    for (int d = 0; d < 3; ++d) {
      const double x = u[d][1] * v[d][2] - u[d][2] * v[d][1], y = u[d][2] * v[d][0] - u[d][0] * v[d][2],
                   z = u[d][0] * v[d][1] - u[d][1] * v[d][0];
      const double thick = vol / sqrt(x * x + y * y + z * z);
      const int periodic = cell_pbc ? cell_pbc[3 * c + d] : 1;
      int r = periodic ? static_cast<int>(ceil(cutoff / thick - 1e-12)) : 0;
      if (periodic && r < 1) r = 1;
      if (r > 2) {
        r = 2;
        atomicExch(err, 1);  // cell thinner than half the cutoff
      }
      cell_reach[3 * c + d] = r;
    }
  }
  for (int code = threadIdx.x; code < 125; code += blockDim.x) {
    const int tx = code / 25 - 2, ty = (code / 5) % 5 - 2, tz = code % 5 - 2;
    for (int k = 0; k < 3; ++k) cell_shift[125 * c + code][k] = tx * h[3 * k] + ty * h[3 * k + 1] + tz * h[3 * k + 2];
  }
}

// Cell of atom i by binary search of the offsets; positions wrapped into the
// cell's periodic directions.
__global__ void k_batch_pack(int N, int ncells, const int* __restrict__ off, const double* __restrict__ x,
                             const int* __restrict__ type, const double* __restrict__ cell_h,
                             const double* __restrict__ cell_hinv, const int* __restrict__ cell_pbc, int species,
                             int* __restrict__ atom_cell, double4* __restrict__ pos4, Status* st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int lo = 0, hi = ncells - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= i) lo = mid;
    else hi = mid - 1;
  }
  const int c = lo;
  const double* h = cell_h + 9 * c;
  const double* hi_ = cell_hinv + 9 * c;
  const double p[3] = {x[i], x[i + N], x[i + 2 * N]};
  double s[3];
  for (int a = 0; a < 3; ++a) {
    s[a] = hi_[3 * a] * p[0] + hi_[3 * a + 1] * p[1] + hi_[3 * a + 2] * p[2];
    const int periodic = cell_pbc ? cell_pbc[3 * c + a] : 1;
    if (periodic) s[a] -= floor(s[a]);
  }
  int t = type[i];
  if (t < 0 || t >= species) {
    st->bad_type = 1;
    t = 0;
  }
  pos4[i] = make_double4(h[0] * s[0] + h[1] * s[1] + h[2] * s[2], h[3] * s[0] + h[4] * s[1] + h[5] * s[2],
                         h[6] * s[0] + h[7] * s[1] + h[8] * s[2], __longlong_as_double(static_cast<long long>(t)));
  atom_cell[i] = c;
}

// Triclinic cells: one thread per atom (orthorhombic cells return at once).
__global__ void __launch_bounds__(128)
    k_batch_fill(int N, const int* __restrict__ off, const int* __restrict__ atom_cell,
                 const double4* __restrict__ pos4, const double* __restrict__ cell_h,
                 const int* __restrict__ cell_reach, double cutoff2, int* __restrict__ nbr,
                 int* __restrict__ ncount, int cap, int count_only, Status* st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  batch::fill_atom_triclinic(i, atom_cell[i], N, off, pos4, cell_h, cell_reach, cutoff2, nbr, ncount, cap,
                             count_only, st);
}

// Orthorhombic cells: one CTA per cell (triclinic cells return at once).
__global__ void __launch_bounds__(128)
    k_batch_fill_ortho(int N, const int* __restrict__ off, const double4* __restrict__ pos4,
                       const double* __restrict__ cell_h, const int* __restrict__ cell_reach, double cutoff2,
                       int* __restrict__ nbr, int* __restrict__ ncount, int cap, int count_only, Status* st) {
  __shared__ batch::FillShared sh;
  batch::fill_cell_ortho(blockIdx.x, N, off, pos4, cell_h, cell_reach, cutoff2, nbr, ncount, cap, count_only, st,
                         sh);
}

// One block per cell: sum of site energies and of per-atom virials.
__global__ void k_cell_reduce(int ncells, const int* __restrict__ off, const double* __restrict__ pe,
                              const double* __restrict__ vir, double* __restrict__ cell_energy,
                              double* __restrict__ cell_virial, int N) {
  const int c = blockIdx.x;
  if (c >= ncells) return;
  __shared__ double red[10][4];
  double v[10];
  for (int q = 0; q < 10; ++q) v[q] = 0.0;
  for (int i = off[c] + threadIdx.x; i < off[c + 1]; i += blockDim.x) {
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
    if (threadIdx.x == 0) {
      if (cell_energy) cell_energy[c] = x;
    } else if (cell_virial) {
      cell_virial[9 * c + threadIdx.x - 1] = x;
    }
  }
}

inline int blocks(int n, int b) { return (n + b - 1) / b; }

}  // namespace

void launch_batch_geometry(cudaStream_t s, int ncells, const double* cell_h, const int* cell_pbc, double cutoff,
                           double* cell_hinv, int* cell_reach, double (*cell_shift)[3], int* status_error) {
  k_batch_geometry<<<ncells, 128, 0, s>>>(ncells, cell_h, cell_pbc, cutoff, cell_hinv, cell_reach, cell_shift,
                                          status_error);
}

void launch_batch_pack(cudaStream_t s, int N, int ncells, const int* off, const double* x, const int* type,
                       const double* cell_h, const double* cell_hinv, const int* cell_pbc, int species,
                       int* atom_cell, double4* pos4, Status* st) {
  k_batch_pack<<<blocks(N, 256), 256, 0, s>>>(N, ncells, off, x, type, cell_h, cell_hinv, cell_pbc, species,
                                              atom_cell, pos4, st);
}

void launch_batch_fill(cudaStream_t s, int N, int ncells, const int* off, const int* atom_cell, const double4* pos4,
                       const double* cell_h, const int* cell_reach, double cutoff2, int* nbr, int* ncount, int cap,
                       int count_only, Status* st) {
  k_batch_fill_ortho<<<ncells, 128, 0, s>>>(N, off, pos4, cell_h, cell_reach, cutoff2, nbr, ncount, cap, count_only,
                                            st);
  k_batch_fill<<<blocks(N, 128), 128, 0, s>>>(N, off, atom_cell, pos4, cell_h, cell_reach, cutoff2, nbr, ncount,
                                              cap, count_only, st);
}

void launch_cell_reduce(cudaStream_t s, int ncells, int N, const int* off, const double* pe, const double* virial,
                        double* cell_energy, double* cell_virial) {
  k_cell_reduce<<<ncells, 128, 0, s>>>(ncells, off, pe, virial, cell_energy, cell_virial, N);
}

}  // namespace sus2sh
