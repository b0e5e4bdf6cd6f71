// Fused evaluation of a batch of small periodic cells: one persistent launch
// does the per-cell neighbour fill, the basic moments, the CG product graph,
// the forces and virials and the per-cell energy and virial sums of every
// atom of the batch.
//
// NVRTC only: the program that includes this header defines, before it,
// sus2sh::batch::cg_atom (the model's straight-line CG contraction on
// register arrays, cg_codegen.cpp) and the model's radial coefficients
// (SUS2_MODEL_COEF).  The stage kernels it replaces for such models are
// k_batch_fill_ortho / k_batch_fill -> k_basic -> CG kernel -> k_force ->
// k_finalize -> k_cell_reduce, each a pass over every atom with the lists,
// moments and adjoints in HBM between them and the neighbour reactions as
// global atomics.
//
// Work split.  The batch's atoms are cut into tiles of whole cells: tile t
// holds the cells whose first atom lies in [t*TA, (t+1)*TA) (TA = tile_atoms),
// so every tile owns its cells' atoms and sums outright.  CTAs stay resident
// and draw tiles from a counter; a CTA first fills its tile's neighbour lists
// (batch_fill.cuh: the stage fill kernels' code, so the same lists in the same
// order), then walks its tile's atoms BLOCK at a time,
// one thread per atom: moments over the atom's list, the CG contraction with
// the moments and adjoints in registers, then its force loop.  Every
// neighbour of an atom lies in its own cell, so the reactions F_j -= dE land
// in a shared-memory force buffer of the tile (FP32, as the stage path's
// scatter buffer), flushed once into the FP64 force array; a tile with more
// atoms than the buffer holds adds them to the force array with FP64 atomics
// instead.  Per-cell energy and virial sums are taken by the tile's warps
// afterwards, in a fixed order (deterministic), over the accumulated outputs
// as k_cell_reduce takes them.
#pragma once

// the neighbour lists are written by this kernel before it reads them
#define SUS2_NBR_WRITTEN_IN_KERNEL 1
#include "batch_fill.cuh"
#include "edge_kernels.cuh"

namespace sus2sh {
namespace batch {

// First cell c in [0, ncells] with off[c] >= v.
__device__ __forceinline__ int first_cell(const int* __restrict__ off, int ncells, long long v) {
  int lo = 0, hi = ncells;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] >= v) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

template <int L, int K, int RB, int BLOCK, int MINB>
__global__ void __launch_bounds__(BLOCK, MINB) k_batch_fused(const EdgeArgs<float> a, const FusedArgs f) {
  using T = float;
  static_assert(BLOCK == 128, "the fill's shared candidate queue has one column per thread of a 128-thread CTA");
  constexpr int C = (L + 1) * (L + 1), NB = K * C;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* s_tab = reinterpret_cast<T*>(smem_raw);
  const int tab_n = a.rs.species * a.rs.species * a.rs.pair_stride;
  float* s_f = reinterpret_cast<float*>(smem_raw) + ((tab_n + 3) & ~3);
  __shared__ int s_tile[3];
  __shared__ FillShared fill_sh;
  edge::load_pair_table(a, s_tab);
  const int N = a.N;
  const int cap = f.buf_atoms;
  for (;;) {
    if (threadIdx.x == 0) {
      const int t = atomicAdd(f.tile_counter, 1);
      s_tile[0] = t;
      if (t < f.ntiles) {
        s_tile[1] = first_cell(f.off, f.ncells, static_cast<long long>(t) * f.tile_atoms);
        s_tile[2] = first_cell(f.off, f.ncells, static_cast<long long>(t + 1) * f.tile_atoms);
      }
    }
    __syncthreads();
    if (s_tile[0] >= f.ntiles) break;
    const int c0 = s_tile[1], c1 = s_tile[2];
    const int a0 = f.off[c0], a1 = f.off[c1];
    if (f.fill) {
      // the tile's cells' neighbour lists: orthorhombic cells by the whole
      // CTA, triclinic ones one thread per atom
      for (int c = c0; c < c1; ++c)
        if (!fill_cell_ortho(c, N, f.off, a.pos4, f.cell_h, f.cell_reach, f.cutoff2, f.nbr, f.ncount, f.cap, 0,
                             f.st, fill_sh))
          for (int i = f.off[c] + threadIdx.x; i < f.off[c + 1]; i += BLOCK)
            fill_atom_triclinic(i, c, N, f.off, a.pos4, f.cell_h, f.cell_reach, f.cutoff2, f.nbr, f.ncount, f.cap,
                                0, f.st);
    }
    const bool buffered = a1 - a0 <= cap;
    if (buffered)
      for (int q = threadIdx.x; q < a1 - a0; q += BLOCK) {
        s_f[q] = 0.0f;
        s_f[cap + q] = 0.0f;
        s_f[2 * cap + q] = 0.0f;
      }
    __syncthreads();
    // neighbour reactions: the tile's buffer, or FP64 atomics on the output
    auto add = [&](int j, T x, T y, T z) {
      if (buffered) {
        const int q = j - a0;
        atomicAdd(s_f + q, x);
        atomicAdd(s_f + cap + q, y);
        atomicAdd(s_f + 2 * cap + q, z);
      } else {
        atomicAdd(f.force + j, static_cast<double>(x));
        atomicAdd(f.force + N + j, static_cast<double>(y));
        atomicAdd(f.force + 2 * N + j, static_cast<double>(z));
      }
    };
    for (int base = a0; base < a1; base += BLOCK) {
      const int i = base + threadIdx.x;
      if (i >= a1) continue;
      T m[NB];
      edge::atom_basic<T, L, K, RB, false>(a, s_tab, i, m);
#pragma unroll
      for (int c = 0; c < NB; ++c) m[c] *= T(sh_poly_norm<L>(c % C));
      const int ti = edge::type_of(a.pos4[i]);
      const double ct = f.species_coeffs[ti];
      T g[NB];
      const double E = cg_atom(m, g, static_cast<T>(ct));
      f.pe[i] += f.shift_coeffs[ti] + ct + ct * E;
#pragma unroll
      for (int c = 0; c < NB; ++c) g[c] *= T(sh_poly_norm<L>(c % C));
      T fx, fy, fz, w[9];
      edge::atom_force<T, L, K, RB, false>(a, s_tab, i, g, fx, fy, fz, w, add);
      add(i, fx, fy, fz);
      if (f.virial) {
#pragma unroll
        for (int q = 0; q < 9; ++q) f.virial[static_cast<size_t>(q) * N + i] += static_cast<double>(w[q]);
      }
    }
    __syncthreads();  // reactions complete; pe and virial of the tile written
    if (buffered)
      for (int q = threadIdx.x; q < a1 - a0; q += BLOCK) {
        f.force[a0 + q] += static_cast<double>(s_f[q]);
        f.force[N + a0 + q] += static_cast<double>(s_f[cap + q]);
        f.force[2 * N + a0 + q] += static_cast<double>(s_f[2 * cap + q]);
      }
    if (f.cell_energy || f.cell_virial) {
      const int lane = threadIdx.x & 31;
      for (int c = c0 + (threadIdx.x >> 5); c < c1; c += BLOCK / 32) {
        double v[10];
#pragma unroll
        for (int q = 0; q < 10; ++q) v[q] = 0.0;
        for (int i = f.off[c] + lane; i < f.off[c + 1]; i += 32) {
          v[0] += f.pe[i];
          if (f.cell_virial)
#pragma unroll
            for (int q = 0; q < 9; ++q) v[q + 1] += f.virial[static_cast<size_t>(q) * N + i];
        }
#pragma unroll
        for (int q = 0; q < 10; ++q)
          for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
        if (lane == 0) {
          if (f.cell_energy) f.cell_energy[c] = v[0];
          if (f.cell_virial)
#pragma unroll
            for (int q = 0; q < 9; ++q) f.cell_virial[9 * c + q] = v[q + 1];
        }
      }
    }
    __syncthreads();  // the buffer and s_tile are free for the next tile
  }
}

}  // namespace batch
}  // namespace sus2sh
