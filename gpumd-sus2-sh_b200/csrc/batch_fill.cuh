// Per-cell neighbour fill of a batch of periodic cells (device code shared
// by the stage fill kernels in batch.cu and the fused batch kernel, which
// builds with NVRTC: no host-only code here).
//
// The reference evaluates one box per call and handles boxes thinner than
// 2 rc by enumerating images for every pair (gpu_count_neighbors_images_on2 /
// gpu_fill_neighbors_images_on2, src/force/sus2_sh.cu:7668-7769); here each
// atom's neighbours are searched among the atoms of its own cell, with the
// candidate images filtered per axis.
#pragma once

#include "edge_args.cuh"

namespace sus2sh {
namespace batch {

// Neighbours of atom i among atoms [j0, j1) of its cell (h, reach r): every
// image within reach gets the FP64 distance test, j ascending, then tz, ty, tx
// ascending.  Writes the list and its count and flags an overflow.
__device__ __forceinline__ void fp64_image_scan(int i, int j0, int j1, const double4* __restrict__ pos4,
                                const double* __restrict__ h, int rx, int ry, int rz, double cutoff2,
                                int* __restrict__ nbr, int* __restrict__ ncount, int N, int cap, int count_only,
                                Status* st) {
  const double4 pi = pos4[i];
  int k = 0;
  for (int j = j0; j < j1; ++j) {
    const double4 pj = pos4[j];
    const double d0x = pj.x - pi.x, d0y = pj.y - pi.y, d0z = pj.z - pi.z;
    for (int tz = -rz; tz <= rz; ++tz) {
      for (int ty = -ry; ty <= ry; ++ty) {
        for (int tx = -rx; tx <= rx; ++tx) {
          if (j == i && tx == 0 && ty == 0 && tz == 0) continue;
          const double dx = d0x + tx * h[0] + ty * h[1] + tz * h[2];
          const double dy = d0y + tx * h[3] + ty * h[4] + tz * h[5];
          const double dz = d0z + tx * h[6] + ty * h[7] + tz * h[8];
          if (dx * dx + dy * dy + dz * dz < cutoff2) {
            if (!count_only && k < cap) {
              const int code = (tx + 2) * 25 + (ty + 2) * 5 + (tz + 2);
              nbr[static_cast<size_t>(k) * N + i] = j | (code << 24);
            }
            ++k;
          }
        }
      }
    }
  }
  ncount[i] = k;
  atomicMax(&st->max_count, k);
  if (k > cap && !count_only) st->overflow = 1;
}

// Atom i of a triclinic cell c: the FP64 image scan over its cell's atoms
// (orthorhombic cells are left to fill_cell_ortho).
__device__ __forceinline__ void fill_atom_triclinic(int i, int c, int N, const int* __restrict__ off,
                                                    const double4* __restrict__ pos4,
                                                    const double* __restrict__ cell_h,
                                                    const int* __restrict__ cell_reach, double cutoff2,
                                                    int* __restrict__ nbr, int* __restrict__ ncount, int cap,
                                                    int count_only, Status* st) {
  const double* h = cell_h + 9 * c;
  const bool ortho = h[1] == 0.0 && h[2] == 0.0 && h[3] == 0.0 && h[5] == 0.0 && h[6] == 0.0 && h[7] == 0.0;
  if (ortho) return;  // orthorhombic cells: fill_cell_ortho
  fp64_image_scan(i, off[c], off[c + 1], pos4, h, cell_reach[3 * c], cell_reach[3 * c + 1], cell_reach[3 * c + 2],
                  cutoff2, nbr, ncount, N, cap, count_only, st);
}

// Orthorhombic cell c, by one CTA of 128 threads (every thread calls it;
// false, with nothing done, for a triclinic or empty cell): the cell's positions are staged in
// shared memory (FP32, relative to its first atom) and every thread tests its
// atom against them.  Cells wider than twice the cutoff take the nearest image
// of each pair only (below); in narrower cells, per axis, only the images that
// can come within the cutoff are visited (computed from the displacement, at
// most `reach` each way).  An FP32 pre-test with a 1e-3 A margin admits a superset of the pairs;
// each admitted pair gets the exact FP64 test of k_batch_fill, so the lists
// (and their order: j ascending, then tz, ty, tx ascending) are the same.
// Both FP32 tests hold their margins for coordinates (relative to the cell's
// first atom) up to kCompact; a cell with an atom farther out (a long periodic
// edge, or atoms far along an open axis) takes the FP64 scan of k_batch_fill.
constexpr int kFillTile = 256;
constexpr double kCompact = 512.0;
// per-thread queue of a tile's near candidates in the wide-cell path
constexpr int kFillQueue = 96;
struct FillShared {
  float4 sp[kFillTile];
  unsigned short queue[kFillQueue][128];  // [slot][thread]: one CTA of 128 threads
};

__device__ __forceinline__ bool fill_cell_ortho(int c, int N, const int* __restrict__ off,
                                                const double4* __restrict__ pos4, const double* __restrict__ cell_h,
                                                const int* __restrict__ cell_reach, double cutoff2,
                                                int* __restrict__ nbr, int* __restrict__ ncount, int cap,
                                                int count_only, Status* st, FillShared& sh) {
  float4* const sp = sh.sp;
  unsigned short(*const s_queue)[128] = sh.queue;
  const double* h = cell_h + 9 * c;
  const bool ortho = h[1] == 0.0 && h[2] == 0.0 && h[3] == 0.0 && h[5] == 0.0 && h[6] == 0.0 && h[7] == 0.0;
  const int a0 = off[c], a1 = off[c + 1];
  if (!ortho || a1 <= a0) return false;  // uniform across the block
  const double4 o = pos4[a0];
  bool spread = false;
  for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) {
    const double4 p = pos4[a];
    spread |= !(fabs(p.x - o.x) <= kCompact && fabs(p.y - o.y) <= kCompact && fabs(p.z - o.z) <= kCompact);
  }
  if (__syncthreads_or(spread)) {  // uniform across the block
    for (int i = a0 + threadIdx.x; i < a1; i += blockDim.x)
      fp64_image_scan(i, a0, a1, pos4, h, cell_reach[3 * c], cell_reach[3 * c + 1], cell_reach[3 * c + 2], cutoff2,
                      nbr, ncount, N, cap, count_only, st);
    return true;
  }
  const float L[3] = {static_cast<float>(h[0]), static_cast<float>(h[4]), static_cast<float>(h[8])};
  const float iL[3] = {1.0f / L[0], 1.0f / L[1], 1.0f / L[2]};
  const int r[3] = {cell_reach[3 * c], cell_reach[3 * c + 1], cell_reach[3 * c + 2]};
  const float cutm = static_cast<float>(sqrt(cutoff2)) + 1.0e-3f;
  const float cutm2 = cutm * cutm;
  // Cells wider than twice the cutoff along every periodic axis: a pair has at
  // most one image within the cutoff, the nearest (positions are wrapped into
  // the cell, so it is -1, 0 or +1 cell away per axis).  Every candidate takes
  // that image by rounding and is classified in FP32: below cutoff2 - m in,
  // above cutoff2 + m out, in between the FP64 test below decides (m = 0.01 +
  // 1e-3 cutoff2 A^2, far above the FP32 rounding of these cell-local
  // coordinates).  The lists, j ascending, are the general path's.
  bool wide = true;
  for (int a = 0; a < 3; ++a)
    if (r[a] > 0 && !(L[a] > 2.0f * cutm)) wide = false;
  if (wide) {
    const float jx = r[0] > 0 ? iL[0] : 0.0f, jy = r[1] > 0 ? iL[1] : 0.0f, jz = r[2] > 0 ? iL[2] : 0.0f;
    const double margin = 0.01 + 1e-3 * cutoff2;
    const float lo2 = static_cast<float>(cutoff2 - margin), hi2 = static_cast<float>(cutoff2 + margin);
    for (int base = a0; base < a1; base += blockDim.x) {
      const int i = base + threadIdx.x;
      const bool act = i < a1;
      double4 pi = make_double4(0.0, 0.0, 0.0, 0.0);
      float fx = 0.0f, fy = 0.0f, fz = 0.0f;
      if (act) {
        pi = pos4[i];
        fx = static_cast<float>(pi.x - o.x);
        fy = static_cast<float>(pi.y - o.y);
        fz = static_cast<float>(pi.z - o.z);
      }
      int k = 0;
      for (int t0 = a0; t0 < a1; t0 += kFillTile) {
        const int tn = min(kFillTile, a1 - t0);
        __syncthreads();  // the previous tile is consumed
        for (int q = threadIdx.x; q < tn; q += blockDim.x) {
          const double4 p = pos4[t0 + q];
          sp[q] = make_float4(static_cast<float>(p.x - o.x), static_cast<float>(p.y - o.y),
                              static_cast<float>(p.z - o.z), 0.0f);
        }
        __syncthreads();
        if (!act) continue;
        // candidate q of the tile: nearest-image FP32 distance, and the full
        // test and list write for one within hi2
        auto dist2 = [&](int q, float& tx, float& ty, float& tz) {
          const float4 pj = sp[q];
          const float dx = pj.x - fx, dy = pj.y - fy, dz = pj.z - fz;
          tx = rintf(dx * jx);
          ty = rintf(dy * jy);
          tz = rintf(dz * jz);
          const float ex = fmaf(-tx, L[0], dx), ey = fmaf(-ty, L[1], dy), ez = fmaf(-tz, L[2], dz);
          return fmaf(ex, ex, fmaf(ey, ey, ez * ez));
        };
        auto accept = [&](int q, float m2, float tx, float ty, float tz) {
          const int j = t0 + q;
          const int ix = -static_cast<int>(tx), iy = -static_cast<int>(ty), iz = -static_cast<int>(tz);
          if (j == i && ix == 0 && iy == 0 && iz == 0) return;
          if (!(m2 <= lo2)) {
            const double4 pjd = pos4[j];
            const double gx = (pjd.x - pi.x) + ix * h[0] + iy * h[1] + iz * h[2];
            const double gy = (pjd.y - pi.y) + ix * h[3] + iy * h[4] + iz * h[5];
            const double gz = (pjd.z - pi.z) + ix * h[6] + iy * h[7] + iz * h[8];
            if (!(gx * gx + gy * gy + gz * gz < cutoff2)) return;
          }
          if (!count_only && k < cap) {
            const int code = (ix + 2) * 25 + (iy + 2) * 5 + (iz + 2);
            nbr[static_cast<size_t>(k) * N + i] = j | (code << 24);
          }
          ++k;
        };
        // two phases keep the lanes busy: a uniform scan queues the tile's
        // candidates within hi2 (a fifth or so), then each thread tests and
        // writes its queue; a queue that would overflow (never at physical
        // densities) is replaced by a direct pass over the tile, same order
        int nq = 0;
#pragma unroll 4
        for (int q = 0; q < tn; ++q) {
          float tx, ty, tz;
          const float m2 = dist2(q, tx, ty, tz);
          if (m2 < hi2) {  // (a NaN distance is rejected, as the FP64 test would)
            if (nq < kFillQueue) s_queue[nq][threadIdx.x] = static_cast<unsigned short>(q);
            ++nq;
          }
        }
        if (nq <= kFillQueue) {
          for (int u = 0; u < nq; ++u) {
            const int q = s_queue[u][threadIdx.x];
            float tx, ty, tz;
            const float m2 = dist2(q, tx, ty, tz);
            accept(q, m2, tx, ty, tz);
          }
        } else {
          for (int q = 0; q < tn; ++q) {
            float tx, ty, tz;
            const float m2 = dist2(q, tx, ty, tz);
            if (m2 < hi2) accept(q, m2, tx, ty, tz);
          }
        }
      }
      if (act) {
        ncount[i] = k;
        atomicMax(&st->max_count, k);
        if (k > cap && !count_only) st->overflow = 1;
      }
    }
    return true;
  }
  for (int base = a0; base < a1; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const bool act = i < a1;
    double4 pi = make_double4(0.0, 0.0, 0.0, 0.0);
    float fx = 0.0f, fy = 0.0f, fz = 0.0f;
    if (act) {
      pi = pos4[i];
      fx = static_cast<float>(pi.x - o.x);
      fy = static_cast<float>(pi.y - o.y);
      fz = static_cast<float>(pi.z - o.z);
    }
    int k = 0;
    for (int t0 = a0; t0 < a1; t0 += kFillTile) {
      const int tn = min(kFillTile, a1 - t0);
      __syncthreads();  // the previous tile is consumed
      for (int q = threadIdx.x; q < tn; q += blockDim.x) {
        const double4 p = pos4[t0 + q];
        sp[q] = make_float4(static_cast<float>(p.x - o.x), static_cast<float>(p.y - o.y),
                            static_cast<float>(p.z - o.z), 0.0f);
      }
      __syncthreads();
      if (!act) continue;
      // candidates in groups of 8: the nearest-image distances of a group are
      // independent (instruction-level parallelism); most of a large cell's
      // candidates are farther than the cutoff in every image and stop there
      for (int q0 = 0; q0 < tn; q0 += 8) {
        unsigned near = 0;
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const float4 pj = sp[min(q0 + u, tn - 1)];
          float m2 = 0.0f;
          const float d[3] = {pj.x - fx, pj.y - fy, pj.z - fz};
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            const float t = r[a] > 0 ? rintf(d[a] * iL[a]) : 0.0f;
            const float e = d[a] - t * L[a];
            m2 = fmaf(e, e, m2);
          }
          if (q0 + u < tn && m2 < cutm2) near |= 1u << u;
        }
        while (near) {
          const int u = __ffs(near) - 1;
          near &= near - 1;
          const int q = q0 + u;
          const int j = t0 + q;
          const float4 pj = sp[q];
          const float d0[3] = {pj.x - fx, pj.y - fy, pj.z - fz};
          int lo[3], hi[3];
#pragma unroll
          for (int a = 0; a < 3; ++a) {
            lo[a] = max(-r[a], static_cast<int>(ceilf((-cutm - d0[a]) * iL[a])));
            hi[a] = min(r[a], static_cast<int>(floorf((cutm - d0[a]) * iL[a])));
          }
          for (int tz = lo[2]; tz <= hi[2]; ++tz) {
            const float ez = d0[2] + tz * L[2];
            const float ez2 = ez * ez;
            if (ez2 >= cutm2) continue;
            for (int ty = lo[1]; ty <= hi[1]; ++ty) {
              const float ey = d0[1] + ty * L[1];
              const float eyz2 = ey * ey + ez2;
              if (eyz2 >= cutm2) continue;
              for (int tx = lo[0]; tx <= hi[0]; ++tx) {
                const float ex = d0[0] + tx * L[0];
                if (ex * ex + eyz2 >= cutm2) continue;
                if (j == i && tx == 0 && ty == 0 && tz == 0) continue;
                const double4 pjd = pos4[j];
                const double dx = (pjd.x - pi.x) + tx * h[0] + ty * h[1] + tz * h[2];
                const double dy = (pjd.y - pi.y) + tx * h[3] + ty * h[4] + tz * h[5];
                const double dz = (pjd.z - pi.z) + tx * h[6] + ty * h[7] + tz * h[8];
                if (dx * dx + dy * dy + dz * dz < cutoff2) {
                  if (!count_only && k < cap) {
                    const int code = (tx + 2) * 25 + (ty + 2) * 5 + (tz + 2);
                    nbr[static_cast<size_t>(k) * N + i] = j | (code << 24);
                  }
                  ++k;
                }
              }
            }
          }
        }
      }
    }
    if (act) {
      ncount[i] = k;
      atomicMax(&st->max_count, k);
      if (k > cap && !count_only) st->overflow = 1;
    }
  }
  return true;
}

}  // namespace batch
}  // namespace sus2sh
