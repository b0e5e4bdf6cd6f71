// SUS2-SH engine kernels for sm_100a.
//
// Kernel map (reference stage in brackets, src/force/sus2_sh.cu):
//   k_pack        positions -> unwrapped double4 + species, displacement max
//   k_decide      rebuild flag (skin/2 displacement rule or host-forced)
//   k_bin/k_scan_*/k_scatter/k_sort_cells/k_fill
//                 cell-list Verlet list with explicit image codes
//                 [build_neighbor_list :9547-9618, image kernels :7668-7769]
//   k_basic       B[k,l,m] = sum_j R_kl(r_ij) Y_lm(r_ij)      [gpu_sh_compute_basic :3486-3550]
//   k_product     layered CG program: forward, site energy, adjoint
//                 [gpu_sh_forward_energy_backward_compact_rows :5592-5964]
//   k_force       dE/dr_ij = sum_b g_b (R' u Y + R grad Y), F_i += dE,
//                 F_j -= dE, W_i -= r_ij (x) dE        [gpu_sh_compute_forces :6347-6446]
//   k_finalize    scatter buffer -> FP64 force          [gpu_accumulate_float_to_double :7629-7655]
// One thread owns one centre atom in the edge kernels (lane = atom), so all
// per-atom sums are private and only the F_j scatter uses atomics (one
// 128-bit vector red per edge in FP32).
#include "edge_common.cuh"
#include "edge_kernels.cuh"
#include "engine.cuh"
#include "sh_math.cuh"
#include "zbl.cuh"

#include <cstdio>

namespace sus2sh {
namespace {
using namespace edge;

// ---------------------------------------------------------------------------
// positions
// ---------------------------------------------------------------------------
__global__ void k_pack(int N, const double* __restrict__ x, const int* __restrict__ type,
                       const double4* __restrict__ ref4, double4* __restrict__ pos4,
                       const BoxGeom* __restrict__ g, int have_ref, int species, Status* st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  float d2 = 0.0f;
  if (i < N) {
    double px = x[i], py = x[i + N], pz = x[i + 2 * N];
    if (have_ref) {
      const double4 r = ref4[i];
      const double dx = px - r.x, dy = py - r.y, dz = pz - r.z;
      double s[3];
      for (int a = 0; a < 3; ++a) {
        s[a] = g->hinv[3 * a] * dx + g->hinv[3 * a + 1] * dy + g->hinv[3 * a + 2] * dz;
        s[a] = g->pbc[a] ? rint(s[a]) : 0.0;
      }
      // u = p - h * round(h^-1 (p - ref)): undo wraps applied by the caller.
      px -= g->h[0] * s[0] + g->h[1] * s[1] + g->h[2] * s[2];
      py -= g->h[3] * s[0] + g->h[4] * s[1] + g->h[5] * s[2];
      pz -= g->h[6] * s[0] + g->h[7] * s[1] + g->h[8] * s[2];
      const double ex = px - r.x, ey = py - r.y, ez = pz - r.z;
      d2 = static_cast<float>(ex * ex + ey * ey + ez * ez);
    }
    int t = type[i];
    if (t < 0 || t >= species) {  // keep every table lookup in bounds
      st->bad_type = 1;
      t = 0;
    }
    pos4[i] = make_double4(px, py, pz, __longlong_as_double(static_cast<long long>(t)));
  }
  // block max of the displacement, one atomic per block
  __shared__ float red[32];
  float v = d2;
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0f;
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0 && v > 0.0f) atomicMax(&st->maxdisp2_bits, __float_as_uint(v));
  }
}

__global__ void k_decide(Status* st, int force, float half_skin2) {
  const float d2 = __uint_as_float(st->maxdisp2_bits);
  const int need = force || (d2 > half_skin2);
  st->rebuilt = need;
  if (need) st->builds += 1;
}

// ---------------------------------------------------------------------------
// neighbour list (all kernels return immediately when no rebuild is due)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int floor_div(int a, int n) {
  return a >= 0 ? a / n : -((-a + n - 1) / n);
}

__global__ void k_bin(int N, const Status* __restrict__ st, const BoxGeom* __restrict__ g,
                      const double4* __restrict__ pos4, double4* __restrict__ ref4,
                      int* __restrict__ cell_count, int* __restrict__ atom_cell,
                      int* __restrict__ atom_rank) {
  if (!st->rebuilt) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double4 p = pos4[i];
  double s[3];
  int c[3];
  for (int a = 0; a < 3; ++a) {
    s[a] = g->hinv[3 * a] * p.x + g->hinv[3 * a + 1] * p.y + g->hinv[3 * a + 2] * p.z;
    double w = g->pbc[a] ? floor(s[a]) : 0.0;
    s[a] -= w;
    int ci = static_cast<int>(floor(s[a] * g->ncell[a]));
    ci = ci < 0 ? 0 : (ci >= g->ncell[a] ? g->ncell[a] - 1 : ci);
    c[a] = ci;
    s[a] = w;  // reuse: wrap count
  }
  const double wx = p.x - (g->h[0] * s[0] + g->h[1] * s[1] + g->h[2] * s[2]);
  const double wy = p.y - (g->h[3] * s[0] + g->h[4] * s[1] + g->h[5] * s[2]);
  const double wz = p.z - (g->h[6] * s[0] + g->h[7] * s[1] + g->h[8] * s[2]);
  ref4[i] = make_double4(wx, wy, wz, p.w);
  const int cell = (c[2] * g->ncell[1] + c[1]) * g->ncell[0] + c[0];
  atom_cell[i] = cell;
  atom_rank[i] = atomicAdd(&cell_count[cell], 1);
}

// Exclusive scan of the cell counts in three passes: per-block sums of 1024
// cells, a scan of the block sums (one block, looping when there are more
// than 1024 of them), and the per-block scans with their offsets.
constexpr int kScanTile = 1024;

__device__ __forceinline__ int block_exclusive_scan(int v, int* warp_sums, int& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < (blockDim.x >> 5) ? warp_sums[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    warp_sums[lane] = w;  // inclusive prefix of the warp sums
  }
  __syncthreads();
  total = warp_sums[(blockDim.x >> 5) - 1];
  const int before = warp > 0 ? warp_sums[warp - 1] : 0;
  __syncthreads();
  return before + x - v;
}

__global__ void __launch_bounds__(kScanTile) k_scan_sums(const Status* __restrict__ st, const int* __restrict__ cnt,
                                                         int ncells, int* __restrict__ block_sums) {
  if (!st->rebuilt) return;
  __shared__ int warp_sums[32];
  const int c = blockIdx.x * kScanTile + threadIdx.x;
  int total;
  block_exclusive_scan(c < ncells ? cnt[c] : 0, warp_sums, total);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanTile) k_scan_top(const Status* __restrict__ st, int nblocks,
                                                        int* __restrict__ block_sums) {
  if (!st->rebuilt) return;
  __shared__ int warp_sums[32];
  int carry = 0;
  for (int b0 = 0; b0 < nblocks; b0 += kScanTile) {
    const int b = b0 + threadIdx.x;
    const int v = b < nblocks ? block_sums[b] : 0;
    int total;
    const int ex = block_exclusive_scan(v, warp_sums, total);
    if (b < nblocks) block_sums[b] = carry + ex;
    carry += total;
  }
}

__global__ void __launch_bounds__(kScanTile) k_scan_apply(const Status* __restrict__ st, const int* __restrict__ cnt,
                                                          int ncells, const int* __restrict__ block_sums,
                                                          int* __restrict__ start) {
  if (!st->rebuilt) return;
  __shared__ int warp_sums[32];
  const int c = blockIdx.x * kScanTile + threadIdx.x;
  const int v = c < ncells ? cnt[c] : 0;
  int total;
  const int ex = block_exclusive_scan(v, warp_sums, total);
  const int s0 = block_sums[blockIdx.x] + ex;
  if (c < ncells) start[c] = s0;
  if (c == ncells - 1) start[ncells] = s0 + v;
}

__global__ void k_scatter(int N, const Status* __restrict__ st, const int* __restrict__ start,
                          const int* __restrict__ atom_cell, const int* __restrict__ atom_rank,
                          int* __restrict__ cell_atoms) {
  if (!st->rebuilt) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  cell_atoms[start[atom_cell[i]] + atom_rank[i]] = i;
}

// Cartesian corner h (cx/ncx, cy/ncy, cz/ncz) of cell (cx, cy, cz); for
// indices outside [0, n) it is the corner of that cell's periodic image.
__device__ __forceinline__ void cell_corner(const BoxGeom* __restrict__ g, int cx, int cy, int cz, double& ox,
                                            double& oy, double& oz) {
  const double* v = g->cellvec;
  ox = v[0] * cx + v[1] * cy + v[2] * cz;
  oy = v[3] * cx + v[4] * cy + v[5] * cz;
  oz = v[6] * cx + v[7] * cy + v[8] * cz;
}

// Largest coordinate (A) of an FP32 position relative to its cell corner, and
// of a cell-to-cell offset, for which the fill's FP32 distance test is used;
// beyond them it takes the FP64 test.
constexpr float kRelLimit = 64.0f;
constexpr double kOffLimit = 256.0;
// CTA size of the fill and its per-thread queue of one cell's near candidates
constexpr int kFillBlock = 128;
constexpr int kFillQueue = 32;

// Sort each cell's atoms by index so the neighbour order (and every FP sum)
// is deterministic, and store their positions in that order relative to the
// cell's corner in FP32 (w = 1 when a coordinate exceeds kRelLimit: such an
// atom always gets the FP64 test), so the fill reads each cell's candidates
// contiguously, 16 bytes each.
__global__ void k_sort_cells(int ncells, const Status* __restrict__ st, const BoxGeom* __restrict__ g,
                             const int* __restrict__ start, int* __restrict__ cell_atoms,
                             const double4* __restrict__ ref4, float4* __restrict__ cell_rel) {
  if (!st->rebuilt) return;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  const int b = start[c], e = start[c + 1];
  for (int a = b + 1; a < e; ++a) {
    const int v = cell_atoms[a];
    int k = a - 1;
    while (k >= b && cell_atoms[k] > v) {
      cell_atoms[k + 1] = cell_atoms[k];
      --k;
    }
    cell_atoms[k + 1] = v;
  }
  double ox, oy, oz;
  cell_corner(g, c % g->ncell[0], (c / g->ncell[0]) % g->ncell[1], c / (g->ncell[0] * g->ncell[1]), ox, oy, oz);
  for (int a = b; a < e; ++a) {
    const double4 q = ref4[cell_atoms[a]];
    const float x = static_cast<float>(q.x - ox), y = static_cast<float>(q.y - oy), z = static_cast<float>(q.z - oz);
    const bool far = !(fabsf(x) <= kRelLimit && fabsf(y) <= kRelLimit && fabsf(z) <= kRelLimit);
    cell_rel[a] = make_float4(x, y, z, far ? 1.0f : 0.0f);
  }
}

// Candidates are classified by an FP32 distance between cell-relative
// positions (cell_rel) plus the FP64 cell-to-cell offset h (ox/ncx, oy/ncy,
// oz/ncz) rounded to FP32: below cutoff2 - margin they are in, above
// cutoff2 + margin out, and in between (or for atoms or offsets beyond the FP32
// limits) the FP64 test on the full positions decides, exactly as the
// distance test of the list has always been taken.  The margin is many times
// the FP32 rounding bound of these short coordinates, so the list (and its
// order) is the one the FP64 test alone gives.  An accepted candidate's
// index is loaded only then.
__global__ void k_fill(int N, Status* __restrict__ st, const BoxGeom* __restrict__ g,
                       double cutoff2, const double4* __restrict__ ref4,
                       const int* __restrict__ start, const int* __restrict__ cell_atoms,
                       const float4* __restrict__ cell_rel, const int* __restrict__ atom_cell,
                       int* __restrict__ nbr, int* __restrict__ ncount, double4* __restrict__ pos4, int cap,
                       int count_only) {
  if (!st->rebuilt) return;
  // offsets of the (image) corners of the scanned cells from the home corner,
  // cellvec (ox, oy, oz) in FP32 (w = 1 beyond kOffLimit), once per CTA
  __shared__ float4 s_off[125];
  __shared__ unsigned short s_queue[kFillQueue][kFillBlock];  // [slot][thread]
  const int rx = g->reach[0], ry = g->reach[1], rz = g->reach[2];
  const int wx = 2 * rx + 1, wy = 2 * ry + 1;
  for (int t = threadIdx.x; t < wx * wy * (2 * rz + 1); t += blockDim.x) {
    double x, y, z;
    cell_corner(g, t % wx - rx, (t / wx) % wy - ry, t / (wx * wy) - rz, x, y, z);
    const bool far = !(fabs(x) <= kOffLimit && fabs(y) <= kOffLimit && fabs(z) <= kOffLimit);
    s_off[t] = make_float4(static_cast<float>(x), static_cast<float>(y), static_cast<float>(z), far ? 1.0f : 0.0f);
  }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double4 p = ref4[i];
  const int cell = atom_cell[i];
  const int cx = cell % g->ncell[0];
  const int cy = (cell / g->ncell[0]) % g->ncell[1];
  const int cz = cell / (g->ncell[0] * g->ncell[1]);
  double hx, hy, hz;
  cell_corner(g, cx, cy, cz, hx, hy, hz);
  const float px = static_cast<float>(p.x - hx), py = static_cast<float>(p.y - hy), pz = static_cast<float>(p.z - hz);
  const bool far_i = !(fabsf(px) <= kRelLimit && fabsf(py) <= kRelLimit && fabsf(pz) <= kRelLimit);
  const double margin = 0.01 + 1e-3 * cutoff2;
  const float lo = static_cast<float>(cutoff2 - margin), hi = static_cast<float>(cutoff2 + margin);
  int k = 0;
  for (int oz = -g->reach[2]; oz <= g->reach[2]; ++oz) {
    int nz = cz + oz, tz = 0;
    if (g->pbc[2]) {
      tz = floor_div(nz, g->ncell[2]);
      nz -= tz * g->ncell[2];
    } else if (nz < 0 || nz >= g->ncell[2]) {
      continue;
    }
    for (int oy = -g->reach[1]; oy <= g->reach[1]; ++oy) {
      int ny = cy + oy, ty = 0;
      if (g->pbc[1]) {
        ty = floor_div(ny, g->ncell[1]);
        ny -= ty * g->ncell[1];
      } else if (ny < 0 || ny >= g->ncell[1]) {
        continue;
      }
      for (int ox = -g->reach[0]; ox <= g->reach[0]; ++ox) {
        int nx = cx + ox, tx = 0;
        if (g->pbc[0]) {
          tx = floor_div(nx, g->ncell[0]);
          nx -= tx * g->ncell[0];
        } else if (nx < 0 || nx >= g->ncell[0]) {
          continue;
        }
        const int code = (tx + 2) * 25 + (ty + 2) * 5 + (tz + 2);
        const double sx = g->shift[code][0], sy = g->shift[code][1], sz = g->shift[code][2];
        const int nc = (nz * g->ncell[1] + ny) * g->ncell[0] + nx;
        const int a1 = start[nc + 1];
        const float4 off = s_off[((oz + rz) * wy + (oy + ry)) * wx + (ox + rx)];
        const bool exact_cell = far_i || off.w != 0.0f;
        const float fx = off.x - px, fy = off.y - py, fz = off.z - pz;
        const int a0 = start[nc];
        // candidate a: FP32 distance, and whether it needs the FP64 test
        auto dist2 = [&](int a, bool& exact) {
          const float4 q = cell_rel[a];
          const float dx = q.x + fx, dy = q.y + fy, dz = q.z + fz;
          exact = exact_cell || q.w != 0.0f;
          return dx * dx + dy * dy + dz * dz;
        };
        auto accept = [&](int a, float d2, bool exact) {
          const int j = cell_atoms[a];
          if (j == i && code == kCenterCode) return;
          if (exact || !(d2 <= lo)) {
            const double4 qq = ref4[j];
            const double ex = qq.x - p.x + sx, ey = qq.y - p.y + sy, ez = qq.z - p.z + sz;
            if (!(ex * ex + ey * ey + ez * ez < cutoff2)) return;
          }
          if (!count_only && k < cap) nbr[static_cast<size_t>(k) * N + i] = j | (code << 24);
          ++k;
        };
        // a uniform scan queues the cell's candidates that may be in (about
        // one in seven), then the accept work runs over the queue, so lanes do
        // not idle on it; a queue that would overflow is replaced by a direct
        // pass over the cell (same order)
        int nq = 0;
        for (int a = a0; a < a1; ++a) {
          bool exact;
          const float d2 = dist2(a, exact);
          if (exact || d2 < hi) {  // (a NaN distance is rejected, as the FP64 test would)
            if (nq < kFillQueue) s_queue[nq][threadIdx.x] = static_cast<unsigned short>(a - a0);
            ++nq;
          }
        }
        if (nq <= kFillQueue && a1 - a0 <= 65535) {
          for (int u = 0; u < nq; ++u) {
            const int a = a0 + s_queue[u][threadIdx.x];
            bool exact;
            const float d2 = dist2(a, exact);
            accept(a, d2, exact);
          }
        } else {
          for (int a = a0; a < a1; ++a) {
            bool exact;
            const float d2 = dist2(a, exact);
            if (exact || d2 < hi) accept(a, d2, exact);
          }
        }
      }
    }
  }
  ncount[i] = k;
  atomicMax(&st->max_count, k);
  if (k > cap && !count_only) st->overflow = 1;
  if (!count_only) pos4[i] = p;
}

// Inner list: the listed pairs within rc + margin, in list order, for the
// basic-moment kernel.  Rebuilt at every full build and on every call whose
// largest displacement since that build exceeds margin / 2 (so it holds every
// pair within rc); otherwise it returns at once.
__global__ void k_inner(int N, const Status* __restrict__ st, float half_margin2, double inner2,
                        const double4* __restrict__ pos4, const int* __restrict__ nbr,
                        const int* __restrict__ ncount, int cap, const BoxGeom* __restrict__ g,
                        int* __restrict__ inner_nbr, int* __restrict__ inner_count) {
  if (!st->rebuilt && !(__uint_as_float(st->maxdisp2_bits) > half_margin2)) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double4 pi = pos4[i];
  const int cnt = min(ncount[i], cap);
  int k = 0;
  for (int n = 0; n < cnt; ++n) {
    const int w = __ldg(nbr + static_cast<size_t>(n) * N + i);
    const double4 pj = pos4[w & 0xFFFFFF];
    double sx, sy, sz;
    image_shift(g->shift, static_cast<unsigned>(w) >> 24, sx, sy, sz);
    const double dx = pj.x - pi.x + sx, dy = pj.y - pi.y + sy, dz = pj.z - pi.z + sz;
    if (dx * dx + dy * dy + dz * dz < inner2) inner_nbr[static_cast<size_t>(k++) * N + i] = w;
  }
  inner_count[i] = k;
}

template <typename T>
__global__ void k_finalize(int N, const void* __restrict__ ftmp, double* __restrict__ force,
                           double sign);
template <>
__global__ void k_finalize<float>(int N, const void* __restrict__ ftmp, double* __restrict__ force,
                                  double sign) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const float4 v = reinterpret_cast<const float4*>(ftmp)[i];
  force[i] += sign * static_cast<double>(v.x);
  force[i + N] += sign * static_cast<double>(v.y);
  force[i + 2 * N] += sign * static_cast<double>(v.z);
}
template <>
__global__ void k_finalize<double>(int N, const void* __restrict__ ftmp, double* __restrict__ force,
                                   double sign) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double4 v = reinterpret_cast<const double4*>(ftmp)[i];
  force[i] += sign * v.x;
  force[i + N] += sign * v.y;
  force[i + 2 * N] += sign * v.z;
}

// ---------------------------------------------------------------------------
// CG product program (lane = atom).  Row header: kind(2) | nterms(14) | dst(16);
// term word: a(16) | b(16).  Kinds:
//   0 FWD   V[dst]  = sum c V[a] V[b]
//   1 TERM  E += sum c V[a] V[b]; G[a] += c V[b]; G[b] += c V[a]
//           (terminal scalar row, c premultiplied by its moment weight)
//   2 SEED  E += c V[a]; G[a] += c              (non-terminal scalar)
//   3 BACK  G[dst] += sum c G[a] V[b]           (a = consumer target slot)
// G[v] lives at slot v + nvalue.
// ---------------------------------------------------------------------------
template <typename T, bool kShared>
__global__ void __launch_bounds__(128)
    k_product(int N, const ProgramDev p, const double4* __restrict__ pos4, const T* __restrict__ B,
              T* __restrict__ G, T* __restrict__ scratch, const double* __restrict__ shift_coeffs,
              const double* __restrict__ species_coeffs, double* __restrict__ pe, int pe_assign) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int atom = blockIdx.x * blockDim.x + threadIdx.x;
  if (atom >= N) return;
  T* S;
  size_t stride;
  if (kShared) {
    S = reinterpret_cast<T*>(smem_raw) + threadIdx.x;
    stride = blockDim.x;
  } else {
    S = scratch + atom;
    stride = static_cast<size_t>(N);
  }
  const int gofs = p.nvalue;
  for (int b = 0; b < p.nbasic; ++b)
    S[b * stride] = B[static_cast<size_t>(__ldg(p.basic_canon + b)) * N + atom];
  for (int v = 0; v < p.nvalue; ++v) S[(gofs + v) * stride] = T(0);
  const uint32_t* __restrict__ code = p.code;
  const T* __restrict__ cf = reinterpret_cast<const T*>(p.coef);
  double E = 0.0;
  for (int r = 0; r < p.nrows; ++r) {
    const uint32_t h = __ldg(code++);
    const int kind = h >> 30;
    const int nt = (h >> 16) & 0x3FFF;
    const int dst = h & 0xFFFF;
    if (kind == 0) {
      T acc = T(0);
      for (int t = 0; t < nt; ++t) {
        const uint32_t w = __ldg(code + t);
        acc = fma(__ldg(cf + t) * S[(w & 0xFFFF) * stride], S[(w >> 16) * stride], acc);
      }
      S[dst * stride] = acc;
    } else if (kind == 1) {
      T acc = T(0);
      for (int t = 0; t < nt; ++t) {
        const uint32_t w = __ldg(code + t);
        const int ia = w & 0xFFFF, ib = w >> 16;
        const T c = __ldg(cf + t);
        const T va = S[ia * stride], vb = S[ib * stride];
        acc = fma(c * va, vb, acc);
        S[(gofs + ia) * stride] += c * vb;
        S[(gofs + ib) * stride] += c * va;
      }
      E += static_cast<double>(acc);
    } else if (kind == 2) {
      const uint32_t w = __ldg(code);
      const int ia = w & 0xFFFF;
      const T c = __ldg(cf);
      E += static_cast<double>(c * S[ia * stride]);
      S[(gofs + ia) * stride] += c;
    } else {
      T acc = T(0);
      for (int t = 0; t < nt; ++t) {
        const uint32_t w = __ldg(code + t);
        acc = fma(__ldg(cf + t) * S[(gofs + (w & 0xFFFF)) * stride], S[(w >> 16) * stride], acc);
      }
      S[(gofs + dst) * stride] += acc;
    }
    code += nt;
    cf += nt;
  }
  const int ti = type_of(pos4[atom]);
  const double ct = species_coeffs[ti];
  const double site = shift_coeffs[ti] + ct + ct * E;
  if (pe) pe[atom] = pe_assign ? site : pe[atom] + site;
  const T sc = static_cast<T>(ct);
  for (int c = 0; c < p.ncanon; ++c) {
    const int b = __ldg(p.canon_basic + c);
    G[static_cast<size_t>(c) * N + atom] = b >= 0 ? sc * S[(gofs + b) * stride] : T(0);
  }
}

// ---------------------------------------------------------------------------
// ZBL pair term (gpu_sh_apply_zbl, src/force/sus2_sh.cu:7522-7627): half of
// each pair energy on each end of the full list, FP64 throughout.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128)
    k_zbl(int mode, int N, int cap, const double4* __restrict__ pos4, const int* __restrict__ nbr,
          const int* __restrict__ ncount, const double (*__restrict__ shift)[3], const int* __restrict__ atom_cell,
          const ZblTables z, const double* __restrict__ weight, double* __restrict__ pe, double* __restrict__ force,
          double* __restrict__ virial, double sign) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double4 pi = pos4[i];
  const double(*cell_shift)[3] = shift + (atom_cell ? 125 * atom_cell[i] : 0);
  const int ti = type_of(pi);
  const int zi = z.z[ti];
  const int cnt = min(ncount[i], cap);
  const double wi = weight ? weight[i] : 1.0;
  double e = 0.0, fx = 0.0, fy = 0.0, fz = 0.0;
  double w[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int n = 0; n < cnt; ++n) {
    const int word = __ldg(nbr + static_cast<size_t>(n) * N + i);
    const int j = word & 0xFFFFFF;
    const double4 pj = pos4[j];
    double sx, sy, sz;
    image_shift(cell_shift, static_cast<unsigned>(word) >> 24, sx, sy, sz);
    const double dx = pj.x - pi.x + sx, dy = pj.y - pi.y + sy, dz = pj.z - pi.z + sz;
    const double r2 = dx * dx + dy * dy + dz * dz;
    const int pair = ti * z.species + type_of(pj);
    const double outer = z.outer[pair];
    if (r2 <= 0.0 || r2 >= outer * outer) continue;
    const double r = sqrt(r2);
    const zbl::PairValue v = zbl::pair(zi, z.z[type_of(pj)], r, z.inner[pair], outer);
    if (v.energy == 0.0 && v.dEdr == 0.0) continue;
    if (mode == 0) {
      e += 0.5 * v.energy;
      continue;
    }
    const double sc = 0.5 * v.dEdr / r * wi;
    const double ex = sc * dx, ey = sc * dy, ez = sc * dz;
    fx += ex;
    fy += ey;
    fz += ez;
    atomicAdd(force + j, -sign * ex);
    atomicAdd(force + j + N, -sign * ey);
    atomicAdd(force + j + 2 * N, -sign * ez);
    w[0] -= dx * ex; w[1] -= dy * ey; w[2] -= dz * ez;
    w[3] -= dx * ey; w[4] -= dx * ez; w[5] -= dy * ez;
    w[6] -= dy * ex; w[7] -= dz * ex; w[8] -= dz * ey;
  }
  if (mode == 0) {
    pe[i] += e;
    return;
  }
  atomicAdd(force + i, sign * fx);
  atomicAdd(force + i + N, sign * fy);
  atomicAdd(force + i + 2 * N, sign * fz);
  if (virial)
    for (int q = 0; q < 9; ++q) virial[static_cast<size_t>(q) * N + i] += w[q];
}

// Sum of per-atom energy (out[0]) and virial (out[1..9]); one FP64 atomic
// per block and component.
__global__ void k_reduce(int N, const double* __restrict__ pe, const double* __restrict__ vir,
                         double* __restrict__ out) {
  __shared__ double red[10][8];
  double v[10];
  for (int q = 0; q < 10; ++q) v[q] = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
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
    atomicAdd(out + threadIdx.x, x);
  }
}

inline int blocks_for(int n, int b) { return (n + b - 1) / b; }

}  // namespace

void launch_reduce(cudaStream_t s, int N, const double* pe, const double* virial, double* out) {
  cudaMemsetAsync(out, 0, 10 * sizeof(double), s);
  int grid = blocks_for(N, 256);
  if (grid > 592) grid = 592;
  if (grid < 1) grid = 1;
  k_reduce<<<grid, 256, 0, s>>>(N, pe, virial, out);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
void launch_pack(cudaStream_t s, int N, const double* x, const int* type, const double4* ref4,
                 double4* pos4, const BoxGeom* geom_dev, int have_ref, int species, Status* st) {
  k_pack<<<blocks_for(N, 256), 256, 0, s>>>(N, x, type, ref4, pos4, geom_dev, have_ref, species, st);
}

void launch_decide(cudaStream_t s, Status* st, int force, float half_skin2) {
  k_decide<<<1, 1, 0, s>>>(st, force, half_skin2);
}

void launch_build(cudaStream_t s, int N, int force, float half_skin2, double cutoff2, const BoxGeom& g,
                  const BoxGeom* geom_dev, double4* pos4, double4* ref4, int* cell_count, int* cell_start,
                  int* cell_atoms, float4* cell_rel, int* atom_cell, int* atom_rank, int ncells, int* nbr,
                  int* ncount, int cap, int count_only, Status* st) {
  (void)g;
  launch_decide(s, st, force, half_skin2);
  launch_rebuild(s, N, cutoff2, geom_dev, pos4, ref4, cell_count, cell_start, cell_atoms, cell_rel, atom_cell,
                 atom_rank, ncells, nbr, ncount, cap, count_only, st);
}

void launch_rebuild(cudaStream_t s, int N, double cutoff2, const BoxGeom* geom_dev, double4* pos4, double4* ref4,
                    int* cell_count, int* cell_start, int* cell_atoms, float4* cell_rel, int* atom_cell,
                    int* atom_rank, int ncells, int* nbr, int* ncount, int cap, int count_only, Status* st) {
  cudaMemsetAsync(cell_count, 0, sizeof(int) * (ncells + 1), s);
  k_bin<<<blocks_for(N, 256), 256, 0, s>>>(N, st, geom_dev, pos4, ref4, cell_count, atom_cell, atom_rank);
  // block sums live in the spare tail of cell_count (sized by the caller)
  const int nblocks = blocks_for(ncells, kScanTile);
  int* block_sums = cell_count + ncells + 1;
  k_scan_sums<<<nblocks, kScanTile, 0, s>>>(st, cell_count, ncells, block_sums);
  k_scan_top<<<1, kScanTile, 0, s>>>(st, nblocks, block_sums);
  k_scan_apply<<<nblocks, kScanTile, 0, s>>>(st, cell_count, ncells, block_sums, cell_start);
  k_scatter<<<blocks_for(N, 256), 256, 0, s>>>(N, st, cell_start, atom_cell, atom_rank, cell_atoms);
  k_sort_cells<<<blocks_for(ncells, 128), 128, 0, s>>>(ncells, st, geom_dev, cell_start, cell_atoms, ref4, cell_rel);
  k_fill<<<blocks_for(N, kFillBlock), kFillBlock, 0, s>>>(N, st, geom_dev, cutoff2, ref4, cell_start, cell_atoms,
                                                           cell_rel, atom_cell, nbr, ncount, pos4, cap, count_only);
}

// The IF conditions of the neighbour graph, from k_decide's decision: a build,
// and a refresh of the inner list (at a build, or once an atom has moved more
// than half the inner margin since it).
__global__ void k_cond(const Status* __restrict__ st, float half_margin2, int use_inner,
                       cudaGraphConditionalHandle build, cudaGraphConditionalHandle inner) {
  const int b = st->rebuilt;
  cudaGraphSetConditional(build, b ? 1u : 0u);
  const bool refresh = use_inner && (b || __uint_as_float(st->maxdisp2_bits) > half_margin2);
  cudaGraphSetConditional(inner, refresh ? 1u : 0u);
}

cudaError_t build_neighbor_graph(cudaStream_t capture, const NeighborGraphArgs& g, cudaGraph_t* graph_out,
                                 cudaGraphExec_t* exec_out) {
  *graph_out = nullptr;
  *exec_out = nullptr;
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaGraphCreate(&graph, 0);
  if (e != cudaSuccess) return e;
  auto fail = [&](cudaError_t err) {
    cudaGraphDestroy(graph);
    return err;
  };
  cudaGraphConditionalHandle hb, hi;
  if ((e = cudaGraphConditionalHandleCreate(&hb, graph, 0, cudaGraphCondAssignDefault)) != cudaSuccess) return fail(e);
  if ((e = cudaGraphConditionalHandleCreate(&hi, graph, 0, cudaGraphCondAssignDefault)) != cudaSuccess) return fail(e);
  // k_cond
  const Status* st = g.st;
  float half_margin2 = g.half_margin2;
  int use_inner = g.use_inner;
  void* cond_args[] = {&st, &half_margin2, &use_inner, &hb, &hi};
  cudaKernelNodeParams kp = {};
  kp.func = reinterpret_cast<void*>(k_cond);
  kp.gridDim = dim3(1);
  kp.blockDim = dim3(1);
  kp.kernelParams = cond_args;
  cudaGraphNode_t ncond;
  if ((e = cudaGraphAddKernelNode(&ncond, graph, nullptr, 0, &kp)) != cudaSuccess) return fail(e);
  // IF build: the rebuild kernels, captured into the body graph
  cudaGraphNodeParams cb = {};
  cb.type = cudaGraphNodeTypeConditional;
  cb.conditional.handle = hb;
  cb.conditional.type = cudaGraphCondTypeIf;
  cb.conditional.size = 1;
  cudaGraphNode_t nbuild;
  if ((e = cudaGraphAddNode(&nbuild, graph, &ncond, 1, &cb)) != cudaSuccess) return fail(e);
  cudaGraph_t body = cb.conditional.phGraph_out[0];
  if ((e = cudaStreamBeginCaptureToGraph(capture, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed)) !=
      cudaSuccess)
    return fail(e);
  launch_rebuild(capture, g.N, g.cutoff2, g.geom, g.pos4, g.ref4, g.cell_count, g.cell_start, g.cell_atoms,
                 g.cell_rel, g.atom_cell, g.atom_rank, g.ncells, g.nbr, g.ncount, g.cap, 0, g.st);
  if ((e = cudaStreamEndCapture(capture, &body)) != cudaSuccess) return fail(e);
  // IF inner refresh: k_inner
  cudaGraphNodeParams ci = {};
  ci.type = cudaGraphNodeTypeConditional;
  ci.conditional.handle = hi;
  ci.conditional.type = cudaGraphCondTypeIf;
  ci.conditional.size = 1;
  cudaGraphNode_t ninner;
  if ((e = cudaGraphAddNode(&ninner, graph, &nbuild, 1, &ci)) != cudaSuccess) return fail(e);
  cudaGraph_t ibody = ci.conditional.phGraph_out[0];
  if ((e = cudaStreamBeginCaptureToGraph(capture, ibody, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed)) !=
      cudaSuccess)
    return fail(e);
  if (g.use_inner)
    launch_inner(capture, g.N, g.st, g.half_margin2, g.inner2, g.pos4, g.nbr, g.ncount, g.cap, g.geom, g.inner_nbr,
                 g.inner_count);
  if ((e = cudaStreamEndCapture(capture, &ibody)) != cudaSuccess) return fail(e);
  cudaGraphExec_t exec = nullptr;
  if ((e = cudaGraphInstantiate(&exec, graph, 0)) != cudaSuccess) return fail(e);
  *graph_out = graph;
  *exec_out = exec;
  return cudaSuccess;
}

void launch_inner(cudaStream_t s, int N, const Status* st, float half_margin2, double inner2, const double4* pos4,
                  const int* nbr, const int* ncount, int cap, const BoxGeom* geom_dev, int* inner_nbr,
                  int* inner_count) {
  k_inner<<<blocks_for(N, 128), 128, 0, s>>>(N, st, half_margin2, inner2, pos4, nbr, ncount, cap, geom_dev,
                                              inner_nbr, inner_count);
}

// Compiled (L, K, RB) shapes of the edge kernels.
#define SUS2_SHAPES(X) \
  X(3, 3, 8)           \
  X(3, 3, 10)          \
  X(4, 4, 10)          \
  X(4, 4, 8)           \
  X(2, 2, 8)           \
  X(1, 1, 4)

bool shape_supported(int l_max, int k_max, int rb) {
#define SUS2_CHECK(L, K, RB) \
  if (l_max == L && k_max == K && rb == RB) return true;
  SUS2_SHAPES(SUS2_CHECK)
#undef SUS2_CHECK
  return false;
}

template <typename T>
static size_t pair_smem(const EdgeArgs<T>& a) {
  return sizeof(T) * static_cast<size_t>(a.rs.species) * a.rs.species * a.rs.pair_stride;
}

// CTA sizes the tile autotuner may choose for the FP32 edge kernels (the FP64
// engine always uses 128).
bool block_supported(int block, bool fp32) { return block == 128 || (fp32 && (block == 64 || block == 256)); }

// Opts a kernel into more than 48 KB of dynamic shared memory (large species
// counts with many radial functions) once per kernel.
template <typename K>
void allow_smem(K kernel, size_t bytes) {
  if (bytes > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
}

template <typename T, int L, int K, int RB>
int launch_basic_shape(cudaStream_t s, const EdgeArgs<T>& a, T* B, int block, bool gate) {
  const size_t sm = pair_smem(a);
  if (gate) {  // gate models: 128-thread CTAs only
    allow_smem(k_basic<T, L, K, RB, 128, true>, sm);
    k_basic<T, L, K, RB, 128, true><<<blocks_for(a.N, 128), 128, sm, s>>>(a, B);
    return 0;
  }
  allow_smem(k_basic<T, L, K, RB, 64>, sm);
  allow_smem(k_basic<T, L, K, RB, 128>, sm);
  allow_smem(k_basic<T, L, K, RB, 256>, sm);
  if (sizeof(T) == 4 && block == 64) {
    k_basic<T, L, K, RB, 64><<<blocks_for(a.N, 64), 64, sm, s>>>(a, B);
  } else if (sizeof(T) == 4 && block == 256) {
    k_basic<T, L, K, RB, 256><<<blocks_for(a.N, 256), 256, sm, s>>>(a, B);
  } else {
    k_basic<T, L, K, RB, 128><<<blocks_for(a.N, 128), 128, sm, s>>>(a, B);
  }
  return 0;
}

template <typename T, int L, int K, int RB>
int launch_force_shape(cudaStream_t s, const EdgeArgs<T>& a, const T* G, const double* weight, void* ftmp,
                       double* force, double* virial, double sign, int block, bool gate) {
  const size_t sm = pair_smem(a);
  if (gate) {
    allow_smem(k_force<T, L, K, RB, 128, true>, sm);
    k_force<T, L, K, RB, 128, true><<<blocks_for(a.N, 128), 128, sm, s>>>(a, G, weight, ftmp, force, virial, sign);
    return 0;
  }
  allow_smem(k_force<T, L, K, RB, 64>, sm);
  allow_smem(k_force<T, L, K, RB, 128>, sm);
  allow_smem(k_force<T, L, K, RB, 256>, sm);
  if (sizeof(T) == 4 && block == 64) {
    k_force<T, L, K, RB, 64><<<blocks_for(a.N, 64), 64, sm, s>>>(a, G, weight, ftmp, force, virial, sign);
  } else if (sizeof(T) == 4 && block == 256) {
    k_force<T, L, K, RB, 256><<<blocks_for(a.N, 256), 256, sm, s>>>(a, G, weight, ftmp, force, virial, sign);
  } else {
    k_force<T, L, K, RB, 128><<<blocks_for(a.N, 128), 128, sm, s>>>(a, G, weight, ftmp, force, virial, sign);
  }
  return 0;
}

template <typename T>
int launch_basic(cudaStream_t s, const EdgeArgs<T>& a, T* B, int block, bool gate) {
#define SUS2_BASIC(L, K, RB) \
  if (a.l_max == L && a.k_max == K && a.rs.rb == RB) return launch_basic_shape<T, L, K, RB>(s, a, B, block, gate);
  SUS2_SHAPES(SUS2_BASIC)
#undef SUS2_BASIC
  return -1;
}

template <typename T>
int launch_force(cudaStream_t s, const EdgeArgs<T>& a, const T* G, const double* weight, void* ftmp,
                 double* force, double* virial, double sign, int block, bool gate) {
#define SUS2_FORCE(L, K, RB)                                                                         \
  if (a.l_max == L && a.k_max == K && a.rs.rb == RB)                                                 \
    return launch_force_shape<T, L, K, RB>(s, a, G, weight, ftmp, force, virial, sign, block, gate);
  SUS2_SHAPES(SUS2_FORCE)
#undef SUS2_FORCE
  return -1;
}

template <typename T>
void launch_product(cudaStream_t s, int N, const ProgramDev& p, const double4* pos4, const T* B, T* G,
                    T* scratch, size_t smem_tile_bytes, int tile, const double* shift_coeffs,
                    const double* species_coeffs, double* pe, int pe_assign) {
  if (scratch == nullptr) {
    static bool configured[2] = {false, false};
    const int which = sizeof(T) == 8;
    if (!configured[which]) {
      cudaFuncSetAttribute(k_product<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
      configured[which] = true;
    }
    k_product<T, true><<<blocks_for(N, tile), tile, smem_tile_bytes, s>>>(
        N, p, pos4, B, G, nullptr, shift_coeffs, species_coeffs, pe, pe_assign);
  } else {
    k_product<T, false><<<blocks_for(N, 128), 128, 0, s>>>(N, p, pos4, B, G, scratch, shift_coeffs,
                                                           species_coeffs, pe, pe_assign);
  }
}

template <typename T>
void launch_finalize(cudaStream_t s, int N, const void* ftmp, double* force, double sign) {
  k_finalize<T><<<blocks_for(N, 256), 256, 0, s>>>(N, ftmp, force, sign);
}


void launch_zbl(cudaStream_t s, int mode, int N, int cap, const double4* pos4, const int* nbr, const int* ncount,
                const double (*shift)[3], const int* atom_cell, const ZblTables& z, const double* weight,
                double* pe, double* force, double* virial, double sign) {
  k_zbl<<<blocks_for(N, 128), 128, 0, s>>>(mode, N, cap, pos4, nbr, ncount, shift, atom_cell, z, weight, pe, force,
                                           virial, sign);
}

template int launch_basic<float>(cudaStream_t, const EdgeArgs<float>&, float*, int, bool);
template int launch_basic<double>(cudaStream_t, const EdgeArgs<double>&, double*, int, bool);
template int launch_force<float>(cudaStream_t, const EdgeArgs<float>&, const float*, const double*, void*,
                                 double*, double*, double, int, bool);
template int launch_force<double>(cudaStream_t, const EdgeArgs<double>&, const double*, const double*, void*,
                                  double*, double*, double, int, bool);
template void launch_product<float>(cudaStream_t, int, const ProgramDev&, const double4*, const float*, float*,
                                    float*, size_t, int, const double*, const double*, double*, int);
template void launch_product<double>(cudaStream_t, int, const ProgramDev&, const double4*, const double*,
                                     double*, double*, size_t, int, const double*, const double*, double*, int);
template void launch_finalize<float>(cudaStream_t, int, const void*, double*, double);
template void launch_finalize<double>(cudaStream_t, int, const void*, double*, double);

}  // namespace sus2sh
