// Parameter gradients of a loss of per-atom energies and forces.
//
// Given upstream weights a_i = dL/dE_i and b_i = dL/dF_i (3-vector per atom),
//   dL/dtheta = sum_k a_k dE_k/dtheta + sum_i b_i . dF_i/dtheta
//             = sum_k a_k dE_k/dtheta - D_b[ dE/dtheta ],
// with F_i = -dE/dr_i and D_b the directional derivative along the position
// perturbation r_i -> r_i + eps b_i (forward-over-reverse).  Moments are
// recomputed (no per-pair intermediates are stored):
//   k_pg_basic   B and its tangent Bdot = sum_j grad_d B(d_kj) . (b_j - b_k)
//   k_pg_product flat products with dual numbers: M, Mdot, adjoints g, gdot;
//                dL/dw_s = sum_k c_t (a_k M_k[s] - Mdot_k[s]);
//                writes alpha = a g - gdot and beta = g per basic
//   k_pg_radial  dL/dc[mu][n] = sum_kj sum_{b in mu} alpha_b phi_b - beta_b grad phi_b . ddot,
//                phi_b = s_pair (r - rc)^2 T_n(xi) Y_b
// The flat product pass follows the reference's simplest form
// (gpu_sh_forward_energy_backward, src/force/sus2_sh.cu:4799-4846).
#include "edge_common.cuh"
#include "engine.cuh"

namespace sus2sh {
namespace {
using namespace edge;

// First-order dual number: value and tangent.
template <typename T>
struct Dual {
  T v, d;
  __device__ __forceinline__ Dual() : v(0), d(0) {}
  __device__ __forceinline__ Dual(double c) : v(static_cast<T>(c)), d(0) {}
  __device__ __forceinline__ Dual(T a, T b) : v(a), d(b) {}
};
template <typename T>
__device__ __forceinline__ Dual<T> operator+(Dual<T> a, Dual<T> b) { return Dual<T>(a.v + b.v, a.d + b.d); }
template <typename T>
__device__ __forceinline__ Dual<T> operator-(Dual<T> a, Dual<T> b) { return Dual<T>(a.v - b.v, a.d - b.d); }
template <typename T>
__device__ __forceinline__ Dual<T> operator*(Dual<T> a, Dual<T> b) {
  return Dual<T>(a.v * b.v, fma(a.d, b.v, a.v * b.d));
}

template <typename T, int L>
__device__ __forceinline__ void harmonics_and_tangent(const Edge<T>& e, T tx, T ty, T tz, T ud, T* Y, T* Yd) {
  constexpr int C = (L + 1) * (L + 1);
  Dual<T> Q[C];
  sh_values<L>(Dual<T>(e.ux, tx), Dual<T>(e.uy, ty), Dual<T>(e.uz, tz), Q);
  // d/deps Y_lm(d + eps t) = (grad P_lm(u) . t - l Y_lm (u . t)) / r
#pragma unroll
  for (int l = 0; l <= L; ++l)
#pragma unroll
    for (int m = 0; m <= 2 * l; ++m) {
      Y[l * l + m] = Q[l * l + m].v;
      Yd[l * l + m] = (Q[l * l + m].d - T(l) * Q[l * l + m].v * ud) * e.rinv;
    }
}

// KIND: the radial basis kind (kRadialLaguerre), or -1 for the Chebyshev
// kinds read at run time.
template <typename T, int L, int K, int RB, int KIND>
__global__ void __launch_bounds__(128)
    k_pg_basic(const EdgeArgs<T> a, const double* __restrict__ fw, T* __restrict__ B, T* __restrict__ Bd) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* s_tab = reinterpret_cast<T*>(smem_raw);
  load_pair_table(a, s_tab);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  constexpr int C = (L + 1) * (L + 1), KMU = K * (L + 1), NB = K * C;
  T acc[NB], accd[NB];
#pragma unroll
  for (int b = 0; b < NB; ++b) acc[b] = accd[b] = T(0);
  const double4 pi = a.pos4[i];
  const double(*cell_shift)[3] = a.shift + (a.atom_cell ? 125 * a.atom_cell[i] : 0);
  const double bix = fw ? fw[i] : 0.0, biy = fw ? fw[i + a.N] : 0.0, biz = fw ? fw[i + 2 * a.N] : 0.0;
  const int row_i = type_of(pi) * a.rs.species;
  const int cnt = min(a.ncount[i], a.cap);
  const double rc = a.rs.rc, rc2 = rc * rc;
  for (int n = 0; n < cnt; ++n) {
    const int w = __ldg(a.nbr + static_cast<size_t>(n) * a.N + i);
    const int j = w & 0xFFFFFF;
    const double4 pj = a.pos4[j];
    double sx, sy, sz;
    image_shift(cell_shift, static_cast<unsigned>(w) >> 24, sx, sy, sz);
    const double dx = pj.x - pi.x + sx, dy = pj.y - pi.y + sy, dz = pj.z - pi.z + sz;
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 >= rc2) continue;
    const Edge<T> e = make_edge<T>(dx, dy, dz, r2, rc, rc2);
    const T tx = fw ? static_cast<T>(fw[j] - bix) : T(0);
    const T ty = fw ? static_cast<T>(fw[j + a.N] - biy) : T(0);
    const T tz = fw ? static_cast<T>(fw[j + 2 * a.N] - biz) : T(0);
    const T ud = e.ux * tx + e.uy * ty + e.uz * tz;
    const T* row = s_tab + (row_i + type_of(pj)) * a.rs.pair_stride;
    T R[KMU], dR[KMU];
    radial_values_ders<T, KMU, RB, KIND>(a, row, e, R, dR);
    T Y[C], Yd[C];
    harmonics_and_tangent<T, L>(e, tx, ty, tz, ud, Y, Yd);
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
      for (int l = 0; l <= L; ++l) {
        const T r = R[k * (L + 1) + l], rd = dR[k * (L + 1) + l] * ud;
#pragma unroll
        for (int m = 0; m <= 2 * l; ++m) {
          acc[k * C + l * l + m] = fma(r, Y[l * l + m], acc[k * C + l * l + m]);
          accd[k * C + l * l + m] = fma(rd, Y[l * l + m], fma(r, Yd[l * l + m], accd[k * C + l * l + m]));
        }
      }
  }
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    B[static_cast<size_t>(b) * a.N + i] = acc[b];
    Bd[static_cast<size_t>(b) * a.N + i] = accd[b];
  }
}

// Warp-sum then one FP64 atomic per warp.
__device__ __forceinline__ void warp_add(double* dst, double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(dst, v);
}

template <typename T>
__global__ void __launch_bounds__(128)
    k_pg_product(int N, int M, const FlatProgram p, const double4* __restrict__ pos4,
                 const double* __restrict__ species_coeffs, const double* __restrict__ ew,
                 const T* __restrict__ B, const T* __restrict__ Bd, T* __restrict__ work,
                 T* __restrict__ Galpha, T* __restrict__ Gbeta, double* __restrict__ grad_w) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = k < N;
  const int kk = active ? k : 0;
  const size_t n = static_cast<size_t>(N);
  T* Mv = work + kk;
  T* Md = work + static_cast<size_t>(M) * n + kk;
  T* gv = work + 2 * static_cast<size_t>(M) * n + kk;
  T* gd = work + 3 * static_cast<size_t>(M) * n + kk;
  double ct = 0.0, ak = 0.0;
  if (active) {
    ct = species_coeffs[type_of(pos4[k])];
    ak = ew ? ew[k] : 0.0;
    for (int m = 0; m < M; ++m) {
      Mv[m * n] = T(0);
      Md[m * n] = T(0);
      gv[m * n] = T(0);
      gd[m * n] = T(0);
    }
    for (int b = 0; b < p.nbasic; ++b) {
      const size_t c = static_cast<size_t>(p.basic_canon[b]);
      Mv[b * n] = B[c * n + k];
      Md[b * n] = Bd[c * n + k];
    }
    for (int q = 0; q < p.nprod; ++q) {
      const int l = p.left[q], r = p.right[q], t = p.target[q];
      const T c = static_cast<T>(p.coeff[q]);
      const T ml = Mv[l * n], mr = Mv[r * n];
      Mv[t * n] += c * ml * mr;
      Md[t * n] += c * (Md[l * n] * mr + ml * Md[r * n]);
    }
  }
  for (int s = 0; s < p.nscalar; ++s) {
    double contrib = 0.0;
    if (active) {
      const int m = p.scalar_map[s];
      const double w = p.scalar_w[s];
      gv[m * n] += static_cast<T>(ct * w);
      contrib = ct * (ak * static_cast<double>(Mv[m * n]) - static_cast<double>(Md[m * n]));
    }
    warp_add(grad_w + s, contrib);
  }
  if (!active) return;
  for (int q = p.nprod - 1; q >= 0; --q) {
    const int l = p.left[q], r = p.right[q], t = p.target[q];
    const T c = static_cast<T>(p.coeff[q]);
    const T gt = c * gv[t * n], gdt = c * gd[t * n];
    const T ml = Mv[l * n], mr = Mv[r * n];
    gv[l * n] += gt * mr;
    gv[r * n] += gt * ml;
    gd[l * n] += gdt * mr + gt * Md[r * n];
    gd[r * n] += gdt * ml + gt * Md[l * n];
  }
  for (int c = 0; c < p.ncanon; ++c) {
    Galpha[static_cast<size_t>(c) * n + k] = T(0);
    Gbeta[static_cast<size_t>(c) * n + k] = T(0);
  }
  const T a = static_cast<T>(ak);
  for (int b = 0; b < p.nbasic; ++b) {
    const size_t c = static_cast<size_t>(p.basic_canon[b]);
    Galpha[c * n + k] = a * gv[b * n] - gd[b * n];
    Gbeta[c * n + k] = gv[b * n];
  }
}

template <typename T, int L, int K, int RB, int KIND>
__global__ void __launch_bounds__(128)
    k_pg_radial(const EdgeArgs<T> a, const double* __restrict__ fw, const T* __restrict__ Galpha,
                const T* __restrict__ Gbeta, double* __restrict__ grad_c) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* s_tab = reinterpret_cast<T*>(smem_raw);
  load_pair_table(a, s_tab);
  constexpr int C = (L + 1) * (L + 1), KMU = K * (L + 1), NB = K * C;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = i < a.N;
  T acc[KMU * RB];
#pragma unroll
  for (int q = 0; q < KMU * RB; ++q) acc[q] = T(0);
  if (active) {
    T al[NB], be[NB];
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      al[b] = Galpha[static_cast<size_t>(b) * a.N + i];
      be[b] = Gbeta[static_cast<size_t>(b) * a.N + i];
    }
    const double4 pi = a.pos4[i];
    const double(*cell_shift)[3] = a.shift + (a.atom_cell ? 125 * a.atom_cell[i] : 0);
    const double bix = fw ? fw[i] : 0.0, biy = fw ? fw[i + a.N] : 0.0, biz = fw ? fw[i + 2 * a.N] : 0.0;
    const int row_i = type_of(pi) * a.rs.species;
    const int cnt = min(a.ncount[i], a.cap);
    const double rc = a.rs.rc, rc2 = rc * rc;
    const int kind = KIND >= 0 ? KIND : (a.rs.kind == kRadialRational ? kRadialRational : kRadialTanh);
    for (int n = 0; n < cnt; ++n) {
      const int w = __ldg(a.nbr + static_cast<size_t>(n) * a.N + i);
      const int j = w & 0xFFFFFF;
      const double4 pj = a.pos4[j];
      double sx, sy, sz;
      image_shift(cell_shift, static_cast<unsigned>(w) >> 24, sx, sy, sz);
      const double dx = pj.x - pi.x + sx, dy = pj.y - pi.y + sy, dz = pj.z - pi.z + sz;
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 >= rc2) continue;
      const Edge<T> e = make_edge<T>(dx, dy, dz, r2, rc, rc2);
      const T tx = fw ? static_cast<T>(fw[j] - bix) : T(0);
      const T ty = fw ? static_cast<T>(fw[j + a.N] - biy) : T(0);
      const T tz = fw ? static_cast<T>(fw[j + 2 * a.N] - biz) : T(0);
      const T ud = e.ux * tx + e.uy * ty + e.uz * tz;
      const T* row = s_tab + (row_i + type_of(pj)) * a.rs.pair_stride;
      const T ps = row[2 * KMU];
      const T fc = e.dr * e.dr, dfc = T(2) * e.dr;
      T Y[C], Yd[C];
      harmonics_and_tangent<T, L>(e, tx, ty, tz, ud, Y, Yd);
      // radial basis of the pair, once per edge when every mu shares (scal,
      // shift): phi_n = env P_n(x) and its r-derivative relative to fc,
      // dphi_n = (denv/env) phi_n + env (dx/dr) P_n'(x), so that the basis
      // function fc phi_n has derivative dfc phi_n + fc dphi_n
      T t0[RB], dt0[RB];
      if (a.rs.shared_xi) {
        T x, dx, env, denv;
        radial_arg<T>(kind, row[0], row[1], e.rd, x, dx, env, denv);
        radial_poly_d<RB>(kind, x, t0, dt0);
#pragma unroll
        for (int q = 0; q < RB; ++q) {
          t0[q] *= env;
          dt0[q] = fma(denv, t0[q], env * dx * dt0[q]);
        }
      }
#pragma unroll
      for (int k = 0; k < K; ++k)
#pragma unroll
        for (int l = 0; l <= L; ++l) {
          const int mu = k * (L + 1) + l;
          T A = T(0), Bm = T(0), Cm = T(0);
#pragma unroll
          for (int m = 0; m <= 2 * l; ++m) {
            A = fma(al[k * C + l * l + m], Y[l * l + m], A);
            Bm = fma(be[k * C + l * l + m], Y[l * l + m], Bm);
            Cm = fma(be[k * C + l * l + m], Yd[l * l + m], Cm);
          }
          T t[RB], dt[RB];
          if (a.rs.shared_xi) {
#pragma unroll
            for (int q = 0; q < RB; ++q) {
              t[q] = t0[q];
              dt[q] = dt0[q];
            }
          } else {
            T x, dx, env, denv;
            radial_arg<T>(kind, row[2 * mu], row[2 * mu + 1], e.rd, x, dx, env, denv);
            radial_poly_d<RB>(kind, x, t, dt);
#pragma unroll
            for (int q = 0; q < RB; ++q) {
              t[q] *= env;
              dt[q] = fma(denv, t[q], env * dx * dt[q]);
            }
          }
          const T p1 = ps * fc * (A - Cm);
          const T p2 = ps * ud * Bm;
#pragma unroll
          for (int q = 0; q < RB; ++q) acc[mu * RB + q] += p1 * t[q] - p2 * (dfc * t[q] + fc * dt[q]);
        }
    }
  }
  // warp sums -> per-warp rows in shared memory -> one FP64 atomic per
  // coefficient per CTA (the CTA has at most 4 warps)
  __shared__ double part[4][KMU * RB];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int q = 0; q < KMU * RB; ++q) {
    double v = static_cast<double>(acc[q]);
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) part[warp][q] = v;
  }
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  for (int q = threadIdx.x; q < KMU * RB; q += blockDim.x) {
    double v = 0.0;
    for (int w = 0; w < nw; ++w) v += part[w][q];
    if (v != 0.0) atomicAdd(grad_c + q, v);
  }
}

inline int blocks(int n, int b) { return (n + b - 1) / b; }

}  // namespace

#define SUS2_PG_SHAPES(X) \
  X(3, 3, 8)              \
  X(3, 3, 10)             \
  X(4, 4, 10)             \
  X(4, 4, 8)              \
  X(2, 2, 8)              \
  X(1, 1, 4)

// dL/dw_s = sum_k contrib[s][k] (the generated product kernel writes the
// per-atom terms), in two deterministic stages: kPgChunks blocks per scalar
// write partial sums, then one thread per scalar adds them in order.
constexpr int kPgChunks = 64;

template <typename T>
__global__ void __launch_bounds__(256) k_pg_reduce(int N, const T* __restrict__ contrib, double* __restrict__ partial) {
  const int s = blockIdx.y, chunk = blockIdx.x;
  const T* row = contrib + static_cast<size_t>(s) * N;
  const int per = (N + kPgChunks - 1) / kPgChunks;
  const int k0 = chunk * per, k1 = min(N, k0 + per);
  double v = 0.0;
  for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) v += static_cast<double>(row[k]);
  __shared__ double red[8];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += red[w];
    partial[static_cast<size_t>(s) * kPgChunks + chunk] = t;
  }
}

__global__ void k_pg_reduce_final(int nscalar, const double* __restrict__ partial, double* __restrict__ grad_w) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nscalar) return;
  double t = 0.0;
  for (int c = 0; c < kPgChunks; ++c) t += partial[static_cast<size_t>(s) * kPgChunks + c];
  grad_w[s] = t;
}

template <typename T>
int launch_pg_basic(cudaStream_t s, const EdgeArgs<T>& a, const double* fw, T* B, T* Bd, double* grad_c) {
  const size_t sm = sizeof(T) * static_cast<size_t>(a.rs.species) * a.rs.species * a.rs.pair_stride;
  const int grid = blocks(a.N, 128);
  cudaMemsetAsync(grad_c, 0, sizeof(double) * a.rs.kmu * a.rs.rb, s);
  bool ok = false;
#define SUS2_PG_BASIC(L, K, RB)                                                     \
  if (!ok && a.l_max == L && a.k_max == K && a.rs.rb == RB) {                       \
    if (a.rs.kind == kRadialLaguerre)                                               \
      k_pg_basic<T, L, K, RB, kRadialLaguerre><<<grid, 128, sm, s>>>(a, fw, B, Bd); \
    else                                                                            \
      k_pg_basic<T, L, K, RB, -1><<<grid, 128, sm, s>>>(a, fw, B, Bd);              \
    ok = true;                                                                      \
  }
  SUS2_PG_SHAPES(SUS2_PG_BASIC)
#undef SUS2_PG_BASIC
  return ok ? 0 : -1;
}

template <typename T>
void launch_pg_product(cudaStream_t s, int N, const FlatProgram& p, int M, const double4* pos4,
                       const double* species_coeffs, const double* ew, const T* B, const T* Bd, T* work, T* Galpha,
                       T* Gbeta, double* grad_w) {
  cudaMemsetAsync(grad_w, 0, sizeof(double) * (p.nscalar > 0 ? p.nscalar : 1), s);
  k_pg_product<T><<<blocks(N, 128), 128, 0, s>>>(N, M, p, pos4, species_coeffs, ew, B, Bd, work, Galpha, Gbeta,
                                                 grad_w);
}

template <typename T>
void launch_pg_reduce(cudaStream_t s, int nscalar, int N, const T* contrib, double* partial, double* grad_w) {
  if (nscalar <= 0) return;
  k_pg_reduce<T><<<dim3(kPgChunks, nscalar), 256, 0, s>>>(N, contrib, partial);
  k_pg_reduce_final<<<blocks(nscalar, 128), 128, 0, s>>>(nscalar, partial, grad_w);
}

template <typename T>
int launch_pg_radial(cudaStream_t s, const EdgeArgs<T>& a, const double* fw, const T* Galpha, const T* Gbeta,
                     double* grad_c) {
  const size_t sm = sizeof(T) * static_cast<size_t>(a.rs.species) * a.rs.species * a.rs.pair_stride;
  const int grid = blocks(a.N, 128);
  bool ok = false;
#define SUS2_PG_RADIAL(L, K, RB)                                                    \
  if (!ok && a.l_max == L && a.k_max == K && a.rs.rb == RB) {                       \
    if (a.rs.kind == kRadialLaguerre)                                               \
      k_pg_radial<T, L, K, RB, kRadialLaguerre><<<grid, 128, sm, s>>>(a, fw, Galpha, Gbeta, grad_c); \
    else                                                                            \
      k_pg_radial<T, L, K, RB, -1><<<grid, 128, sm, s>>>(a, fw, Galpha, Gbeta, grad_c); \
    ok = true;                                                                      \
  }
  SUS2_PG_SHAPES(SUS2_PG_RADIAL)
#undef SUS2_PG_RADIAL
  return ok ? 0 : -1;
}

#define SUS2_PG_INSTANTIATE(T)                                                                                      \
  template int launch_pg_basic<T>(cudaStream_t, const EdgeArgs<T>&, const double*, T*, T*, double*);               \
  template void launch_pg_product<T>(cudaStream_t, int, const FlatProgram&, int, const double4*, const double*,     \
                                     const double*, const T*, const T*, T*, T*, T*, double*);                        \
  template void launch_pg_reduce<T>(cudaStream_t, int, int, const T*, double*, double*);                            \
  template int launch_pg_radial<T>(cudaStream_t, const EdgeArgs<T>&, const double*, const T*, const T*, double*);
SUS2_PG_INSTANTIATE(float)
SUS2_PG_INSTANTIATE(double)
#undef SUS2_PG_INSTANTIATE

}  // namespace sus2sh
