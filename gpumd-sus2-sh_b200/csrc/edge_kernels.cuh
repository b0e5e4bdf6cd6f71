// Per-edge kernels of the SUS2-SH engine, one template per model shape
// (working precision T, sh_l_max L, sh_k_max K, radial_basis_size RB, CTA
// size BLOCK).  Shapes listed in engine.cu are compiled ahead of time; any
// other shape the model format allows is compiled from this same header with
// NVRTC when the model is loaded (edge_jit.cpp), so this file and the headers
// it includes stay free of host-only code.
//
//   k_basic  B[k,l,m](i) = sum_j R_kl(r_ij) Y_lm(r_ij)   [gpu_sh_compute_basic, src/force/sus2_sh.cu:3486-3550]
//   k_force  dE/dr_ij = sum_b g_b (R' u Y + R grad Y); F_i += dE, F_j -= dE,
//            W_i -= r_ij (x) dE                         [gpu_sh_compute_forces, :6347-6446]
// One thread owns one centre atom (lane = atom), so all per-atom sums are
// private and only the F_j scatter uses atomics (one 128-bit vector red per
// edge in FP32).
#pragma once

#include "edge_common.cuh"
#include "sh_math.cuh"

// Minimum resident CTAs per SM of the FP32 edge kernels (register caps, for
// shapes with at most 64 basic moments).  Measured on the 1.024M-atom l3k3
// workload: k_force at 4 CTAs (128 registers, 32 B spill) runs 1.38 ms vs
// 1.54 ms at 3 CTAs; k_basic at 4 CTAs 0.71 ms vs 0.75 ms at its natural 140
// registers.
#ifndef SUS2_BASIC_MIN_BLOCKS
#define SUS2_BASIC_MIN_BLOCKS 4
#endif
#ifndef SUS2_FORCE_MIN_BLOCKS
#define SUS2_FORCE_MIN_BLOCKS 4
#endif
namespace sus2sh {
namespace edge {

// ---------------------------------------------------------------------------
// basic moments
// ---------------------------------------------------------------------------
// GATE: two-layer gate models' main pass, every R_mu of neighbour j scaled by
// the gate multiplier G_{j,mu} (gpu_sh_compute_basic_gate_main, sus2_sh.cu:4247-4314).
// Unnormalised basic moments acc[k*C + l*l + m] = sum_j R_kl P_lm of centre
// i over its list (the inner list when the engine keeps one); the pairs
// inside rc are appended to the atom's cut_nbr column when it is set.
template <typename T, int L, int K, int RB, bool GATE>
__device__ __forceinline__ void atom_basic(const EdgeArgs<T>& a, const T* __restrict__ s_tab, int i,
                                           T (&acc)[K * (L + 1) * (L + 1)]) {
  constexpr int C = (L + 1) * (L + 1), KMU = K * (L + 1), NB = K * C;
#pragma unroll
  for (int b = 0; b < NB; ++b) acc[b] = T(0);
  const double4 pi = a.pos4[i];
  const double(*cell_shift)[3] = a.shift + (a.atom_cell ? 125 * a.atom_cell[i] : 0);
  const int S = a.rs.species;
  const int row_i = type_of(pi) * S;
  // the inner list (pairs within rc + margin) when the engine keeps one
  const bool inner = a.inner_nbr != nullptr;
  const int cnt = inner ? a.inner_count[i] : min(a.ncount[i], a.cap);
  const double rc = a.rs.rc, rc2 = rc * rc;
  NeighborStream ns(inner ? a.inner_nbr : a.nbr, a.pos4, a.N, i, cnt);
  int* const cut = a.cut_nbr ? a.cut_nbr + i : nullptr;
  int ncut = 0;
  // the build specialised to one model (no spills there) runs two edges per
  // unrolled iteration: 0.470 -> 0.459 ms at 1.024M atoms; the parameter build
  // measured slower unrolled
#ifdef SUS2_MODEL_COEF
#pragma unroll 2
#endif
  for (int n = 0; n < cnt; ++n) {
    int w;
    double4 pj;
    ns.next(n, w, pj);
    double sx, sy, sz;
    image_shift(cell_shift, static_cast<unsigned>(w) >> 24, sx, sy, sz);
    const double dx = pj.x - pi.x + sx;
    const double dy = pj.y - pi.y + sy;
    const double dz = pj.z - pi.z + sz;
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 >= rc2) continue;
    if (cut) cut[static_cast<size_t>(ncut++) * a.N] = w;
    const Edge<T> e = make_edge<T>(dx, dy, dz, r2, rc, rc2);
    const T* row = s_tab + (row_i + type_of(pj)) * a.rs.pair_stride;
    T R[KMU];
    radial_values<T, KMU, RB>(a, row, e, R);
    if constexpr (GATE) {
      const int j = w & 0xFFFFFF;
#pragma unroll
      for (int mu = 0; mu < KMU; ++mu) R[mu] *= a.gate_mult[static_cast<size_t>(mu) * a.N + j];
    }
    T P[C];  // harmonic polynomials; their normalisation is applied once per atom below
    sh_poly<L>(e.ux, e.uy, e.uz, P);
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
      for (int l = 0; l <= L; ++l)
#pragma unroll
        for (int m = 0; m <= 2 * l; ++m)
          acc[k * C + l * l + m] = fma(R[k * (L + 1) + l], P[l * l + m], acc[k * C + l * l + m]);
  }
  if (cut) a.cut_count[i] = ncut;
}

template <typename T, int L, int K, int RB, int BLOCK, bool GATE = false>
__global__ void __launch_bounds__(BLOCK, sizeof(T) == 4 && K * (L + 1) * (L + 1) <= 64 &&
                                                 SUS2_BASIC_MIN_BLOCKS * 128 / BLOCK > 1
                                             ? SUS2_BASIC_MIN_BLOCKS * 128 / BLOCK
                                             : 1)
    k_basic(const EdgeArgs<T> a, T* __restrict__ B) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* s_tab = reinterpret_cast<T*>(smem_raw);
  load_pair_table(a, s_tab);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  constexpr int C = (L + 1) * (L + 1), NB = K * C;
  T acc[NB];
  atom_basic<T, L, K, RB, GATE>(a, s_tab, i, acc);
  const unsigned long long pol = l2_evict_first();
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int c = 0; c < C; ++c)
      st_stream(B + static_cast<size_t>(k * C + c) * a.N + i, T(sh_poly_norm<L>(c)) * acc[k * C + c], pol);
}

// ---------------------------------------------------------------------------
// forces and virial
// ---------------------------------------------------------------------------
template <typename T>
struct Scatter;
template <>
struct Scatter<float> {
  __device__ __forceinline__ static void add(void* buf, int j, float x, float y, float z) {
    atomicAdd(reinterpret_cast<float4*>(buf) + j, make_float4(x, y, z, 0.0f));
  }
};
template <>
struct Scatter<double> {
  __device__ __forceinline__ static void add(void* buf, int j, double x, double y, double z) {
    double* p = reinterpret_cast<double*>(reinterpret_cast<double4*>(buf) + j);
    atomicAdd(p, x);
    atomicAdd(p + 1, y);
    atomicAdd(p + 2, z);
  }
};

// GATE: the main pass of a gate model (gpu_sh_compute_forces_gate_main_cached_grads,
// sus2_sh.cu:6555-6693 with compute_sh_edge_derivative_gate_main_cached_grads
// :6077-6121): R, R' scaled by G_{j,mu}, and dE/dh_{j,mu} += dG/dh_{j,mu}
// R_mu sum_m g_{mu,m} Y_m accumulated on the neighbour.
// The register cap applies to shapes whose adjoints fit it (K (L+1)^2 <= 64);
// larger shapes keep up to 255 registers.  The same holds for k_basic.
// Force and virial of centre i's edges from its adjoints g, pre-scaled by the
// harmonic normalisation (g'_klm = c_lm g_klm, so every edge works with the
// bare polynomials P_lm): the self force is summed into fx, fy, fz, the
// per-atom virial into w, and each neighbour's reaction -dE goes to
// scatter(j, x, y, z).
template <typename T, int L, int K, int RB, bool GATE, class Scatter_>
__device__ __forceinline__ void atom_force(const EdgeArgs<T>& a, const T* __restrict__ s_tab, int i,
                                           const T (&g)[K * (L + 1) * (L + 1)], T& fx, T& fy, T& fz, T (&w)[9],
                                           Scatter_ scatter) {
  constexpr int C = (L + 1) * (L + 1), KMU = K * (L + 1);
  fx = fy = fz = T(0);
#pragma unroll
  for (int q = 0; q < 9; ++q) w[q] = T(0);
  const double4 pi = a.pos4[i];
  const double(*cell_shift)[3] = a.shift + (a.atom_cell ? 125 * a.atom_cell[i] : 0);
  const int S = a.rs.species;
  const int row_i = type_of(pi) * S;
  // the in-cutoff sub-list written by k_basic when available (every pair in
  // it passes the test below, so no lane idles on a listed pair outside rc),
  // else the full list
  const bool sub = a.use_cut != 0;
  const int cnt = sub ? a.cut_count[i] : min(a.ncount[i], a.cap);
  const double rc = a.rs.rc, rc2 = rc * rc;
  NeighborStream ns(sub ? a.cut_nbr : a.nbr, a.pos4, a.N, i, cnt);
  for (int n = 0; n < cnt; ++n) {
    int wd;
    double4 pj;
    ns.next(n, wd, pj);
    const int j = wd & 0xFFFFFF;
    double sx, sy, sz;
    image_shift(cell_shift, static_cast<unsigned>(wd) >> 24, sx, sy, sz);
    const double dx = pj.x - pi.x + sx;
    const double dy = pj.y - pi.y + sy;
    const double dz = pj.z - pi.z + sz;
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 >= rc2) continue;
    const Edge<T> e = make_edge<T>(dx, dy, dz, r2, rc, rc2);
    const T* row = s_tab + (row_i + type_of(pj)) * a.rs.pair_stride;
    // R_mu = fS s_mu, dR_mu = dfS s_mu + fS fac sd_mu.  Shared argument: fS =
    // f env, dfS = env (df + f denv/env), fac = dx/dr, s_mu = sum_n c[mu][n]
    // P_n, sd_mu = sum_n d[mu][n] P_n (derivative series).  Per-mu arguments:
    // fS = f, dfS = df, fac = 1, with env and dx/dr folded into s_mu, sd_mu.
    // f = s_pair (r-rc)^2; the common factors are applied after the
    // contractions below.
    const T ps = row[2 * KMU];
    const T f = ps * e.dr * e.dr;
    const T df = T(2) * ps * e.dr;
    const int kind = SUS2_RADIAL_KIND(a);
    T t[RB], fac = T(1), fS = f, dfS = df, xarg = T(0);
    if (SUS2_SHARED_XI(a)) {
      T env, denv;
      radial_arg<T>(kind, row[0], row[1], e.rd, xarg, fac, env, denv);
      fS = f * env;
      dfS = env * fma(f, denv, df);
      radial_poly<RB>(kind, xarg, t);
    }
    T P[C];
    sh_poly<L>(e.ux, e.uy, e.uz, P);
    // Gt_lm = sum_k g_klm s_kl, Ht_lm = sum_k g_klm sd_kl; sG = P.Gt, sH = P.Ht;
    // the radial sums of one l at a time
    T Gt[C];
    T sG = T(0), sH = T(0);
#pragma unroll
    for (int l = 0; l <= L; ++l) {
      T sk[K], sdk[K];
#pragma unroll
      for (int k = 0; k < K; ++k) {
        const int mu = k * (L + 1) + l;
        T scale = T(1), env = T(1), denv = T(0);
        if (!SUS2_SHARED_XI(a)) {
          radial_arg<T>(kind, row[2 * mu], row[2 * mu + 1], e.rd, xarg, scale, env, denv);
          radial_poly<RB>(kind, xarg, t);
        }
        T v = T(0), d = T(0);
        if constexpr (2 * KMU * RB <= kMaxCoef) {
          // derivative series stored after the coefficients
#pragma unroll
          for (int n = 0; n < RB; ++n) {
            v = fma(SUS2_COEF(a, mu * RB + n), t[n], v);
            if (n + 1 < RB) d = fma(SUS2_COEF(a, KMU * RB + mu * RB + n), t[n], d);
          }
        } else {
          T tt[RB], dt[RB];
          radial_poly_d<RB>(kind, xarg, tt, dt);
#pragma unroll
          for (int n = 0; n < RB; ++n) {
            v = fma(SUS2_COEF(a, mu * RB + n), t[n], v);
            d = fma(SUS2_COEF(a, mu * RB + n), dt[n], d);
          }
        }
        if (SUS2_SHARED_XI(a)) {
          sk[k] = v;
          sdk[k] = d;
        } else {
          sk[k] = env * v;
          sdk[k] = env * fma(denv, v, scale * d);
        }
        if constexpr (GATE) {
          T p = T(0);
#pragma unroll
          for (int m = 0; m <= 2 * l; ++m) p = fma(g[k * C + l * l + m], P[l * l + m], p);
          const size_t at = static_cast<size_t>(mu) * a.N + j;
          atomicAdd(a.gate_adj + at, p * (fS * sk[k]) * a.gate_deriv[at]);
          const T gm = a.gate_mult[at];
          sk[k] *= gm;
          sdk[k] *= gm;
        }
      }
#pragma unroll
      for (int m = 0; m <= 2 * l; ++m) {
        T gv = T(0), hv = T(0);
#pragma unroll
        for (int k = 0; k < K; ++k) {
          gv = fma(g[k * C + l * l + m], sk[k], gv);
          hv = fma(g[k * C + l * l + m], sdk[k], hv);
        }
        Gt[l * l + m] = gv;
        sG = fma(gv, P[l * l + m], sG);
        sH = fma(hv, P[l * l + m], sH);
      }
    }
    // radial part s = dE/dr along u; tangential part f (V - (u.V) u) / r
    const T s = dfS * sG + (fS * fac) * sH;
    T vx, vy, vz;
    sh_poly_grad_contract<L>(e.ux, e.uy, e.uz, Gt, vx, vy, vz);
    const T uv = e.ux * vx + e.uy * vy + e.uz * vz;
    const T ft = fS * e.rinv;
    const T dEx = s * e.ux + (vx - uv * e.ux) * ft;
    const T dEy = s * e.uy + (vy - uv * e.uy) * ft;
    const T dEz = s * e.uz + (vz - uv * e.uz) * ft;
    fx += dEx;
    fy += dEy;
    fz += dEz;
    scatter(j, -dEx, -dEy, -dEz);
    w[0] -= e.dx * dEx;
    w[1] -= e.dy * dEy;
    w[2] -= e.dz * dEz;
    w[3] -= e.dx * dEy;
    w[4] -= e.dx * dEz;
    w[5] -= e.dy * dEz;
    w[6] -= e.dy * dEx;
    w[7] -= e.dz * dEx;
    w[8] -= e.dz * dEy;
  }
}

template <typename T, int L, int K, int RB, int BLOCK, bool GATE = false>
__global__ void __launch_bounds__(BLOCK, sizeof(T) == 4 && K * (L + 1) * (L + 1) <= 64 &&
                                                 SUS2_FORCE_MIN_BLOCKS * 128 / BLOCK > 1
                                             ? SUS2_FORCE_MIN_BLOCKS * 128 / BLOCK
                                             : 1)
    k_force(const EdgeArgs<T> a, const T* __restrict__ G, const double* __restrict__ weight,
            void* __restrict__ ftmp, double* __restrict__ force, double* __restrict__ virial,
            double sign) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* s_tab = reinterpret_cast<T*>(smem_raw);
  load_pair_table(a, s_tab);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  constexpr int C = (L + 1) * (L + 1), NB = K * C;
  const T wscale = weight ? static_cast<T>(weight[i]) : T(1);
  T g[NB];
  const unsigned long long pol = l2_evict_first();
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int c = 0; c < C; ++c)
      g[k * C + c] = (wscale * T(sh_poly_norm<L>(c))) * ld_stream(G + static_cast<size_t>(k * C + c) * a.N + i, pol);
  T fx, fy, fz;
  T w[9];
  atom_force<T, L, K, RB, GATE>(a, s_tab, i, g, fx, fy, fz, w,
                                [ftmp](int j, T x, T y, T z) { Scatter<T>::add(ftmp, j, x, y, z); });
  force[i] += sign * static_cast<double>(fx);
  force[i + a.N] += sign * static_cast<double>(fy);
  force[i + 2 * a.N] += sign * static_cast<double>(fz);
  if (virial) {
#pragma unroll
    for (int q = 0; q < 9; ++q) virial[static_cast<size_t>(q) * a.N + i] += static_cast<double>(w[q]);
  }
}

}  // namespace edge
}  // namespace sus2sh
