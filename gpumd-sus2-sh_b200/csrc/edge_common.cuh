// Per-edge device helpers shared by the engine's kernels: species bits,
// neighbour stream, image shifts, FP64-to-working-precision edge geometry and
// the radial basis (values, and values + derivatives).
#pragma once

#include "edge_args.cuh"
#include "sh_math.cuh"

namespace sus2sh {
namespace edge {

constexpr int kCenterCode = 62;  // image (0,0,0) in base-5 codes

// Radial coefficient X (c[mu][n], then the derivative series), whether all
// radial functions of a pair share one radial argument, and the radial basis
// kind: from the kernel parameters, or, in a build specialised to one model,
// compiled in (model_coef() table and the SUS2_MODEL_SHARED_XI /
// SUS2_MODEL_RADIAL_KIND constants), so every coefficient of an unrolled loop
// is an immediate operand and the per-edge tests of the radial setup
// disappear.
#ifdef SUS2_MODEL_COEF
#define SUS2_COEF(a, X) (::sus2sh::edge::model_coef(X))
#define SUS2_SHARED_XI(a) (SUS2_MODEL_SHARED_XI != 0)
#define SUS2_RADIAL_KIND(a) (SUS2_MODEL_RADIAL_KIND)
#else
#define SUS2_COEF(a, X) ((a).coef[X])
#define SUS2_SHARED_XI(a) ((a).rs.shared_xi != 0)
#ifdef SUS2_SHAPE_RADIAL_KIND
// NVRTC build of a shape for one radial basis kind
#define SUS2_RADIAL_KIND(a) (SUS2_SHAPE_RADIAL_KIND)
#else
// other builds (ahead of time, or NVRTC for a shape): the Chebyshev kinds,
// tanh or rational map read at run time; Laguerre models get a build with
// SUS2_SHAPE_RADIAL_KIND, so these kernels carry no Laguerre code
#define SUS2_RADIAL_KIND(a) ((a).rs.kind == ::sus2sh::kRadialRational ? ::sus2sh::kRadialRational \
                                                                      : ::sus2sh::kRadialTanh)
#endif
#endif

// Basic moments and their adjoints ([K*C][N]: hundreds of MB at large N)
// pass through L2 once per kernel.  They are stored and loaded with an L2
// evict-first policy, so they do not push out of L2 the code of a large
// generated CG kernel, which every launch fetches through L2 again (the
// component-split kernel of an l4k4 body-5 graph on 262,144 atoms: 3.07 ms
// with its code resident, 3.63 ms with it evicted by plain traffic, 3.17 ms
// when the same traffic is evict-first).
__device__ __forceinline__ unsigned long long l2_evict_first() {
  unsigned long long p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ void st_stream(float* a, float v, unsigned long long pol) {
  asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(a), "f"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_stream(double* a, double v, unsigned long long pol) {
  asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(a), "d"(v), "l"(pol) : "memory");
}
// read-only data (not written while the kernel runs)
__device__ __forceinline__ float ld_stream(const float* a, unsigned long long pol) {
  float v;
  asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ double ld_stream(const double* a, unsigned long long pol) {
  double v;
  asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
  return v;
}

__device__ __forceinline__ int type_of(const double4& p) {
  return static_cast<int>(__double_as_longlong(p.w));
}

// ---------------------------------------------------------------------------
// per-edge geometry and radial basis
// ---------------------------------------------------------------------------
template <typename T>
struct Edge {
  T r, rinv, ux, uy, uz, dr;  // dr = r - rc (formed in FP64)
  T dx, dy, dz;
  double rd;                  // r in FP64: the radial argument scal (r - shift) / 2 is formed from it
};

template <typename T>
__device__ __forceinline__ Edge<T> make_edge(double dx, double dy, double dz, double r2, double rc,
                                             double rc2);

template <>
__device__ __forceinline__ Edge<float> make_edge<float>(double dx, double dy, double dz, double r2,
                                                        double rc, double rc2) {
  Edge<float> e;
  const float r2f = static_cast<float>(r2);
  e.rinv = rsqrtf(r2f);
  const float r32 = r2f * e.rinv;
  // one Newton step on the FP64 r^2 gives r to FP64 accuracy: the radial
  // argument and (r - rc) near the cutoff are formed from it in FP64
  e.rd = fma(r2 - static_cast<double>(r32) * static_cast<double>(r32), 0.5 * static_cast<double>(e.rinv),
             static_cast<double>(r32));
  e.r = static_cast<float>(e.rd);
  e.dx = static_cast<float>(dx);
  e.dy = static_cast<float>(dy);
  e.dz = static_cast<float>(dz);
  e.ux = e.dx * e.rinv;
  e.uy = e.dy * e.rinv;
  e.uz = e.dz * e.rinv;
  e.dr = static_cast<float>(e.rd - rc);
  (void)rc2;
  return e;
}

template <>
__device__ __forceinline__ Edge<double> make_edge<double>(double dx, double dy, double dz, double r2,
                                                          double rc, double rc2) {
  Edge<double> e;
  e.r = sqrt(r2);
  e.rd = e.r;
  e.rinv = 1.0 / e.r;
  e.dx = dx;
  e.dy = dy;
  e.dz = dz;
  e.ux = dx * e.rinv;
  e.uy = dy * e.rinv;
  e.uz = dz * e.rinv;
  e.dr = (r2 - rc2) / (e.r + rc);
  return e;
}

// R_mu for every mu; the pair table row holds KMU (scal, shift) pairs then
// the LK pair scale.  R_mu = s_pair (r - rc)^2 env(x) sum_n c[mu][n] P_n(x)
// with x the kind's argument (radial_arg).
// KIND >= 0 fixes the basis kind at compile time (kernels instantiated per
// kind); -1 takes SUS2_RADIAL_KIND.
template <typename T, int KMU, int RB, int KIND = -1>
__device__ __forceinline__ void radial_values(const EdgeArgs<T>& a, const T* __restrict__ row,
                                              const Edge<T>& e, T* R) {
  const T f = row[2 * KMU] * e.dr * e.dr;
  const int kind = KIND >= 0 ? KIND : SUS2_RADIAL_KIND(a);
  if (SUS2_SHARED_XI(a)) {
    T x, dx, env, denv;
    radial_arg<T>(kind, row[0], row[1], e.rd, x, dx, env, denv);
    T t[RB];
    radial_poly<RB>(kind, x, t);
    const T fe = f * env;
#pragma unroll
    for (int mu = 0; mu < KMU; ++mu) {
      T s = T(0);
#pragma unroll
      for (int n = 0; n < RB; ++n) s = fma(SUS2_COEF(a, mu * RB + n), t[n], s);
      R[mu] = fe * s;
    }
  } else {
#pragma unroll
    for (int mu = 0; mu < KMU; ++mu) {
      T x, dx, env, denv;
      radial_arg<T>(kind, row[2 * mu], row[2 * mu + 1], e.rd, x, dx, env, denv);
      T t[RB];
      radial_poly<RB>(kind, x, t);
      T s = T(0);
#pragma unroll
      for (int n = 0; n < RB; ++n) s = fma(SUS2_COEF(a, mu * RB + n), t[n], s);
      R[mu] = f * env * s;
    }
  }
}

// R_mu and dR_mu/dr: with f = s_pair (r - rc)^2, s = sum c P_n(x),
// sd = sum c P_n'(x): dR = (df + f denv/env) env s + f env (dx/dr) sd.
template <typename T, int KMU, int RB, int KIND = -1>
__device__ __forceinline__ void radial_values_ders(const EdgeArgs<T>& a, const T* __restrict__ row,
                                                   const Edge<T>& e, T* R, T* dR) {
  const T ps = row[2 * KMU];
  const T f = ps * e.dr * e.dr;
  const T df = T(2) * ps * e.dr;
  const int kind = KIND >= 0 ? KIND : SUS2_RADIAL_KIND(a);
  if (SUS2_SHARED_XI(a)) {
    T x, dx, env, denv;
    radial_arg<T>(kind, row[0], row[1], e.rd, x, dx, env, denv);
    const T fe = f * env;
    const T dfe = env * fma(f, denv, df);
    const T g = fe * dx;  // f env dx/dr
    T t[RB], dt[RB];
    radial_poly_d<RB>(kind, x, t, dt);
#pragma unroll
    for (int mu = 0; mu < KMU; ++mu) {
      T s = T(0), sd = T(0);
#pragma unroll
      for (int n = 0; n < RB; ++n) {
        s = fma(SUS2_COEF(a, mu * RB + n), t[n], s);
        sd = fma(SUS2_COEF(a, mu * RB + n), dt[n], sd);
      }
      R[mu] = fe * s;
      dR[mu] = dfe * s + g * sd;
    }
  } else {
#pragma unroll
    for (int mu = 0; mu < KMU; ++mu) {
      T x, dx, env, denv;
      radial_arg<T>(kind, row[2 * mu], row[2 * mu + 1], e.rd, x, dx, env, denv);
      T t[RB], dt[RB];
      radial_poly_d<RB>(kind, x, t, dt);
      T s = T(0), sd = T(0);
#pragma unroll
      for (int n = 0; n < RB; ++n) {
        s = fma(SUS2_COEF(a, mu * RB + n), t[n], s);
        sd = fma(SUS2_COEF(a, mu * RB + n), dt[n], sd);
      }
      R[mu] = f * env * s;
      dR[mu] = env * (fma(f, denv, df) * s + f * dx * sd);
    }
  }
}

template <typename T>
__device__ __forceinline__ void load_pair_table(const EdgeArgs<T>& a, T* s_tab) {
  const int n = a.rs.species * a.rs.species * a.rs.pair_stride;
  const T* src = reinterpret_cast<const T*>(a.pair_table);
  for (int t = threadIdx.x; t < n; t += blockDim.x) s_tab[t] = src[t];
  __syncthreads();
}

// Software-pipelined neighbour stream of one centre atom: the neighbour word
// is fetched two edges ahead and the neighbour's position one edge ahead, so
// the dependent gathers overlap the previous edge's arithmetic.
struct NeighborStream {
  const int* __restrict__ nbr;
  const double4* __restrict__ pos4;
  size_t stride;
  int cnt;
  int w_next, w_next2;
  double4 p_next;

  __device__ __forceinline__ NeighborStream(const int* nb, const double4* p4, int N, int i, int count)
      : nbr(nb + i), pos4(p4), stride(static_cast<size_t>(N)), cnt(count) {
    w_next = cnt > 0 ? word(nbr) : 0;
    w_next2 = cnt > 1 ? word(nbr + stride) : 0;
    p_next = cnt > 0 ? pos4[w_next & 0xFFFFFF] : make_double4(0.0, 0.0, 0.0, 0.0);
  }
  // Returns edge n's word and position and issues the loads for n+1 / n+2.
  __device__ __forceinline__ void next(int n, int& w, double4& pj) {
    w = w_next;
    pj = p_next;
    w_next = w_next2;
    if (n + 1 < cnt) p_next = pos4[w_next & 0xFFFFFF];
    if (n + 2 < cnt) w_next2 = word(nbr + static_cast<size_t>(n + 2) * stride);
  }
  // Neighbour words through the read-only data path, or, in a kernel that
  // writes the lists itself before reading them (SUS2_NBR_WRITTEN_IN_KERNEL),
  // through plain loads, which see the kernel's own earlier writes.
  __device__ __forceinline__ static int word(const int* p) {
#ifdef SUS2_NBR_WRITTEN_IN_KERNEL
    return *p;
#else
    return __ldg(p);
#endif
  }
};

// Image shift of a neighbour word (zero for the home image, which is most).
__device__ __forceinline__ void image_shift(const double (*shift)[3], int code, double& sx, double& sy,
                                            double& sz) {
  if (code == kCenterCode) {
    sx = sy = sz = 0.0;
  } else {
    sx = shift[code][0];
    sy = shift[code][1];
    sz = shift[code][2];
  }
}

}  // namespace edge
}  // namespace sus2sh
