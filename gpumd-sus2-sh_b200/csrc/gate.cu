// Two-layer mu-body gate models (two_layer_gate_enabled = 1), neighbour site
// mode with shared radial (scal, shift) tables.  Per evaluation:
//
//   1. first-layer basics Bg = k_basic with the gate radial coefficients;
//   2. k_gate_forward: the needed part of the saved product graph on Bg, the
//      gate scalars s_q = M[moment(q)], the signals
//        mu-body-linear-combo  b_p = sum_{q: body(q) = p} w_q s_q,
//                              h_mu = sum_p c_{mu,p} b_p
//        mu-scalar-full        h_mu = sum_q W_{mu,q} s_q
//      and the multipliers G_mu = 1 + A tanh(a_t h_mu), dG/dh = A a_t (1 - tanh^2)
//      (gpu_sh_gate_values_from_moments :4565-4610, gpu_sh_gate_precompute_tanh
//      :4641-4662, src/force/sus2_sh.cu);
//   3. main basics with R_mu(r_ij) G_{j,mu} (k_basic<GATE>), products, energy;
//   4. k_force<GATE>: main forces and dE/dh_{j,mu};
//   5. k_gate_backward: seeds dE/ds_q (gpu_sh_seed_gate_moment_grads_from_mu_adjoints
//      :4664-4727), reverse through the needed products, first-layer basic
//      adjoints;
//   6. k_force with the gate radial coefficients on those adjoints
//      (gpu_sh_compute_forces_gate_first_layer_cached_grads :6695-6790).
//
// Lane = atom; the first-layer moments and their adjoints live in [slot][N]
// scratch (coalesced per slot), only the moments the gate signals need.
#include "edge_common.cuh"
#include "engine.cuh"

namespace sus2sh {
namespace {

constexpr int kGateMaxMu = 48;

template <typename T>
__global__ void __launch_bounds__(128)
    k_gate_forward(int N, const GateProgDev p, const double4* __restrict__ pos4, const T* __restrict__ Bg,
                   T* __restrict__ M, T* __restrict__ gmult, T* __restrict__ gderiv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const size_t n = static_cast<size_t>(N);
  for (int b = 0; b < p.nbasic; ++b) M[b * n + i] = Bg[static_cast<size_t>(p.basic_canon[b]) * n + i];
  for (int s = p.nbasic; s < p.nslots; ++s) M[s * n + i] = T(0);
  for (int q = 0; q < p.nprod; ++q) {
    const int l = __ldg(p.prod + 3 * q), r = __ldg(p.prod + 3 * q + 1), t = __ldg(p.prod + 3 * q + 2);
    const T c = static_cast<T>(__ldg(p.coef + q));
    M[t * n + i] = fma(c * M[l * n + i], M[r * n + i], M[t * n + i]);
  }
  T h[kGateMaxMu];
  if (p.mode == 1) {
    T body[kGateMaxMu];
    for (int b = 0; b < p.nbody; ++b) body[b] = T(0);
    for (int q = 0; q < p.nq; ++q)
      body[p.q_body[q]] += static_cast<T>(p.weights[q]) * M[static_cast<size_t>(p.q_slot[q]) * n + i];
    for (int mu = 0; mu < p.kmu; ++mu) {
      T v = T(0);
      for (int b = 0; b < p.nbody; ++b) v += static_cast<T>(p.body_mix[mu * p.nbody + b]) * body[b];
      h[mu] = v;
    }
  } else {
    for (int mu = 0; mu < p.kmu; ++mu) h[mu] = T(0);
    for (int q = 0; q < p.nq; ++q) {
      const T s = M[static_cast<size_t>(p.q_slot[q]) * n + i];
      for (int mu = 0; mu < p.kmu; ++mu) h[mu] += static_cast<T>(p.weights[mu * p.nq + q]) * s;
    }
  }
  const int t = static_cast<int>(__double_as_longlong(pos4[i].w));
  const T a = static_cast<T>(p.additive[t]);
  const T A = static_cast<T>(p.amplitude);
  for (int mu = 0; mu < p.kmu; ++mu) {
    const T th = tanh(a * h[mu]);
    gmult[mu * n + i] = T(1) + A * th;
    gderiv[mu * n + i] = A * a * (T(1) - th * th);
  }
}

template <typename T>
__global__ void __launch_bounds__(128)
    k_gate_backward(int N, const GateProgDev p, const T* __restrict__ M, T* __restrict__ gM,
                    const T* __restrict__ adjh, T* __restrict__ Gg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const size_t n = static_cast<size_t>(N);
  for (int s = 0; s < p.nslots; ++s) gM[s * n + i] = T(0);
  if (p.mode == 1) {
    T body[kGateMaxMu];
    for (int b = 0; b < p.nbody; ++b) body[b] = T(0);
    for (int mu = 0; mu < p.kmu; ++mu) {
      const T adj = adjh[mu * n + i];
      for (int b = 0; b < p.nbody; ++b) body[b] += adj * static_cast<T>(p.body_mix[mu * p.nbody + b]);
    }
    for (int q = 0; q < p.nq; ++q) {
      const size_t at = static_cast<size_t>(p.q_slot[q]) * n + i;
      gM[at] += body[p.q_body[q]] * static_cast<T>(p.weights[q]);
    }
  } else {
    for (int q = 0; q < p.nq; ++q) {
      T seed = T(0);
      for (int mu = 0; mu < p.kmu; ++mu) seed += adjh[mu * n + i] * static_cast<T>(p.weights[mu * p.nq + q]);
      const size_t at = static_cast<size_t>(p.q_slot[q]) * n + i;
      gM[at] += seed;
    }
  }
  for (int q = p.nprod - 1; q >= 0; --q) {
    const int l = __ldg(p.prod + 3 * q), r = __ldg(p.prod + 3 * q + 1), t = __ldg(p.prod + 3 * q + 2);
    const T gt = gM[t * n + i] * static_cast<T>(__ldg(p.coef + q));
    if (gt == T(0)) continue;
    const T ml = M[l * n + i], mr = M[r * n + i];
    gM[l * n + i] = fma(gt, mr, gM[l * n + i]);
    gM[r * n + i] = fma(gt, ml, gM[r * n + i]);
  }
  for (int b = 0; b < p.nbasic; ++b) Gg[static_cast<size_t>(p.basic_canon[b]) * n + i] = gM[b * n + i];
}

inline int blocks(int n, int b) { return (n + b - 1) / b; }

}  // namespace

template <typename T>
void launch_gate_forward(cudaStream_t s, int N, const GateProgDev& p, const double4* pos4, const T* Bg, T* M,
                         T* gmult, T* gderiv) {
  k_gate_forward<T><<<blocks(N, 128), 128, 0, s>>>(N, p, pos4, Bg, M, gmult, gderiv);
}

template <typename T>
void launch_gate_backward(cudaStream_t s, int N, const GateProgDev& p, const T* M, T* gM, const T* adjh, T* Gg) {
  k_gate_backward<T><<<blocks(N, 128), 128, 0, s>>>(N, p, M, gM, adjh, Gg);
}

template void launch_gate_forward<float>(cudaStream_t, int, const GateProgDev&, const double4*, const float*,
                                         float*, float*, float*);
template void launch_gate_forward<double>(cudaStream_t, int, const GateProgDev&, const double4*, const double*,
                                          double*, double*, double*);
template void launch_gate_backward<float>(cudaStream_t, int, const GateProgDev&, const float*, float*,
                                          const float*, float*);
template void launch_gate_backward<double>(cudaStream_t, int, const GateProgDev&, const double*, double*,
                                           const double*, double*);

}  // namespace sus2sh
