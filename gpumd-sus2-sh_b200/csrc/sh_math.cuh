// Per-edge math of the SUS2-SH descriptor, shared by the CUDA kernels and by
// host-side unit tests (every function is __host__ __device__).
//
//  * Real spherical harmonics Y_lm(u), l <= 6, orthonormal, no Condon-Shortley
//    phase, flat index l*l + l + m (same basis and ordering as the reference's
//    eval_real_sh, src/force/sus2_sh.cu:3032-3169, and its solid-harmonic
//    path for l_max > 4, :2880-3030).  For L <= 4 the polynomial forms are the
//    standard real-harmonic table evaluated on the unit vector u = d/|d|; for
//    L = 5, 6 every l comes from the associated-Legendre recurrences of the
//    complex solid harmonics (sh_values_solid below).
//  * Gradients use the tangential projection: for Y(d) = F(d/r),
//        dY/dd = (grad F(u) - (u . grad F(u)) u) / r,
//    with F the homogeneous Cartesian polynomial of each harmonic.  The force
//    kernel contracts the adjoint first and projects once per edge.
//  * Chebyshev-sss radial basis (sus2_sh.cu:3171-3220):
//        xi = tanh(z) or z/sqrt(1+z^2) (rational map, README.md:45,55-56),
//        z = scal (r - shift) / 2,
//        R_mu = s_pair (r-rc)^2 sum_n c[mu][n] T_n(xi),
//    T_0 = 1, T_1 = xi, T_n = 2 xi T_{n-1} - T_{n-2}; dT_n/dxi by the paired
//    recurrence.  s_pair = scaling * rtc[t_i] * rtc[t_j] is the LK species
//    scaling folded per pair (build_direct_radial_tables, sus2_sh.cu:2484-2517).
#pragma once

#if !defined(__CUDACC_RTC__)
#include <cmath>
#endif

#if defined(__CUDACC__)
#define SUS2_HD __host__ __device__ __forceinline__
#else
#define SUS2_HD inline
#endif

namespace sus2sh {

// Normalisation constants of the real harmonics.
struct YC {
  static constexpr double c00 = 0.28209479177387814347;   // 1/2 sqrt(1/pi)
  static constexpr double c1 = 0.48860251190291992159;    // 1/2 sqrt(3/pi)
  static constexpr double c2a = 1.09254843059207907054;   // 1/2 sqrt(15/pi)
  static constexpr double c20 = 0.31539156525252000603;   // 1/4 sqrt(5/pi)
  static constexpr double c22 = 0.54627421529603953527;   // 1/4 sqrt(15/pi)
  static constexpr double c33 = 0.59004358992664351035;   // 1/4 sqrt(35/(2pi))
  static constexpr double c32 = 2.89061144264055405539;   // 1/2 sqrt(105/pi)
  static constexpr double c31 = 0.45704579946446573616;   // 1/4 sqrt(21/(2pi))
  static constexpr double c30 = 0.37317633259011539141;   // 1/4 sqrt(7/pi)
  static constexpr double c3p2 = 1.44530572132027702770;  // 1/4 sqrt(105/pi)
  static constexpr double c44m = 2.50334294179670453835;  // 3/4 sqrt(35/pi)
  static constexpr double c43 = 1.77013076977993053104;   // 3/4 sqrt(35/(2pi))
  static constexpr double c42m = 0.94617469575756001810;  // 3/4 sqrt(5/pi)
  static constexpr double c41 = 0.66904654355728916795;   // 3/4 sqrt(5/(2pi))
  static constexpr double c40 = 0.10578554691520430380;   // 3/16 sqrt(1/pi)
  static constexpr double c42 = 0.47308734787878000905;   // 3/8 sqrt(5/pi)
  static constexpr double c44 = 0.62583573544917613459;   // 3/16 sqrt(35/pi)
};

// Normalisation of the solid-harmonic path: N_l0 for m = 0 and sqrt(2) N_lm
// for m > 0, N_lm^2 = (2l+1)/(4 pi) (l-m)!/(l+m)!, keyed by 8 l + m.
SUS2_HD constexpr double solid_norm(int key) {
  switch (key) {
    case 0: return 0.28209479177387814;
    case 8: return 0.4886025119029199;
    case 9: return 0.48860251190292;
    case 16: return 0.6307831305050401;
    case 17: return 0.36418281019735976;
    case 18: return 0.18209140509867988;
    case 24: return 0.7463526651802308;
    case 25: return 0.3046971996429772;
    case 26: return 0.09635371475468515;
    case 27: return 0.03933623932844291;
    case 32: return 0.8462843753216345;
    case 33: return 0.2676186174229157;
    case 34: return 0.063078313050504;
    case 35: return 0.016858388283618388;
    case 36: return 0.005960340337611203;
    case 40: return 0.9356025796273888;
    case 41: return 0.2415715473043717;
    case 42: return 0.045652731285460234;
    case 43: return 0.009318824751147628;
    case 44: return 0.002196468058075176;
    case 45: return 0.0006945841871324552;
    case 48: return 1.0171072362820548;
    case 49: return 0.22195099524523101;
    case 50: return 0.03509353369580661;
    case 51: return 0.005848922282634435;
    case 52: return 0.0010678622237644956;
    case 53: return 0.00022766899107568562;
    case 54: return 6.57223766418388e-05;
    default: return 0.0;
  }
}

// Every Y_lm, l <= L, from the complex solid harmonics
// Q_l^m = r^l P_l^m(cos t) e^{i m p} (associated Legendre without the
// Condon-Shortley phase), built by the standard recurrences
//   Q_m^m = (2m-1) (x + i y) Q_{m-1}^{m-1},   Q_{m+1}^m = (2m+1) z Q_m^m,
//   (l-m) Q_l^m = (2l-1) z Q_{l-1}^m - (l+m-1) r^2 Q_{l-2}^m,
// with Y_l0 = N_l0 Re Q_l^0 and (Y_l,m, Y_l,-m) = sqrt2 N_lm (Re, Im) Q_l^m.
// r^2 is formed from (x, y, z), so the polynomials stay homogeneous and their
// gradients (sh_grad_solid) obey the tangential-projection identity.
template <int L, typename T>
SUS2_HD void sh_values_solid(T x, T y, T z, T* Y) {
  const T r2 = x * x + y * y + z * z;
  T dre = T(1), dim = T(0);
#pragma unroll
  for (int m = 0; m <= L; ++m) {
    if (m > 0) {
      const T c = T(2 * m - 1);
      const T re = c * (x * dre - y * dim), im = c * (x * dim + y * dre);
      dre = re;
      dim = im;
    }
    T p1re = dre, p1im = dim, p2re = T(0), p2im = T(0);
#pragma unroll
    for (int l = m; l <= L; ++l) {
      if (l == m + 1) {
        const T c = T(2 * m + 1) * z;
        p2re = p1re;
        p2im = p1im;
        p1re = c * p2re;
        p1im = c * p2im;
      } else if (l > m + 1) {
        const T a = T(2 * l - 1) * z, b = T(l + m - 1) * r2, inv = T(1.0 / (l - m));
        const T qre = (a * p1re - b * p2re) * inv, qim = (a * p1im - b * p2im) * inv;
        p2re = p1re;
        p2im = p1im;
        p1re = qre;
        p1im = qim;
      }
      const T nrm = T(solid_norm(8 * l + m));
      Y[l * l + l + m] = nrm * p1re;
      if (m > 0) Y[l * l + l - m] = nrm * p1im;
    }
  }
}

// V = sum_lm G[lm] grad P_lm on the solid-harmonic path (forward-mode
// derivatives carried through the same recurrences).
template <int L, typename T>
SUS2_HD void sh_grad_solid(T x, T y, T z, const T* G, T& vx, T& vy, T& vz) {
  const T r2 = x * x + y * y + z * z;
  vx = vy = vz = T(0);
  // diagonal Q_m^m: value and gradient (re, im)
  T dre = T(1), dim = T(0);
  T dgre[3] = {T(0), T(0), T(0)}, dgim[3] = {T(0), T(0), T(0)};
#pragma unroll
  for (int m = 0; m <= L; ++m) {
    if (m > 0) {
      const T c = T(2 * m - 1);
      T gre[3], gim[3];
      gre[0] = c * (x * dgre[0] - y * dgim[0] + dre);
      gre[1] = c * (x * dgre[1] - y * dgim[1] - dim);
      gre[2] = c * (x * dgre[2] - y * dgim[2]);
      gim[0] = c * (x * dgim[0] + y * dgre[0] + dim);
      gim[1] = c * (x * dgim[1] + y * dgre[1] + dre);
      gim[2] = c * (x * dgim[2] + y * dgre[2]);
      const T re = c * (x * dre - y * dim), im = c * (x * dim + y * dre);
      dre = re;
      dim = im;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        dgre[a] = gre[a];
        dgim[a] = gim[a];
      }
    }
    T p1re = dre, p1im = dim, p2re = T(0), p2im = T(0);
    T g1re[3], g1im[3], g2re[3] = {T(0), T(0), T(0)}, g2im[3] = {T(0), T(0), T(0)};
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      g1re[a] = dgre[a];
      g1im[a] = dgim[a];
    }
#pragma unroll
    for (int l = m; l <= L; ++l) {
      if (l == m + 1) {
        const T c = T(2 * m + 1);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          g2re[a] = g1re[a];
          g2im[a] = g1im[a];
          g1re[a] = c * (z * g2re[a] + (a == 2 ? p1re : T(0)));
          g1im[a] = c * (z * g2im[a] + (a == 2 ? p1im : T(0)));
        }
        p2re = p1re;
        p2im = p1im;
        p1re = c * z * p2re;
        p1im = c * z * p2im;
      } else if (l > m + 1) {
        const T a2 = T(2 * l - 1), b2 = T(l + m - 1), inv = T(1.0 / (l - m));
        const T q[3] = {x, y, z};
        T nre[3], nim[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          nre[a] = (a2 * (z * g1re[a] + (a == 2 ? p1re : T(0))) -
                    b2 * (r2 * g2re[a] + T(2) * q[a] * p2re)) * inv;
          nim[a] = (a2 * (z * g1im[a] + (a == 2 ? p1im : T(0))) -
                    b2 * (r2 * g2im[a] + T(2) * q[a] * p2im)) * inv;
        }
        const T qre = (a2 * z * p1re - b2 * r2 * p2re) * inv, qim = (a2 * z * p1im - b2 * r2 * p2im) * inv;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          g2re[a] = g1re[a];
          g2im[a] = g1im[a];
          g1re[a] = nre[a];
          g1im[a] = nim[a];
        }
        p2re = p1re;
        p2im = p1im;
        p1re = qre;
        p1im = qim;
      }
      const T nrm = T(solid_norm(8 * l + m));
      const T cre = nrm * G[l * l + l + m];
      vx = fma(cre, g1re[0], vx);
      vy = fma(cre, g1re[1], vy);
      vz = fma(cre, g1re[2], vz);
      if (m > 0) {
        const T cim = nrm * G[l * l + l - m];
        vx = fma(cim, g1im[0], vx);
        vy = fma(cim, g1im[1], vy);
        vz = fma(cim, g1im[2], vz);
      }
    }
  }
}

// Normalisation c_i of the polynomial forms, Y_i = c_i P_i (flat index
// i = l*l + l + m, L <= 4).  Models with L > 4 take every harmonic from the
// solid-harmonic path, already normalised (c_i = 1).
template <int L>
SUS2_HD constexpr double sh_poly_norm(int i) {
  if (L > 4) return 1.0;
  switch (i) {
    case 0: return YC::c00;
    case 1: case 2: case 3: return YC::c1;
    case 4: case 5: case 7: return YC::c2a;
    case 6: return YC::c20;
    case 8: return YC::c22;
    case 9: case 15: return YC::c33;
    case 10: return YC::c32;
    case 11: case 13: return YC::c31;
    case 12: return YC::c30;
    case 14: return YC::c3p2;
    case 16: return YC::c44m;
    case 17: case 23: return YC::c43;
    case 18: return YC::c42m;
    case 19: case 21: return YC::c41;
    case 20: return YC::c40;
    case 22: return YC::c42;
    case 24: return YC::c44;
    default: return 1.0;
  }
}

// P_i(x, y, z), the homogeneous polynomial of Y_i without its normalisation
// (L <= 4; L > 4: the normalised solid-harmonic values).
template <int L, typename T>
SUS2_HD void sh_poly(T x, T y, T z, T* P) {
  if constexpr (L > 4) {
    sh_values_solid<L>(x, y, z, P);
    return;
  }
  P[0] = T(1);
  if (L < 1) return;
  P[1] = y;
  P[2] = z;
  P[3] = x;
  if (L < 2) return;
  const T x2 = x * x, y2 = y * y, z2 = z * z;
  P[4] = x * y;
  P[5] = y * z;
  P[6] = T(2) * z2 - x2 - y2;
  P[7] = x * z;
  P[8] = x2 - y2;
  if (L < 3) return;
  const T a31 = T(4) * z2 - x2 - y2;
  P[9] = y * (T(3) * x2 - y2);
  P[10] = x * y * z;
  P[11] = y * a31;
  P[12] = z * (T(2) * z2 - T(3) * x2 - T(3) * y2);
  P[13] = x * a31;
  P[14] = z * (x2 - y2);
  P[15] = x * (x2 - T(3) * y2);
  if (L < 4) return;
  const T r2 = x2 + y2;
  P[16] = x * y * (x2 - y2);
  P[17] = y * z * (T(3) * x2 - y2);
  P[18] = x * y * (T(6) * z2 - r2);
  P[19] = y * z * (T(4) * z2 - T(3) * r2);
  P[20] = T(8) * z2 * z2 - T(24) * z2 * r2 + T(3) * r2 * r2;
  P[21] = x * z * (T(4) * z2 - T(3) * r2);
  P[22] = (x2 - y2) * (T(6) * z2 - r2);
  P[23] = x * z * (x2 - T(3) * y2);
  P[24] = x2 * x2 - T(6) * x2 * y2 + y2 * y2;
}

// V = sum_i G[i] grad P_i (L <= 4; L > 4: gradients of the normalised solid
// harmonics).
template <int L, typename T>
SUS2_HD void sh_poly_grad_contract(T x, T y, T z, const T* G, T& vx, T& vy, T& vz) {
  if constexpr (L > 4) {
    sh_grad_solid<L>(x, y, z, G, vx, vy, vz);
    return;
  }
  vx = T(0);
  vy = T(0);
  vz = T(0);
  if (L < 1) return;
  vx = G[3];
  vy = G[1];
  vz = G[2];
  if (L < 2) return;
  const T x2 = x * x, y2 = y * y, z2 = z * z;
  {
    const T g4 = G[4], g5 = G[5], g6 = G[6], g7 = G[7], g8 = G[8];
    vx += g4 * y + g7 * z + T(2) * x * (g8 - g6);
    vy += g4 * x + g5 * z - T(2) * y * (g6 + g8);
    vz += g5 * y + g7 * x + T(4) * z * g6;
  }
  if (L < 3) return;
  {
    const T g9 = G[9], g10 = G[10], g11 = G[11], g12 = G[12], g13 = G[13], g14 = G[14], g15 = G[15];
    const T xy = x * y, xz = x * z, yz = y * z;
    // P9 = y(3x^2-y^2): (6xy, 3x^2-3y^2, 0)
    // P10 = xyz: (yz, xz, xy)
    // P11 = y(4z^2-x^2-y^2): (-2xy, 4z^2-x^2-3y^2, 8yz)
    // P12 = z(2z^2-3x^2-3y^2): (-6xz, -6yz, 6z^2-3x^2-3y^2)
    // P13 = x(4z^2-x^2-y^2): (4z^2-3x^2-y^2, -2xy, 8xz)
    // P14 = z(x^2-y^2): (2xz, -2yz, x^2-y^2)
    // P15 = x(x^2-3y^2): (3x^2-3y^2, -6xy, 0)
    vx += T(6) * xy * g9 + yz * g10 - T(2) * xy * g11 - T(6) * xz * g12 +
          (T(4) * z2 - T(3) * x2 - y2) * g13 + T(2) * xz * g14 + T(3) * (x2 - y2) * g15;
    vy += T(3) * (x2 - y2) * g9 + xz * g10 + (T(4) * z2 - x2 - T(3) * y2) * g11 -
          T(6) * yz * g12 - T(2) * xy * g13 - T(2) * yz * g14 - T(6) * xy * g15;
    vz += xy * g10 + T(8) * yz * g11 + (T(6) * z2 - T(3) * x2 - T(3) * y2) * g12 +
          T(8) * xz * g13 + (x2 - y2) * g14;
  }
  if (L < 4) return;
  {
    const T g16 = G[16], g17 = G[17], g18 = G[18], g19 = G[19], g20 = G[20];
    const T g21 = G[21], g22 = G[22], g23 = G[23], g24 = G[24];
    const T xyz = x * y * z, r2 = x2 + y2;
    // P16 = x^3 y - x y^3
    vx += g16 * (T(3) * x2 * y - y * y2);
    vy += g16 * (x * x2 - T(3) * x * y2);
    // P17 = 3x^2 yz - y^3 z
    vx += g17 * T(6) * xyz;
    vy += g17 * (T(3) * x2 * z - T(3) * y2 * z);
    vz += g17 * (T(3) * x2 * y - y * y2);
    // P18 = 6xyz^2 - x^3 y - x y^3
    vx += g18 * (T(6) * y * z2 - T(3) * x2 * y - y * y2);
    vy += g18 * (T(6) * x * z2 - x * x2 - T(3) * x * y2);
    vz += g18 * T(12) * xyz;
    // P19 = 4yz^3 - 3x^2 yz - 3y^3 z
    vx += g19 * (-T(6) * xyz);
    vy += g19 * (T(4) * z * z2 - T(3) * x2 * z - T(9) * y2 * z);
    vz += g19 * (T(12) * y * z2 - T(3) * x2 * y - T(3) * y * y2);
    // P20 = 8z^4 - 24 z^2 r2 + 3 r2^2, r2 = x^2 + y^2
    const T a40 = T(12) * r2 - T(48) * z2;
    vx += g20 * a40 * x;
    vy += g20 * a40 * y;
    vz += g20 * (T(32) * z * z2 - T(48) * z * r2);
    // P21 = 4xz^3 - 3x^3 z - 3x y^2 z
    vx += g21 * (T(4) * z * z2 - T(9) * x2 * z - T(3) * y2 * z);
    vy += g21 * (-T(6) * xyz);
    vz += g21 * (T(12) * x * z2 - T(3) * x * x2 - T(3) * x * y2);
    // P22 = 6x^2 z^2 - 6y^2 z^2 - x^4 + y^4
    vx += g22 * (T(12) * x * z2 - T(4) * x * x2);
    vy += g22 * (T(4) * y * y2 - T(12) * y * z2);
    vz += g22 * (T(12) * (x2 - y2) * z);
    // P23 = x^3 z - 3x y^2 z
    vx += g23 * (T(3) * x2 * z - T(3) * y2 * z);
    vy += g23 * (-T(6) * xyz);
    vz += g23 * (x * x2 - T(3) * x * y2);
    // P24 = x^4 - 6x^2 y^2 + y^4
    vx += g24 * (T(4) * x * x2 - T(12) * x * y2);
    vy += g24 * (T(4) * y * y2 - T(12) * x2 * y);
  }
}

// Y[l*l+l+m] for l <= L at unit vector (x, y, z).
template <int L, typename T>
SUS2_HD void sh_values(T x, T y, T z, T* Y) {
  constexpr int C = (L + 1) * (L + 1);
  sh_poly<L>(x, y, z, Y);
  if constexpr (L <= 4) {
#pragma unroll
    for (int i = 0; i < C; ++i) Y[i] = T(sh_poly_norm<L>(i)) * Y[i];
  }
}

// V = sum_lm G[lm] * grad P_lm(u), P_lm the homogeneous polynomial of Y_lm
// (normalisation included).
template <int L, typename T>
SUS2_HD void sh_grad_contract(T x, T y, T z, const T* G, T& vx, T& vy, T& vz) {
  if constexpr (L > 4) {
    sh_grad_solid<L>(x, y, z, G, vx, vy, vz);
  } else {
    constexpr int C = (L + 1) * (L + 1);
    T Gs[C];
#pragma unroll
    for (int i = 0; i < C; ++i) Gs[i] = T(sh_poly_norm<L>(i)) * G[i];
    sh_poly_grad_contract<L>(x, y, z, Gs, vx, vy, vz);
  }
}

// Radial argument map xi(z) and d xi / dz.
template <typename T>
SUS2_HD void radial_map(T z, bool rational, T& xi, T& dxi_dz) {
  if (rational) {
    const T q = T(1) / sqrt(T(1) + z * z);
    xi = z * q;
    dxi_dz = q * q * q;
  } else {
    xi = tanh(z);
    dxi_dz = T(1) - xi * xi;
  }
}

// Radial basis kinds (RadialSetup::kind): the Chebyshev basis of the tanh map
// (RBChebyshev_sss), of the rational map (RBChebyshev_sss_rational), and the
// Laguerre basis of u = scal log(1 + r / rho) under the envelope exp(-u/2)
// (RBLaguerre_log1p, src/force/sus2_sh.cu:363-374,3299-3352: the reference's
// phi_n = (r - rc)^2 exp(-u/2) L_n(u), rho = max(shift, 1e-8)).
constexpr int kRadialTanh = 0;
constexpr int kRadialRational = 1;
constexpr int kRadialLaguerre = 2;
constexpr double kLaguerreMinRho = 1.0e-8;

// The polynomial argument x of one radial function at distance r (FP64), with
// dx/dr, the envelope env (1 for the Chebyshev kinds) and (d env / dr) / env.
template <typename T>
SUS2_HD void radial_arg(int kind, T scal, T shift, double r, T& x, T& dx_dr, T& env, T& denv_rel) {
  if (kind == kRadialLaguerre) {
    const double rho = static_cast<double>(shift) > kLaguerreMinRho ? static_cast<double>(shift) : kLaguerreMinRho;
    const T u = scal * log1p(static_cast<T>(r / rho));
    x = u;
    dx_dr = scal / static_cast<T>(rho + r);
    env = exp(T(-0.5) * u);
    denv_rel = T(-0.5) * dx_dr;
  } else {
    const T half = T(0.5) * scal;
    T dxi;
    radial_map<T>(half * static_cast<T>(r - static_cast<double>(shift)), kind == kRadialRational, x, dxi);
    dx_dr = half * dxi;
    env = T(1);
    denv_rel = T(0);
  }
}

// Chebyshev T_n(xi), n < RB.
template <int RB, typename T>
SUS2_HD void chebyshev(T xi, T* t) {
  t[0] = T(1);
  if (RB > 1) t[1] = xi;
#pragma unroll
  for (int n = 2; n < RB; ++n) t[n] = T(2) * xi * t[n - 1] - t[n - 2];
}

// T_n(xi) and dT_n/dxi, n < RB.
template <int RB, typename T>
SUS2_HD void chebyshev_d(T xi, T* t, T* dt) {
  t[0] = T(1);
  dt[0] = T(0);
  if (RB > 1) {
    t[1] = xi;
    dt[1] = T(1);
  }
#pragma unroll
  for (int n = 2; n < RB; ++n) {
    t[n] = T(2) * xi * t[n - 1] - t[n - 2];
    dt[n] = T(2) * (t[n - 1] + xi * dt[n - 1]) - dt[n - 2];
  }
}

// Laguerre L_n(u), n < RB: L_0 = 1, L_1 = 1 - u,
// (n+1) L_{n+1} = (2n+1-u) L_n - n L_{n-1}.
template <int RB, typename T>
SUS2_HD void laguerre(T u, T* t) {
  t[0] = T(1);
  if (RB > 1) t[1] = T(1) - u;
#pragma unroll
  for (int n = 1; n + 1 < RB; ++n)
    t[n + 1] = ((T(2 * n + 1) - u) * t[n] - T(n) * t[n - 1]) * T(1.0 / (n + 1));
}

// L_n(u) and dL_n/du, n < RB.
template <int RB, typename T>
SUS2_HD void laguerre_d(T u, T* t, T* dt) {
  t[0] = T(1);
  dt[0] = T(0);
  if (RB > 1) {
    t[1] = T(1) - u;
    dt[1] = T(-1);
  }
#pragma unroll
  for (int n = 1; n + 1 < RB; ++n) {
    const T inv = T(1.0 / (n + 1));
    t[n + 1] = ((T(2 * n + 1) - u) * t[n] - T(n) * t[n - 1]) * inv;
    dt[n + 1] = ((T(2 * n + 1) - u) * dt[n] - t[n] - T(n) * dt[n - 1]) * inv;
  }
}

// The basis polynomials of a kind at argument x (and their x-derivatives).
template <int RB, typename T>
SUS2_HD void radial_poly(int kind, T x, T* t) {
  if (kind == kRadialLaguerre) laguerre<RB>(x, t);
  else chebyshev<RB>(x, t);
}
template <int RB, typename T>
SUS2_HD void radial_poly_d(int kind, T x, T* t, T* dt) {
  if (kind == kRadialLaguerre) laguerre_d<RB>(x, t, dt);
  else chebyshev_d<RB>(x, t, dt);
}

}  // namespace sus2sh
