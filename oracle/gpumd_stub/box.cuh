// Test infrastructure only (oracle): a minimal stand-in for GPUMD's simulation
// box, written for compiling the reference's SUS2-SH engine
// (src/force/sus2_sh.cu) without the GPUMD tree.  It carries exactly what that
// file reads: cpu_h (h row-major, the box vectors as columns, then h^-1),
// pbc_x/y/z, thickness_x/y/z, get_area, get_volume, and the device
// minimum-image function apply_mic (sus2_sh.cu:3483).
#pragma once
#include <cmath>

class Box {
public:
  double cpu_h[18] = {};  // [0..8] h, [9..17] h^-1
  int pbc_x = 1;
  int pbc_y = 1;
  int pbc_z = 1;
  double thickness_x = 0.0;
  double thickness_y = 0.0;
  double thickness_z = 0.0;

  // Sets h (row-major 3x3, columns a, b, c) and derives h^-1 and thicknesses.
  void set(const double h[9], int px, int py, int pz) {
    for (int k = 0; k < 9; ++k) cpu_h[k] = h[k];
    const double* m = cpu_h;
    const double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                       m[2] * (m[3] * m[7] - m[4] * m[6]);
    double* inv = cpu_h + 9;
    inv[0] = (m[4] * m[8] - m[5] * m[7]) / det;
    inv[1] = (m[2] * m[7] - m[1] * m[8]) / det;
    inv[2] = (m[1] * m[5] - m[2] * m[4]) / det;
    inv[3] = (m[5] * m[6] - m[3] * m[8]) / det;
    inv[4] = (m[0] * m[8] - m[2] * m[6]) / det;
    inv[5] = (m[2] * m[3] - m[0] * m[5]) / det;
    inv[6] = (m[3] * m[7] - m[4] * m[6]) / det;
    inv[7] = (m[1] * m[6] - m[0] * m[7]) / det;
    inv[8] = (m[0] * m[4] - m[1] * m[3]) / det;
    pbc_x = px;
    pbc_y = py;
    pbc_z = pz;
    const double v = get_volume();
    thickness_x = v / get_area(0);
    thickness_y = v / get_area(1);
    thickness_z = v / get_area(2);
  }

  double get_volume() const {
    const double* m = cpu_h;
    return std::fabs(m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                     m[2] * (m[3] * m[7] - m[4] * m[6]));
  }

  // Area of the face spanned by the two box vectors other than vector d.
  double get_area(int d) const {
    const int a = (d + 1) % 3, b = (d + 2) % 3;
    const double ux = cpu_h[a], uy = cpu_h[3 + a], uz = cpu_h[6 + a];
    const double wx = cpu_h[b], wy = cpu_h[3 + b], wz = cpu_h[6 + b];
    const double cx = uy * wz - uz * wy, cy = uz * wx - ux * wz, cz = ux * wy - uy * wx;
    return std::sqrt(cx * cx + cy * cy + cz * cz);
  }
};

// Minimum image of a displacement: fractional coordinates rounded to the
// nearest integer along periodic axes, in the precision of the arguments (the
// reference calls it with float and with double displacements).
template <typename T>
static __host__ __device__ __forceinline__ void apply_mic(const Box& box, T& x12, T& y12, T& z12) {
  const double* h = box.cpu_h;
  T sx = T(h[9]) * x12 + T(h[10]) * y12 + T(h[11]) * z12;
  T sy = T(h[12]) * x12 + T(h[13]) * y12 + T(h[14]) * z12;
  T sz = T(h[15]) * x12 + T(h[16]) * y12 + T(h[17]) * z12;
  if (box.pbc_x == 1) sx -= rint(sx);
  if (box.pbc_y == 1) sy -= rint(sy);
  if (box.pbc_z == 1) sz -= rint(sz);
  x12 = T(h[0]) * sx + T(h[1]) * sy + T(h[2]) * sz;
  y12 = T(h[3]) * sx + T(h[4]) * sy + T(h[5]) * sz;
  z12 = T(h[6]) * sx + T(h[7]) * sy + T(h[8]) * sz;
}
