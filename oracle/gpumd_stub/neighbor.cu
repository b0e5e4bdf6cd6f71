// Test infrastructure only (oracle): the neighbour search behind the stand-in
// Neighbor class (neighbor.cuh).  Cell list in fractional coordinates: cells
// at least rc thick along each periodic axis with three or more cells, one
// cell spanning the axis otherwise (open axes, thin axes); atoms sorted by
// cell with a stable radix sort, so lists are deterministic; each atom scans
// its cell's neighbourhood once per distinct cell and tests the
// minimum-image r^2 < rc^2 in FP64.
#include "neighbor.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstdio>

namespace {

__device__ __forceinline__ int stub_cell_coord(double s, int n, int periodic) {
  if (n == 1) return 0;
  if (periodic) s -= floor(s);
  int c = static_cast<int>(floor(s * n));
  return c < 0 ? 0 : (c >= n ? n - 1 : c);
}

__global__ void k_stub_bin(int N, Box box, int nx, int ny, int nz, const double* __restrict__ x,
                           const double* __restrict__ y, const double* __restrict__ z, int* __restrict__ cell,
                           int* __restrict__ count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double* g = box.cpu_h + 9;
  const double sx = g[0] * x[i] + g[1] * y[i] + g[2] * z[i];
  const double sy = g[3] * x[i] + g[4] * y[i] + g[5] * z[i];
  const double sz = g[6] * x[i] + g[7] * y[i] + g[8] * z[i];
  const int c = stub_cell_coord(sx, nx, box.pbc_x) +
                nx * (stub_cell_coord(sy, ny, box.pbc_y) + ny * stub_cell_coord(sz, nz, box.pbc_z));
  cell[i] = c;
  atomicAdd(count + c, 1);
}

__global__ void k_stub_search(int N, Box box, int nx, int ny, int nz, double rc2, const double* __restrict__ x,
                              const double* __restrict__ y, const double* __restrict__ z,
                              const int* __restrict__ cell_of_atom, const int* __restrict__ order,
                              const int* __restrict__ start, const int* __restrict__ count, int max_nbr,
                              int* __restrict__ NN, int* __restrict__ NL, int* __restrict__ overflow) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int c = cell_of_atom[i];
  const int cx = c % nx, cy = (c / nx) % ny, cz = c / (nx * ny);
  // an axis with fewer than three cells is scanned once over all its cells
  const int x0 = nx >= 3 ? -1 : -cx, x1 = nx >= 3 ? 1 : nx - 1 - cx;
  const int y0 = ny >= 3 ? -1 : -cy, y1 = ny >= 3 ? 1 : ny - 1 - cy;
  const int z0 = nz >= 3 ? -1 : -cz, z1 = nz >= 3 ? 1 : nz - 1 - cz;
  const double xi = x[i], yi = y[i], zi = z[i];
  int n = 0;
  for (int dz = z0; dz <= z1; ++dz) {
    const int kz = (cz + dz + nz) % nz;
    for (int dy = y0; dy <= y1; ++dy) {
      const int ky = (cy + dy + ny) % ny;
      for (int dx = x0; dx <= x1; ++dx) {
        const int kx = (cx + dx + nx) % nx;
        const int k = kx + nx * (ky + ny * kz);
        const int b = start[k], e = b + count[k];
        for (int p = b; p < e; ++p) {
          const int j = order[p];
          if (j == i) continue;
          double ddx = x[j] - xi, ddy = y[j] - yi, ddz = z[j] - zi;
          apply_mic(box, ddx, ddy, ddz);
          if (ddx * ddx + ddy * ddy + ddz * ddz < rc2) {
            if (n < max_nbr) NL[static_cast<size_t>(n) * N + i] = j;
            else *overflow = 1;
            ++n;
          }
        }
      }
    }
  }
  NN[i] = n < max_nbr ? n : max_nbr;
}

__global__ void k_stub_iota(int N, int* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N) out[i] = i;
}

}  // namespace

void Neighbor::initialize(double, int, int max_nbr) { max_nbr_ = max_nbr; }

void Neighbor::find_neighbor_global(double rc, Box& box, const GPU_Vector<int>& type,
                                    const GPU_Vector<double>& position) {
  const int N = static_cast<int>(type.size());
  const double thick[3] = {box.thickness_x, box.thickness_y, box.thickness_z};
  const int pbc[3] = {box.pbc_x, box.pbc_y, box.pbc_z};
  for (int d = 0; d < 3; ++d) {
    int n = pbc[d] ? static_cast<int>(std::floor(thick[d] / rc)) : 1;
    n = std::min(std::max(n, 1), 512);
    nb_[d] = n >= 3 ? n : 1;
  }
  const int ncell = nb_[0] * nb_[1] * nb_[2];
  if (cell_.size() != static_cast<size_t>(N)) {
    cell_.resize(N);
    keys_.resize(N);
    index_.resize(N);
    order_.resize(N);
  }
  if (start_.size() < static_cast<size_t>(ncell)) {
    start_.resize(ncell);
    count_.resize(ncell);
  }
  // scratch of the radix sort and the scan, sized once for this N and ncell
  size_t sort_bytes = 0, scan_bytes = 0;
  CHECK(cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, cell_.data(), keys_.data(), index_.data(),
                                        order_.data(), N));
  CHECK(cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, count_.data(), start_.data(), ncell));
  const size_t need = std::max(sort_bytes, scan_bytes);
  if (temp_.size() < need) temp_.resize(need);
  CHECK(cudaMemset(count_.data(), 0, sizeof(int) * ncell));
  const double* x = position.data();
  const int grid = (N + 127) / 128;
  k_stub_bin<<<grid, 128>>>(N, box, nb_[0], nb_[1], nb_[2], x, x + N, x + 2 * N, cell_.data(), count_.data());
  CHECK(cudaGetLastError());
  k_stub_iota<<<grid, 128>>>(N, index_.data());
  CHECK(cudaGetLastError());
  size_t bytes = temp_.size();
  CHECK(cub::DeviceScan::ExclusiveSum(temp_.data(), bytes, count_.data(), start_.data(), ncell));
  bytes = temp_.size();
  CHECK(cub::DeviceRadixSort::SortPairs(temp_.data(), bytes, cell_.data(), keys_.data(), index_.data(),
                                        order_.data(), N));
}

void Neighbor::find_local_neighbor_from_global(double rc, Box& box, const GPU_Vector<double>& position,
                                               GPU_Vector<int>& NN, GPU_Vector<int>& NL) {
  const int N = static_cast<int>(NN.size());
  if (overflow_.size() != 1) overflow_.resize(1);
  CHECK(cudaMemset(overflow_.data(), 0, sizeof(int)));
  // the cell grid of find_neighbor_global is reused (same box and positions)
  const double* x = position.data();
  const int grid = (N + 127) / 128;
  k_stub_search<<<grid, 128>>>(N, box, nb_[0], nb_[1], nb_[2], rc * rc, x, x + N, x + 2 * N, cell_.data(),
                               order_.data(), start_.data(), count_.data(), max_nbr_, NN.data(), NL.data(),
                               overflow_.data());
  CHECK(cudaGetLastError());
  int flag = 0;
  overflow_.copy_to_host(&flag);
  if (flag) {
    std::printf("Error: more than %d neighbours of one atom within %g A.\n", max_nbr_, rc);
    std::exit(1);
  }
}
