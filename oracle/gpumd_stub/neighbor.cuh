// Test infrastructure only (oracle): a stand-in for GPUMD's neighbour search
// with the three members the reference's SUS2-SH engine calls
// (src/force/sus2_sh.cu:9336,9583-9585).  It writes GPUMD's full-list layout:
// NN[i] neighbours of atom i, NL[k * N + i] the k-th one, every pair listed
// from both ends, r^2 < rc^2 by the minimum image.  The engine uses it only
// for boxes at least twice the cutoff thick along every periodic axis (it
// switches to its own image kernels otherwise), so the minimum image is the
// only image within rc.  Buffers are kept between calls and grow only with
// N, so a call allocates nothing in the steady state.
#pragma once
#include "box.cuh"
#include "utilities/gpu_vector.cuh"

class Neighbor {
public:
  void initialize(double rc, int N, int max_nbr);
  void find_neighbor_global(double rc, Box& box, const GPU_Vector<int>& type,
                            const GPU_Vector<double>& position);
  void find_local_neighbor_from_global(double rc, Box& box, const GPU_Vector<double>& position,
                                       GPU_Vector<int>& NN, GPU_Vector<int>& NL);

private:
  int max_nbr_ = 512;
  int nb_[3] = {1, 1, 1};     // cells per axis
  GPU_Vector<int> cell_;        // cell of each atom
  GPU_Vector<int> keys_;        // cell keys sorted along with order_
  GPU_Vector<int> index_;       // 0..N-1
  GPU_Vector<int> order_;       // atoms sorted by cell (stable: by index within a cell)
  GPU_Vector<int> start_;       // first sorted position of each cell
  GPU_Vector<int> count_;       // atoms per cell
  GPU_Vector<int> overflow_;    // [0] overflow flag
  GPU_Vector<unsigned char> temp_;  // sort/scan scratch, kept between calls
};
