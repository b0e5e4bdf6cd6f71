// Test infrastructure only (oracle): the abstract potential interface the
// reference's SUS2-SH class derives from (src/force/sus2_sh.cuh:7-25): one
// virtual compute over the box, species, SoA positions and the FP64
// potential/force/virial arrays, which the caller zeroes before the call.
#pragma once
#include "box.cuh"
#include "utilities/gpu_vector.cuh"

class Potential {
public:
  int N1 = 0;
  int N2 = 0;
  double rc = 0.0;
  virtual ~Potential() = default;
  virtual void compute(Box& box, const GPU_Vector<int>& type, const GPU_Vector<double>& position,
                       GPU_Vector<double>& potential, GPU_Vector<double>& force,
                       GPU_Vector<double>& virial) = 0;
};
