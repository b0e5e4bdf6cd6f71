// GPUMD drop-in for src/force/sus2_sh.cuh: the SUS2_SH potential class with
// the reference's constructor and compute signatures (src/force/sus2_sh.cuh:
// 7-25), forwarding to this repository's engine through its C-ABI
// (include/sus2sh.h).  Force::parse_potential (src/force/force.cu:113-119)
// selects and constructs it unchanged.
#pragma once
#include "potential.cuh"
#include "utilities/gpu_vector.cuh"

#include "sus2sh.h"

class SUS2_SH : public Potential
{
public:
  using Potential::compute;

  SUS2_SH(
    const char* file_potential,
    int num_atoms,
    int num_potential_options = 0,
    const char** potential_options = nullptr);
  virtual ~SUS2_SH(void);

  // Accumulates per-atom energies, forces and virials (GPUMD zeroes the
  // arrays before the first potential, src/force/force.cu:513-519).
  virtual void compute(
    Box& box,
    const GPU_Vector<int>& type,
    const GPU_Vector<double>& position,
    GPU_Vector<double>& potential,
    GPU_Vector<double>& force,
    GPU_Vector<double>& virial);

  // Steps recomputed because a neighbour rebuild outgrew the list capacity.
  int recomputed_steps() const { return recomputed_steps_; }

private:
  sus2sh_handle* handle_ = nullptr;
  int recomputed_steps_ = 0;
};

// src/force/sus2_sh.cu:7771-7780
bool is_sus2_sh_potential_file(const char* file_potential);
