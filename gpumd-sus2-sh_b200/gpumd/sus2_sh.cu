// GPUMD drop-in for src/force/sus2_sh.cu (see sus2_sh.cuh).  Input errors end
// the run through PRINT_INPUT_ERROR with the engine's message, as the
// reference's sh_input_error does (src/force/sus2_sh.cu:269-273).
#include "sus2_sh.cuh"
#include "utilities/error.cuh"

#include <cstdio>

bool is_sus2_sh_potential_file(const char* file_potential)
{
  return sus2sh_is_sus2_sh_file(file_potential) == 1;
}

SUS2_SH::SUS2_SH(
  const char* file_potential,
  int num_atoms,
  int num_potential_options,
  const char** potential_options)
{
  if (sus2sh_create(file_potential, num_atoms, num_potential_options, potential_options, &handle_) !=
      SUS2SH_OK) {
    PRINT_INPUT_ERROR(sus2sh_last_error());
  }
  rc = sus2sh_cutoff(handle_);
}

SUS2_SH::~SUS2_SH(void) { sus2sh_destroy(handle_); }

void SUS2_SH::compute(
  Box& box,
  const GPU_Vector<int>& type,
  const GPU_Vector<double>& position,
  GPU_Vector<double>& potential,
  GPU_Vector<double>& force,
  GPU_Vector<double>& virial)
{
  const int N = static_cast<int>(type.size());
  const int pbc[3] = {box.pbc_x, box.pbc_y, box.pbc_z};
  // GPUMD launches on the default stream; so does the engine here
  if (sus2sh_compute(handle_, N, box.cpu_h, pbc, type.data(), position.data(), potential.data(),
                     force.data(), virial.data(), nullptr) != SUS2SH_OK) {
    PRINT_INPUT_ERROR(sus2sh_last_error());
  }
  int flags = 0;
  const int status = sus2sh_sync(handle_, &flags);
  if (status == SUS2SH_E_NEIGHBOR) {
    // A rebuild found more neighbours than the list holds; the engine has
    // grown it.  The arrays hold this step's partial contribution: in GPUMD's
    // single-potential ("observe") mode they held nothing before this call,
    // so they are cleared and the step is computed again.
    ++recomputed_steps_;
    std::printf("SUS2_SH: neighbour list capacity grown; step recomputed.\n");
    potential.fill(0.0);
    force.fill(0.0);
    virial.fill(0.0);
    if (sus2sh_compute(handle_, N, box.cpu_h, pbc, type.data(), position.data(), potential.data(),
                       force.data(), virial.data(), nullptr) != SUS2SH_OK ||
        sus2sh_sync(handle_, &flags) != SUS2SH_OK) {
      PRINT_INPUT_ERROR(sus2sh_last_error());
    }
  } else if (status != SUS2SH_OK) {
    PRINT_INPUT_ERROR(sus2sh_last_error());
  }
}
