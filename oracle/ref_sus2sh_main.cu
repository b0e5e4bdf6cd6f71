// Test infrastructure only (oracle): a command-line driver around the
// reference's own SUS2-SH engine (src/force/sus2_sh.cu, compiled unmodified
// against the GPUMD stand-ins in gpumd_stub/).  It calls the engine the way
// GPUMD's Force::compute does (src/force/force.cu:513-519): the potential,
// force and virial arrays are zeroed, then SUS2_SH::compute accumulates into
// them.  The reference reports input errors by printing the message and
// exiting with status 1 (sus2_sh.cu:269-273); this driver keeps that.
//
//   ref_sus2sh load <model.mtp> [options...]
//       constructs the potential (model reading, graph set-up) in host
//       memory and prints "SUS2SH_REF_LOADED"; needs no GPU.
//   ref_sus2sh run <model.mtp> <in.bin> <out.bin> <steps> <warmup> [options...]
//       in.bin : int32 N, int32 pbc[3], double h[9] (row-major, box vectors as
//                columns), int32 type[N], double position[3N] (SoA x, y, z)
//       out.bin: double potential[N], force[3N], virial[9N] of the last call
//       prints {"ref_ms_per_step": mean, "ref_ms_median", "ref_ms_min",
//       "ref_ms_max", "steps": K, "N": N}: CUDA-event times of SUS2_SH::compute
//       over the K calls after `warmup` untimed ones.
// Options are the run.in tokens after the file name: species symbols first,
// then the reference's own switches (sus2_float=0|1, sus2_sh_profile=1, ...).
#include "sus2_sh.cuh"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace {

template <typename T>
void read_exact(std::FILE* f, T* p, size_t n) {
  if (std::fread(p, sizeof(T), n, f) != n) {
    std::printf("ref_sus2sh: short input file\n");
    std::exit(2);
  }
}

int usage() {
  std::printf("usage: ref_sus2sh load <model> [opts...] | run <model> <in.bin> <out.bin> <steps> <warmup> [opts...]\n");
  return 2;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) return usage();
  const std::string mode = argv[1];
  const char* model = argv[2];
  if (mode == "load") {
    gpumd_stub_host_memory() = true;
    std::vector<const char*> opts(argv + 3, argv + argc);
    SUS2_SH pot(model, 1, static_cast<int>(opts.size()), opts.empty() ? nullptr : opts.data());
    std::printf("SUS2SH_REF_LOADED\n");
    return 0;
  }
  if (mode != "run" || argc < 7) return usage();
  const int steps = std::atoi(argv[5]);
  const int warmup = std::atoi(argv[6]);
  std::vector<const char*> opts(argv + 7, argv + argc);

  std::FILE* in = std::fopen(argv[3], "rb");
  if (!in) {
    std::printf("ref_sus2sh: cannot open %s\n", argv[3]);
    return 2;
  }
  int N = 0, pbc[3];
  double h[9];
  read_exact(in, &N, 1);
  read_exact(in, pbc, 3);
  read_exact(in, h, 9);
  std::vector<int> type(N);
  std::vector<double> pos(3 * static_cast<size_t>(N));
  read_exact(in, type.data(), type.size());
  read_exact(in, pos.data(), pos.size());
  std::fclose(in);

  Box box;
  box.set(h, pbc[0], pbc[1], pbc[2]);
  GPU_Vector<int> d_type(N);
  GPU_Vector<double> d_pos(3 * static_cast<size_t>(N));
  GPU_Vector<double> d_pe(N), d_f(3 * static_cast<size_t>(N)), d_vir(9 * static_cast<size_t>(N));
  d_type.copy_from_host(type.data());
  d_pos.copy_from_host(pos.data());

  SUS2_SH pot(model, N, static_cast<int>(opts.size()), opts.empty() ? nullptr : opts.data());
  cudaEvent_t e0, e1;
  CHECK(cudaEventCreate(&e0));
  CHECK(cudaEventCreate(&e1));
  double total_ms = 0.0;
  std::vector<float> step_ms;
  for (int s = 0; s < warmup + steps; ++s) {
    CHECK(cudaMemset(d_pe.data(), 0, sizeof(double) * d_pe.size()));
    CHECK(cudaMemset(d_f.data(), 0, sizeof(double) * d_f.size()));
    CHECK(cudaMemset(d_vir.data(), 0, sizeof(double) * d_vir.size()));
    CHECK(cudaEventRecord(e0));
    pot.compute(box, d_type, d_pos, d_pe, d_f, d_vir);
    CHECK(cudaEventRecord(e1));
    CHECK(cudaEventSynchronize(e1));
    float ms = 0.0f;
    CHECK(cudaEventElapsedTime(&ms, e0, e1));
    if (s >= warmup) {
      total_ms += ms;
      step_ms.push_back(ms);
    }
  }
  CHECK(cudaGetLastError());
  std::vector<double> pe(N), f(3 * static_cast<size_t>(N)), vir(9 * static_cast<size_t>(N));
  d_pe.copy_to_host(pe.data());
  d_f.copy_to_host(f.data());
  d_vir.copy_to_host(vir.data());
  std::FILE* out = std::fopen(argv[4], "wb");
  if (!out) {
    std::printf("ref_sus2sh: cannot write %s\n", argv[4]);
    return 2;
  }
  std::fwrite(pe.data(), sizeof(double), pe.size(), out);
  std::fwrite(f.data(), sizeof(double), f.size(), out);
  std::fwrite(vir.data(), sizeof(double), vir.size(), out);
  std::fclose(out);
  std::vector<float> sorted = step_ms;
  std::sort(sorted.begin(), sorted.end());
  const double med = sorted.empty() ? 0.0 : sorted[sorted.size() / 2];
  const double lo = sorted.empty() ? 0.0 : sorted.front(), hi = sorted.empty() ? 0.0 : sorted.back();
  std::printf("{\"ref_ms_per_step\": %.6f, \"ref_ms_median\": %.6f, \"ref_ms_min\": %.6f, \"ref_ms_max\": %.6f, "
              "\"steps\": %d, \"N\": %d}\n",
              steps > 0 ? total_ms / steps : 0.0, med, lo, hi, steps, N);
  return 0;
}
