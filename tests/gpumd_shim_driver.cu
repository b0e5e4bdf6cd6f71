// Test driver of the engine's GPUMD shim (gpumd-sus2-sh_b200/gpumd/sus2_sh.cu),
// built against the GPUMD stand-ins of oracle/gpumd_stub and libsus2sh.so.
// It calls the shim as GPUMD's Force::compute does (src/force/force.cu:
// 513-519: the per-atom arrays zeroed, then SUS2_SH::compute), once per frame:
//   gpumd_shim_driver <model.mtp> <in.bin> <out.bin> [options...]
//   in.bin : int32 N, int32 pbc[3], double h[9], int32 type[N], int32 frames,
//            then per frame double position[3N] (SoA)
//   out.bin: per frame double potential[N], force[3N], virial[9N]
// and prints {"recomputed_steps": n, "rc": rc}.
#include "sus2_sh.cuh"

#include <cstdio>
#include <vector>

int main(int argc, char** argv) {
  if (argc < 4) {
    std::printf("usage: gpumd_shim_driver <model> <in.bin> <out.bin> [options...]\n");
    return 2;
  }
  std::FILE* in = std::fopen(argv[2], "rb");
  if (!in) return 2;
  int N = 0, pbc[3], frames = 0;
  double h[9];
  bool ok = std::fread(&N, sizeof(int), 1, in) == 1 && std::fread(pbc, sizeof(int), 3, in) == 3 &&
            std::fread(h, sizeof(double), 9, in) == 9;
  std::vector<int> type(N);
  ok = ok && std::fread(type.data(), sizeof(int), N, in) == static_cast<size_t>(N) &&
       std::fread(&frames, sizeof(int), 1, in) == 1;
  std::vector<double> pos(3 * static_cast<size_t>(N) * frames);
  ok = ok && std::fread(pos.data(), sizeof(double), pos.size(), in) == pos.size();
  std::fclose(in);
  if (!ok) {
    std::printf("gpumd_shim_driver: short input\n");
    return 2;
  }
  std::vector<const char*> opts(argv + 4, argv + argc);
  Box box;
  box.set(h, pbc[0], pbc[1], pbc[2]);
  GPU_Vector<int> d_type(N);
  d_type.copy_from_host(type.data());
  GPU_Vector<double> d_pos(3 * static_cast<size_t>(N)), d_pe(N), d_f(3 * static_cast<size_t>(N)),
    d_vir(9 * static_cast<size_t>(N));
  SUS2_SH pot(argv[1], N, static_cast<int>(opts.size()), opts.empty() ? nullptr : opts.data());
  std::FILE* out = std::fopen(argv[3], "wb");
  if (!out) return 2;
  std::vector<double> pe(N), f(3 * static_cast<size_t>(N)), vir(9 * static_cast<size_t>(N));
  for (int s = 0; s < frames; ++s) {
    d_pos.copy_from_host(pos.data() + 3 * static_cast<size_t>(N) * s);
    d_pe.fill(0.0);
    d_f.fill(0.0);
    d_vir.fill(0.0);
    pot.compute(box, d_type, d_pos, d_pe, d_f, d_vir);
    d_pe.copy_to_host(pe.data());
    d_f.copy_to_host(f.data());
    d_vir.copy_to_host(vir.data());
    std::fwrite(pe.data(), sizeof(double), pe.size(), out);
    std::fwrite(f.data(), sizeof(double), f.size(), out);
    std::fwrite(vir.data(), sizeof(double), vir.size(), out);
  }
  std::fclose(out);
  std::printf("{\"recomputed_steps\": %d, \"rc\": %.17g}\n", pot.recomputed_steps(), pot.rc);
  return 0;
}
