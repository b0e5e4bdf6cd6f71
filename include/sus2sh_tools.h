/*
 * sus2sh_tools.h - libsus2sh_tools.so, a library beside the engine (not part
 * of libsus2sh.so): helpers that GPUMD itself provides in a real run
 * (structure set-up, the NVE integrator) or that the tests and the benchmark
 * need (seeded synthetic models, graph statistics, the CUDA-core FMA peak).
 * None of these are part of the drop-in boundary in sus2sh.h.  Errors:
 * return codes of sus2sh.h; the message of the last failed call from
 * sus2sh_tools_last_error().
 */
#ifndef SUS2SH_TOOLS_H
#define SUS2SH_TOOLS_H

#ifdef __cplusplus
extern "C" {
#endif

const char* sus2sh_tools_last_error(void);

/* Writes a seeded SUS2-SH v1.1.0 model with the standard real-CG product
 * graph for (l_max, k_max, body_order[, body_l_max]) and random coefficients:
 * radial ~ N(0, radial_sigma), moment weights ~ N(0, moment_sigma),
 * species_coeffs = 1, every radial (scal, shift) = (scal, rshift) with
 * rshift < 0 meaning (r_min + rc)/2, radial type coefficients = 1.
 * rational selects the radial basis: 0 RBChebyshev_sss, 1
 * RBChebyshev_sss_rational, 2 RBLaguerre_log1p (shift is then rho).
 * body_l_max may be NULL (n_body_l_max = 0). */
int sus2sh_write_synthetic_model(const char* path, int species, int l_max, int k_max,
                                 int body_order, const int* body_l_max, int n_body_l_max,
                                 int rb_size, double r_min, double rc, int rational,
                                 const double* shift_coeffs, double radial_sigma,
                                 double moment_sigma, double scal, double rshift,
                                 unsigned long long seed);

/* Counts of the standard graph (no file): out[0..7] = node_count, basics,
 * products, scalars, tensor_blocks, cg_blocks, cg_terms, max_layer.
 * body_l_max may be NULL. */
int sus2sh_standard_graph_counts(int l_max, int k_max, int body_order, const int* body_l_max,
                                 int n_body_l_max, int* out);

/* Velocity-Verlet halves on device arrays (SoA, A / fs / amu / eV):
 * kick_drift: v += dt/2 F/m; x += dt v; then force (and potential, virial
 * when not NULL) are zeroed for the next accumulating force call.
 * kick: v += dt/2 F/m. */
int sus2sh_md_kick_drift(int N, double dt, const double* inv_mass_type, const int* type,
                         double* force, double* velocity, double* position, double* potential,
                         double* virial, void* stream);
int sus2sh_md_kick(int N, double dt, const double* inv_mass_type, const int* type,
                   const double* force, double* velocity, void* stream);

/* Sum of per-atom energy (out[0]) and per-atom virial (out[1..9]) on device;
 * out is a device array of 10 doubles; virial may be NULL. */
int sus2sh_reduce(int N, const double* potential, const double* virial, double* out, void* stream);

/* FMA-chain microbenchmark of the current device: measured FP32 (fp64 = 0)
 * or FP64 (fp64 = 1) CUDA-core throughput in TFLOP/s (2 flops per FMA).  It is
 * the roofline denominator of the SIMT kernels. */
int sus2sh_measure_fma_peak(int fp64, double* tflops);

/* Random sequential insertion of N points with minimum distance dmin in the
 * orthorhombic box lx*ly*lz (periodic), seeded; writes SoA positions (3N).
 * Returns 0, or a negative value when the insertion budget runs out. */
int sus2sh_random_insertion(int N, double lx, double ly, double lz, double dmin,
                            unsigned long long seed, double* position);

#ifdef __cplusplus
}
#endif

#endif /* SUS2SH_TOOLS_H */
