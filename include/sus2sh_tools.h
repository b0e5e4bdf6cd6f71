/*
 * sus2sh_tools.h - helpers around the engine that GPUMD itself provides in a
 * real run (structure set-up, the NVE integrator) or that the tests and the
 * benchmark need (seeded synthetic models, graph statistics).  None of these
 * are part of the drop-in boundary in sus2sh.h.
 */
#ifndef SUS2SH_TOOLS_H
#define SUS2SH_TOOLS_H

#ifdef __cplusplus
extern "C" {
#endif

/* Writes a seeded SUS2-SH v1.1.0 model with the standard real-CG product
 * graph for (l_max, k_max, body_order[, body_l_max]) and random coefficients:
 * radial ~ N(0, radial_sigma), moment weights ~ N(0, moment_sigma),
 * species_coeffs = 1, every radial (scal, shift) = (scal, rshift) with
 * rshift < 0 meaning (r_min + rc)/2, radial type coefficients = 1.
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

/* Generates and NVRTC-compiles (sm_100a, no GPU needed) the model-specialised
 * CG product kernel the engine would build for a model file (split: -1 as the
 * engine chooses, 0 never / 1 always the component-split kernel, 2 the
 * forward-over-reverse product kernel of the parameter gradients): info[0]
 * registers per thread, [1] spill store bytes, [2] emitted multiply-add terms,
 * [3] generate+compile ms, [4] cubin bytes, [5] 1 for a component-split
 * kernel, [6] device functions, [7] components, [8] threads per CTA, [9]
 * dynamic shared memory bytes.  text (if not NULL) receives the ptxas report
 * (use_float < 0: the generated FP32 source instead).  Graphs that get no CG
 * kernel (the engine runs the row interpreter) return SUS2SH_E_INPUT. */
int sus2sh_cg_kernel_info(const char* path, int use_float, int split, int* info, char* text,
                          size_t text_size);

/* Compiles the per-edge kernels (k_basic, k_force, 128-thread CTAs) of one
 * model shape with NVRTC for sm_100a, as model load does for shapes without
 * an ahead-of-time build, and reports their register counts, the compile time
 * and the compiler log (truncated to log_len).  Needs no GPU.  No reference
 * counterpart (the reference dispatches among fixed kernels). */
int sus2sh_edge_kernel_info(int fp32, int l_max, int k_max, int rb, int* basic_registers, int* force_registers,
                            double* compile_ms, char* log, size_t log_len);

/* Compiles, as FP32 model load does (option sus2_sh_model_edges, on by
 * default), the per-edge kernels specialised to the radial coefficients of a
 * model file (k_basic, k_force at 64, 128 and 256 threads per CTA; each
 * coefficient and derivative-series coefficient an immediate operand).
 * info[0] k_basic and [1] k_force registers per thread (64-thread CTAs),
 * [2] compile ms, [3] bytes of module data in global memory (as for the
 * shape's build without the table: every coefficient folded into the
 * instructions), [4] coefficient-table entries, [5] cubin bytes.  log (if not NULL) receives the ptxas report.  Needs no
 * GPU.  No reference counterpart. */
int sus2sh_model_edge_kernel_info(const char* path, int* info, char* log, size_t log_len);

/* The engine's real spherical harmonics, evaluated on the host in FP64: Y at
 * the unit vector (x, y, z) for every l <= l_max (l_max <= 6, flat index
 * l*l + l + m) and, when G and V are non-NULL, V = sum_lm G[lm] grad P_lm
 * (P_lm the homogeneous polynomial of Y_lm).  No reference counterpart; the
 * reference evaluates them inside its kernels (eval_real_sh,
 * src/force/sus2_sh.cu:2880-3169). */
int sus2sh_real_sh(int l_max, double x, double y, double z, double* Y, const double* G, double* V);

/* The engine's ZBL pair function (energy and dE/dr at distance r for atomic
 * numbers zi, zj and the pair's inner/outer cutoffs), for checks against the
 * reference's sus2_zbl_pair. */
int sus2sh_zbl_pair(int zi, int zj, double r, double inner, double outer, double* energy, double* dEdr);

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
