/*
 * sus2sh_diag.h - diagnostics of libsus2sh.so: reports of the kernels the
 * engine compiles for a model and host evaluations of the engine's own
 * harmonics and ZBL pair function, for tests and profiling.  None is needed
 * by the GPUMD shim.
 */
#ifndef SUS2SH_DIAG_H
#define SUS2SH_DIAG_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Generates and NVRTC-compiles (sm_100a, no GPU needed) the model-specialised
 * CG product kernel the engine would build for a model file (split: -1 as the
 * engine chooses, 0 never / 1 always the component-split kernel, 2 the
 * forward-over-reverse product kernel of the parameter gradients, 3 the
 * component-split kernel compiled as parallel relocatable units, as option
 * sus2_sh_cg_whole=0 does; otherwise one program, through the engine's
 * on-disk cache of one-program builds): info[0]
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

/* Compiles, as the first sus2sh_compute_batch of an FP32 handle with option
 * sus2_sh_batch_fused=1 does, the fused persistent batch kernel of a model
 * file (its radial coefficients and
 * straight-line CG contraction compiled in; 128-thread CTAs with 3 and with
 * 2 resident CTAs per SM).  info[0] [1] registers per thread of the two
 * variants, [2] compile ms, [3] cubin bytes.  An input error for models whose
 * graph takes the component-split CG kernel.  log (if not NULL) receives the
 * ptxas report.  Needs no GPU.  No reference counterpart. */
int sus2sh_batch_kernel_info(const char* path, int* info, char* log, size_t log_len);

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

#ifdef __cplusplus
}
#endif

#endif /* SUS2SH_DIAG_H */
