/*
 * sus2sh.h - C ABI of the B200 SUS2-SH energy/force/virial engine.
 *
 * This is the drop-in boundary for GPUMD's potential dispatch.  Each entry
 * point names the reference (hu-yanxiao/GPUMD-SUS2-SH) interface it replaces.
 * All device arrays use GPUMD's layouts:
 *   position  double[3N]  SoA  x0..x_{N-1}, y..., z...
 *   type      int[N]      species index in [0, species_count)
 *   potential double[N]   per-atom energy (eV)
 *   force     double[3N]  SoA (eV/A)
 *   virial    double[9N]  SoA, component order xx yy zz xy xz yz yx zx zy
 *   box_h     double[9]   GPUMD Box::cpu_h: columns a=(h0,h3,h6), b=(h1,h4,h7), c=(h2,h5,h8)
 *   pbc       int[3]      1 = periodic
 * sus2sh_compute ACCUMULATES (+=) into potential/force/virial exactly like
 * SUS2_SH::compute; the caller zeroes them (GPUMD's Force::compute does,
 * src/force/force.cu:513-519).
 *
 * Return codes: 0 success, negative error (message via sus2sh_last_error()).
 * A handle is not re-entrant; all work is enqueued on the stream passed in
 * (cudaStream_t given as void*, NULL = legacy default stream).
 */
#ifndef SUS2SH_H
#define SUS2SH_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sus2sh_handle sus2sh_handle;

#define SUS2SH_OK 0
#define SUS2SH_E_INPUT (-1)     /* malformed/unsupported model or options */
#define SUS2SH_E_CUDA (-2)      /* CUDA runtime error */
#define SUS2SH_E_ARG (-3)       /* invalid argument */
#define SUS2SH_E_NEIGHBOR (-4)  /* neighbour capacity exceeded; recompute */

/* status flags returned by sus2sh_sync */
#define SUS2SH_STATUS_OVERFLOW 1
#define SUS2SH_STATUS_BAD_TYPE 2  /* a type was outside [0, species_count) */
#define SUS2SH_STATUS_THIN_CELL 4 /* a batch cell is thinner than half the cutoff */

/* Replaces is_sus2_sh_potential_file (src/force/sus2_sh.cu:7771-7780,
 * declared src/force/sus2_sh.cuh:205): 1 if the file contains
 * "potential_tag = SUS2-SH", else 0. */
int sus2sh_is_sus2_sh_file(const char* path);

/* Replaces SUS2_SH::SUS2_SH(const char* file_potential, int num_atoms,
 * int num_potential_options, const char** potential_options)
 * (src/force/sus2_sh.cuh:12-16, src/force/sus2_sh.cu:7782-9469).
 * opts are the run.in tokens after the model file: the species symbols first,
 * then key=value options (sus2_float=0|1; the reference's tuning switches are
 * accepted and ignored; sus2_sh_skin=<A>, sus2_sh_rebuild_interval=<n>). */
int sus2sh_create(const char* path, int num_atoms, int nopts, const char** opts,
                  sus2sh_handle** out);

/* Replaces SUS2_SH::compute(Box&, const GPU_Vector<int>& type,
 * const GPU_Vector<double>& position, GPU_Vector<double>& potential,
 * GPU_Vector<double>& force, GPU_Vector<double>& virial)
 * (src/force/sus2_sh.cuh:19-25, src/force/sus2_sh.cu:9620-10675).
 * Device pointers; accumulates into potential, force, virial. */
int sus2sh_compute(sus2sh_handle* h, int N, const double box_h[9], const int pbc[3],
                   const int* type, const double* position, double* potential,
                   double* force, double* virial, void* stream);

/* Replaces SUS2_SH::~SUS2_SH (src/force/sus2_sh.cuh:17). */
void sus2sh_destroy(sus2sh_handle* h);

/* Replaces the Potential::rc member the reference sets from max_dist
 * (src/force/sus2_sh.cu:7814). */
double sus2sh_cutoff(const sus2sh_handle* h);

/* Message of the last error on this thread (the reference prints it and
 * exits, src/force/sus2_sh.cu:269-273). */
const char* sus2sh_last_error(void);

/* Waits for the handle's queued work and reports neighbour-list status
 * (SUS2SH_STATUS_OVERFLOW when a list was truncated; the next call then
 * rebuilds with a larger capacity).  The reference has no counterpart: its
 * neighbour capacity is fixed at 512 (src/force/sus2_sh.cuh:68). */
int sus2sh_sync(sus2sh_handle* h, int* status_flags);

/* Forward/backward pair behind the force path (the explicit adjoint of
 * SUS2_SH::compute's basic -> product -> force stages,
 * src/force/sus2_sh.cu:10258-10469).
 * forward:  potential[i] = E_i (assigned, not accumulated).
 * backward: grad_position = sum_i w_i dE_i/dr (assigned; w = grad_potential,
 *           NULL means all ones) and, if virial != NULL, the per-atom virial
 *           of sum_i w_i E_i (assigned).  Uses the state of the last forward. */
int sus2sh_forward(sus2sh_handle* h, int N, const double box_h[9], const int pbc[3],
                   const int* type, const double* position, double* potential, void* stream);
int sus2sh_backward(sus2sh_handle* h, const double* grad_potential, double* grad_position,
                    double* virial, void* stream);

/* Gradient of a loss L(E_i, F_i) with respect to the model's linear weights
 * (moment_coeffs, [alpha_scalar_moments]) and radial coefficients
 * (radial_coeffs without the species columns, [radial_funcs_count][rb], the
 * .mtp order).  The caller passes the upstream weights energy_weight[i] =
 * dL/dE_i ([N], NULL = 0) and force_weight = dL/dF_i ([3N] SoA, NULL = 0);
 * the force part is the forward-over-reverse derivative of dE/dtheta along
 * force_weight (moments recomputed, nothing stored per pair).  Outputs are
 * device arrays, assigned.  The reference has no counterpart (its trainer
 * lives in a separate project); this is the gradient path of the engine. */
int sus2sh_param_grad(sus2sh_handle* h, int N, const double box_h[9], const int pbc[3],
                      const int* type, const double* position, const double* energy_weight,
                      const double* force_weight, double* grad_moment_coeffs,
                      double* grad_radial_coeffs, void* stream);

/* Batch of independent periodic cells in one call (many small training or
 * screening structures).  All arrays are device arrays: cell c holds atoms
 * [cell_offset[c], cell_offset[c+1]) of the concatenated SoA position/type
 * arrays (N = cell_offset[ncells]); cell_h[9c..9c+8] is its box in the
 * box_h layout; cell_pbc[3c..3c+2] its periodicity (NULL = periodic).  Each
 * cell may be as thin as half of rc (images are explicit).  Outputs accumulate
 * like sus2sh_compute; cell_energy [ncells] and cell_virial [9 ncells] (NULL
 * to skip) are assigned.  After the first call with a given (N, ncells) the
 * call neither allocates nor synchronises, so it can be captured in a CUDA
 * graph and replayed.  With the option sus2_sh_batch_fused=1, FP32 models
 * with the straight-line CG kernel (no gate, no ZBL) are evaluated by one
 * persistent kernel instead of the stage kernels (neighbour fill, moments,
 * CG products, forces, per-cell sums), built with NVRTC and tuned at the
 * first batch call.  The reference evaluates one box per call
 * (SUS2_SH::compute, src/force/sus2_sh.cu:9620). */
int sus2sh_compute_batch(sus2sh_handle* h, int N, int ncells, const int* cell_offset,
                         const double* cell_h, const int* cell_pbc, const int* type,
                         const double* position, double* potential, double* force, double* virial,
                         double* cell_energy, double* cell_virial, void* stream);

/* sus2sh_param_grad over a batch of cells (arguments as in
 * sus2sh_compute_batch and sus2sh_param_grad). */
int sus2sh_param_grad_batch(sus2sh_handle* h, int N, int ncells, const int* cell_offset,
                            const double* cell_h, const int* cell_pbc, const int* type,
                            const double* position, const double* energy_weight,
                            const double* force_weight, double* grad_moment_coeffs,
                            double* grad_radial_coeffs, void* stream);

/* Host-buffer variant of sus2sh_compute for callers without device arrays:
 * copies type/position in, evaluates, and copies per-atom energy, forces and
 * the total virial (9 values, xx yy zz xy xz yz yx zx zy) out.  Outputs are
 * assigned.  Pinned host buffers make the copies asynchronous-capable. */
int sus2sh_compute_host(sus2sh_handle* h, int N, const double box_h[9], const int pbc[3],
                        const int* type, const double* position, double* potential,
                        double* force, double* virial_total, void* stream);

/* Stage profiler (the reference's sus2_sh_profile=1 stage times,
 * src/force/sus2_sh.cu:9631-9645,10638-10674, measured here with CUDA events
 * on the caller's stream instead of device-wide syncs).  sus2sh_profile turns
 * it on/off and clears it; sus2sh_profile_read waits for the recorded calls
 * and returns up to n values: total ms of [0] neighbour (pack + conditional
 * build) [1] basic [2] product [3] force [4] accumulate, and [5] the number
 * of profiled calls.  The option token sus2_sh_profile=1 enables it at
 * creation. */
int sus2sh_profile(sus2sh_handle* h, int enable);
int sus2sh_profile_read(sus2sh_handle* h, double* out, int n);

/* No counterpart in the reference.  The CG product stage alone (forward
 * contraction, site energy E_i and adjoints dE_i/dB_b(i)) on basic moments the
 * caller provides, for callers that cannot allocate device memory at call
 * time: MD codes that reserve all device memory up front in their own pools
 * and forbid allocations during a run, and real-time loops that cannot take
 * the synchronisation an allocation or free may imply.  It calls no
 * cudaMalloc, cudaFree or allocating library routine.
 *   basics        [alpha_index_basic_count][N], the model's basic order,
 *                 float for an FP32 handle (sus2_float=1), double otherwise
 *   potential     [N] double, assigned
 *   basic_adjoint [alpha_index_basic_count][N], same type as basics, assigned
 * An atom whose species lies outside [0, species_count) gets NaN energy and
 * NaN adjoints.  The device current at the call must be the one the handle
 * was created on (SUS2SH_E_ARG otherwise).
 * Its work area is one fixed 16 MiB device array inside the library (held by
 * every GPU that loads the library until the process exits), so
 * N * 2 * (program value slots) * sizeof(element) must be at most 16 MiB;
 * larger N is rejected with SUS2SH_E_ARG and a message giving the limit.  The
 * first call on each device resolves that array's device address with the
 * device current; make that first call before any stream capture.  All calls
 * share the array: calls that overlap on the GPU race, so serialise them.  A
 * CUDA error left pending by the caller's earlier work is not consumed. */
int sus2sh_cg_energy_noalloc(const sus2sh_handle* h, int N, const int* type, const void* basics,
                             double* potential, void* basic_adjoint, void* stream);

/* Model/graph statistics for logging (the reference prints them at
 * construction, src/force/sus2_sh.cu:9339-9466).  Fills up to n ints:
 * [0] species [1] l_max [2] k_max [3] body_order [4] rb_size [5] basics
 * [6] moments [7] products [8] scalars [9] rows [10] layers
 * [11] terminal scalar rows [12] program value slots [13] program rows
 * [14] standard graph matched [15] use_float [16] neighbour capacity
 * [17] neighbour builds so far (valid after sus2sh_sync) [18] kernels
 * launched by this handle [19] shared radial argument [20] product slots in
 * HBM [21] model-specialised CG kernel in use [22] its registers per thread
 * [23] its NVRTC compile time (ms) [24] CTA size of the basic-moment kernel
 * [25] CTA size of the force kernel (both picked by the tile autotuner at the
 * first evaluation; option sus2_sh_autotune=0 keeps 128) [26] edge kernels
 * compiled with NVRTC at load: 0 no (ahead-of-time build), 1 for the shape
 * (shape without an ahead-of-time build, FP64 or gate model; or
 * sus2_sh_edge_jit=1), 2 specialised to the model's radial coefficients (FP32
 * non-gate models; sus2_sh_model_edges=0 turns it off) [27] [28] their
 * registers per thread (basic, force; first CTA size)
 * [29] their compile time (ms) [30] two-layer gate mode (0 none,
 * 1 mu-body-linear-combo, 2 mu-scalar-full) [31] CG kernel kind (0 row
 * interpreter, 1 one straight-line function, 2 component-split) [32] [33]
 * registers and local-memory bytes per thread of the loaded CG kernel, call
 * tree included (-1 before the first evaluation) [34] how the CG kernel was
 * compiled (0 none, 1 one NVRTC program, 2 parallel relocatable units joined
 * by nvJitLink: option sus2_sh_cg_whole=0 for component-split kernels)
 * [35] 1 when that program was read from the on-disk cache of one-program
 * builds ($SUS2SH_CACHE_DIR, else $XDG_CACHE_HOME/sus2sh or
 * ~/.cache/sus2sh; SUS2SH_CACHE_DIR=off disables it)
 * [36] 1 when batches run the fused persistent kernel (valid after the first
 * sus2sh_compute_batch: option sus2_sh_batch_fused=1, FP32 models with the
 * straight-line CG kernel and model-specialised edge kernels, no gate, no
 * ZBL) [37] its registers per thread [38] its CTA shape (threads x
 * 100 + minimum resident CTAs per SM) [39] its tile size in atoms (picked by
 * timing at the first batch call, or sus2_sh_batch_tile=<atoms>) [40] its
 * NVRTC compile time (ms).  Returns the number written. */
int sus2sh_model_info(const sus2sh_handle* h, int* out, int n);

#ifdef __cplusplus
}
#endif

#endif /* SUS2SH_H */
